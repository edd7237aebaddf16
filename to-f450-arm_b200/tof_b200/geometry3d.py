"""The production F450 arm domain (the reference's ArmGeometry3D), vectorised.

The reference builds its production voxel domain in src/mesh3d.py:43-389:
a 216 x 42 x 54 mm bounding box at 2 mm voxels with six body-side screw
holes (four from the top plate, two from the bottom plate, each over its own
engaged z span), a motor-mount hole through the top pad, keep-solid collars
around the screws and the motor pad, clamps on the screw bearing annuli, the
motor + propeller tip mass on the top-face pad nodes, and thrust / in-plane
bearing / motor-torque loads on the pad and the hole wall.  Its clamp and
load builders walk every node in Python loops.  This class produces the same
masks, node sets (in the same order) and load vectors with array operations,
so the production domain runs through tof_b200.fem.FEM3D.  The dimensions,
screw table and ring sizes are the reference's (they define the domain).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Tuple

import numpy as np


@dataclass
class ArmGeometry3D:
    """Production F450 arm voxel domain (src/mesh3d.py:43-110)."""

    L_x: float = 216e-3
    L_y: float = 42e-3
    L_z: float = 54e-3
    dx: float = 2e-3
    dy: float = 2e-3
    dz: float = 2e-3
    screw_dia: float = 2.5e-3
    # (x, y, z0, z1): screw axis and the z span it engages (src/mesh3d.py:74-87)
    screws: Tuple[Tuple[float, float, float, float], ...] = (
        (25.8e-3, 9.5e-3, 33.2e-3, 53.2e-3),
        (25.8e-3, 32.5e-3, 33.2e-3, 53.2e-3),
        (5.8e-3, 12.7e-3, 46.9e-3, 53.2e-3),
        (5.8e-3, 29.2e-3, 46.9e-3, 53.2e-3),
        (25.5e-3, 10.5e-3, 15.2e-3, 35.2e-3),
        (25.5e-3, 31.5e-3, 15.2e-3, 35.2e-3),
    )
    motor_dia: float = 10e-3
    motor_centre: Tuple[float, float] = (195.6e-3, 21e-3)
    keep_solid_ring: float = 4.0e-3
    motor_keep_ring: float = 8.0e-3
    motor_pad_depth: float = 4e-3
    nx: int = field(init=False)
    ny: int = field(init=False)
    nz: int = field(init=False)
    n_elements: int = field(init=False)
    n_nodes: int = field(init=False)
    n_dofs: int = field(init=False)

    def __post_init__(self):
        self.nx = int(round(self.L_x / self.dx))
        self.ny = int(round(self.L_y / self.dy))
        self.nz = int(round(self.L_z / self.dz))
        self.n_elements = self.nx * self.ny * self.nz
        self.n_nodes = (self.nx + 1) * (self.ny + 1) * (self.nz + 1)
        self.n_dofs = 3 * self.n_nodes

    @property
    def screw_centres(self):
        return tuple((s[0], s[1]) for s in self.screws)

    # -- indexing (src/mesh3d.py:126-146) --------------------------------- #
    def element_centre(self, ex, ey, ez):
        return ((ex + 0.5) * self.dx, (ey + 0.5) * self.dy, (ez + 0.5) * self.dz)

    def node_coord(self, ix, iy, iz):
        return (ix * self.dx, iy * self.dy, iz * self.dz)

    def node_index(self, ix, iy, iz):
        return iz * (self.nx + 1) * (self.ny + 1) + iy * (self.nx + 1) + ix

    def element_index(self, ex, ey, ez):
        return ez * self.nx * self.ny + ey * self.nx + ex

    def element_nodes(self, ex, ey, ez) -> np.ndarray:
        """8 node indices, bottom face counter-clockwise then top face."""
        return np.array([self.node_index(ex + ox, ey + oy, ez + oz)
                         for oz in (0, 1) for oy, ox in ((0, 0), (0, 1), (1, 1), (1, 0))], dtype=np.int64)

    # -- helpers ------------------------------------------------------------ #
    def _node_xy(self):
        """(NX, NY) node x and y coordinates, indexed [ix, iy]."""
        x = np.arange(self.nx + 1) * self.dx
        y = np.arange(self.ny + 1) * self.dy
        return np.meshgrid(x, y, indexing="ij")

    def _stack_z(self, ixy, iz0, iz1):
        """Node indices for each selected (ix, iy) (in row-major [ix, iy]
        order) times iz = iz0..iz1, iz fastest, as the reference's loops."""
        ix, iy = ixy
        iz = np.arange(iz0, iz1 + 1)
        return (iz[None, :] * (self.nx + 1) * (self.ny + 1) + (iy * (self.nx + 1) + ix)[:, None]).ravel()

    def _pad_wall(self):
        """(ix, iy, d) of the nodes on the motor hole wall annulus and the
        first z layer of the pad (src/mesh3d.py:253-270)."""
        cx, cy = self.motor_centre
        X, Y = self._node_xy()
        d = np.hypot(X - cx, Y - cy)
        r_in, r_out = self.motor_dia / 2.0, self.motor_dia / 2.0 + self.motor_keep_ring
        ix, iy = np.nonzero((r_in <= d) & (d <= r_out))
        iz0 = int(round((self.L_z - self.motor_pad_depth) / self.dz))
        return ix, iy, d[ix, iy], X[ix, iy], Y[ix, iy], iz0

    # -- masks (src/mesh3d.py:149-200) --------------------------------------- #
    def build_masks(self) -> dict:
        XC, YC, ZC = np.meshgrid((np.arange(self.nx) + 0.5) * self.dx, (np.arange(self.ny) + 0.5) * self.dy,
                                 (np.arange(self.nz) + 0.5) * self.dz, indexing="ij")
        in_screw = np.zeros(XC.shape, bool)
        keep_screw = np.zeros(XC.shape, bool)
        r_keep = (self.screw_dia / 2.0 + self.keep_solid_ring) ** 2
        for cx, cy, z0, z1 in self.screws:
            r2 = (XC - cx) ** 2 + (YC - cy) ** 2
            in_screw |= (r2 <= (self.screw_dia / 2.0) ** 2) & (ZC >= z0) & (ZC <= z1)
            keep_screw |= (r2 <= r_keep) & (ZC >= z0 - self.dz) & (ZC <= z1 + self.dz)
        z_top = self.L_z - self.motor_pad_depth
        rm2 = (XC - self.motor_centre[0]) ** 2 + (YC - self.motor_centre[1]) ** 2
        in_motor = (rm2 <= (self.motor_dia / 2.0) ** 2) & (ZC > z_top)
        in_arm = ~in_screw & ~in_motor
        keep_screw &= in_arm
        keep_motor = (rm2 <= (self.motor_dia / 2.0 + self.motor_keep_ring) ** 2) & (ZC > z_top) & in_arm
        keep_solid = keep_screw | keep_motor
        return dict(in_arm=in_arm, keep_solid=keep_solid, design=in_arm & ~keep_solid, keep_screw=keep_screw,
                    keep_motor=keep_motor)

    # -- boundary conditions (src/mesh3d.py:203-228) --------------------------- #
    def fixed_nodes(self) -> np.ndarray:
        """Nodes on each screw's bearing annulus over its span +- one voxel."""
        X, Y = self._node_xy()
        r_out, r_in = self.screw_dia / 2.0 + self.keep_solid_ring, self.screw_dia / 2.0
        z = np.arange(self.nz + 1) * self.dz
        out = []
        for cx, cy, z0, z1 in self.screws:
            d = np.hypot(X - cx, Y - cy)
            ix, iy = np.nonzero((r_in <= d) & (d <= r_out))
            izs = np.nonzero((z0 - self.dz <= z) & (z <= z1 + self.dz))[0]
            if len(ix) and len(izs):
                out.append((izs[None, :] * (self.nx + 1) * (self.ny + 1) + (iy * (self.nx + 1) + ix)[:, None]).ravel())
        return np.unique(np.concatenate(out)) if out else np.array([], dtype=np.int64)

    # -- motor mount (src/mesh3d.py:231-250) ----------------------------------- #
    def motor_mount_top_nodes(self) -> np.ndarray:
        """Top-face nodes within the motor pad radius, [ix, iy] order."""
        X, Y = self._node_xy()
        d = np.hypot(X - self.motor_centre[0], Y - self.motor_centre[1])
        ix, iy = np.nonzero(d <= self.motor_dia / 2.0 + self.motor_keep_ring)
        return (self.nz * (self.nx + 1) * (self.ny + 1) + iy * (self.nx + 1) + ix).astype(np.int64)

    # -- loads (src/mesh3d.py:273-365) ----------------------------------------- #
    def load_dofs_for_force(self, F_xyz):
        """Fz spread evenly over the pad's top-face nodes; (Fx, Fy) as a
        cosine-weighted bearing load on the hole wall (pad layers)."""
        Fx, Fy, Fz = F_xyz
        dofs, mags = [], []
        if abs(Fz) > 1e-12:
            top = self.motor_mount_top_nodes()
            dofs.append(3 * top + 2)
            mags.append((Fz / len(top)) * np.ones(len(top)))
        if abs(Fx) + abs(Fy) > 1e-12:
            ix, iy, d, x, y, iz0 = self._pad_wall()
            cx, cy = self.motor_centre
            ld = np.asarray((Fx, Fy), float)
            ld = ld / np.linalg.norm(ld)
            cos_t = -(((x - cx) / d) * ld[0] + ((y - cy) / d) * ld[1])
            keep = cos_t > 1e-6
            if keep.any():
                nl = self.nz - iz0 + 1
                nodes = self._stack_z((ix[keep], iy[keep]), iz0, self.nz)
                w = np.repeat(cos_t[keep], nl)
                w = w / w.sum()
                dofs += [3 * nodes, 3 * nodes + 1]
                mags += [Fx * w, Fy * w]
        if not dofs:
            return np.array([], dtype=np.int64), np.array([])
        return np.concatenate(dofs), np.concatenate(mags)

    def load_dofs_for_moment_Mz(self, Mz):
        """Moment about the motor axis as tangential forces on the hole wall."""
        ix, iy, d, x, y, iz0 = self._pad_wall()
        cx, cy = self.motor_centre
        nl = self.nz - iz0 + 1
        nodes = self._stack_z((ix, iy), iz0, self.nz)
        r = np.repeat(d, nl)
        c = np.repeat((x - cx) / d, nl)
        s = np.repeat((y - cy) / d, nl)
        Ft = Mz / r.sum()
        return np.concatenate([3 * nodes, 3 * nodes + 1]), np.concatenate([-Ft * s, Ft * c])

    def load_vector(self, F=None, Mz=None) -> np.ndarray:
        """Full-length load vector from a force and / or a motor-axis moment."""
        out = np.zeros(self.n_dofs)
        if F is not None:
            d, v = self.load_dofs_for_force(F)
            np.add.at(out, d, v)
        if Mz is not None:
            d, v = self.load_dofs_for_moment_Mz(Mz)
            np.add.at(out, d, v)
        return out

    def summary(self) -> str:
        m = self.build_masks()
        return (f"ArmGeometry3D: {self.L_x*1e3:.1f} x {self.L_y*1e3:.1f} x {self.L_z*1e3:.1f} mm, "
                f"grid {self.nx} x {self.ny} x {self.nz}, {int(m['in_arm'].sum())} elements in the arm, "
                f"{int(m['design'].sum())} design, {int(m['keep_solid'].sum())} keep-solid")
