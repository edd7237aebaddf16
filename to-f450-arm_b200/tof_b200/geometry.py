"""Synthetic voxel geometries implementing the reference's geometry interface.

The solver consumes geometry through a duck type, the one `ArmGeometry3D`
exposes (src/mesh3d.py:117-365) and `FEM3D` / `SIMPOptimizer` read
(src/fem.py:225-290, src/topopt.py:127-158):

    nx, ny, nz, dx, dy, dz, n_elements, n_nodes, n_dofs
    node_index(i, j, k), element_nodes(ex, ey, ez)
    build_masks() -> {"in_arm", "design", "keep_solid"}   (nx, ny, nz) bool
    fixed_nodes() -> node ids clamped in all three DOFs
    motor_mount_top_nodes() -> tip-mass attachment node ids
    load_dofs_for_force((Fx, Fy, Fz)) -> (dofs, magnitudes)
    load_dofs_for_moment_Mz(Mz) -> (dofs, magnitudes)

`BoxGeometry` is a rectangular voxel block with configurable clamps, a
load/mount node set and optional holes, which covers the benchmark domains:
a root-clamped cantilever and a bolted arm with a motor-mount face at the tip.
Node numbering is the reference's: node = k*(nx+1)*(ny+1) + j*(nx+1) + i
(src/mesh3d.py:134-135), element nodes bottom face CCW then top face
(src/mesh3d.py:140-146).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np


@dataclass
class BoxGeometry:
    nx: int
    ny: int
    nz: int
    dx: float = 2e-3
    dy: float = 2e-3
    dz: float = 2e-3
    # "root_face": every node on x = 0.  "bolt_patches": four 2x2-node patches
    # on the x = 0 face at y ~ ny/4, 3ny/4 and z ~ nz/4, 3nz/4.
    clamp: str = "root_face"
    # Nodes that carry the vertical load and the tip mass.  "tip_face": all
    # nodes on x = nx.  "mount_top": nodes on the top face (k = nz) of the
    # last `mount_cols` voxel columns.
    mount: str = "tip_face"
    mount_cols: int = 4
    # Optional (nx, ny, nz) bool masks; default: whole box active, no keep-solid.
    in_arm_mask: Optional[np.ndarray] = None
    keep_solid_mask: Optional[np.ndarray] = None

    n_elements: int = field(init=False)
    n_nodes: int = field(init=False)
    n_dofs: int = field(init=False)

    def __post_init__(self):
        self.n_elements = self.nx * self.ny * self.nz
        self.n_nodes = (self.nx + 1) * (self.ny + 1) * (self.nz + 1)
        self.n_dofs = 3 * self.n_nodes

    # ------------------------------------------------------------------ #
    @property
    def L_x(self):
        return self.nx * self.dx

    @property
    def L_y(self):
        return self.ny * self.dy

    @property
    def L_z(self):
        return self.nz * self.dz

    def node_index(self, i, j, k):
        return (np.asarray(k) * (self.nx + 1) * (self.ny + 1)
                + np.asarray(j) * (self.nx + 1) + np.asarray(i))

    def node_coord(self, i, j, k):
        return (i * self.dx, j * self.dy, k * self.dz)

    def element_index(self, ex, ey, ez):
        return ez * self.nx * self.ny + ey * self.nx + ex

    def element_nodes(self, ex: int, ey: int, ez: int) -> np.ndarray:
        di = np.array([0, 1, 1, 0, 0, 1, 1, 0])
        dj = np.array([0, 0, 1, 1, 0, 0, 1, 1])
        dk = np.array([0, 0, 0, 0, 1, 1, 1, 1])
        return self.node_index(ex + di, ey + dj, ez + dk).astype(np.int64)

    # ------------------------------------------------------------------ #
    def build_masks(self) -> dict:
        shape = (self.nx, self.ny, self.nz)
        in_arm = (np.ones(shape, bool) if self.in_arm_mask is None
                  else np.asarray(self.in_arm_mask, bool).copy())
        keep = (np.zeros(shape, bool) if self.keep_solid_mask is None
                else np.asarray(self.keep_solid_mask, bool).copy())
        keep &= in_arm
        return dict(in_arm=in_arm, keep_solid=keep, design=in_arm & ~keep)

    # ------------------------------------------------------------------ #
    def _face_nodes_x(self, i: int) -> np.ndarray:
        J, K = np.meshgrid(np.arange(self.ny + 1), np.arange(self.nz + 1), indexing="ij")
        return np.sort(self.node_index(i, J.ravel(), K.ravel()).astype(np.int64))

    @staticmethod
    def _patch_starts(n: int):
        lo = int(np.floor(n / 4.0 - 0.5))
        return lo, n - lo - 1

    def bolt_patches(self):
        """(j0, k0) lower corners of the four 2x2-node clamp patches on x = 0."""
        jl, jh = self._patch_starts(self.ny)
        kl, kh = self._patch_starts(self.nz)
        return [(jl, kl), (jh, kl), (jl, kh), (jh, kh)]

    def fixed_nodes(self) -> np.ndarray:
        if self.clamp == "root_face":
            return self._face_nodes_x(0)
        if self.clamp == "bolt_patches":
            nodes = []
            for j0, k0 in self.bolt_patches():
                for dj in (0, 1):
                    for dk in (0, 1):
                        nodes.append(self.node_index(0, j0 + dj, k0 + dk))
            return np.unique(np.asarray(nodes, dtype=np.int64))
        raise ValueError(f"unknown clamp {self.clamp!r}")

    def motor_mount_top_nodes(self) -> np.ndarray:
        if self.mount == "tip_face":
            return self._face_nodes_x(self.nx)
        if self.mount == "mount_top":
            I, J = np.meshgrid(np.arange(self.nx - self.mount_cols, self.nx + 1),
                               np.arange(self.ny + 1), indexing="ij")
            return np.sort(self.node_index(I.ravel(), J.ravel(), self.nz).astype(np.int64))
        raise ValueError(f"unknown mount {self.mount!r}")

    def tip_face_nodes(self) -> np.ndarray:
        return self._face_nodes_x(self.nx)

    def _node_ijk(self, nodes):
        nodes = np.asarray(nodes, dtype=np.int64)
        i = nodes % (self.nx + 1)
        j = (nodes // (self.nx + 1)) % (self.ny + 1)
        k = nodes // ((self.nx + 1) * (self.ny + 1))
        return i, j, k

    # ------------------------------------------------------------------ #
    def load_dofs_for_force(self, F_xyz):
        """Vertical component spread evenly over the mount nodes; in-plane
        components spread evenly over the tip face (x = nx)."""
        Fx, Fy, Fz = (float(v) for v in F_xyz)
        dofs, mags = [], []
        if abs(Fz) > 1e-12:
            top = self.motor_mount_top_nodes()
            dofs.append(3 * top + 2)
            mags.append(np.full(len(top), Fz / len(top)))
        if abs(Fx) + abs(Fy) > 1e-12:
            face = self.tip_face_nodes()
            dofs += [3 * face, 3 * face + 1]
            mags += [np.full(len(face), Fx / len(face)), np.full(len(face), Fy / len(face))]
        if not dofs:
            return np.array([], dtype=np.int64), np.array([])
        return np.concatenate(dofs), np.concatenate(mags)

    def load_dofs_for_moment_Mz(self, Mz: float):
        """Moment about the vertical axis through the mount-node centroid, as
        tangential in-plane nodal forces F_t = Mz / sum(r) on the mount nodes
        (the construction of src/mesh3d.py:340-365 on this node set)."""
        nodes = self.motor_mount_top_nodes()
        i, j, _ = self._node_ijk(nodes)
        x, y = i * self.dx, j * self.dy
        cx, cy = x.mean(), y.mean()
        r = np.hypot(x - cx, y - cy)
        keep = r > 1e-12
        nodes, r = nodes[keep], r[keep]
        c, s = (x[keep] - cx) / r, (y[keep] - cy) / r
        Ft = Mz / r.sum()
        return np.concatenate([3 * nodes, 3 * nodes + 1]), np.concatenate([-Ft * s, Ft * c])

    def load_dofs_for_moment_Mx(self, Mx: float):
        """Torque about the arm (x) axis through the tip-face centroid, as
        tangential nodal forces F_t = Mx / sum(r) in the y-z plane of the tip
        face."""
        nodes = self.tip_face_nodes()
        _, j, k = self._node_ijk(nodes)
        y, z = j * self.dy, k * self.dz
        cy, cz = y.mean(), z.mean()
        r = np.hypot(y - cy, z - cz)
        keep = r > 1e-12
        nodes, r = nodes[keep], r[keep]
        c, s = (y[keep] - cy) / r, (z[keep] - cz) / r
        Ft = Mx / r.sum()
        return np.concatenate([3 * nodes + 1, 3 * nodes + 2]), np.concatenate([-Ft * s, Ft * c])

    def load_vector(self, F=None, Mz=None, Mx=None) -> np.ndarray:
        out = np.zeros(self.n_dofs)
        if F is not None:
            d, m = self.load_dofs_for_force(F)
            np.add.at(out, d, m)
        if Mz is not None:
            d, m = self.load_dofs_for_moment_Mz(Mz)
            np.add.at(out, d, m)
        if Mx is not None:
            d, m = self.load_dofs_for_moment_Mx(Mx)
            np.add.at(out, d, m)
        return out

    def summary(self) -> str:
        m = self.build_masks()
        return (f"BoxGeometry {self.nx}x{self.ny}x{self.nz} @ {self.dx*1e3:.2f} mm, "
                f"{int(m['in_arm'].sum())} active, {int(m['design'].sum())} design, "
                f"{self.n_dofs} DOF, clamp={self.clamp}, mount={self.mount}")


def shell_mask(nx, ny, nz) -> np.ndarray:
    """(nx, ny, nz) bool: voxels on any of the six faces of the box."""
    m = np.zeros((nx, ny, nz), bool)
    m[0, :, :] = m[-1, :, :] = True
    m[:, 0, :] = m[:, -1, :] = True
    m[:, :, 0] = m[:, :, -1] = True
    return m


def arm_keep_solid(geom: BoxGeometry) -> np.ndarray:
    """Keep-solid voxels of the bolted arm: the root voxels touching a clamp
    patch and the top voxel layer under the motor-mount face."""
    keep = np.zeros((geom.nx, geom.ny, geom.nz), bool)
    for j0, k0 in geom.bolt_patches():
        # voxels (ex=0) sharing a node with the patch nodes j0..j0+1, k0..k0+1
        keep[0, max(j0 - 1, 0):min(j0 + 2, geom.ny), max(k0 - 1, 0):min(k0 + 2, geom.nz)] = True
    keep[geom.nx - geom.mount_cols:, :, geom.nz - 1] = True
    return keep
