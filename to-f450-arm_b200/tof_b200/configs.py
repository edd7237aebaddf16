"""Benchmark workloads: material, geometry, densities and load cases.

Five synthetic workloads exercise the voxel SIMP path (sizes in voxels):

* cantilever 40x8x8 @ 2 mm: root face clamped, -10 N z over the tip face,
  density 0.5 + U(-0.05, 0.05) (seed 0); one static solve and 6 modes.
* arm 110x14x12 @ 2 mm: four 2x2-node bolt patches on the root face, -15 N z
  over the motor-mount face (top face of the last 4 voxel columns), hollow
  box density (1-voxel shell 1.0, interior 1e-3), 60 g tip mass on the mount.
* the arm grid with design density 0.08 + U(-0.02, 0.02) (seed 0) for
  differentiation and SIMP iterations at vf = 0.08, filter radius 1.5 voxels.
* the arm grid with four load cases solved together (thrust; 0.3 N m torque
  about the arm axis plus 10 N lateral; both; 3 g -z inertial body load).
* five arm designs (vf 0.08 / 0.10 / 0.20 / 0.30 / 0.50) plus one 1 mm arm
  (220x28x24) batched together.

PA12 material: E = 1.7 GPa, nu = 0.39, rho = 1010 kg/m^3.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .geometry import BoxGeometry, arm_keep_solid, shell_mask


@dataclass
class Material:
    """Linear-elastic material; field names follow src/fem.py:182-188."""
    E: float = 1700e6
    nu: float = 0.39
    sigma_y: float = 38e6
    sigma_u: float = 48e6
    rho: float = 930.0


PA12 = Material(E=1.7e9, nu=0.39, sigma_y=38e6, sigma_u=48e6, rho=1010.0)
TIP_MASS_KG = 0.060
G0 = 9.81


def active_element_ids(in_arm: np.ndarray) -> np.ndarray:
    """Flat element ids e = ez*nx*ny + ey*nx + ex of active voxels, ascending.

    This is the order of the reference's `rho_active` vector, whose element
    loop runs z outermost and x innermost (src/fem.py:244-246)."""
    return np.flatnonzero(np.asarray(in_arm, bool).transpose(2, 1, 0).ravel())


def grid_to_active(grid: np.ndarray, in_arm: np.ndarray) -> np.ndarray:
    """(nx, ny, nz) grid values -> rho_active order."""
    return np.asarray(grid).transpose(2, 1, 0).ravel()[active_element_ids(in_arm)]


def active_to_grid(vals: np.ndarray, in_arm: np.ndarray) -> np.ndarray:
    """rho_active-ordered values -> (nx, ny, nz) grid with zeros elsewhere."""
    nx, ny, nz = in_arm.shape
    flat = np.zeros(nx * ny * nz, dtype=np.asarray(vals).dtype)
    flat[active_element_ids(in_arm)] = vals
    return flat.reshape(nz, ny, nx).transpose(2, 1, 0).copy()


# ---------------------------------------------------------------------- #
def cantilever_geometry(nx=40, ny=8, nz=8, h=2e-3) -> BoxGeometry:
    return BoxGeometry(nx, ny, nz, h, h, h, clamp="root_face", mount="tip_face")


def cantilever_density(geom: BoxGeometry, seed: int = 0) -> np.ndarray:
    n = int(geom.build_masks()["in_arm"].sum())
    return 0.5 + np.random.default_rng(seed).uniform(-0.05, 0.05, n)


def cantilever_loads(geom: BoxGeometry):
    return [geom.load_vector(F=(0.0, 0.0, -10.0))]


def arm_geometry(nx=110, ny=14, nz=12, h=2e-3, mount_cols=None,
                 keep_solid: bool = True) -> BoxGeometry:
    if mount_cols is None:
        mount_cols = max(1, int(round(8e-3 / h)))      # 8 mm motor-mount face
    g = BoxGeometry(nx, ny, nz, h, h, h, clamp="bolt_patches", mount="mount_top",
                    mount_cols=mount_cols)
    if keep_solid:
        g.keep_solid_mask = arm_keep_solid(g)
    return g


def arm_hollow_density(geom: BoxGeometry, wall=1.0, core=1e-3) -> np.ndarray:
    m = geom.build_masks()
    grid = np.where(shell_mask(geom.nx, geom.ny, geom.nz), wall, core)
    return grid_to_active(grid, m["in_arm"])


def arm_design_start(geom: BoxGeometry, vf=0.08, spread=0.02, seed=0) -> np.ndarray:
    """Design-cell start values vf + U(-spread, spread), FP32, in the
    reference's design-cell order (grid[design] on the (nx, ny, nz) array)."""
    n = int(geom.build_masks()["design"].sum())
    x = vf + np.random.default_rng(seed).uniform(-spread, spread, n)
    return x.astype(np.float32)


def arm_static_loads(geom: BoxGeometry):
    """The three surface-load cases on the arm: thrust; torque about the arm
    axis plus lateral; both together."""
    lc1 = geom.load_vector(F=(0.0, 0.0, -15.0))
    lc2 = geom.load_vector(F=(0.0, 10.0, 0.0), Mx=0.3)
    return [lc1, lc2, lc1 + lc2]


def body_load_from_Mr(M_times_ez: np.ndarray, n_g: float = 3.0) -> np.ndarray:
    """Inertial load -n_g * g0 * M e_z, given M e_z (the consistent mass
    applied to a unit z translation)."""
    return -n_g * G0 * np.asarray(M_times_ez)


SWEEP_VFS = (0.08, 0.10, 0.20, 0.30, 0.50)
