"""Hex8 element matrices for the structured voxel grid (host side, FP64).

These are the constants the device kernels are parameterised with: one 24x24
stiffness matrix and one 24x24 consistent mass matrix for a unit-density voxel,
scaled per element on the device by the SIMP factors.

Conventions follow the reference solver so that matrices are interchangeable
with its `FEM3D.Ke_solid` / `FEM3D.Me_solid` (src/fem.py:99-152):

* local node order: bottom face (zeta=-1) counter-clockwise from (-1,-1), then
  the top face in the same order (src/fem.py:35-46);
* DOF order per node is [ux, uy, uz], so local DOF = 3*node + component
  (src/fem.py:119-130);
* Voigt strain order [exx, eyy, ezz, gxy, gyz, gxz] (src/fem.py:63);
* 2x2x2 Gauss quadrature with unit weights (src/fem.py:29-33).

The integration here is vectorised over the eight Gauss points instead of the
reference's per-point Python loop; results agree to FP64 round-off.
"""
from __future__ import annotations

import numpy as np

# Corner signs of the reference hexahedron, in the local node order above.
CORNER_SIGNS = np.array([
    [-1, -1, -1], [+1, -1, -1], [+1, +1, -1], [-1, +1, -1],
    [-1, -1, +1], [+1, -1, +1], [+1, +1, +1], [-1, +1, +1],
], dtype=np.float64)

# Offsets (di, dj, dk) of each local node from the element's lowest corner
# node on the structured grid.
CORNER_OFFSETS = ((CORNER_SIGNS + 1) // 2).astype(np.int64)

_G = 1.0 / np.sqrt(3.0)
# 2x2x2 Gauss points, weights all 1.
GAUSS_POINTS = np.array([[a, b, c] for a in (-_G, _G) for b in (-_G, _G)
                         for c in (-_G, _G)], dtype=np.float64)


def _shape(points: np.ndarray):
    """Trilinear shape functions and their parametric gradients.

    points: (P, 3) parametric coordinates.
    Returns N (P, 8) and dN (P, 8, 3) = dN_a / d(xi, eta, zeta).
    """
    s = CORNER_SIGNS[None, :, :]              # (1, 8, 3)
    p = points[:, None, :]                    # (P, 1, 3)
    f = 1.0 + s * p                           # (P, 8, 3) one linear factor per axis
    N = 0.125 * f[..., 0] * f[..., 1] * f[..., 2]
    dN = np.empty(points.shape[:1] + (8, 3))
    dN[..., 0] = 0.125 * s[..., 0] * f[..., 1] * f[..., 2]
    dN[..., 1] = 0.125 * f[..., 0] * s[..., 1] * f[..., 2]
    dN[..., 2] = 0.125 * f[..., 0] * f[..., 1] * s[..., 2]
    return N, dN


def isotropic_D(E: float, nu: float) -> np.ndarray:
    """6x6 isotropic elasticity matrix in Voigt order [xx, yy, zz, xy, yz, xz]."""
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] += 2.0 * mu
    D[np.arange(3, 6), np.arange(3, 6)] = mu
    return D


def orthotropic_D(Ex, Ey, Ez, nu_xy, nu_yz, nu_xz, Gxy, Gyz, Gxz) -> np.ndarray:
    """6x6 orthotropic elasticity matrix from engineering constants.

    Built by inverting the symmetric compliance matrix, the same construction
    as the reference's anisotropy study helper (src/fem.py:75-96).
    """
    S = np.diag([1.0 / Ex, 1.0 / Ey, 1.0 / Ez, 1.0 / Gxy, 1.0 / Gyz, 1.0 / Gxz])
    S[0, 1] = S[1, 0] = -nu_xy / Ex
    S[1, 2] = S[2, 1] = -nu_yz / Ey
    S[0, 2] = S[2, 0] = -nu_xz / Ex
    return np.linalg.inv(S)


def strain_displacement(dN_phys: np.ndarray) -> np.ndarray:
    """Voigt B matrices from physical shape-function gradients.

    dN_phys: (P, 8, 3). Returns B (P, 6, 24).
    """
    P = dN_phys.shape[0]
    B = np.zeros((P, 6, 8, 3))
    gx, gy, gz = dN_phys[..., 0], dN_phys[..., 1], dN_phys[..., 2]
    B[:, 0, :, 0] = gx
    B[:, 1, :, 1] = gy
    B[:, 2, :, 2] = gz
    B[:, 3, :, 0] = gy
    B[:, 3, :, 1] = gx
    B[:, 4, :, 1] = gz
    B[:, 4, :, 2] = gy
    B[:, 5, :, 0] = gz
    B[:, 5, :, 2] = gx
    return B.reshape(P, 6, 24)


def element_stiffness(dx: float, dy: float, dz: float, D: np.ndarray) -> np.ndarray:
    """24x24 stiffness of a dx*dy*dz brick: sum_gp B^T D B |J| (weights 1)."""
    half = np.array([dx, dy, dz], dtype=np.float64) / 2.0
    detJ = half.prod()
    _, dN = _shape(GAUSS_POINTS)
    B = strain_displacement(dN / half[None, None, :])
    Ke = np.einsum("pik,ij,pjl->kl", B, D, B) * detJ
    return 0.5 * (Ke + Ke.T)


def element_mass(rho: float, dx: float, dy: float, dz: float) -> np.ndarray:
    """24x24 consistent mass: rho * sum_gp (N N^T kron I3) |J| (weights 1)."""
    half = np.array([dx, dy, dz], dtype=np.float64) / 2.0
    detJ = half.prod()
    N, _ = _shape(GAUSS_POINTS)
    NN = np.einsum("pa,pb->ab", N, N) * (rho * detJ)
    return np.kron(NN, np.eye(3))


def element_B_centre(dx: float, dy: float, dz: float) -> np.ndarray:
    """6x24 strain-displacement matrix at the element centre (stress recovery)."""
    half = np.array([dx, dy, dz], dtype=np.float64) / 2.0
    _, dN = _shape(np.zeros((1, 3)))
    return strain_displacement(dN / half[None, None, :])[0]
