"""Oracle restatement of the reference FEM core (src/fem.py) — test infrastructure.

Everything is FP64 on the host with SciPy sparse matrices assembled exactly as
the reference assembles them, so `K_ff @ x`, `M_ff @ x`, solves and eigenpairs
are the reference's own operators.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

GP = 1.0 / np.sqrt(3.0)
# Local node order: bottom face CCW from (-1,-1), then top face (src/fem.py:37-46).
LOCAL = np.array([(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1),
                  (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)], dtype=float)


def shape(xi, eta, zeta):
    """N (8,), dN/dxi (8, 3): src/fem.py:49-59."""
    xs, ys, zs = LOCAL[:, 0], LOCAL[:, 1], LOCAL[:, 2]
    N = 0.125 * (1 + xs * xi) * (1 + ys * eta) * (1 + zs * zeta)
    dN = np.stack([0.125 * xs * (1 + ys * eta) * (1 + zs * zeta),
                   0.125 * (1 + xs * xi) * ys * (1 + zs * zeta),
                   0.125 * (1 + xs * xi) * (1 + ys * eta) * zs], axis=1)
    return N, dN


def D_iso(E, nu):
    """src/fem.py:62-72."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    for i in range(3):
        for j in range(3):
            D[i, j] = lam + (2 * mu if i == j else 0.0)
        D[i + 3, i + 3] = mu
    return D


def _B(dN_dx):
    B = np.zeros((6, 24))
    for n in range(8):
        gx, gy, gz = dN_dx[n]
        c = 3 * n
        B[0, c], B[1, c + 1], B[2, c + 2] = gx, gy, gz
        B[3, c], B[3, c + 1] = gy, gx
        B[4, c + 1], B[4, c + 2] = gz, gy
        B[5, c], B[5, c + 2] = gz, gx
    return B


def Ke_unit(E, nu, dx, dy, dz, D=None):
    """src/fem.py:99-132."""
    D = D_iso(E, nu) if D is None else D
    inv_half = 2.0 / np.array([dx, dy, dz])
    detJ = dx * dy * dz / 8.0
    Ke = np.zeros((24, 24))
    for a in (-GP, GP):
        for b in (-GP, GP):
            for c in (-GP, GP):
                B = _B(shape(a, b, c)[1] * inv_half)
                Ke += B.T @ D @ B * detJ
    return Ke


def Me_unit(rho, dx, dy, dz):
    """src/fem.py:135-152."""
    detJ = dx * dy * dz / 8.0
    Me = np.zeros((24, 24))
    for a in (-GP, GP):
        for b in (-GP, GP):
            for c in (-GP, GP):
                N = shape(a, b, c)[0]
                Me += np.kron(np.outer(N, N), np.eye(3)) * rho * detJ
    return Me


class OracleFEM:
    """FP64 restatement of `FEM3D` (src/fem.py:191-625)."""

    SIMP_PENALTY = 3.0          # src/fem.py:204
    E_MIN_FRAC = 1e-9           # src/fem.py:205
    MASS_THRESHOLD = 0.1        # src/fem.py:331
    MASS_PENALTY_Q = 6.0        # src/fem.py:332

    def __init__(self, geom, E, nu, rho_mat, Ke=None, Me=None):
        self.geom = geom
        self.Ke = Ke_unit(E, nu, geom.dx, geom.dy, geom.dz) if Ke is None else np.asarray(Ke)
        self.Me = Me_unit(rho_mat, geom.dx, geom.dy, geom.dz) if Me is None else np.asarray(Me)
        self.rho_mat = rho_mat
        masks = geom.build_masks()
        in_arm = masks["in_arm"].astype(bool)
        nx, ny, nz = geom.nx, geom.ny, geom.nz
        # Active elements in the reference's loop order: ez outer, ex inner
        # (src/fem.py:244-263), vectorised.
        EZ, EY, EX = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        EX, EY, EZ = EX.ravel(), EY.ravel(), EZ.ravel()
        act = in_arm[EX, EY, EZ]
        EX, EY, EZ = EX[act], EY[act], EZ[act]
        di = np.array([0, 1, 1, 0, 0, 1, 1, 0])
        dj = np.array([0, 0, 1, 1, 0, 0, 1, 1])
        dk = np.array([0, 0, 0, 0, 1, 1, 1, 1])
        NX, NY = nx + 1, ny + 1
        nodes = ((EZ[:, None] + dk) * NX * NY + (EY[:, None] + dj) * NX + (EX[:, None] + di))
        self.elem_node_ids = nodes.astype(np.int64)
        self.elem_dof_ids = (3 * nodes[:, :, None] + np.arange(3)).reshape(-1, 24)
        self.elem_grid_idx = np.stack([EX, EY, EZ], axis=1)
        self.n_active = len(EX)
        ndof = geom.n_dofs
        rr = np.repeat(self.elem_dof_ids, 24, axis=1)
        cc = np.tile(self.elem_dof_ids, (1, 24))
        self.rows, self.cols = rr.ravel(), cc.ravel()
        # Fixed DOFs (src/fem.py:282-290) plus ghost DOFs (src/fem.py:292-305).
        fixed_nodes = np.asarray(geom.fixed_nodes(), dtype=np.int64)
        fixed = np.concatenate([3 * fixed_nodes, 3 * fixed_nodes + 1, 3 * fixed_nodes + 2])
        used = np.zeros(geom.n_nodes, bool)
        used[self.elem_node_ids.ravel()] = True
        ghost = np.flatnonzero(~used)
        fixed = np.concatenate([fixed, 3 * ghost, 3 * ghost + 1, 3 * ghost + 2])
        self.fixed_dofs = np.unique(fixed)
        free = np.ones(ndof, bool)
        free[self.fixed_dofs] = False
        self.free_dofs = np.flatnonzero(free)

    # -- assembly --------------------------------------------------------- #
    def stiffness_factor(self, rho):
        """emin + (1-emin) rho^p: src/fem.py:316-320."""
        return self.E_MIN_FRAC + (1.0 - self.E_MIN_FRAC) * rho ** self.SIMP_PENALTY

    def mass_factor(self, rho):
        """src/fem.py:334-349."""
        t, q = self.MASS_THRESHOLD, self.MASS_PENALTY_Q
        return np.where(rho >= t, rho, t * (np.maximum(rho, 0.0) / t) ** q)

    def mass_factor_grad(self, rho):
        """src/fem.py:351-360."""
        t, q = self.MASS_THRESHOLD, self.MASS_PENALTY_Q
        return np.where(rho >= t, 1.0, q * (np.maximum(rho, 0.0) / t) ** (q - 1.0))

    def _assemble(self, fac, Ae):
        vals = (fac[:, None] * Ae.ravel()[None, :]).ravel()
        n = self.geom.n_dofs
        return sp.coo_matrix((vals, (self.rows, self.cols)), shape=(n, n)).tocsr()

    def assemble_K(self, rho):
        """src/fem.py:311-325."""
        return self._assemble(self.stiffness_factor(np.asarray(rho, float)), self.Ke)

    def assemble_M(self, rho, tip_mass_kg=0.0, tip_nodes=None):
        """src/fem.py:362-398: consistent SIMP mass plus an even lumped tip mass
        on the three translational DOFs of each tip node."""
        M = self._assemble(self.mass_factor(np.asarray(rho, float)), self.Me)
        if tip_mass_kg > 0.0 and tip_nodes is not None and len(tip_nodes) > 0:
            tip_nodes = np.asarray(tip_nodes, dtype=np.int64)
            d = np.concatenate([3 * tip_nodes, 3 * tip_nodes + 1, 3 * tip_nodes + 2])
            n = self.geom.n_dofs
            M = (M + sp.coo_matrix((np.full(len(d), tip_mass_kg / len(tip_nodes)), (d, d)),
                                   shape=(n, n)).tocsr()).tocsr()
        return M

    def reduce(self, A):
        f = self.free_dofs
        return A[f][:, f].tocsr()

    # -- static ----------------------------------------------------------- #
    def solve(self, rho, F, rtol=1e-8, x0=None, exact=False, maxiter=20000):
        """Jacobi PCG on K_ff (src/fem.py:529-561); `exact` uses a sparse LU
        (the reference's `method="lu"` branch).  Returns (u, info)."""
        K = self.reduce(self.assemble_K(rho))
        f = self.free_dofs
        Ff = np.asarray(F, float)[f]
        if exact:
            uf, info = spla.spsolve(K.tocsc(), Ff), 0
        else:
            d = K.diagonal()
            Minv = sp.diags(1.0 / np.where(d != 0, d, 1.0))
            uf, info = spla.cg(K, Ff, M=Minv, rtol=rtol, atol=0.0, maxiter=maxiter,
                               x0=None if x0 is None else np.asarray(x0)[f])
        u = np.zeros(self.geom.n_dofs)
        u[f] = uf
        return u, info

    # -- modal ------------------------------------------------------------ #
    def modal(self, rho, n_modes=6, tip_mass_kg=0.0, tip_nodes=None, tol=1e-12):
        """Lowest eigenpairs of K_ff v = lam M_ff v by shift-invert Lanczos
        about 0 (the reference's eigsh fallback, src/fem.py:455-461, run to a
        tight tolerance).  Modes are M-normalised; post-processing (sort,
        clamp, Hz, padding) follows src/fem.py:462-470."""
        K = self.reduce(self.assemble_K(rho))
        M = self.reduce(self.assemble_M(rho, tip_mass_kg, tip_nodes))
        lam, V = spla.eigsh(K.tocsc(), k=n_modes, M=M.tocsc(), sigma=0.0, which="LM",
                            tol=tol, maxiter=20000)
        order = np.argsort(lam)
        lam = np.maximum(lam[order], 0.0)
        V = V[:, order]
        V /= np.sqrt(np.einsum("ik,ik->k", V, M @ V))[None, :]
        modes = np.zeros((self.geom.n_dofs, n_modes))
        modes[self.free_dofs] = V
        return np.sqrt(lam) / (2 * np.pi), modes, lam

    # -- element quantities ---------------------------------------------- #
    def elem_quadform(self, v, Ae):
        ve = np.asarray(v)[self.elem_dof_ids]
        return np.einsum("ij,jk,ik->i", ve, Ae, ve)

    def elem_compliance(self, u):
        """u_e^T Ke u_e per active element: src/fem.py:605-615."""
        return self.elem_quadform(u, self.Ke)

    def eigenvalue_sensitivity(self, rho, lam, v, tip_mass_kg=0.0, tip_nodes=None):
        """d lam / d rho_e: src/fem.py:472-526 (rho_safe = max(rho, 1e-9) for
        the stiffness term, raw rho for the mass term, tip mass only in v^T M v)."""
        rho = np.asarray(rho, float)
        p, emin = self.SIMP_PENALTY, self.E_MIN_FRAC
        fKp = (1.0 - emin) * p * np.maximum(rho, 1e-9) ** (p - 1.0)
        fMp = self.mass_factor_grad(rho)
        vKv = self.elem_quadform(v, self.Ke)
        vMv_e = self.elem_quadform(v, self.Me)
        vMv = float(np.sum(self.mass_factor(rho) * vMv_e))
        if tip_mass_kg > 0.0 and tip_nodes is not None and len(tip_nodes) > 0:
            tip_nodes = np.asarray(tip_nodes, dtype=np.int64)
            d = np.concatenate([3 * tip_nodes, 3 * tip_nodes + 1, 3 * tip_nodes + 2])
            vMv += float(tip_mass_kg / len(tip_nodes) * np.sum(np.asarray(v)[d] ** 2))
        if vMv <= 0.0:
            vMv = 1.0
        return (fKp * vKv - lam * fMp * vMv_e) / vMv

    def total_mass(self, rho):
        """src/fem.py:618-621."""
        g = self.geom
        return float(np.sum(rho) * g.dx * g.dy * g.dz * self.rho_mat)
