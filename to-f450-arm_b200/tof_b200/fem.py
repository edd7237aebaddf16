"""`FEM3D` with the reference's interface, computed on the B200 through libtof.

Mirrors `FEM3D` of the reference (src/fem.py:191-625): same constructor
arguments, same attributes (Ke_solid, Me_solid, D_solid, B_centre,
elem_dof_ids, elem_grid_idx, free_dofs, fixed_dofs, n_active, rho_active),
same method signatures and return shapes (NumPy FP64 in, NumPy FP64 out).
Nothing is assembled: `assemble_K` / `assemble_M` return operator handles
bound to the densities, and every solve / product / element contraction runs
in the CUDA library.  There is no CPU fallback: without a GPU or without the
built library every compute method raises.

Solver selection (`mode`):
  "fp64"  - the reference's algorithms in FP64: Jacobi PCG, Jacobi LOBPCG.
  "mixed" - FP64 Krylov / LOBPCG preconditioned by an FP32 geometric
            multigrid V-cycle; all load cases solved as one block.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from .configs import active_element_ids
from .element import element_B_centre, element_mass, element_stiffness, isotropic_D
from .engine import DesignContext


class _Operator:
    """Matrix-free K(rho) or M(rho) bound to a density (the value
    `assemble_K` / `assemble_M` return)."""

    def __init__(self, fem, kind, rho, tip_mass_kg=0.0, tip_mass_nodes=None):
        self.fem, self.kind = fem, kind
        self.rho = np.array(rho, dtype=np.float64, copy=True)
        self.tip_mass_kg, self.tip_mass_nodes = tip_mass_kg, tip_mass_nodes
        n = fem.geom.n_dofs
        self.shape = (n, n)

    def __matmul__(self, x):
        """A_ff x for a full-length vector (N,) or block (N, k); zeros at fixed DOFs."""
        return self.fem._apply(self, np.asarray(x, dtype=np.float64))

    dot = __matmul__

    def diagonal(self):
        fem = self.fem
        ctx = fem._prepare(self.rho, self.tip_mass_kg if self.kind == "M" else None, self.tip_mass_nodes)
        d = ctx.diag(L.OP_K if self.kind == "K" else L.OP_M)[:, :3].reshape(-1)
        return d.cpu().numpy()


class FEM3D:
    SIMP_PENALTY = 3.0          # src/fem.py:204
    E_MIN_FRAC = 1e-9           # src/fem.py:205
    MASS_THRESHOLD = 0.1        # src/fem.py:331
    MASS_PENALTY_Q = 6.0        # src/fem.py:332
    SOLVE_RTOL = 1e-5           # default of apply_BCs_and_solve (src/fem.py:532)
    SOLVE_MAXITER = 5000        # src/fem.py:546
    LU_RTOL = 1e-12             # method="lu" is served by PCG to this tolerance
    MODAL_TOL_CAP = 1e-5        # LOBPCG relative residual cap (eigenvalues to ~1e-10)

    def __init__(self, geom, mat, mode: str = "fp64", max_rhs: int = 8, max_modes: int = 8, tile=None):
        if mode not in ("fp64", "mixed"):
            raise ValueError("mode must be 'fp64' or 'mixed'")
        self.geom, self.mat, self.mode = geom, mat, mode
        self.max_rhs, self.max_modes, self.tile = max_rhs, max_modes, tile
        self.D_solid = isotropic_D(mat.E, mat.nu)
        self.Ke_solid = element_stiffness(geom.dx, geom.dy, geom.dz, self.D_solid)
        self.B_centre = element_B_centre(geom.dx, geom.dy, geom.dz)
        self.Me_solid = element_mass(mat.rho, geom.dx, geom.dy, geom.dz)
        masks = geom.build_masks()
        self.in_arm = np.asarray(masks["in_arm"], bool)
        self.active_ids = active_element_ids(self.in_arm)      # rho_active order -> grid element id
        nx, ny, nz = geom.nx, geom.ny, geom.nz
        ex = self.active_ids % nx
        ey = (self.active_ids // nx) % ny
        ez = self.active_ids // (nx * ny)
        self.elem_grid_idx = np.stack([ex, ey, ez], axis=1)
        di = np.array([0, 1, 1, 0, 0, 1, 1, 0])
        dj = np.array([0, 0, 1, 1, 0, 0, 1, 1])
        dk = np.array([0, 0, 0, 0, 1, 1, 1, 1])
        NX, NY = nx + 1, ny + 1
        self.elem_node_ids = ((ez[:, None] + dk) * NX * NY + (ey[:, None] + dj) * NX + (ex[:, None] + di))
        self.elem_dof_ids = (3 * self.elem_node_ids[:, :, None] + np.arange(3)).reshape(-1, 24)
        self.n_active = len(self.active_ids)
        # fixed DOFs (src/fem.py:282-290) plus ghost nodes of no active element (:292-305)
        fixed_nodes = np.asarray(geom.fixed_nodes(), dtype=np.int64)
        used = np.zeros(geom.n_nodes, bool)
        used[self.elem_node_ids.ravel()] = True
        ghost = np.flatnonzero(~used)
        nodes = np.concatenate([fixed_nodes, ghost])
        self.fixed_dofs = np.unique(np.concatenate([3 * nodes, 3 * nodes + 1, 3 * nodes + 2]))
        free = np.ones(geom.n_dofs, bool)
        free[self.fixed_dofs] = False
        self.free_dofs = np.flatnonzero(free)
        self.rho_active = np.ones(self.n_active)
        self._ctx = None
        self._ctx_key = None
        self._rho_dev = None
        self._tip_key = None
        self.last_stats = None

    # -- flattened templates, as the reference exposes them ---------------- #
    @property
    def Ke_flat(self):
        return self.Ke_solid.ravel()

    @property
    def Me_flat(self):
        return self.Me_solid.ravel()

    # -- device context ------------------------------------------------------ #
    def device(self) -> DesignContext:
        """The libtof context; rebuilt if Ke_solid / Me_solid were replaced
        (the reference's callers may overwrite them, e.g. an orthotropic D)."""
        key = (self.Ke_solid.tobytes(), self.Me_solid.tobytes(), self.SIMP_PENALTY, self.E_MIN_FRAC,
               self.MASS_THRESHOLD, self.MASS_PENALTY_Q)
        if self._ctx is None or key != self._ctx_key:
            g = self.geom
            if self.tile == "auto":                       # measured once per grid (tof_b200.autotune)
                from .autotune import tune_tile
                self.tile = tune_tile(self)
            self._ctx = DesignContext(g.nx, g.ny, g.nz, (g.dx, g.dy, g.dz), self.Ke_solid, self.Me_solid,
                                      active_grid=self.in_arm, fixed_dofs=self.fixed_dofs,
                                      simp=(self.SIMP_PENALTY, self.E_MIN_FRAC, self.MASS_THRESHOLD,
                                            self.MASS_PENALTY_Q),
                                      max_rhs=self.max_rhs, max_modes=self.max_modes, tile=self.tile)
            self._ctx_key = key
            self._rho_dev = None
            self._tip_key = None
        return self._ctx

    def rho_to_grid(self, rho_active) -> torch.Tensor:
        """rho_active (n_active,) -> device FP64 element grid (NE,), x fastest."""
        ctx = self.device()
        r = torch.as_tensor(np.asarray(rho_active, dtype=np.float64)).to(ctx.device)
        grid = torch.zeros(ctx.NE, dtype=torch.float64, device=ctx.device)
        grid[torch.as_tensor(self.active_ids, device=ctx.device)] = r
        return grid

    def _tip_nodes(self, tip_mass_nodes):
        if tip_mass_nodes is not None:
            return np.asarray(tip_mass_nodes, dtype=np.int64)
        if hasattr(self.geom, "motor_mount_top_nodes"):                  # src/fem.py:426-432
            return np.asarray(self.geom.motor_mount_top_nodes(), dtype=np.int64)
        if hasattr(self.geom, "_motor_top_boundary_nodes"):
            return np.asarray(self.geom._motor_top_boundary_nodes(), dtype=np.int64)
        return np.array([], dtype=np.int64)

    def tip_lump(self, tip_mass_kg, tip_mass_nodes):
        """Per-DOF lumped mass mass_kg / n_nodes on each tip node's three DOFs
        (src/fem.py:383-398); None when there is no tip mass."""
        nodes = self._tip_nodes(tip_mass_nodes)
        if not tip_mass_kg or tip_mass_kg <= 0.0 or len(nodes) == 0:
            return None
        t = np.zeros(self.geom.n_dofs)
        for c in range(3):
            np.add.at(t, 3 * nodes + c, tip_mass_kg / len(nodes))
        return t

    def _prepare(self, rho_active, tip_mass_kg=None, tip_mass_nodes=None) -> DesignContext:
        ctx = self.device()
        rho = np.asarray(rho_active, dtype=np.float64)
        if self._rho_dev is None or not np.array_equal(self._rho_dev, rho):
            ctx.set_density(self.rho_to_grid(rho))
            self._rho_dev = rho.copy()
        if tip_mass_kg is not None:
            t = self.tip_lump(tip_mass_kg, tip_mass_nodes)
            key = None if t is None else t.tobytes()
            if key != self._tip_key:
                ctx.set_tip_lump(t)
                self._tip_key = key
        return ctx

    def _apply(self, op: _Operator, x):
        ctx = self._prepare(op.rho, op.tip_mass_kg if op.kind == "M" else None, op.tip_mass_nodes)
        vec = x.ndim == 1
        X = x[:, None] if vec else x
        dev = ctx.pack(torch.from_numpy(np.ascontiguousarray(X.T)))
        y = ctx.unpack(ctx.matvec(L.OP_K if op.kind == "K" else L.OP_M, dev)).cpu().numpy().T
        return y[:, 0] if vec else y

    def _mode_id(self, mode=None):
        return L.MODE_MIXED if (mode or self.mode) == "mixed" else L.MODE_FP64

    # -- assembly (operators, no matrices) ------------------------------------ #
    def stiffness_factor(self, rho_active):
        """emin + (1 - emin) rho^p (src/fem.py:316-320)."""
        return self.E_MIN_FRAC + (1.0 - self.E_MIN_FRAC) * np.asarray(rho_active, float) ** self.SIMP_PENALTY

    def _mass_simp_factor(self, rho_active):
        """src/fem.py:334-349."""
        r = np.asarray(rho_active, float)
        t, q = self.MASS_THRESHOLD, self.MASS_PENALTY_Q
        return np.where(r >= t, r, t * (np.maximum(r, 0.0) / t) ** q)

    def _mass_simp_factor_grad(self, rho_active):
        """src/fem.py:351-360."""
        r = np.asarray(rho_active, float)
        t, q = self.MASS_THRESHOLD, self.MASS_PENALTY_Q
        return np.where(r >= t, 1.0, q * (np.maximum(r, 0.0) / t) ** (q - 1.0))

    def assemble_K(self, rho_active):
        """Matrix-free K(rho) handle (replaces src/fem.py:311-325)."""
        return _Operator(self, "K", rho_active)

    def assemble_M(self, rho_active, tip_mass_kg=0.0, tip_mass_nodes=None):
        """Matrix-free M(rho) handle with the lumped tip mass (src/fem.py:362-398)."""
        return _Operator(self, "M", rho_active, tip_mass_kg, tip_mass_nodes)

    # -- static ---------------------------------------------------------------- #
    def apply_BCs_and_solve(self, K, F, method="cg", x0=None, rtol=1e-5):
        """Solve K_ff u_f = F_f, u = 0 at fixed DOFs (src/fem.py:529-555).
        K must be the handle `assemble_K` returned."""
        if not isinstance(K, _Operator) or K.kind != "K":
            raise TypeError("apply_BCs_and_solve needs the operator returned by assemble_K "
                            "(no assembled matrix exists on this path)")
        u, = self.solve_block(K.rho, [F], [x0], rtol=self.LU_RTOL if method == "lu" else rtol)[0]
        return u

    def solve(self, rho_active, F, method="cg", x0=None):
        """src/fem.py:558-561."""
        rtol = self.LU_RTOL if method == "lu" else self.SOLVE_RTOL
        u, = self.solve_block(rho_active, [F], [x0], rtol=rtol)[0]
        return u

    def solve_block(self, rho_active, F_list, x0_list=None, rtol=None, mode=None, maxiter=None):
        """All load cases at once: returns ([u_i], stats).  Extension of `solve`."""
        ctx = self._prepare(rho_active)
        F = np.stack([np.asarray(f, dtype=np.float64) for f in F_list])
        b = ctx.pack(torch.from_numpy(F))
        x0 = None
        if x0_list is not None and any(x is not None for x in x0_list):
            X = np.stack([np.zeros(self.geom.n_dofs) if x is None else np.asarray(x, float) for x in x0_list])
            x0 = ctx.pack(torch.from_numpy(X))
        mid = self._mode_id(mode)
        R = len(F_list)
        us = []
        stats = []
        step = R if mid == L.MODE_MIXED else 1
        for s in range(0, R, step):
            xs, st = ctx.pcg(b[s:s + step], None if x0 is None else x0[s:s + step],
                             rtol=self.SOLVE_RTOL if rtol is None else rtol,
                             maxiter=maxiter or max(self.SOLVE_MAXITER, 20000), mode=mid)
            us.append(ctx.unpack(xs))
            stats += st
        u = torch.cat(us).cpu().numpy()
        self.last_stats = stats
        return [u[i] for i in range(R)], stats

    # -- modal ------------------------------------------------------------------ #
    def modal_analysis(self, rho_active, n_modes=6, tip_mass_kg=0.060, tip_mass_nodes=None, X0_free=None,
                       tol=1e-4, maxiter=500):
        """Lowest n_modes of K v = omega^2 M v (src/fem.py:400-470).
        Returns (frequencies_Hz (m,), mode_shapes (N, m) M-normalised, zero at
        fixed DOFs, omega_sq (m,))."""
        ctx = self._prepare(rho_active, tip_mass_kg, tip_mass_nodes)
        nb = min(self.max_modes, n_modes + 2)
        if n_modes > nb:
            raise ValueError(f"n_modes={n_modes} exceeds max_modes={self.max_modes}")
        n_free = len(self.free_dofs)
        if X0_free is not None and np.shape(X0_free) == (n_free, n_modes):
            X0 = np.asarray(X0_free, dtype=np.float64)
        else:
            X0 = np.random.default_rng(0).standard_normal((n_free, n_modes))     # src/fem.py:448-449
        extra = np.random.default_rng(1).standard_normal((n_free, nb - n_modes))
        full = np.zeros((nb, self.geom.n_dofs))
        full[:, self.free_dofs] = np.concatenate([X0, extra], axis=1).T
        X = ctx.pack(torch.from_numpy(full))
        mid = self._mode_id()
        modes4, lam, st = ctx.lobpcg(X, n_modes, tol=min(tol, self.MODAL_TOL_CAP),
                                     maxiter=max(maxiter, 1000 if mid == L.MODE_MIXED else 6000),
                                     mode=mid, precond=L.PRECOND_MG if mid == L.MODE_MIXED else L.PRECOND_JACOBI)
        self.last_stats = st
        lam = np.maximum(lam, 0.0)                                                  # src/fem.py:462-466
        modes = ctx.unpack(modes4).cpu().numpy().T
        return np.sqrt(lam) / (2.0 * np.pi), modes, lam

    def eigenvalue_sensitivity(self, rho_active, omega_sq_k, v_k, tip_mass_kg=0.060, tip_mass_nodes=None):
        """d(omega^2)/d(rho_e) per active element (src/fem.py:472-526)."""
        ctx = self._prepare(rho_active)
        v = np.asarray(v_k, dtype=np.float64)
        v4 = ctx.pack(torch.from_numpy(v))
        qK = ctx.quadform(L.OP_K, v4)[0]
        qM = ctx.quadform(L.OP_M, v4)[0]
        nodes = self._tip_nodes(tip_mass_nodes)
        vmv_tip = 0.0
        if tip_mass_kg > 0.0 and len(nodes) > 0:
            dofs = np.concatenate([3 * nodes, 3 * nodes + 1, 3 * nodes + 2])
            vmv_tip = float(tip_mass_kg / len(nodes) * np.sum(v[dofs] ** 2))
        out = ctx.eig_sens(qK, qM, float(omega_sq_k), vmv_tip)
        return out[torch.as_tensor(self.active_ids, device=ctx.device)].cpu().numpy()

    # -- element quantities --------------------------------------------------- #
    def elem_compliance(self, u, rho_active=None):
        """u_e^T Ke u_e per active element (src/fem.py:605-615)."""
        ctx = self.device()
        u4 = ctx.pack(torch.from_numpy(np.asarray(u, dtype=np.float64)))
        ce = ctx.quadform(L.OP_K, u4)[0]
        return ce[torch.as_tensor(self.active_ids, device=ctx.device)].cpu().numpy()

    def compute_stress(self, u, rho_active):
        """Voigt stress (n_active, 6) at the element centres,
        rho_e D B_c u_e (src/fem.py:564-579)."""
        sig, _, _ = self.stress_fields(u, rho_active, vm=False, smax=False)
        return sig

    def stress_fields(self, u, rho_active, sigma=True, vm=True, smax=True):
        """(sigma (n_active, 6), von Mises (n_active,), largest principal
        (n_active,)) in one kernel pass; u may be one (N,) vector or (R, N)."""
        ctx = self.device()
        U = np.asarray(u, dtype=np.float64)
        one = U.ndim == 1
        u4 = ctx.pack(torch.from_numpy(U))
        rho = self.rho_to_grid(rho_active)
        s, v, m = ctx.stress(u4, self.B_centre, self.D_solid, rho, sigma=sigma, vm=vm, smax=smax)
        ids = torch.as_tensor(self.active_ids, device=ctx.device)
        pick = (lambda t: None if t is None else (t[0, ids] if one else t[:, ids]).cpu().numpy())
        return pick(s), pick(v), pick(m)

    def von_mises(self, stress):
        """von Mises equivalent of (..., 6) Voigt stresses (src/fem.py:582-589)."""
        return self._invariants(stress)[0]

    def principal_stress_max(self, stress):
        """Largest principal stress per row (src/fem.py:592-602)."""
        return self._invariants(stress)[1]

    def _invariants(self, stress):
        from .engine import stress_invariants
        dev = self.device().device
        vm, sm = stress_invariants(torch.as_tensor(np.asarray(stress, dtype=np.float64), device=dev))
        return vm.cpu().numpy(), sm.cpu().numpy()

    def total_mass(self, rho_active):
        """src/fem.py:618-621."""
        g = self.geom
        return float(np.sum(rho_active) * g.dx * g.dy * g.dz * self.mat.rho)

    def total_solid_mass(self):
        return self.total_mass(np.ones(self.n_active))
