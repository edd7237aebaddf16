"""The reference's SIMP design iteration on the host cores, timed for real —
TEST / BASELINE INFRASTRUCTURE ONLY (bench.py's cpu_baseline leg and its
`--impl reference` arm).

`ReferenceSIMPRun.step()` performs one whole iteration of the reference's
loop body (src/topopt.py:267-411) with the reference's own solver calls, on
the same workload as the device arm (same start design, four load cases,
tip mass, six tracked modes, filter, 500 Hz frequency penalty):

* each load case: assemble K (src/fem.py:311-325), Jacobi-preconditioned
  SciPy CG warm-started from the previous iteration's u, maxiter 5000, with
  the reference's fall-back to a sparse direct solve when CG reports
  failure (src/fem.py:529-555), at the workload's relative residual 1e-8
  (the reference's default is 1e-5);
* the modes: assemble K and M with the tip mass, Jacobi-preconditioned SciPy
  LOBPCG with the reference's defaults tol 1e-4, maxiter 500, warm-started
  from the previous iteration's modes (src/fem.py:400-470; on these designs
  it runs all 500 iterations);
* element compliances, sensitivities, the filter, MAC tracking, the
  eigenvalue sensitivity and penalty, OC and the change measure in the main
  process (src/topopt.py:287-390).

The four static solves and the modal solve are independent given the
density, and SciPy's sparse products use one core each, so they run at the
same time in five worker processes (spawned, each with its own copy of the
FEM set-up and one BLAS thread): every step's time is the wall time of one
complete iteration, nothing is extrapolated.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .fem import OracleFEM
from .topopt import cone_kernel, filter_field, oc_update, select_mode_by_mac

_W = {}


def _worker_init(geom, E, nu, rho_mat, tip_mass_kg, tip_nodes):
    from threadpoolctl import threadpool_limits
    _W["blas"] = threadpool_limits(1)          # one core per worker
    _W["fem"] = OracleFEM(geom, E, nu, rho_mat)
    _W["tip"] = (tip_mass_kg, np.asarray(tip_nodes, dtype=np.int64))


def _static(rho, F, x0, rtol):
    """src/fem.py:558-561 -> 529-555 (K assembled per call, as the reference)."""
    fem = _W["fem"]
    t0 = time.perf_counter()
    K = fem.assemble_K(rho)
    f = fem.free_dofs
    Kff = K[f][:, f].tocsc()
    Ff = F[f]
    d = Kff.diagonal()
    Minv = sp.diags(1.0 / np.where(d != 0, d, 1.0))
    it = [0]

    def cb(_):
        it[0] += 1
    uf, info = spla.cg(Kff, Ff, M=Minv, rtol=rtol, atol=0.0, maxiter=5000,
                       x0=None if x0 is None else x0[f], callback=cb)
    direct = info != 0
    if direct:
        uf = spla.spsolve(Kff, Ff)
    u = np.zeros(fem.geom.n_dofs)
    u[f] = uf
    rel = float(np.linalg.norm(Ff - Kff @ uf) / max(np.linalg.norm(Ff), 1e-300))
    return u, dict(iters=it[0], direct=bool(direct), relres=rel, s=time.perf_counter() - t0)


def _modal(rho, n_modes, X0_free):
    """src/fem.py:400-470 with its defaults (tol 1e-4, maxiter 500)."""
    fem = _W["fem"]
    tip_mass_kg, tip_nodes = _W["tip"]
    t0 = time.perf_counter()
    K = fem.assemble_K(rho)
    M = fem.assemble_M(rho, tip_mass_kg, tip_nodes)
    f = fem.free_dofs
    Kff = K[f][:, f].tocsc()
    Mff = M[f][:, f].tocsc()
    dK = Kff.diagonal()
    Minv = sp.diags(1.0 / np.where(dK > 0, dK, 1.0))
    if X0_free is not None and X0_free.shape == (len(f), n_modes):
        X0 = X0_free.copy()
    else:
        X0 = np.random.default_rng(0).standard_normal((len(f), n_modes))
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        try:
            lam, V = spla.lobpcg(Kff, X0, B=Mff, M=Minv, tol=1e-4, largest=False, maxiter=500)
        except Exception:
            lam, V = spla.eigsh(Kff, k=n_modes, M=Mff, sigma=1.0, which="LM", mode="normal", tol=1e-5,
                                maxiter=2000)
    order = np.argsort(lam)
    lam = np.maximum(lam[order], 0.0)
    V = V[:, order]
    modes = np.zeros((fem.geom.n_dofs, n_modes))
    modes[f] = V
    return np.sqrt(lam) / (2 * np.pi), modes, lam, time.perf_counter() - t0


class ReferenceSIMPRun:
    """The reference's SIMP loop (src/topopt.py:217-427) with its solves on
    a pool of worker processes.  `step()` runs one iteration and returns its
    wall time and solver statistics."""

    def __init__(self, geom, E, nu, rho_mat, F_list, x0_design, vol_frac=0.08, r_min_mm=3.0, move=0.2,
                 min_freq_Hz=500.0, tip_mass_kg=0.06, n_modes_track=6, mu_freq_init=0.2, mu_freq_max=50.0,
                 mu_freq_ramp_every=5, mu_freq_ramp_factor=1.5, rtol=1e-8, workers=None):
        self.geom = geom
        self.fem = OracleFEM(geom, E, nu, rho_mat)
        self.F_list = [np.asarray(F, float) for F in F_list]
        self.rtol = rtol
        n = len(self.F_list)
        self.weights = np.full(n, 1.0 / n)                                 # src/topopt.py:121-124
        m = geom.build_masks()
        self.in_arm, self.design = m["in_arm"], m["design"]
        self.active_idx = self.fem.elem_grid_idx
        ex, ey, ez = self.active_idx.T
        self.is_design_active = self.design[ex, ey, ez]
        self.kernel = cone_kernel(max(1.0, r_min_mm / (geom.dx * 1e3)))   # src/topopt.py:109
        self.V_e = geom.dx * geom.dy * geom.dz
        self.design_volume = int(self.is_design_active.sum()) * self.V_e
        self.target_volume = vol_frac * self.design_volume
        self.move = move
        self.lam_t = (2 * np.pi * min_freq_Hz) ** 2
        self.tip_mass_kg = tip_mass_kg
        self.tip_nodes = np.asarray(geom.motor_mount_top_nodes(), dtype=np.int64)
        self.n_modes = n_modes_track
        self.mu, self.mu_max = mu_freq_init, mu_freq_max
        self.ramp_every, self.ramp_factor = mu_freq_ramp_every, mu_freq_ramp_factor
        rho_active = np.where(self.is_design_active, vol_frac, 1.0)       # src/topopt.py:231-235
        self.rho_grid = self._to_grid(rho_active)
        self.rho_grid[self.design] = np.asarray(x0_design, float)
        self.rho_phys_grid = self.rho_grid.copy()
        self.u_prev = [None] * n
        self.X0_free = None
        self.v_prev = None
        self.it = 0
        self.workers = workers or min(n + 1, os.cpu_count() or 1)
        ctx = mp.get_context("spawn")
        self.pool = ProcessPoolExecutor(max_workers=self.workers, mp_context=ctx, initializer=_worker_init,
                                        initargs=(geom, E, nu, rho_mat, tip_mass_kg, self.tip_nodes))

    def close(self):
        self.pool.shutdown(wait=True, cancel_futures=True)

    def _to_grid(self, vals):
        g = np.zeros((self.geom.nx, self.geom.ny, self.geom.nz))
        ex, ey, ez = self.active_idx.T
        g[ex, ey, ez] = vals
        return g

    def _to_active(self, g):
        ex, ey, ez = self.active_idx.T
        return g[ex, ey, ez]

    def step(self):
        t0 = time.perf_counter()
        self.it += 1
        fem, p, emin = self.fem, self.fem.SIMP_PENALTY, self.fem.E_MIN_FRAC
        f = filter_field(self.rho_grid, self.design, self.kernel)             # src/topopt.py:270-281
        f[~self.design] = 0.0
        rho = self._to_active(np.where(self.design, f, np.where(self.in_arm, 1.0, 0.0)))
        fut_modal = self.pool.submit(_modal, rho, self.n_modes, self.X0_free)
        futs = [self.pool.submit(_static, rho, F, self.u_prev[i], self.rtol) for i, F in enumerate(self.F_list)]
        sens = np.zeros_like(self.rho_grid)
        c_total = 0.0
        stats = []
        for i, fu in enumerate(futs):                                        # src/topopt.py:287-306
            u, st = fu.result()
            self.u_prev[i] = u
            stats.append(st)
            ce = fem.elem_compliance(u)
            c_total += self.weights[i] * float(((emin + (1 - emin) * rho ** p) * ce).sum())
            sens += self.weights[i] * self._to_grid(-p * (1 - emin) * rho ** (p - 1) * ce)
        sens_filt = filter_field(sens, self.design, self.kernel)             # src/topopt.py:311
        freqs, modes, lam, t_modal = fut_modal.result()                      # src/topopt.py:315-330
        self.X0_free = modes[fem.free_dofs].copy()
        k = 0 if self.v_prev is None else select_mode_by_mac(modes, self.v_prev)
        lam1, v1 = float(lam[k]), modes[:, k]
        self.v_prev = v1.copy()
        viol = max(0.0, 1.0 - lam1 / self.lam_t)                              # src/topopt.py:339-361
        if viol > 0.0:
            dlam = fem.eigenvalue_sensitivity(rho, lam1, v1, self.tip_mass_kg, self.tip_nodes)
            dlam_f = filter_field(self._to_grid(dlam), self.design, self.kernel)
            s_c = float(np.mean(np.abs(sens_filt[self.design])))
            s_m = float(np.mean(np.abs(dlam_f[self.design])))
            sens_filt = sens_filt - self.mu * viol * (s_c / max(s_m, 1e-30)) * dlam_f
        if self.it % self.ramp_every == 0 and viol > 0.0 and self.mu < self.mu_max:
            self.mu = min(self.mu_max, self.mu * self.ramp_factor)
        x = self.rho_grid[self.design]                                        # src/topopt.py:377-390
        x_new = oc_update(x, sens_filt[self.design], self.V_e, self.target_volume, self.move)
        new_grid = self.rho_grid.copy()
        new_grid[self.design] = x_new
        check = filter_field(new_grid, self.design, self.kernel)
        change = float(np.max(np.abs(check - self.rho_phys_grid)))
        self.rho_grid, self.rho_phys_grid = new_grid, check
        return dict(t_s=time.perf_counter() - t0, compliance=c_total, omega1_Hz=float(np.sqrt(lam1) / (2 * np.pi)),
                    change=change, cg_iters=[s["iters"] for s in stats], cg_direct=[s["direct"] for s in stats],
                    cg_relres=max(s["relres"] for s in stats), t_static_s=max(s["s"] for s in stats),
                    t_modal_s=t_modal)


def arm_workload(vf=0.08, seed=0):
    """Host-only inputs of the arm design-iteration workload: (geom, x0 on
    the design cells, the four load vectors).  The inertial case is -3 g
    times the reference-assembled M(rho_start) e_z at the start design's
    physical density (src/fem.py:362-398, src/topopt.py:270-281)."""
    from tof_b200 import configs as C
    geom = C.arm_geometry()
    x0 = C.arm_design_start(geom, vf=vf, seed=seed).astype(np.float64)
    fem = OracleFEM(geom, C.PA12.E, C.PA12.nu, C.PA12.rho)
    m = geom.build_masks()
    ex, ey, ez = fem.elem_grid_idx.T
    g = np.zeros((geom.nx, geom.ny, geom.nz))
    g[ex, ey, ez] = 1.0
    g[m["design"]] = x0
    f = filter_field(g, m["design"], cone_kernel(1.5))
    f[~m["design"]] = 0.0
    rho = np.where(m["design"], f, np.where(m["in_arm"], 1.0, 0.0))[ex, ey, ez]
    ezv = np.zeros(geom.n_dofs)
    ezv[2::3] = 1.0
    Mr = fem.assemble_M(rho, C.TIP_MASS_KG, geom.motor_mount_top_nodes()) @ ezv
    return geom, x0, C.arm_static_loads(geom) + [C.body_load_from_Mr(Mr, 3.0)]
