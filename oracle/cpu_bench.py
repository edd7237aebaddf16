"""CPU timing of the reference algorithm for one SIMP design iteration —
TEST / BASELINE INFRASTRUCTURE ONLY (bench.py's cpu_baseline leg and its
`--impl reference` arm).

One SIMP iteration of the reference (src/topopt.py:267-411) on the arm grid
costs 4 Jacobi-CG static solves (src/fem.py:529-561, here at rtol 1e-8), one
Jacobi-LOBPCG modal solve (src/fem.py:400-470, tol 1e-4, maxiter 500 — the
reference's defaults; on this grid it exhausts the 500 iterations) and
element/filter/OC work.  A bounded sample times one full static solve, the
first `lob_iters` LOBPCG iterations and the element/filter/OC work, and
extrapolates: t_iter = n_lc * t_static + (500 / lob_iters) * t_lobpcg + t_rest.
"""
from __future__ import annotations

import os
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .fem import OracleFEM
from .topopt import cone_kernel, filter_field, oc_update


def simp_iteration_sample(geom, E, nu, rho_mat, rho_active, F_list, tip_mass_kg, tip_nodes, n_modes=6,
                          lob_iters=25, design_mask=None, rtol=1e-8):
    fem = OracleFEM(geom, E, nu, rho_mat)
    t0 = time.perf_counter()
    K = fem.reduce(fem.assemble_K(rho_active))
    M = fem.reduce(fem.assemble_M(rho_active, tip_mass_kg, tip_nodes))
    t_asm = time.perf_counter() - t0
    f = fem.free_dofs
    d = K.diagonal()
    Minv = sp.diags(1.0 / np.where(d != 0, d, 1.0))
    t0 = time.perf_counter()
    uf, info = spla.cg(K, np.asarray(F_list[0])[f], M=Minv, rtol=rtol, atol=0.0, maxiter=20000)
    t_static = time.perf_counter() - t0
    X0 = np.random.default_rng(0).standard_normal((len(f), n_modes))
    t0 = time.perf_counter()
    try:
        spla.lobpcg(K, X0, B=M, M=sp.diags(1.0 / np.where(d > 0, d, 1.0)), tol=1e-4, largest=False,
                    maxiter=lob_iters)
    except Exception:
        pass
    t_lob = time.perf_counter() - t0
    t0 = time.perf_counter()
    u = np.zeros(geom.n_dofs)
    u[f] = uf
    ce = fem.elem_compliance(u)
    grid = np.zeros((geom.nx, geom.ny, geom.nz))
    ex, ey, ez = fem.elem_grid_idx.T
    grid[ex, ey, ez] = ce
    mask = design_mask if design_mask is not None else np.ones_like(grid, bool)
    k = cone_kernel(1.5)
    for _ in range(4):
        filter_field(grid, mask, k)
    x = np.full(int(mask.sum()), 0.08)
    oc_update(x, -np.abs(grid[mask]) - 1e-12, geom.dx * geom.dy * geom.dz,
              0.08 * x.size * geom.dx * geom.dy * geom.dz, 0.2)
    t_rest = time.perf_counter() - t0
    n_lc = len(F_list)
    t_iter = t_asm * (n_lc + 1) + n_lc * t_static + (500.0 / lob_iters) * t_lob + n_lc * t_rest
    return dict(t_iter_s=t_iter, t_static_s=t_static, static_info=int(info), t_lobpcg_sample_s=t_lob,
                lob_iters=lob_iters, t_assembly_s=t_asm, t_rest_s=t_rest, cores=os.cpu_count(),
                sample_wall_s=t_asm + t_static + t_lob + t_rest)
