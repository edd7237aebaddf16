"""Tile-shape autotuner for the matrix-free operator.

`k_matvec` stages one node tile (plus a one-node halo) of every vector with a
single TMA box per CTA, so the tile shape sets the threads per CTA, the halo
re-read ratio and the shared memory per CTA, and the best shape depends on the
grid (the arm's short y and z axes favour long x tiles; a 1 mm grid can use
larger tiles).  `tune_tile` times the fine-level FP32 and FP64 block products
(the multigrid smoother / residual and the Krylov operator) for each
candidate on a throw-away context of the same grid and returns the fastest.
Results are cached per grid and active mask for the process.
"""
from __future__ import annotations

import hashlib

import numpy as np
import torch

from . import _lib as L
from .engine import DesignContext

# candidate (TX, TY, TZ): TX*TY*TZ threads per CTA (<= 256), one node each
CANDIDATES = [(8, 4, 4), (16, 4, 2), (8, 8, 2), (4, 4, 8), (16, 2, 4), (32, 2, 2), (8, 4, 8), (16, 4, 4),
              (8, 8, 4), (32, 4, 2)]

_cache: dict = {}


def _time_ms(fn, reps):
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    e.synchronize()
    return s.elapsed_time(e) / reps


def tune_tile(fem, R: int = 4, candidates=None, reps: int = 20, return_timings: bool = False):
    """Fastest tile for `fem`'s grid (a tof_b200.fem.FEM3D)."""
    g = fem.geom
    key = (g.nx, g.ny, g.nz, R, fem.max_rhs, fem.max_modes,
           hashlib.sha1(np.asarray(fem.in_arm, bool).tobytes()).hexdigest())
    if key in _cache and not return_timings:
        return _cache[key][0]
    rng = np.random.default_rng(0)
    rho = np.zeros(g.nx * g.ny * g.nz)
    act = np.asarray(fem.in_arm, bool).transpose(2, 1, 0).ravel()
    rho[act] = rng.uniform(0.05, 1.0, int(act.sum()))
    timings = {}
    for tile in (candidates or CANDIDATES):
        if tile[0] * tile[1] * tile[2] > 256:
            continue
        try:        # the design's own vector counts, so the shared-memory limit check is the same
            ctx = DesignContext(g.nx, g.ny, g.nz, (g.dx, g.dy, g.dz), fem.Ke_solid, fem.Me_solid,
                                active_grid=fem.in_arm, fixed_dofs=fem.fixed_dofs, max_rhs=fem.max_rhs,
                                max_modes=fem.max_modes, tile=tile)
        except L.SolverError:
            continue                                 # tile too large for this many vectors
        try:
            ctx.set_density(torch.from_numpy(rho))
            x = ctx.pack(torch.from_numpy(rng.standard_normal((R, ctx.N))))
            x32 = x.to(torch.float32)
            for _ in range(3):
                ctx.matvec(L.OP_K, x32)
                ctx.matvec(L.OP_K, x)
            t32 = _time_ms(lambda: ctx.matvec(L.OP_K, x32), reps)
            t64 = _time_ms(lambda: ctx.matvec(L.OP_K, x), reps)
            timings[tile] = (t32, t64, t32 + t64)
        finally:
            ctx.close()
    best = min(timings, key=lambda t: timings[t][2])
    _cache[key] = (best, timings)
    return (best, timings) if return_timings else best
