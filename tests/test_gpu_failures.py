"""Failure statuses of the solvers, driven without faulting the GPU.

The reference signals a failed solve by `info != 0` from SciPy's cg and by
falling back to another solver (src/fem.py:548-550, src/fem_gpu.py:84-91,
src/fem.py:455-461).  libtof returns a status instead and never falls back:
non-finite input (NaN / Inf in the load or in the density) gives
TOF_ERR_NONFINITE, an iteration cap gives TOF_NOT_CONVERGED with the
statistics filled, an unconstrained (singular) problem ends with a status
rather than a hang, and a device-side wait that nobody releases gives up
after the context's wait budget with TOF_ERR_TIMEOUT and leaves the context
usable.  The waits here are bounded by construction (a barrier that expects
one more arrival than the launch has; every CTA gives up after the budget).
"""
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _cantilever(nx=12, ny=4, nz=4, clamp=True, rho=0.5):
    from tof_b200 import configs as C
    from tof_b200.configs import active_element_ids
    from tof_b200.element import element_mass, element_stiffness, isotropic_D
    from tof_b200.engine import DesignContext
    geom = C.cantilever_geometry(nx=nx, ny=ny, nz=nz)
    h = (geom.dx, geom.dy, geom.dz)
    Ke = element_stiffness(*h, isotropic_D(C.PA12.E, C.PA12.nu))
    Me = element_mass(C.PA12.rho, *h)
    fixed = ()
    if clamp:
        n = geom.fixed_nodes()
        fixed = np.concatenate([3 * n, 3 * n + 1, 3 * n + 2])
    ctx = DesignContext(geom.nx, geom.ny, geom.nz, h, Ke, Me, fixed_dofs=fixed, max_rhs=4, max_modes=8)
    grid = np.zeros(geom.n_elements)
    grid[active_element_ids(geom.build_masks()["in_arm"])] = rho
    ctx.set_density(torch.from_numpy(grid))
    F = C.cantilever_loads(geom)[0]
    return geom, ctx, grid, F


def _start_block(ctx, nb, seed=0):
    X = np.random.default_rng(seed).standard_normal((nb, ctx.N))
    return ctx.pack(torch.from_numpy(X))


@pytest.fixture(scope="module")
def cant():
    return _cantilever()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_nonfinite_load(cant, mode, bad):
    from tof_b200 import _lib as L
    _, ctx, _, F = cant
    b = F.copy()
    b[np.flatnonzero(b)[0]] = bad
    b4 = ctx.pack(torch.from_numpy(b))
    mid = L.MODE_FP64 if mode == "fp64" else L.MODE_MIXED
    _, st = ctx.pcg(b4, rtol=1e-8, maxiter=500, mode=mid, raise_on_error=False)
    assert ctx.last_rc == L.TOF_ERR_NONFINITE
    assert st[0]["status"] == L.TOF_ERR_NONFINITE
    with pytest.raises(L.SolverError):
        ctx.pcg(b4, rtol=1e-8, maxiter=500, mode=mid)


def test_nonfinite_density():
    """A NaN density poisons K: PCG (both forms) and LOBPCG report it."""
    from tof_b200 import _lib as L
    _, ctx, grid, F = _cantilever()
    g = grid.copy()
    g[np.flatnonzero(g)[5]] = np.nan
    ctx.set_density(torch.from_numpy(g))
    b4 = ctx.pack(torch.from_numpy(F))
    for mid in (L.MODE_FP64, L.MODE_MIXED):
        _, st = ctx.pcg(b4, rtol=1e-8, maxiter=500, mode=mid, raise_on_error=False)
        assert ctx.last_rc == L.TOF_ERR_NONFINITE, (mid, st)
    _, _, st = ctx.lobpcg(_start_block(ctx, 4), 2, tol=1e-6, maxiter=50, mode=L.MODE_FP64,
                          precond=L.PRECOND_JACOBI, raise_on_error=False)
    assert ctx.last_rc == L.TOF_ERR_NONFINITE
    assert st["status"] == L.TOF_ERR_NONFINITE
    # a finite density afterwards: the same context solves again
    ctx.set_density(torch.from_numpy(grid))
    _, st = ctx.pcg(b4, rtol=1e-8, maxiter=5000, mode=L.MODE_FP64)
    assert st[0]["status"] == L.TOF_OK


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_pcg_maxiter_one(cant, mode):
    from tof_b200 import _lib as L
    _, ctx, _, F = cant
    b4 = ctx.pack(torch.from_numpy(F))
    mid = L.MODE_FP64 if mode == "fp64" else L.MODE_MIXED
    _, st = ctx.pcg(b4, rtol=1e-8, maxiter=1, mode=mid, raise_on_error=False)
    assert ctx.last_rc == L.TOF_NOT_CONVERGED
    s = st[0]
    assert s["status"] == L.TOF_NOT_CONVERGED
    assert s["iters"] == 1
    assert s["relres"] > 1e-8 and np.isfinite(s["relres"])        # CG residuals may grow at first


@pytest.mark.parametrize("precond", ["jacobi", "mg"])
def test_lobpcg_maxiter_one(cant, precond):
    from tof_b200 import _lib as L
    _, ctx, _, _ = cant
    pc = L.PRECOND_JACOBI if precond == "jacobi" else L.PRECOND_MG
    mid = L.MODE_FP64 if precond == "jacobi" else L.MODE_MIXED
    modes, lam, st = ctx.lobpcg(_start_block(ctx, 6), 4, tol=1e-8, maxiter=1, mode=mid, precond=pc,
                                raise_on_error=False)
    assert ctx.last_rc == L.TOF_NOT_CONVERGED
    assert st["status"] == L.TOF_NOT_CONVERGED
    assert st["iters"] == 1
    assert np.all(np.isfinite(lam)) and np.all(lam > 0)
    assert st["relres"] > 1e-8 and np.all(np.isfinite(st["resid"]))


def test_unconstrained_domain_returns_a_status():
    """No clamp: K is singular (six rigid-body modes) and a net force makes
    K u = F inconsistent.  Both PCG forms stop with a status; LOBPCG finds
    the rigid-body modes (eigenvalues ~0) or stops at its cap."""
    from tof_b200 import _lib as L
    _, ctx, _, F = _cantilever(clamp=False)
    b4 = ctx.pack(torch.from_numpy(F))
    for mid in (L.MODE_FP64, L.MODE_MIXED):
        t0 = time.time()
        _, st = ctx.pcg(b4, rtol=1e-8, maxiter=400, mode=mid, raise_on_error=False)
        assert time.time() - t0 < 30.0
        assert ctx.last_rc in (L.TOF_NOT_CONVERGED, L.TOF_ERR_BREAKDOWN, L.TOF_ERR_NONFINITE), (mid, st)
        assert st[0]["status"] == ctx.last_rc or ctx.last_rc == L.TOF_NOT_CONVERGED
        assert st[0]["iters"] <= 400
    t0 = time.time()
    _, lam, st = ctx.lobpcg(_start_block(ctx, 8), 6, tol=1e-6, maxiter=60, mode=L.MODE_FP64,
                            precond=L.PRECOND_JACOBI, raise_on_error=False)
    assert time.time() - t0 < 30.0
    assert ctx.last_rc in (L.TOF_OK, L.TOF_NOT_CONVERGED, L.TOF_ERR_BREAKDOWN), st
    assert st["iters"] <= 60


def test_wait_budget_expires_and_context_stays_usable():
    from tof_b200 import _lib as L
    lib = L.load()
    _, ctx, _, F = _cantilever()
    s = torch.cuda.current_stream().cuda_stream
    import ctypes
    cs = ctypes.c_void_p(s)
    assert lib.tof_ctx_set_wait_limit(ctx.h, 10) == L.TOF_ERR_ARG           # below 1 us
    assert lib.tof_ctx_set_wait_limit(ctx.h, 20_000) == L.TOF_OK            # 20 us
    assert lib.tof_wait_selftest(ctx.h, 0, cs) == L.TOF_OK                  # everybody arrives
    t0 = time.time()
    rc = lib.tof_wait_selftest(ctx.h, 1, cs)                                # one arrival short
    dt = time.time() - t0
    assert rc == L.TOF_ERR_TIMEOUT
    assert b"wait budget" in lib.tof_last_error(ctx.h)
    assert dt < 1.0
    # back to the default budget: the barrier was reset, solves work
    assert lib.tof_ctx_set_wait_limit(ctx.h, 2_000_000_000) == L.TOF_OK
    assert lib.tof_wait_selftest(ctx.h, 0, cs) == L.TOF_OK
    b4 = ctx.pack(torch.from_numpy(F))
    for mid in (L.MODE_FP64, L.MODE_MIXED):
        _, st = ctx.pcg(b4, rtol=1e-8, maxiter=5000, mode=mid)
        assert st[0]["status"] == L.TOF_OK and st[0]["relres"] <= 1.01e-8
