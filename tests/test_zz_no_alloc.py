"""tof_gram_noalloc: the Gram matrix for callers that cannot allocate device
memory (an application whose memory pool owns the GPU, work issued during
CUDA-graph capture, loops that must avoid cudaMalloc's implicit sync).

Called through the C ABI and checked against tof_gram (the context-based
entry point) on two calls in a row with different shapes and dtypes, to
1e-12 relative (both accumulate in FP64; only the summation grouping
differs).  Also checks the size limit is enforced.  This file is collected
last on purpose."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _ctx():
    from tof_b200 import configs as C
    from tof_b200.configs import active_element_ids
    from tof_b200.element import element_mass, element_stiffness, isotropic_D
    from tof_b200.engine import DesignContext
    geom = C.cantilever_geometry(nx=20, ny=6, nz=5)
    h = (geom.dx, geom.dy, geom.dz)
    Ke = element_stiffness(*h, isotropic_D(C.PA12.E, C.PA12.nu))
    Me = element_mass(C.PA12.rho, *h)
    n = geom.fixed_nodes()
    fixed = np.concatenate([3 * n, 3 * n + 1, 3 * n + 2])
    ctx = DesignContext(geom.nx, geom.ny, geom.nz, h, Ke, Me, fixed_dofs=fixed, max_rhs=8, max_modes=8)
    grid = np.zeros(geom.n_elements)
    grid[active_element_ids(geom.build_masks()["in_arm"])] = 0.5
    ctx.set_density(torch.from_numpy(grid))
    return ctx


def _noalloc(lib, ctx, A, B):
    from tof_b200 import _lib as L
    G = torch.empty((A.shape[0], B.shape[0]), dtype=torch.float64, device=ctx.device)
    dt = L.F64 if A.dtype == torch.float64 else L.F32
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.tof_gram_noalloc(ctx.NN, dt, L.ptr(A), A.shape[0], L.ptr(B), B.shape[0], L.ptr(G), s)
    assert rc == L.TOF_OK, lib.tof_last_error(None)
    return G


def test_gram_noalloc_matches_gram_two_calls():
    from tof_b200 import _lib as L
    lib = L.load()
    ctx = _ctx()
    g = torch.Generator(device="cpu").manual_seed(7)
    # call 1: FP64, 6 x 6
    A = ctx.pack(torch.randn(6, ctx.N, generator=g, dtype=torch.float64))
    B = ctx.pack(torch.randn(6, ctx.N, generator=g, dtype=torch.float64))
    G1 = _noalloc(lib, ctx, A, B)
    R1 = ctx.gram(A, B)
    # call 2 right after: FP32, 24 x 3 (reuses the same scratch array)
    A2 = ctx.pack(torch.randn(24, ctx.N, generator=g, dtype=torch.float64), dtype=torch.float32)
    B2 = ctx.pack(torch.randn(3, ctx.N, generator=g, dtype=torch.float64), dtype=torch.float32)
    G2 = _noalloc(lib, ctx, A2, B2)
    R2 = ctx.gram(A2, B2)
    torch.cuda.synchronize()
    for G, R in ((G1, R1), (G2, R2)):
        G, R = G.cpu().numpy(), R.cpu().numpy()
        assert np.linalg.norm(G - R) <= 1e-12 * np.linalg.norm(R), (G, R)


def test_gram_noalloc_rejects_sizes_beyond_limit():
    from tof_b200 import _lib as L
    lib = L.load()
    ctx = _ctx()
    A = torch.zeros((25, ctx.NN, 4), dtype=torch.float64, device=ctx.device)
    G = torch.empty((25, 25), dtype=torch.float64, device=ctx.device)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.tof_gram_noalloc(ctx.NN, L.F64, L.ptr(A), 25, L.ptr(A), 25, L.ptr(G), s)
    assert rc == L.TOF_ERR_ARG
    assert b"<= 24" in lib.tof_last_error(None)
