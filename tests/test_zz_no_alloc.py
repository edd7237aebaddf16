"""tof_gram_noalloc: the Gram matrix for callers that cannot allocate device
memory at the point they need it (an application whose memory pool owns the
whole GPU, or a loop that must not take cudaMalloc's implicit sync).

Called through the C ABI and checked, on two calls in a row with different
shapes and dtypes, against tof_gram (the context-based entry point) and
against an independent FP64 product in torch, to 1e-12 relative (all
accumulate in FP64; only the summation grouping differs).  A third case has
more nodes than the 256 fixed partial-sum slots cover one chunk each, and a
node count that is not a multiple of the chunk, so CTAs loop over several
chunks and the trailing CTAs publish empty partials.  Also checks that the
size limit is enforced.  This file is collected last on purpose."""
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


def _noalloc(lib, A, B):
    from tof_b200 import _lib as L
    NN = A.shape[1]
    G = torch.empty((A.shape[0], B.shape[0]), dtype=torch.float64, device=A.device)
    dt = L.F64 if A.dtype == torch.float64 else L.F32
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.tof_gram_noalloc(NN, dt, L.ptr(A), A.shape[0], L.ptr(B), B.shape[0], L.ptr(G), s)
    assert rc == L.TOF_OK, lib.tof_last_error(None)
    return G


def _fp64(A, B):
    """Independent FP64 product over the three displacement components."""
    return torch.einsum("anc,bnc->ab", A[..., :3].double(), B[..., :3].double())


def _close(G, R, tol=1e-12):
    G, R = G.cpu().numpy(), R.cpu().numpy()
    assert np.linalg.norm(G - R) <= tol * np.linalg.norm(R), (G, R)


def test_gram_noalloc_matches_gram_two_calls():
    from tof_b200 import _lib as L
    lib = L.load()
    ctx = _ctx()
    g = torch.Generator(device="cpu").manual_seed(7)
    # call 1: FP64, 6 x 6
    A = ctx.pack(torch.randn(6, ctx.N, generator=g, dtype=torch.float64))
    B = ctx.pack(torch.randn(6, ctx.N, generator=g, dtype=torch.float64))
    G1 = _noalloc(lib, A, B)
    R1 = ctx.gram(A, B)
    # call 2 right after: FP32, 24 x 3 (reuses the same scratch array)
    A2 = ctx.pack(torch.randn(24, ctx.N, generator=g, dtype=torch.float64), dtype=torch.float32)
    B2 = ctx.pack(torch.randn(3, ctx.N, generator=g, dtype=torch.float64), dtype=torch.float32)
    G2 = _noalloc(lib, A2, B2)
    R2 = ctx.gram(A2, B2)
    torch.cuda.synchronize()
    _close(G1, R1)
    _close(G2, R2)
    _close(G1, _fp64(A, B))
    _close(G2, _fp64(A2, B2))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_gram_noalloc_many_chunks_ragged(dtype):
    """20 011 nodes: more chunks than the 256 partial-sum slots (FP32 chunks
    of 32 nodes, FP64 of 16), the last chunk partial, idle trailing CTAs."""
    from tof_b200 import _lib as L
    lib = L.load()
    g = torch.Generator(device="cpu").manual_seed(11)
    NN = 20011
    A = torch.randn(7, NN, 4, generator=g, dtype=torch.float64)
    B = torch.randn(5, NN, 4, generator=g, dtype=torch.float64)
    A[..., 3] = 0.0
    B[..., 3] = 0.0
    A = A.to("cuda", dtype)
    B = B.to("cuda", dtype)
    G1 = _noalloc(lib, A, B)
    G2 = _noalloc(lib, B, A)
    torch.cuda.synchronize()
    _close(G1, _fp64(A, B))
    _close(G2, _fp64(B, A))


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
