"""Parity of the CUDA path (through the C ABI) against the reference's own
outputs (golden fixtures) and the oracle.  Tolerances: FP64 paths 1e-12..1e-10
relative, FP32 operators 1e-6 relative, solves to the residual they target."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def make_ctx(g, rho=None, tip_mass=0.0, **kw):
    from tof_b200.configs import active_element_ids
    from tof_b200.engine import DesignContext
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    tip = None
    if tip_mass > 0:
        nodes = g["tip_nodes"]
        tip = np.zeros(3 * (nx + 1) * (ny + 1) * (nz + 1))
        for c in range(3):
            tip[3 * nodes + c] += tip_mass / len(nodes)
    ctx = DesignContext(nx, ny, nz, g["h"], g["Ke"], g["Me"], active_grid=g["in_arm"],
                        fixed_dofs=g["fixed_dofs"], tip_lump=tip, **kw)
    if rho is not None:
        grid = np.zeros(nx * ny * nz)
        grid[active_element_ids(g["in_arm"])] = rho
        ctx.set_density(torch.from_numpy(grid))
    return ctx


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


@pytest.fixture(scope="module")
def tiny(golden):
    g = golden("tiny")
    return g, make_ctx(g, g["rho"], tip_mass=0.06)


def test_free_dof_count(tiny):
    g, ctx = tiny
    assert ctx.n_free == len(g["free_dofs"])


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 2e-6)])
def test_matvec_K_M(tiny, dtype, tol):
    from tof_b200 import _lib as L
    g, ctx = tiny
    X4 = ctx.pack(to_dev(g["X"].T), dtype=dtype)
    KX = ctx.unpack(ctx.matvec(L.OP_K, X4)).cpu().numpy().T
    MX = ctx.unpack(ctx.matvec(L.OP_M, X4)).cpu().numpy().T
    fr = g["free_dofs"]
    assert rel(KX[fr], g["KX"][fr]) < tol
    assert rel(MX[fr], g["MX"][fr]) < tol
    assert np.all(KX[g["fixed_dofs"]] == 0)


def test_diag(tiny):
    from tof_b200 import _lib as L
    g, ctx = tiny
    fr = g["free_dofs"]
    dK = ctx.diag(L.OP_K)[:, :3].reshape(-1).cpu().numpy()
    dM = ctx.diag(L.OP_M)[:, :3].reshape(-1).cpu().numpy()
    assert rel(dK[fr], g["diagK"][fr]) < 1e-14
    assert rel(dM[fr], g["diagM"][fr]) < 1e-14


@pytest.mark.parametrize("mode", [0, 1])
def test_pcg_tiny(tiny, mode):
    g, ctx = tiny
    b = ctx.pack(to_dev(np.stack([g["F1"], g["F2"]])))
    x, st = ctx.pcg(b, rtol=1e-10, mode=mode)
    u = ctx.unpack(x).cpu().numpy()
    assert all(s["status"] == 0 for s in st), st
    assert rel(u[0], g["u1"]) < 1e-8
    assert rel(u[1], g["u2"]) < 1e-8


def test_quadform_compliance(tiny):
    from tof_b200 import _lib as L
    from tof_b200.configs import active_element_ids
    g, ctx = tiny
    u4 = ctx.pack(to_dev(g["u1"]))
    ce = ctx.quadform(L.OP_K, u4)[0].cpu().numpy()[active_element_ids(g["in_arm"])]
    assert rel(ce, g["ce1"]) < 1e-12


@pytest.mark.parametrize("mode", [0, 1])
def test_lobpcg_tiny(tiny, mode):
    from tof_b200 import _lib as L
    g, ctx = tiny
    rng = np.random.default_rng(0)
    X0 = ctx.pack(to_dev(rng.standard_normal((6, 3 * ctx.NN))))
    X, lam, st = ctx.lobpcg(X0, 4, tol=1e-6, maxiter=300, mode=mode)
    freqs = np.sqrt(lam) / (2 * np.pi)
    assert rel(freqs, g["freqs"]) < 1e-7, (freqs, g["freqs"], st)
    eff = ctx.effective_mass(X)
    assert np.max(np.abs(eff - g["eff"])) < 1e-6
    # all block Ritz vectors come back (the warm start of the next solve):
    # M-orthonormal, Rayleigh quotients ascending, the first four the modes
    B = ctx.last_block
    assert B.shape[0] == 6 and torch.equal(B[:4], X)
    GM = ctx.gram(B, ctx.matvec(L.OP_M, B)).cpu().numpy()
    GK = ctx.gram(B, ctx.matvec(L.OP_K, B)).cpu().numpy()
    assert np.max(np.abs(GM - np.eye(6))) < 1e-8
    rq = np.diag(GK) / np.diag(GM)
    assert np.all(np.diff(rq) >= -1e-8 * rq[-1])
    assert rel(rq[:4], lam) < 1e-8


def test_filter_and_oc(golden):
    from tof_b200.configs import active_element_ids  # noqa: F401
    from tof_b200.engine import DensityFilter, oc_update
    g = golden("tiny")
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    for key, mask, k in (("filt15", g["design"], g["k15"]), ("filt23", g["in_arm"], g["k23"])):
        f = DensityFilter((nx, ny, nz), k, mask)
        field = to_dev(g["field"].transpose(2, 1, 0).ravel())
        out = f.apply(field).cpu().numpy().reshape(nz, ny, nx).transpose(2, 1, 0)
        assert rel(out, g[key]) < 1e-14
    o = golden("oc")
    x_new = oc_update(to_dev(o["x"]), to_dev(o["dc"]), float(o["V_e"]), float(o["target_volume"]),
                      float(o["move"])).cpu().numpy()
    assert np.max(np.abs(x_new - o["x_new"])) < 1e-12


def test_cantilever_static_and_modes(golden):
    g = golden("cantilever")
    ctx = make_ctx(g, g["rho"])
    b = ctx.pack(to_dev(g["F"]))
    for mode in (0, 1):
        x, st = ctx.pcg(b, rtol=1e-8, mode=mode)
        assert st[0]["status"] == 0 and st[0]["relres"] <= 1e-8, st
        u = ctx.unpack(x)[0].cpu().numpy()
        c = float(g["F"] @ u)
        assert abs(c - float(g["compliance"])) < 1e-7 * float(g["compliance"])
    rng = np.random.default_rng(0)
    X0 = ctx.pack(to_dev(rng.standard_normal((8, 3 * ctx.NN))))
    for mode in (1,):
        X, lam, st = ctx.lobpcg(X0, 6, tol=1e-5, maxiter=400, mode=mode)
        freqs = np.sqrt(lam) / (2 * np.pi)
        assert np.max(np.abs(freqs / g["freqs"] - 1)) < 1e-6, (freqs, g["freqs"], st)
