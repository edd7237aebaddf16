"""Geometric multigrid preconditioner: Galerkin operators against an explicit
P^T (D K D) P, V-cycle symmetry / positivity, and multigrid-preconditioned PCG
parity with the reference's compliance."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mg_model import assemble_elements, levels, prolongation  # noqa: E402
from test_gpu_core import make_ctx, rel, to_dev  # noqa: E402

pytestmark = pytest.mark.gpu


def oracle_for(name, g):
    from oracle.fem import OracleFEM
    from tof_b200 import configs as C
    from tof_b200.geometry import BoxGeometry
    if name == "tiny":
        geom = BoxGeometry(int(g["nx"]), int(g["ny"]), int(g["nz"]), *g["h"], clamp="root_face", mount="tip_face",
                           in_arm_mask=g["in_arm"], keep_solid_mask=g["keep_solid"])
    elif name == "cantilever":
        geom = C.cantilever_geometry()
    else:
        geom = C.arm_geometry()
    return OracleFEM(geom, C.PA12.E, C.PA12.nu, C.PA12.rho)


@pytest.mark.parametrize("name", ["tiny", "cantilever"])
def test_hierarchy(golden, name):
    g = golden(name)
    ctx = make_ctx(g, g["rho"])
    lv = ctx.mg_levels()
    expect = levels(int(g["nx"]), int(g["ny"]), int(g["nz"]))
    assert [l[:3] for l in lv] == [e[:3] for e in expect]
    assert all(0.0 < l[3] < 0.6 for l in lv[:-1])          # first-sweep weight 1.76 / lambda_max, lambda ~ 3.5..6


def test_single_level_is_exact_coarse_solve(golden):
    """A grid at or below the coarsest-level size is one level: the V-cycle is
    the dense FP64 inverse, so mg_apply(r) = K_ff^-1 r (FP32 in and out)."""
    import scipy.sparse.linalg as spla
    g = golden("tiny")
    ctx = make_ctx(g, g["rho"])
    assert len(ctx.mg_levels()) == 1
    fem = oracle_for("tiny", g)
    K = fem.assemble_K(g["rho"]).tocsr()
    fd = fem.free_dofs
    rng = np.random.default_rng(3)
    r = np.zeros((2, K.shape[0]))
    r[:, fd] = rng.standard_normal((2, len(fd)))
    r32 = ctx.pack(to_dev(r), dtype=torch.float32)
    e = ctx.unpack(ctx.mg_apply(r32).double()).cpu().numpy()
    rq = ctx.unpack(r32.double()).cpu().numpy()            # the FP32-rounded right-hand sides
    Kff = K[fd][:, fd].tocsc()
    for k in range(2):
        ref = spla.spsolve(Kff, rq[k, fd])
        assert rel(e[k, fd], ref) < 1e-5
        assert np.all(e[k, np.setdiff1d(np.arange(K.shape[0]), fd)] == 0.0)


def test_galerkin_level1(golden):
    name = "cantilever"
    g = golden(name)
    ctx = make_ctx(g, g["rho"])
    expect = levels(int(g["nx"]), int(g["ny"]), int(g["nz"]))
    assert len(expect) >= 2
    fem = oracle_for(name, g)
    K = fem.assemble_K(g["rho"]).tocsr()
    free = np.zeros(K.shape[0])
    free[fem.free_dofs] = 1.0
    D = np.asarray(free)
    P = prolongation(expect[0], expect[1])
    P = (P.multiply(D[:, None])).tocsr()
    A1_ref = (P.T @ (K.multiply(D[:, None]).multiply(D[None, :])) @ P).toarray()
    Ae = ctx.mg_element_matrices(1).cpu().numpy()
    A1 = assemble_elements(Ae, *expect[1][:3]).toarray()
    assert rel(A1, A1_ref) < 2e-6


def test_vcycle_symmetric_positive(golden):
    g = golden("cantilever")
    ctx = make_ctx(g, g["rho"])
    rng = np.random.default_rng(1)
    r = ctx.pack(to_dev(rng.standard_normal((2, ctx.N))), dtype=torch.float32)
    e = ctx.mg_apply(r)
    a = float((e[0].double() * r[1].double()).sum())
    b = float((r[0].double() * e[1].double()).sum())
    assert abs(a - b) <= 1e-4 * max(abs(a), abs(b))
    assert float((e[0].double() * r[0].double()).sum()) > 0
    assert float((e[1].double() * r[1].double()).sum()) > 0


@pytest.mark.parametrize("name,max_it", [("cantilever", 60), ("arm", 200)])
def test_mg_pcg_parity(golden, name, max_it):
    from tof_b200 import configs as C
    g = golden(name)
    ctx = make_ctx(g, g["rho"], tip_mass=C.TIP_MASS_KG if name == "arm" else 0.0)
    b = ctx.pack(to_dev(np.stack([g["F"]] * 4)))
    x, st = ctx.pcg(b, rtol=1e-8, mode=1)
    for s in st:
        assert s["status"] == 0 and s["relres"] <= 1e-8 and s["iters"] <= max_it, st
    u = ctx.unpack(x).cpu().numpy()
    for k in range(4):
        c = float(g["F"] @ u[k])
        assert abs(c - float(g["compliance"])) < 1e-7 * float(g["compliance"])
