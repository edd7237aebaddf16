"""CPU model of the library's multigrid V-cycle (same coarsening, masked
trilinear transfers, Galerkin coarse operators, 10-step power estimate of
lambda_max(D^-1 A) per level, degree-2 Chebyshev smoothing on
[lambda / 30, 1.3 lambda] before and after the coarse correction, direct
coarsest solve): on a high-contrast SIMP density the cycle, written out as a
matrix B, is symmetric positive definite -- so it is a valid preconditioner
for CG and LOBPCG -- and conditions K better than damped Jacobi with the same
two sweeps (omega = 1.3333 / lambda), the smoother it replaced.  An interval
whose upper end falls below lambda_max makes the cycle indefinite, which is
why the library keeps a margin above the power estimate."""
import numpy as np
import scipy.sparse as sp

from mg_model import levels, prolongation
from oracle.fem import OracleFEM
from tof_b200 import configs as C
from tof_b200.geometry import BoxGeometry

CHEB_RATIO, OMEGA_SCALE, POWER_ITERS = 30.0, 1.3333, 10


def hierarchy(geom, rho):
    fem = OracleFEM(geom, C.PA12.E, C.PA12.nu, C.PA12.rho)
    free = np.zeros(geom.n_dofs)
    free[fem.free_dofs] = 1.0
    D = sp.diags(free)
    A = [(D @ fem.assemble_K(rho) @ D).tocsr()]
    fix = [free == 0]
    P = []
    lv = levels(geom.nx, geom.ny, geom.nz)
    for l in range(1, len(lv)):
        Pl = (sp.diags((~fix[-1]).astype(float)) @ prolongation(lv[l - 1], lv[l])).tocsr()
        Ac = (Pl.T @ A[-1] @ Pl).tocsr()
        P.append(Pl)
        A.append(Ac)
        fix.append(np.abs(Ac.diagonal()) == 0)
    dinv = [np.where(f, 0.0, 1.0 / np.where(f, 1.0, a.diagonal())) for a, f in zip(A, fix)]
    rng = np.random.default_rng(0)
    lam = []
    for l in range(len(A) - 1):
        x = rng.uniform(-1, 1, A[l].shape[0]) * (~fix[l])
        for _ in range(POWER_ITERS):
            y = dinv[l] * (A[l] @ x)
            est = np.linalg.norm(y) / np.linalg.norm(x)
            x = y
        lam.append(est)
    nf = ~fix[-1]
    return dict(A=A, P=P, fix=fix, dinv=dinv, lam=lam, nf=nf, Ainv=np.linalg.inv(A[-1][nf][:, nf].toarray()),
                free=np.flatnonzero(free))


def smooth(H, l, x, b, kind, upper):
    A, dinv, lam = H["A"][l], H["dinv"][l], H["lam"][l]
    if kind == "jacobi":
        w = OMEGA_SCALE / lam
        for _ in range(2):
            x = x + w * dinv * (b - A @ x)
        return x
    bu = upper * lam
    al = bu / CHEB_RATIO
    th, de = 0.5 * (bu + al), 0.5 * (bu - al)
    sg = th / de
    d = dinv * (b - A @ x) / th
    x = x + d
    rho0 = 1.0 / sg
    rho1 = 1.0 / (2.0 * sg - rho0)
    d = rho1 * rho0 * d + (2.0 * rho1 / de) * dinv * (b - A @ x)
    return x + d


def vcycle(H, l, b, kind, upper):
    if l == len(H["A"]) - 1:
        e = np.zeros_like(b)
        e[H["nf"]] = H["Ainv"] @ b[H["nf"]]
        return e
    x = smooth(H, l, np.zeros_like(b), b, kind, upper)
    rc = (H["P"][l].T @ (b - H["A"][l] @ x)) * (~H["fix"][l + 1])
    x = x + (H["P"][l] @ vcycle(H, l + 1, rc, kind, upper)) * (~H["fix"][l])
    return smooth(H, l, x, b, kind, upper)


def cycle_matrix(H, kind, upper=1.3):
    f = H["free"]
    cols = []
    for k in f:
        e = np.zeros(H["A"][0].shape[0])
        e[k] = 1.0
        cols.append(vcycle(H, 0, e, kind, upper)[f])
    return np.array(cols).T


def test_chebyshev_cycle_is_spd_and_better_conditioned():
    geom = BoxGeometry(12, 4, 4, clamp="root_face", mount="tip_face")
    rng = np.random.default_rng(5)
    rho = np.clip(rng.uniform(-0.4, 1.0, geom.n_elements), 1e-3, 1.0)     # voids next to solid
    H = hierarchy(geom, rho)
    assert len(H["A"]) == 2
    Kf = H["A"][0][H["free"]][:, H["free"]].toarray()
    kappa = {}
    for kind in ("chebyshev", "jacobi"):
        B = cycle_matrix(H, kind)
        assert np.linalg.norm(B - B.T) <= 1e-9 * np.linalg.norm(B)
        assert np.linalg.eigvalsh(0.5 * (B + B.T)).min() > 0.0
        ev = np.sort(np.linalg.eigvals(B @ Kf).real)
        assert ev[0] > 0.0
        kappa[kind] = ev[-1] / ev[0]
    assert kappa["chebyshev"] < kappa["jacobi"]
    # an interval that stops below lambda_max amplifies the top of the spectrum
    B = cycle_matrix(H, "chebyshev", upper=0.8)
    assert np.sort(np.linalg.eigvals(B @ Kf).real)[0] < 0.0
