"""Differentiable SIMP objective (compliance + augmented-Lagrangian frequency
penalty, 4 load cases, 500 Hz target, filter r = 1.5 voxels) on a small arm.

* The hand-written adjoint (exact filter transpose) against FP64 central
  finite differences, h = 1e-4, on seeded design cells; solves at 5e-9
  (statics: about the FP64 true-residual floor of this high-contrast design;
  the objective's stationary compliance form makes J second-order in that
  error) and 1e-6 (modes; eigenvalues are second-order in it).  Tolerance: 1e-4 of the largest gradient entry
  (the FD truncation and solver noise are ~1e-6 of it here).
* The reference-form sensitivity (normalised filter of dJ/drho, the
  reference's src/topopt.py:311, 361) against the oracle's analytic
  sensitivity of the same iterate, to 1e-6 relative.
* An FP32 input field gives an FP32 gradient.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _setup():
    from tof_b200.workloads import arm_simp
    from tof_b200.autograd import SIMPObjective
    geom, fem, opt = arm_simp(mode="mixed", nx=24, ny=6, nz=6)
    obj = SIMPObjective(opt, pcg_rtol=5e-9, modal_tol=1e-6)
    return geom, fem, opt, obj


def test_adjoint_matches_central_differences():
    geom, fem, opt, obj = _setup()
    x = opt.x.clone().requires_grad_(True)
    J = obj(x)
    J.backward()
    g = x.grad.detach()
    assert obj.last["viol"] > 0.0 and obj.last["P"] > 0.0          # the penalty is active
    design = opt.design_ids.cpu().numpy()
    rng = np.random.default_rng(0)
    cells = rng.choice(design, size=12, replace=False)
    h = 1e-4
    gmax = float(g[opt.design_ids].abs().max())
    for e in cells:
        xp = x.detach().clone(); xp[int(e)] += h
        xm = x.detach().clone(); xm[int(e)] -= h
        fd = (obj.evaluate(xp)["J"] - obj.evaluate(xm)["J"]) / (2 * h)
        assert abs(fd - float(g[int(e)])) <= 1e-4 * gmax, (int(e), fd, float(g[int(e)]))
    # cells off the design domain get no gradient
    off = torch.ones(opt.ctx.NE, dtype=torch.bool, device=g.device)
    off[opt.design_ids] = False
    assert float(g[off].abs().max()) == 0.0


def test_reference_sensitivity_matches_oracle():
    from oracle.fem import OracleFEM
    from oracle.topopt import OracleSIMP
    from tof_b200 import configs as C
    geom, fem, opt, obj = _setup()
    obj.evaluate(opt.x)
    mine = obj.reference_sensitivity()[opt.design_ids].cpu().numpy()
    ofem = OracleFEM(geom, C.PA12.E, C.PA12.nu, C.PA12.rho)
    ref = OracleSIMP(geom, ofem, opt.F_list, vol_frac=0.08, r_min_mm=3.0, min_freq_Hz=500.0, tip_mass_kg=0.06,
                     n_modes_track=6, mu_freq_init=0.2, x0_design=C.arm_design_start(geom).astype(float))
    r = ref.step()
    theirs = r["sens_final"][ref.design]
    assert np.linalg.norm(mine - theirs) <= 1e-6 * np.linalg.norm(theirs)
    assert abs(obj.last["c"] / r["compliance"] - 1.0) < 1e-9


def test_fp32_field_gives_fp32_gradient():
    geom, fem, opt, obj = _setup()
    x = opt.x.to(torch.float32).clone().requires_grad_(True)
    J = obj(x)
    J.backward()
    assert x.grad.dtype == torch.float32
    g64 = obj.gradient()
    d = opt.design_ids
    assert torch.allclose(x.grad[d].double(), g64[d], rtol=1e-6, atol=1e-6 * float(g64[d].abs().max()))
