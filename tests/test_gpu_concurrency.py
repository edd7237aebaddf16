"""Static and modal solves of a design iteration issued at the same time on
two streams (SIMPOptimizer concurrent=True, the default in the mixed form):
the library keeps separate scratch and multigrid vectors for the two solver
families, so the iterations are bit-identical to issuing them one after the
other."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_concurrent_static_and_modal_match_sequential():
    from tof_b200.workloads import arm_simp
    runs = []
    for concurrent in (True, False):
        geom, fem, opt = arm_simp(mode="mixed", nx=48, ny=8, nz=8)
        opt.concurrent = concurrent
        for _ in range(4):
            opt.step()
        torch.cuda.synchronize()
        runs.append((opt.history, opt.x.cpu().numpy(), opt.u4.cpu().numpy(), opt.X4.cpu().numpy()))
    (h1, x1, u1, m1), (h2, x2, u2, m2) = runs
    for key in ("compliance", "omega_1_Hz", "change", "pcg_iters", "modal_iters", "modal_converged"):
        assert h1[key] == h2[key], key
    assert np.array_equal(x1, x2)
    assert np.array_equal(u1, u2)
    assert np.array_equal(m1, m2)
