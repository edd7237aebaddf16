"""Independent designs advanced concurrently (one stream and host thread
each) give bit-identical histories to running them one after another, and
each design's modes are ranked by effective mass.  Also: the tile
autotuner returns a candidate that a context accepts."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _designs():
    from tof_b200.workloads import arm_simp
    out = []
    for name, kw in (("a", dict(nx=24, ny=6, nz=6, vf=0.08)), ("b", dict(nx=30, ny=8, nz=6, vf=0.2))):
        geom, fem, opt = arm_simp(mode="mixed", n_modes=4, **kw)
        out.append((name, geom, fem, opt))
    return out


def test_concurrent_equals_sequential():
    from tof_b200.batch import DesignSweep
    conc = DesignSweep(_designs())
    seq = DesignSweep(_designs())
    for _ in range(2):
        conc.step(concurrent=True)
        seq.step(concurrent=False)
    hc, hs = conc.histories(), seq.histories()
    for name in hc:
        for key in ("compliance", "omega_1_Hz", "change"):
            assert np.array_equal(np.asarray(hc[name][key]), np.asarray(hs[name][key])), (name, key)
        r = conc.ranking[name][-1]
        assert sorted(r["order"]) == list(range(4))
        eff = np.asarray(r["eff"])
        assert np.all(np.diff(eff[r["order"]]) <= 0.0)


def test_autotuned_tile_is_usable():
    from tof_b200 import configs as C
    from tof_b200.autotune import tune_tile
    from tof_b200.fem import FEM3D
    geom = C.arm_geometry(nx=24, ny=6, nz=6)
    fem = FEM3D(geom, C.PA12, mode="mixed", tile="auto")
    best, timings = tune_tile(fem, return_timings=True)
    assert best in timings and len(timings) >= 3
    ctx = fem.device()                       # the context accepts the tuned tile
    assert tuple(ctx.tile) == tuple(best)
