"""The drop-in on the reference's own classes.

`enable_b200_solver` is applied to the reference's `src.fem.FEM3D` and
`src.topopt` (the reference package installed into baseline/_ref with pip's
`--target`) and
the reference's own code runs on top of it:

* its `SIMPOptimizer.run` (src/topopt.py:217-427) for four iterations of the
  small arm case, against the fixture of the same run with exact solves
  (tests/golden/simp_small.npz): histories to 1e-6;
* its self-test path `K = assemble_K(rho); u = apply_BCs_and_solve(K, F)`
  (src/fem.py:674-680) with the reference's own assembled CSR, against the
  reference's unpatched direct solve; a CSR changed after assembly, or one
  that assemble_K did not build, is rejected.

The patch is undone after each test.  Fails when the reference is not
installed in baseline/_ref.
"""
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from conftest import ROOT  # noqa: E402
from test_gpu_api import tiny_geom  # noqa: E402
from test_gpu_core import rel  # noqa: E402

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "baseline", "_ref")


@pytest.fixture(scope="module")
def ref():
    if not os.path.isfile(os.path.join(REF, "src", "fem.py")):
        pytest.fail("the reference is not installed in baseline/_ref (pip install --target baseline/_ref <checkout>)")
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import src.fem as rfem
    import src.topopt as rtop
    return rfem, rtop


def _material(rfem):
    from tof_b200 import configs as C
    return rfem.Material(E=C.PA12.E, nu=C.PA12.nu, sigma_y=C.PA12.sigma_y, sigma_u=C.PA12.sigma_u, rho=C.PA12.rho)


def test_reference_simp_run_on_b200(ref, golden):
    from tof_b200 import configs as C
    from tof_b200.fem_b200 import disable_b200_solver, enable_b200_solver
    rfem, rtop = ref
    g = golden("simp_small")
    geom = C.arm_geometry(nx=int(g["nx"]), ny=int(g["ny"]), nz=int(g["nz"]), h=2e-3, mount_cols=2)
    filt0 = rtop.filter_field
    assert enable_b200_solver(rfem.FEM3D, rtop, mode="fp64", rtol=1e-12)
    try:
        assert rtop.filter_field is not filt0
        fem = rfem.FEM3D(geom, _material(rfem))
        opt = rtop.SIMPOptimizer(geom, fem, load_cases=[dict(F=(0, 0, 0))] * 2, weights=list(g["weights"]),
                                 vol_frac=float(g["vol_frac"]), r_min_mm=float(g["r_min_mm"]),
                                 max_iter=int(g["n_iter"]), tol_change=0.0, min_freq_Hz=float(g["min_freq_Hz"]),
                                 tip_mass_kg=0.06, n_modes_track=int(g["n_modes"]),
                                 mu_freq_init=float(g["mu_init"]), mu_freq_ramp_every=int(g["ramp_every"]))
        opt.F_list = [g["F1"].copy(), g["F2"].copy()]
        res = opt.run(verbose=False)
        assert "fp64" in fem._b200_twins                      # the device twin did the work
    finally:
        disable_b200_solver(rfem.FEM3D)
    assert rtop.filter_field is filt0 and "_b200_originals" not in rfem.FEM3D.__dict__
    h = res["history"]
    assert rel(h["compliance"], g["compliance"]) < 1e-6
    assert np.max(np.abs(np.array(h["change"]) - g["change"])) < 1e-5
    assert rel(h["omega_1_Hz"], g["omega1"]) < 1e-6
    assert np.allclose(h["mu_freq"], g["mu_hist"])
    assert rel(h["vol_frac"], g["vf_hist"]) < 1e-6
    assert rel(res["rho_active"], g["rho_final"]) < 1e-5


def test_reference_assembled_csr_through_apply_bcs_and_solve(ref, golden):
    from tof_b200.fem_b200 import disable_b200_solver, enable_b200_solver
    rfem, _ = ref
    g = golden("tiny")
    geom = tiny_geom(g)
    fem = rfem.FEM3D(geom, _material(rfem))
    rho = g["rho"]
    u_ref = fem.apply_BCs_and_solve(fem.assemble_K(rho), g["F2"], method="lu")   # the reference, unpatched
    assert enable_b200_solver(rfem.FEM3D, None, mode="fp64")
    try:
        K = fem.assemble_K(rho)                                # the reference's CSR (tagged)
        assert K.nnz > 0 and hasattr(K, "tocsc")
        u = fem.apply_BCs_and_solve(K, g["F2"], rtol=1e-10)
        assert rel(u, u_ref) < 1e-8
        assert rel(u, g["u2"]) < 1e-8
        u_lu = fem.apply_BCs_and_solve(K, g["F2"], method="lu")
        assert rel(u_lu, u_ref) < 1e-9
        K2 = fem.assemble_K(rho)
        K2.data[0] *= 2.0                                      # changed after assembly
        with pytest.raises(TypeError):
            fem.apply_BCs_and_solve(K2, g["F2"])
        with pytest.raises(TypeError):                         # a CSR assemble_K did not build
            fem.apply_BCs_and_solve(K.copy(), g["F2"])
    finally:
        disable_b200_solver(rfem.FEM3D)
