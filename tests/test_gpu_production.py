"""The reference's production domain (ArmGeometry3D: 108 x 21 x 27 voxels at
2 mm, six screw clamps, motor-mount tip mass, ~198k free DOF) through this
package: the six lowest frequencies of the solid arm with the 60 g tip mass
against the reference's own exact FP64 eigenpairs (tests/golden/
arm3d_modes.npz), to 1e-8 relative, and a static thrust solve whose
compliance is consistent between the two forms."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_production_domain_frequencies(golden):
    from tof_b200 import configs as C
    from tof_b200.fem import FEM3D
    from tof_b200.geometry3d import ArmGeometry3D
    d = golden("arm3d_modes")
    g = ArmGeometry3D()
    fem = FEM3D(g, C.PA12, mode="mixed")
    assert len(fem.free_dofs) == int(d["n_free"])
    freqs, modes, lam = fem.modal_analysis(np.ones(fem.n_active), n_modes=6, tip_mass_kg=0.06, tol=1e-8)
    assert np.max(np.abs(freqs / d["freqs"] - 1.0)) < 1e-8, (freqs, d["freqs"])


def test_production_domain_static_forms_agree():
    from tof_b200 import configs as C
    from tof_b200.fem import FEM3D
    from tof_b200.geometry3d import ArmGeometry3D
    g = ArmGeometry3D()
    F = g.load_vector(F=(0.0, 0.0, -15.0), Mz=0.3)
    rho = np.ones(int(g.build_masks()["in_arm"].sum()))
    out = {}
    for mode in ("mixed", "fp64"):
        fem = FEM3D(g, C.PA12, mode=mode)
        fem.SOLVE_RTOL = 1e-10
        u = fem.solve(rho, F)
        out[mode] = float(F @ u)
    assert abs(out["mixed"] / out["fp64"] - 1.0) < 1e-8, out
