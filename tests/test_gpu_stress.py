"""Element stress (Voigt sigma at the centres, von Mises, largest principal)
and the Goodman / S-N fatigue field on the device, against the reference's
own outputs (tests/golden/stress.npz) and, at the arm size, against the
oracle.  Tolerances: 1e-12 relative to the field's largest entry (FP64; the
closed-form principal stress 1e-10)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _tiny_fem(t):
    from tof_b200 import configs as C
    from tof_b200.fem import FEM3D
    from tof_b200.geometry import BoxGeometry
    geom = BoxGeometry(int(t["nx"]), int(t["ny"]), int(t["nz"]), *t["h"], clamp="root_face", mount="tip_face",
                       in_arm_mask=t["in_arm"], keep_solid_mask=t["keep_solid"])
    return FEM3D(geom, C.PA12)


def _close(a, b, tol):
    scale = max(float(np.abs(b).max()), 1e-300)
    assert float(np.abs(np.asarray(a) - b).max()) <= tol * scale


def test_stress_fields_match_reference(golden):
    d, t = golden("stress"), golden("tiny")
    fem = _tiny_fem(t)
    np.testing.assert_allclose(fem.B_centre, d["B_centre"], rtol=1e-15)
    for i in (1, 2):
        sig, vm, sm = fem.stress_fields(d[f"u{i}"], d["rho"])
        _close(sig, d[f"sigma{i}"], 1e-12)
        _close(vm, d[f"vm{i}"], 1e-12)
        _close(sm, d[f"smax{i}"], 1e-10)
        _close(fem.compute_stress(d[f"u{i}"], d["rho"]), d[f"sigma{i}"], 1e-12)
    # two vectors in one launch
    sig2, _, _ = fem.stress_fields(np.stack([d["u1"], d["u2"]]), d["rho"])
    _close(sig2[1], d["sigma2"], 1e-12)


def test_invariants_of_given_stress(golden):
    d, t = golden("stress"), golden("tiny")
    fem = _tiny_fem(t)
    _close(fem.von_mises(d["sigma1"]), d["vm1"], 1e-12)
    _close(fem.principal_stress_max(d["sigma2"]), d["smax2"], 1e-10)


def test_fatigue_matches_reference(golden):
    from tof_b200 import fatigue as F
    d = golden("stress")
    f = F.fatigue_life_field(d["fat_s1"], d["fat_s2"], 48e6)
    for k, v in f.items():
        np.testing.assert_allclose(v, d["fat_" + k], rtol=1e-12, err_msg=k)
    np.testing.assert_allclose(F.sn_life(d["fat_sigma_alt_eq"]), d["fat_life"], rtol=1e-12)
    assert F.sn_alt_stress_at(1e6) == float(d["sn_alt_1e6"])
    # every branch of the S-N lookup is present in the sample
    life = d["fat_life"]
    assert (life == 1e9).any() and (life == 1.0).any() and ((life > 1.0) & (life < 1e9)).any()


def test_arm_stress_matches_oracle():
    """Device stress of an arm static solution against the oracle's
    restatement on the same displacements (18 480 elements, 4 load cases)."""
    from oracle import stress as S
    from tof_b200.workloads import arm_simp
    geom, fem, opt = arm_simp(mode="mixed")
    rho_a = opt.physical_density()[torch.as_tensor(fem.active_ids, device=opt.dev)].cpu().numpy()
    U = np.stack([fem.solve(rho_a, F) for F in opt.F_list[:2]])
    sig, vm, sm = fem.stress_fields(U, rho_a)
    for k in range(2):
        ref = S.compute_stress(U[k], fem.elem_dof_ids, S.B_centre(geom.dx, geom.dy, geom.dz), fem.D_solid, rho_a)
        _close(sig[k], ref, 1e-12)
        _close(vm[k], S.von_mises(ref), 1e-12)
        _close(sm[k], S.principal_stress_max(ref), 1e-10)


def test_modal_frf_matches_reference(golden):
    """Modal-superposition FRF (src/plotting.py:378-399) on the device against
    the reference's own output, one DOF at a time and batched over DOFs."""
    from tof_b200.modal import modal_frf, modal_frf_at_dof
    d = golden("frf")
    for i, dof in enumerate(d["dofs"]):
        f, H = modal_frf_at_dof(d["freqs"], d["modes"], int(dof))
        np.testing.assert_array_equal(f, d[f"f{i}"])
        np.testing.assert_allclose(H, d[f"H{i}"], rtol=1e-12)
    f, H = modal_frf_at_dof(d["freqs"], d["modes"], int(d["dofs"][0]), (50.0, 4000.0), 257, 0.05)
    np.testing.assert_allclose(H, d["H_alt"], rtol=1e-12)
    Hb = modal_frf(d["freqs"], d["modes"][d["dofs"], :], d["f0"]).cpu().numpy()
    for i in range(3):
        np.testing.assert_allclose(Hb[i], d[f"H{i}"], rtol=1e-12)
