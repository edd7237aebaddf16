"""The oracle against fixtures produced by the reference itself (CPU only)."""
import numpy as np
import pytest

from oracle import fem as ofem
from oracle import modal as omodal
from oracle import topopt as otop
from tof_b200 import configs as C
from tof_b200.geometry import BoxGeometry


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def tiny_geom(g):
    return BoxGeometry(int(g["nx"]), int(g["ny"]), int(g["nz"]), *g["h"], clamp="root_face",
                       mount="tip_face", in_arm_mask=g["in_arm"], keep_solid_mask=g["keep_solid"])


@pytest.fixture(scope="module")
def tiny(golden):
    g = golden("tiny")
    geom = tiny_geom(g)
    fem = ofem.OracleFEM(geom, C.PA12.E, C.PA12.nu, C.PA12.rho)
    return g, geom, fem


def test_element_matrices(tiny):
    g, geom, fem = tiny
    assert rel(fem.Ke, g["Ke"]) < 1e-14
    assert rel(fem.Me, g["Me"]) < 1e-14


def test_dof_bookkeeping(tiny):
    g, geom, fem = tiny
    np.testing.assert_array_equal(fem.fixed_dofs, g["fixed_dofs"])
    np.testing.assert_array_equal(fem.free_dofs, g["free_dofs"])
    np.testing.assert_array_equal(fem.elem_dof_ids, g["elem_dof_ids"])
    # the removed corner voxel leaves node (6,3,3) in no element: a ghost
    ghost = int(geom.node_index(6, 3, 3))
    assert 3 * ghost in set(g["fixed_dofs"].tolist())


def test_operators(tiny):
    g, geom, fem = tiny
    rho = g["rho"]
    K = fem.assemble_K(rho)
    M = fem.assemble_M(rho, 0.06, g["tip_nodes"])
    fr = fem.free_dofs
    X = g["X"]
    assert rel((K[fr][:, fr] @ X[fr]), g["KX"][fr]) < 1e-14
    assert rel((M[fr][:, fr] @ X[fr]), g["MX"][fr]) < 1e-14
    assert rel(K.diagonal(), g["diagK"]) < 1e-14
    assert rel(M.diagonal(), g["diagM"]) < 1e-14


def test_static_and_compliance(tiny):
    g, geom, fem = tiny
    for F, u_ref in ((g["F1"], g["u1"]), (g["F2"], g["u2"])):
        u, _ = fem.solve(g["rho"], F, exact=True)
        assert rel(u, u_ref) < 1e-10
        u_cg, info = fem.solve(g["rho"], F, rtol=1e-12)
        assert info == 0 and rel(u_cg, u_ref) < 1e-7
    assert rel(fem.elem_compliance(g["u1"]), g["ce1"]) < 1e-13


def test_modal_sensitivity_effective_mass(tiny):
    g, geom, fem = tiny
    freqs, modes, lam = fem.modal(g["rho"], 4, 0.06, g["tip_nodes"])
    assert rel(freqs, g["freqs"]) < 1e-10
    mac = np.abs(np.sum(modes * g["modes"], axis=0))
    mac /= np.linalg.norm(modes, axis=0) * np.linalg.norm(g["modes"], axis=0)
    assert np.all(mac > 1 - 1e-8)
    dlam = fem.eigenvalue_sensitivity(g["rho"], lam[0], modes[:, 0], 0.06, g["tip_nodes"])
    assert rel(dlam, g["dlam0"]) < 1e-8
    eff = omodal.effective_mass(fem, g["rho"], modes, 0.06, g["tip_nodes"])
    assert rel(eff, g["eff"]) < 1e-8
    assert abs(fem.total_mass(g["rho"]) - float(g["total_mass"])) < 1e-15


def test_filter(tiny):
    g, geom, fem = tiny
    assert rel(otop.cone_kernel(1.5), g["k15"]) == 0.0
    assert rel(otop.cone_kernel(2.3), g["k23"]) == 0.0
    assert rel(otop.filter_field(g["field"], g["design"], g["k15"]), g["filt15"]) < 1e-15
    assert rel(otop.filter_field(g["field"], g["in_arm"], g["k23"]), g["filt23"]) < 1e-15


def test_filter_adjoint_is_transpose(tiny):
    g, geom, fem = tiny
    rng = np.random.default_rng(0)
    mask = g["design"]
    a = rng.standard_normal(mask.shape) * mask
    b = rng.standard_normal(mask.shape) * mask
    lhs = np.sum(otop.filter_field(a, mask, g["k15"]) * b)
    rhs = np.sum(a * otop.filter_adjoint(b, mask, g["k15"]))
    assert abs(lhs - rhs) < 1e-12 * max(abs(lhs), 1.0)


def test_oc(golden):
    g = golden("oc")
    x_new = otop.oc_update(g["x"], g["dc"], float(g["V_e"]), float(g["target_volume"]),
                           float(g["move"]))
    assert np.array_equal(x_new, g["x_new"])


def test_simp_iterations(golden):
    g = golden("simp_small")
    geom = C.arm_geometry(nx=int(g["nx"]), ny=int(g["ny"]), nz=int(g["nz"]), h=2e-3,
                          mount_cols=2)
    fem = ofem.OracleFEM(geom, C.PA12.E, C.PA12.nu, C.PA12.rho)
    opt = otop.OracleSIMP(geom, fem, [g["F1"], g["F2"]], vol_frac=float(g["vol_frac"]),
                          r_min_mm=float(g["r_min_mm"]), weights=g["weights"],
                          min_freq_Hz=float(g["min_freq_Hz"]), tip_mass_kg=0.06,
                          n_modes_track=int(g["n_modes"]), mu_freq_init=float(g["mu_init"]),
                          mu_freq_ramp_every=int(g["ramp_every"]))
    for it in range(int(g["n_iter"])):
        r = opt.step()
        assert rel(r["compliance"], g["compliance"][it]) < 1e-9
        assert abs(r["change"] - g["change"][it]) < 1e-9
        assert abs(r["freqs"][r["track_idx"]] - g["omega1"][it]) < 1e-8 * g["omega1"][it]
        assert r["mu"] == g["mu_hist"][it]
    assert rel(opt.physical_density(opt.rho_grid), g["rho_final"]) < 1e-9


def test_cantilever(golden):
    g = golden("cantilever")
    geom = C.cantilever_geometry()
    fem = ofem.OracleFEM(geom, C.PA12.E, C.PA12.nu, C.PA12.rho)
    np.testing.assert_array_equal(fem.free_dofs, g["free_dofs"])
    rho = C.cantilever_density(geom)
    assert np.array_equal(rho, g["rho"])
    assert np.array_equal(C.cantilever_loads(geom)[0], g["F"])
    u, info = fem.solve(rho, g["F"], rtol=1e-8)
    assert info == 0
    assert abs(float(g["F"] @ u) - float(g["compliance"])) < 1e-7 * float(g["compliance"])
    assert abs(float(g["compliance"]) - 1.449978e-2) < 1e-8


def test_arm_inputs(golden):
    g = golden("arm")
    geom = C.arm_geometry()
    fem = ofem.OracleFEM(geom, C.PA12.E, C.PA12.nu, C.PA12.rho)
    np.testing.assert_array_equal(fem.fixed_dofs, g["fixed_dofs"])
    assert np.array_equal(C.arm_hollow_density(geom), g["rho"])
    assert np.array_equal(C.arm_static_loads(geom)[0], g["F"])
    # operator check on a sample (the full sparse-LU solve takes ~80 s here;
    # the GPU parity tests compare against the stored compliance instead)
    K = fem.reduce(fem.assemble_K(g["rho"]))
    assert K.shape[0] == len(g["free_dofs"])
    assert np.all(K.diagonal() > 0)


def test_oracle_stress_and_fatigue(golden):
    """The stress / fatigue restatement reproduces the reference's own outputs."""
    from oracle import stress as S
    d = golden("stress")
    t = golden("tiny")
    B = S.B_centre(*t["h"])
    assert np.array_equal(B, d["B_centre"])
    for i in (1, 2):
        sig = S.compute_stress(d[f"u{i}"], t["elem_dof_ids"], B, d["D"], d["rho"])
        np.testing.assert_allclose(sig, d[f"sigma{i}"], rtol=1e-13, atol=1e-13 * np.abs(sig).max())
        np.testing.assert_allclose(S.von_mises(sig), d[f"vm{i}"], rtol=1e-13)
        np.testing.assert_allclose(S.principal_stress_max(sig), d[f"smax{i}"], rtol=1e-12,
                                   atol=1e-12 * np.abs(d[f"smax{i}"]).max())
    f = S.fatigue_life_field(d["fat_s1"], d["fat_s2"], 48e6)
    for k, v in f.items():
        np.testing.assert_allclose(v, d["fat_" + k], rtol=1e-13)
    assert S.sn_alt_stress_at(1e6) == float(d["sn_alt_1e6"])


def test_oracle_frf(golden):
    from oracle.modal import modal_frf_at_dof
    d = golden("frf")
    for i, dof in enumerate(d["dofs"]):
        f, H = modal_frf_at_dof(d["freqs"], d["modes"], int(dof))
        np.testing.assert_array_equal(f, d[f"f{i}"])
        np.testing.assert_allclose(H, d[f"H{i}"], rtol=1e-13)
    f, H = modal_frf_at_dof(d["freqs"], d["modes"], int(d["dofs"][0]), (50.0, 4000.0), 257, 0.05)
    np.testing.assert_allclose(H, d["H_alt"], rtol=1e-13)


def test_production_domain_default_material_known_answer(golden):
    """The fixture generator's exact FP64 eigensolve of the reference's
    production domain (ArmGeometry3D, solid, 60 g tip mass, 198 093 free DOF)
    with the reference's default Material() (rho 930 kg/m^3) gives the known
    exact frequencies of that domain, 203.891, 247.267, 801.087, 1234.547,
    1249.151 and 1636.433 Hz.  arm3d_modes.npz, which the production-domain
    GPU test uses, is the same computation for the PA12 of the configs
    (rho 1010), hence its lower frequencies."""
    g = golden("arm3d_modes_930")
    known = np.array([203.891, 247.267, 801.087, 1234.547, 1249.151, 1636.433])
    assert int(g["n_free"]) == 198093
    assert np.allclose(np.round(g["freqs"], 3), known, rtol=0, atol=1e-9)
    g1010 = golden("arm3d_modes")
    assert int(g1010["n_free"]) == 198093
    assert np.all(g1010["freqs"] < g["freqs"])
