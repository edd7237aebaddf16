"""Generate golden fixtures by running the reference solver itself.

Run in a container that has the reference source tree (read-only), passing
its root directory:

    python tests/golden/make_golden.py --ref <reference checkout> [--skip-arm] [--only stress|frf|arm3d|arm3d_modes]

The reference (NinhGhoster/TO-F450-arm, pure Python + SciPy) is imported from
its own `src/` and `sims/` packages and driven with the synthetic geometries of
`tof_b200.geometry` / `tof_b200.configs` (inputs only).  Two solver branches of
the reference are made exact for the fixtures:

* static solves call `FEM3D.apply_BCs_and_solve(..., method="lu")`, the
  reference's own direct branch (src/fem.py:551-552);
* `scipy.sparse.linalg.lobpcg` as seen by src/fem.py is replaced by a tight
  shift-invert `eigsh` (sigma = 0, tol 1e-13) on the same K_ff / M_ff, because
  the reference's LOBPCG at tol 1e-4 is not an accuracy oracle (it misses f1
  by up to 16 % on the production domain).  Everything else in
  `modal_analysis` (assembly, tip mass, sorting, clamping, padding) is the
  reference's code.

Fixtures are written next to this script.  Nothing on the GPU test path reads
the reference; only these .npz files travel.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "to-f450-arm_b200"))

from tof_b200 import configs as C  # noqa: E402
from tof_b200.geometry import BoxGeometry  # noqa: E402


def exact_eigs(K, X, B=None, M=None, tol=None, largest=False, maxiter=None, **kw):
    k = X.shape[1]
    lam, V = spla.eigsh(K.tocsc(), k=k, M=B.tocsc(), sigma=0.0, which="LM", tol=1e-13,
                        maxiter=50000)
    return lam, V


def sign_fix(modes):
    """Make the largest-magnitude entry of each mode positive."""
    out = modes.copy()
    for k in range(out.shape[1]):
        i = np.argmax(np.abs(out[:, k]))
        if out[i, k] < 0:
            out[:, k] *= -1
    return out


def setup_reference(ref):
    sys.path.insert(0, ref)
    import src.fem as rfem
    import src.topopt as rtop
    rfem.spla.lobpcg = exact_eigs          # exact eigenpairs, see module docstring
    from sims import modal_participation as rmp
    return rfem, rtop, rmp


def mat_ref(rfem):
    return rfem.Material(E=C.PA12.E, nu=C.PA12.nu, sigma_y=C.PA12.sigma_y,
                         sigma_u=C.PA12.sigma_u, rho=C.PA12.rho)


def geom_arrays(geom, fem):
    m = geom.build_masks()
    return dict(nx=geom.nx, ny=geom.ny, nz=geom.nz, h=np.array([geom.dx, geom.dy, geom.dz]),
                in_arm=m["in_arm"], design=m["design"], keep_solid=m["keep_solid"],
                fixed_dofs=fem.fixed_dofs, free_dofs=fem.free_dofs,
                tip_nodes=geom.motor_mount_top_nodes(),
                Ke=fem.Ke_solid, Me=fem.Me_solid)


def tiny_geometry():
    nx, ny, nz = 6, 3, 3
    in_arm = np.ones((nx, ny, nz), bool)
    in_arm[5, 2, 2] = False            # corner voxel removed -> node (6,3,3) is a ghost
    in_arm[2, 1, 1] = False            # interior hole
    keep = np.zeros_like(in_arm)
    keep[0, :, :] = True
    g = BoxGeometry(nx, ny, nz, 2e-3, 2e-3, 2e-3, clamp="root_face", mount="tip_face",
                    in_arm_mask=in_arm, keep_solid_mask=keep)
    return g


def make_tiny(rfem, rtop, rmp):
    g = tiny_geometry()
    fem = rfem.FEM3D(g, mat_ref(rfem))
    rng = np.random.default_rng(1)
    rho = rng.uniform(0.03, 1.0, fem.n_active)
    rho[:3] = [0.05, 0.1, 0.0999]            # both branches of the mass penalty
    F1 = g.load_vector(F=(0.0, 0.0, -5.0))
    F2 = g.load_vector(F=(0.0, 3.0, 1.0), Mz=0.05)
    K = fem.assemble_K(rho)
    M = fem.assemble_M(rho, tip_mass_kg=0.06, tip_mass_nodes=g.motor_mount_top_nodes())
    fr = fem.free_dofs
    X = np.zeros((g.n_dofs, 3))
    X[fr] = rng.standard_normal((len(fr), 3))
    KX = np.zeros_like(X)
    MX = np.zeros_like(X)
    KX[fr] = K[fr][:, fr] @ X[fr]
    MX[fr] = M[fr][:, fr] @ X[fr]
    u1 = fem.apply_BCs_and_solve(K, F1, method="lu")
    u2 = fem.apply_BCs_and_solve(K, F2, method="lu")
    ce1 = fem.elem_compliance(u1, rho)
    freqs, modes, lam = fem.modal_analysis(rho, n_modes=4, tip_mass_kg=0.06)
    dlam0 = fem.eigenvalue_sensitivity(rho, lam[0], modes[:, 0], tip_mass_kg=0.06)
    eff = rmp.effective_mass_voxel(fem, g, rho, modes, 0.06, direction=2)
    masks = g.build_masks()
    field = rng.standard_normal((g.nx, g.ny, g.nz))
    k15 = rtop.cone_kernel(1.5)
    k23 = rtop.cone_kernel(2.3)
    filt15 = rtop.filter_field(field, masks["design"], k15)
    filt23 = rtop.filter_field(field, masks["in_arm"], k23)
    return dict(geom_arrays(g, fem), rho=rho, F1=F1, F2=F2, X=X, KX=KX, MX=MX,
                diagK=K.diagonal(), diagM=M.diagonal(),
                u1=u1, u2=u2, ce1=ce1, freqs=freqs, lam=lam, modes=sign_fix(modes),
                dlam0=dlam0, eff=eff, field=field, k15=k15, k23=k23,
                filt15=filt15, filt23=filt23, total_mass=fem.total_mass(rho),
                elem_dof_ids=fem.elem_dof_ids)


def make_oc(rtop):
    """The OC update on its own (src/topopt.py:190-214) via a stub optimiser."""
    rng = np.random.default_rng(2)
    x = rng.uniform(0.001, 1.0, 500)
    dc = -rng.uniform(1e-6, 1e-2, 500)

    class Stub:
        V_e = 8e-9
        move = 0.2
        target_volume = 0.3 * 500 * 8e-9
    x_new = rtop.SIMPOptimizer._oc_update(Stub(), x, dc)
    return dict(x=x, dc=dc, V_e=Stub.V_e, move=Stub.move, target_volume=Stub.target_volume,
                x_new=x_new)


def simp_geometry():
    return C.arm_geometry(nx=16, ny=4, nz=4, h=2e-3, mount_cols=2)


def make_simp(rfem, rtop):
    g = simp_geometry()
    fem = rfem.FEM3D(g, mat_ref(rfem))
    orig = rfem.FEM3D.apply_BCs_and_solve

    def lu_solve(self, K, F, method="cg", x0=None, rtol=1e-5):
        return orig(self, K, F, method="lu")
    rfem.FEM3D.apply_BCs_and_solve = lu_solve
    try:
        F = C.arm_static_loads(g)[:2]
        opt = rtop.SIMPOptimizer(g, fem, load_cases=[dict(F=(0, 0, 0))] * 2,
                                 weights=[0.6, 0.4], vol_frac=0.3, r_min_mm=3.0, max_iter=4,
                                 tol_change=0.0, min_freq_Hz=1500.0, tip_mass_kg=0.06,
                                 n_modes_track=3, mu_freq_init=0.2, mu_freq_ramp_every=2)
        opt.F_list = [f.copy() for f in F]
        res = opt.run(verbose=False)
    finally:
        rfem.FEM3D.apply_BCs_and_solve = orig
    h = res["history"]
    return dict(geom_arrays(g, fem), F1=F[0], F2=F[1], weights=np.array([0.6, 0.4]),
                vol_frac=0.3, r_min_mm=3.0, min_freq_Hz=1500.0, mu_init=0.2, ramp_every=2,
                n_iter=4, n_modes=3,
                compliance=np.array(h["compliance"]), change=np.array(h["change"]),
                vf_hist=np.array(h["vol_frac"]), omega1=np.array(h["omega_1_Hz"]),
                mu_hist=np.array(h["mu_freq"]), viol=np.array(h["freq_violation"]),
                rho_final=res["rho_active"])


def make_cantilever(rfem, rmp):
    g = C.cantilever_geometry()
    fem = rfem.FEM3D(g, mat_ref(rfem))
    rho = C.cantilever_density(g)
    F = C.cantilever_loads(g)[0]
    K = fem.assemble_K(rho)
    t = time.time()
    u = fem.apply_BCs_and_solve(K, F, method="lu")
    t_lu = time.time() - t
    t = time.time()
    u_cg = fem.apply_BCs_and_solve(K, F, method="cg", rtol=1e-8)
    t_cg = time.time() - t
    fr = fem.free_dofs
    Kff = K[fr][:, fr]
    relres_cg = np.linalg.norm(F[fr] - Kff @ u_cg[fr]) / np.linalg.norm(F[fr])
    t = time.time()
    freqs, modes, lam = fem.modal_analysis(rho, n_modes=6, tip_mass_kg=0.0)
    t_eig = time.time() - t
    eff = rmp.effective_mass_voxel(fem, g, rho, modes, 0.0, direction=2)
    ce = fem.elem_compliance(u, rho)
    dlam0 = fem.eigenvalue_sensitivity(rho, lam[0], modes[:, 0], tip_mass_kg=0.0)
    print(f"cantilever: lu {t_lu:.2f}s  cg(1e-8) {t_cg:.2f}s relres {relres_cg:.2e}  eig {t_eig:.1f}s")
    return dict(geom_arrays(g, fem), rho=rho, F=F, u=u, compliance=float(F @ u), ce=ce,
                freqs=freqs, lam=lam, eff=eff, dlam0=dlam0, relres_cg=relres_cg,
                t_cg=t_cg)


def make_arm(rfem, rmp):
    g = C.arm_geometry()
    fem = rfem.FEM3D(g, mat_ref(rfem))
    rho = C.arm_hollow_density(g)
    F = C.arm_static_loads(g)[0]
    K = fem.assemble_K(rho)
    t = time.time()
    u = fem.apply_BCs_and_solve(K, F, method="lu")
    t_lu = time.time() - t
    t = time.time()
    freqs, modes, lam = fem.modal_analysis(rho, n_modes=6, tip_mass_kg=C.TIP_MASS_KG)
    t_eig = time.time() - t
    eff = rmp.effective_mass_voxel(fem, g, rho, modes, C.TIP_MASS_KG, direction=2)
    ce = fem.elem_compliance(u, rho)
    dlam0 = fem.eigenvalue_sensitivity(rho, lam[0], modes[:, 0], tip_mass_kg=C.TIP_MASS_KG)
    rng = np.random.default_rng(3)
    sample = np.sort(rng.choice(fem.n_active, 512, replace=False))
    dof_sample = np.sort(rng.choice(fem.free_dofs, 2048, replace=False))
    print(f"arm: lu {t_lu:.1f}s  eig {t_eig:.1f}s  freqs {freqs}")
    return dict(geom_arrays(g, fem), rho=rho, F=F, compliance=float(F @ u),
                u_sample=u[dof_sample], dof_sample=dof_sample,
                ce_sample=ce[sample], dlam0_sample=dlam0[sample], elem_sample=sample,
                freqs=freqs, lam=lam, eff=eff, umax=np.abs(u).max())


def make_stress(rfem):
    """Element stress (src/fem.py:564-602) on the tiny domain for both load
    cases, and the Goodman / S-N fatigue field (src/fatigue.py:24-112) on the
    von Mises pair plus a sweep that reaches every branch of sn_life."""
    from src import fatigue as rfat
    g = tiny_geometry()
    fem = rfem.FEM3D(g, mat_ref(rfem))
    rng = np.random.default_rng(1)
    rho = rng.uniform(0.03, 1.0, fem.n_active)
    rho[:3] = [0.05, 0.1, 0.0999]
    K = fem.assemble_K(rho)
    out = dict(rho=rho, B_centre=fem.B_centre, D=fem.D_solid)
    for i, F in enumerate((g.load_vector(F=(0.0, 0.0, -5.0)), g.load_vector(F=(0.0, 3.0, 1.0), Mz=0.05)), 1):
        u = fem.apply_BCs_and_solve(K, F, method="lu")
        sig = fem.compute_stress(u, rho)
        out[f"u{i}"] = u
        out[f"sigma{i}"] = sig
        out[f"vm{i}"] = fem.von_mises(sig)
        out[f"smax{i}"] = fem.principal_stress_max(sig)
    # fatigue: stresses in Pa spanning below endurance .. static overload
    a = rng.uniform(0.0, 90e6, 400)
    b = rng.uniform(0.0, 90e6, 400)
    a[:4] = [0.0, 11.9e6, 12.0e6, 30e6]
    b[:4] = [0.0, 0.0, 5e6, 30e6]
    fat = rfat.fatigue_life_field(a, b, C.PA12.sigma_u)
    out.update(fat_s1=a, fat_s2=b, **{f"fat_{k}": v for k, v in fat.items()})
    out["sn_alt_1e6"] = rfat.sn_alt_stress_at(1e6)
    return out


def make_frf(rfem):
    """Modal-superposition FRF |H_dd(f)| (src/plotting.py:378-399) of the tiny
    domain's modes at three DOFs.  src/plotting.py imports matplotlib at module
    level; only `modal_frf_at_dof` (pure NumPy) is used, so matplotlib is
    stubbed for the import when it is absent."""
    import types
    if "matplotlib" not in sys.modules:
        try:
            import matplotlib  # noqa: F401
        except ImportError:
            mpl = types.ModuleType("matplotlib")
            mpl.pyplot = types.ModuleType("matplotlib.pyplot")
            mpl.pyplot.rcParams = {}            # module-level style settings only
            mpl.colors = types.ModuleType("matplotlib.colors")
            for n in ("LogNorm", "Normalize", "BoundaryNorm"):
                setattr(mpl.colors, n, object)
            sys.modules.update({"matplotlib": mpl, "matplotlib.pyplot": mpl.pyplot,
                                "matplotlib.colors": mpl.colors})
    from src import plotting as rplot
    g = tiny_geometry()
    fem = rfem.FEM3D(g, mat_ref(rfem))
    rho = np.random.default_rng(1).uniform(0.03, 1.0, fem.n_active)
    freqs, modes, lam = fem.modal_analysis(rho, n_modes=4, tip_mass_kg=0.06)
    tip = g.motor_mount_top_nodes()
    dofs = np.array([3 * tip[0] + 2, 3 * tip[-1] + 1, fem.free_dofs[7]])
    out = dict(freqs=freqs, modes=modes, dofs=dofs)
    for i, d in enumerate(dofs):
        f, H = rplot.modal_frf_at_dof(freqs, modes, int(d))
        out[f"f{i}"], out[f"H{i}"] = f, H
    f, H = rplot.modal_frf_at_dof(freqs, modes, int(dofs[0]), freq_range_Hz=(50.0, 4000.0), n_pts=257,
                                  modal_damping=0.05)
    out["f_alt"], out["H_alt"] = f, H
    return out


def make_arm3d(with_modes=False, default_material=False):
    """The reference's production domain (src/mesh3d.py ArmGeometry3D):
    masks, clamped nodes, tip-mass nodes and load vectors; with_modes: the
    lowest 6 exact FP64 frequencies of the solid domain with the 60 g tip
    mass (src/fem.py:400-470 with the exact eigensolver), for the PA12 of the
    configs (rho 1010) or, with default_material, for the reference's default
    Material() (src/fem.py:183-188, rho 930)."""
    from src.mesh3d import ArmGeometry3D
    g = ArmGeometry3D()
    m = g.build_masks()
    out = {k: v for k, v in m.items()}
    out["fixed_nodes"] = g.fixed_nodes()
    out["motor_nodes"] = g.motor_mount_top_nodes()
    for tag, F in (("thrust", (0.0, 0.0, -15.0)), ("inplane", (3.0, -4.0, 2.0))):
        d, v = g.load_dofs_for_force(F)
        out[f"{tag}_dofs"], out[f"{tag}_vals"] = d, v
    d, v = g.load_dofs_for_moment_Mz(0.3)
    out["mz_dofs"], out["mz_vals"] = d, v
    if with_modes:
        import src.fem as rfem
        fem = rfem.FEM3D(g, rfem.Material() if default_material else mat_ref(rfem))
        t0 = time.time()
        freqs, modes, lam = fem.modal_analysis(np.ones(fem.n_active), n_modes=6, tip_mass_kg=0.06)
        out = dict(freqs=freqs, lam=lam, n_free=len(fem.free_dofs), seconds=time.time() - t0)
    return out


def make_arm_c3(rfem, rtop, rmp, n_iter=50):
    """The differentiation / SIMP workload on the 2 mm arm grid, run by the
    reference's own SIMPOptimizer.run (src/topopt.py:217-427) with exact
    solves: start design vf 0.08 + U(-0.02, 0.02) (seed 0), filter radius
    3 mm, 500 Hz augmented-Lagrangian target with mu 0.2, 6 tracked modes,
    60 g tip mass, four load cases (thrust; torque about the arm axis plus
    lateral; both; 3 g inertial from the reference's assembled M at the start
    design).  Records the first iteration's physical density, per-load-case
    compliances, frequencies and effective masses (6 and 8 modes), the
    sensitivity handed to the OC update in iterations 1 and 2, and the
    history of all n_iter iterations.

    The inputs (geometry, start values, surface loads) come from
    tof_b200.configs; the start values enter through the one place the
    reference reads vol_frac for them (src/topopt.py:231, an element-wise
    np.where), after target_volume has been computed from the scalar."""
    from scipy.sparse.linalg import splu
    g = C.arm_geometry()
    fem = rfem.FEM3D(g, mat_ref(rfem))
    masks = g.build_masks()
    x0 = C.arm_design_start(g, vf=0.08, seed=0).astype(np.float64)
    fr = fem.free_dofs
    lu_cache = {}

    def factor(Kff):
        """One sparse LU of K_ff per density, shared by the four static
        solves and the shift-invert eigensolve of that iteration."""
        key = hash(Kff.data.tobytes())
        if key not in lu_cache:
            lu_cache.clear()
            lu_cache[key] = splu(Kff, permc_spec="MMD_AT_PLUS_A")
        return lu_cache[key]

    def lu_solve(self, K, F, method="cg", x0=None, rtol=1e-5):
        u = np.zeros(self.geom.n_dofs)
        u[fr] = factor(K[fr][:, fr].tocsc()).solve(F[fr])
        return u

    def eigs_shared_lu(K, X, B=None, M=None, tol=None, largest=False, maxiter=None, **kw):
        lu = factor(K.tocsc())
        op = spla.LinearOperator(K.shape, matvec=lu.solve, dtype=np.float64)
        return spla.eigsh(K, k=X.shape[1], M=B.tocsc(), sigma=0.0, which="LM", tol=1e-13, maxiter=50000,
                          OPinv=op)

    rec = dict(solves=[], modal=[], dc=[], x=[], xs=[])
    orig_solve = rfem.FEM3D.apply_BCs_and_solve
    orig_solve_fn = rfem.FEM3D.solve
    orig_modal = rfem.FEM3D.modal_analysis
    orig_oc = rtop.SIMPOptimizer._oc_update

    def solve(self, rho_active, F, method="cg", x0=None):
        u = orig_solve_fn(self, rho_active, F, method, x0)
        if len(rec["solves"]) < 4:
            rec["solves"].append((rho_active.copy(), u.copy()))
        return u

    def modal(self, rho_active, *a, **kw):
        out = orig_modal(self, rho_active, *a, **kw)
        if not rec["modal"]:
            rec["modal"].append(out)
        return out

    def oc(self, x, dc):
        print(f"  arm_c3 iteration {len(rec['x']) + 1}: {time.time() - t0:.0f}s", flush=True)
        rec["x"].append(None)
        if len(rec["dc"]) < 2:
            rec["dc"].append(dc.copy())
            rec["xs"].append(x.copy())
        return orig_oc(self, x, dc)

    orig_lobpcg = rfem.spla.lobpcg
    rfem.spla.lobpcg = eigs_shared_lu
    rfem.FEM3D.apply_BCs_and_solve = lu_solve
    rfem.FEM3D.solve = solve
    rfem.FEM3D.modal_analysis = modal
    rtop.SIMPOptimizer._oc_update = oc
    t0 = time.time()
    try:
        F3 = C.arm_static_loads(g)
        opt = rtop.SIMPOptimizer(g, fem, load_cases=[dict(F=(0, 0, 0))] * 4, vol_frac=0.08, r_min_mm=3.0,
                                 move=0.2, max_iter=n_iter, tol_change=0.0, min_freq_Hz=500.0,
                                 tip_mass_kg=C.TIP_MASS_KG, n_modes_track=6, mu_freq_init=0.2,
                                 mu_freq_max=50.0, mu_freq_ramp_every=5, mu_freq_ramp_factor=1.5)
        # start values on the design cells (reference design-cell order)
        grid = np.zeros((g.nx, g.ny, g.nz))
        grid[masks["design"]] = x0
        ex, ey, ez = fem.elem_grid_idx.T
        v0 = np.ones(fem.n_active)
        dsg = opt.is_design_active
        v0[dsg] = grid[ex, ey, ez][dsg]
        # start physical density as run() forms it, for the inertial load
        rg = np.zeros((g.nx, g.ny, g.nz))
        rg[ex, ey, ez] = np.where(dsg, v0, 1.0)
        ph = rtop.filter_field(rg, opt.design_mask_grid, opt.kernel)
        ph[~opt.design_mask_grid] = 0.0
        ph = np.where(opt.design, ph, np.where(opt.in_arm, 1.0, 0.0))
        rho_start = ph[ex, ey, ez]
        ez_vec = np.zeros(g.n_dofs)
        ez_vec[2::3] = 1.0
        Mr = fem.assemble_M(rho_start, C.TIP_MASS_KG, g.motor_mount_top_nodes()) @ ez_vec
        F_list = F3 + [C.body_load_from_Mr(Mr, 3.0)]
        opt.F_list = [f.copy() for f in F_list]
        opt.vol_frac = v0
        res = opt.run(verbose=False)
        t_run = time.time() - t0
        freqs8, modes8, lam8 = rfem.FEM3D.modal_analysis(fem, rec["solves"][0][0], n_modes=8,
                                                         tip_mass_kg=C.TIP_MASS_KG)
    finally:
        rfem.spla.lobpcg = orig_lobpcg
        rfem.FEM3D.apply_BCs_and_solve = orig_solve
        rfem.FEM3D.solve = orig_solve_fn
        rfem.FEM3D.modal_analysis = orig_modal
        rtop.SIMPOptimizer._oc_update = orig_oc
    rho1 = rec["solves"][0][0]
    comp1 = np.array([float(F @ u) for F, (_, u) in zip(F_list, rec["solves"])])
    freqs1, modes1, lam1 = rec["modal"][0]
    eff1 = rmp.effective_mass_voxel(fem, g, rho1, modes1, C.TIP_MASS_KG, direction=2)
    eff8 = rmp.effective_mass_voxel(fem, g, rho1, modes8, C.TIP_MASS_KG, direction=2)
    h = res["history"]
    print(f"arm_c3: {n_iter} iterations in {t_run:.0f}s; c {h['compliance'][0]:.6e} -> {h['compliance'][-1]:.6e}")
    return dict(x0=x0, F=np.stack(F_list), rho1=rho1, compliance_lc1=comp1, freqs1=freqs1, lam1=lam1, eff1=eff1,
                freqs8=freqs8, lam8=lam8, eff8=eff8, dc1=rec["dc"][0], dc2=rec["dc"][1], x2=rec["xs"][1],
                compliance=np.array(h["compliance"]), change=np.array(h["change"]),
                vf_hist=np.array(h["vol_frac"]), omega1=np.array(h["omega_1_Hz"]),
                mu_hist=np.array(h["mu_freq"]), viol=np.array(h["freq_violation"]),
                rho_final=res["rho_active"], n_iter=n_iter, seconds=t_run)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference checkout (holds src/ and sims/)")
    ap.add_argument("--skip-arm", action="store_true")
    ap.add_argument("--only", default=None, help="write just this fixture (e.g. stress)")
    ap.add_argument("--iters", type=int, default=50, help="SIMP iterations of the arm_c3 fixture")
    a = ap.parse_args()
    rfem, rtop, rmp = setup_reference(a.ref)
    if a.only == "stress":
        np.savez_compressed(os.path.join(HERE, "stress.npz"), **make_stress(rfem))
        return
    if a.only == "arm3d":
        np.savez_compressed(os.path.join(HERE, "arm3d.npz"), **make_arm3d())
        return
    if a.only == "arm3d_modes":
        np.savez_compressed(os.path.join(HERE, "arm3d_modes.npz"), **make_arm3d(with_modes=True))
        return
    if a.only == "arm3d_modes_930":
        np.savez_compressed(os.path.join(HERE, "arm3d_modes_930.npz"),
                            **make_arm3d(with_modes=True, default_material=True))
        return
    if a.only == "arm_c3":
        np.savez_compressed(os.path.join(HERE, "arm_c3.npz"), **make_arm_c3(rfem, rtop, rmp, n_iter=a.iters))
        return
    if a.only == "frf":
        np.savez_compressed(os.path.join(HERE, "frf.npz"), **make_frf(rfem))
        return
    np.savez_compressed(os.path.join(HERE, "tiny.npz"), **make_tiny(rfem, rtop, rmp))
    np.savez_compressed(os.path.join(HERE, "oc.npz"), **make_oc(rtop))
    np.savez_compressed(os.path.join(HERE, "simp_small.npz"), **make_simp(rfem, rtop))
    np.savez_compressed(os.path.join(HERE, "cantilever.npz"), **make_cantilever(rfem, rmp))
    np.savez_compressed(os.path.join(HERE, "stress.npz"), **make_stress(rfem))
    np.savez_compressed(os.path.join(HERE, "frf.npz"), **make_frf(rfem))
    np.savez_compressed(os.path.join(HERE, "arm3d.npz"), **make_arm3d())
    if not a.skip_arm:
        np.savez_compressed(os.path.join(HERE, "arm3d_modes.npz"), **make_arm3d(with_modes=True))
        np.savez_compressed(os.path.join(HERE, "arm.npz"), **make_arm(rfem, rmp))


if __name__ == "__main__":
    main()
