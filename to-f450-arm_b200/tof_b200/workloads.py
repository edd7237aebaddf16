"""Ready-made workloads on the synthetic arm / cantilever domains.

`arm_simp(...)` builds the design-iteration workload: the 2 mm arm grid
(110 x 14 x 12 voxels), four load cases (15 N -z thrust on the motor-mount
face; 0.3 N m torque about the arm axis plus 10 N lateral on the tip face;
both together; a 3 g -z inertial load from the consistent mass at the
starting design), 6 tracked modes with a 500 Hz augmented-Lagrangian target,
60 g tip mass, filter radius 1.5 voxels, vf 0.08, design start
0.08 + U(-0.02, 0.02) (seed 0), static solves to a 1e-8 relative residual.
The inertial load is evaluated once at the starting design and then held
fixed, as the reference's optimiser supports design-independent loads only;
it is the full consistent mass applied to a unit z translation of every
node (clamped ones included), restricted to the free DOFs by the solver,
i.e. the rows (M @ e_z)[free] of the reference's assembled M.
"""
from __future__ import annotations

import numpy as np
import torch

from . import configs as C
from .fem import FEM3D
from .topopt import SIMPOptimizer


def arm_simp(mode="mixed", nx=110, ny=14, nz=12, h=2e-3, vf=0.08, n_modes=6, min_freq_Hz=500.0,
             solve_rtol=1e-8, modal_tol=1e-5, batch_loads=True, seed=0, tile=None):
    geom = C.arm_geometry(nx=nx, ny=ny, nz=nz, h=h)
    fem = FEM3D(geom, C.PA12, mode=mode, tile=tile)
    F3 = C.arm_static_loads(geom)
    x0 = C.arm_design_start(geom, vf=vf, seed=seed).astype(np.float64)
    opt = SIMPOptimizer(geom, fem, load_cases=[], vol_frac=vf, r_min_mm=3.0 * h / 2e-3, move=0.2,
                        max_iter=50, tol_change=0.0, min_freq_Hz=min_freq_Hz, tip_mass_kg=C.TIP_MASS_KG,
                        n_modes_track=n_modes, mu_freq_init=0.2, mu_freq_max=50.0, mu_freq_ramp_every=5,
                        mu_freq_ramp_factor=1.5, batch_loads=batch_loads, solve_rtol=solve_rtol,
                        modal_tol=modal_tol, x0_design=x0, F_list=F3 + [np.zeros(geom.n_dofs)])
    rho0 = opt.physical_density()
    rho_active = rho0[torch.as_tensor(fem.active_ids, device=rho0.device)].cpu().numpy()
    Mr = consistent_mass_times_translation(fem, rho_active, C.TIP_MASS_KG, geom.motor_mount_top_nodes())
    opt.set_loads(F3 + [C.body_load_from_Mr(Mr, 3.0)])
    return geom, fem, opt


def consistent_mass_times_translation(fem, rho_active, tip_mass_kg, tip_nodes, direction=2):
    """M(rho) r for the unit translation r along `direction` on every DOF:
    the SIMP / Pedersen-scaled consistent element masses (src/fem.py:362-381)
    plus the lumped tip mass (src/fem.py:383-398), assembled on the host
    (set-up only).  Equal to the reference's assemble_M(...) @ r."""
    r_loc = np.zeros(24)
    r_loc[direction::3] = 1.0
    me_r = fem.Me_solid @ r_loc                                  # (24,)
    m = fem._mass_simp_factor(rho_active)
    out = np.zeros(fem.geom.n_dofs)
    np.add.at(out, fem.elem_dof_ids, m[:, None] * me_r[None, :])
    nodes = np.asarray(tip_nodes, dtype=np.int64)
    if tip_mass_kg and tip_mass_kg > 0.0 and len(nodes):
        np.add.at(out, 3 * nodes + direction, tip_mass_kg / len(nodes))
    return out


def arm_hollow_analysis(mode="mixed", tile=None):
    """The hollow-box arm (1-voxel walls at 1.0, core 1e-3), thrust load,
    60 g tip mass: (geom, fem, rho_active, F)."""
    geom = C.arm_geometry()
    fem = FEM3D(geom, C.PA12, mode=mode, tile=tile)
    return geom, fem, C.arm_hollow_density(geom), C.arm_static_loads(geom)[0]


SWEEP_VFS = (0.08, 0.10, 0.20, 0.30, 0.50)


def sweep_designs(vfs=SWEEP_VFS, fine=True, n_modes=8, tile="auto"):
    """The uneven design sweep: arm designs on the 2 mm grid (110 x 14 x 12)
    at the given volume fractions, plus (fine=True) one design on the 1 mm
    grid (220 x 28 x 24, ~480k DOF) at vf 0.08; each with the four load cases
    and the n_modes lowest modes.  Returns [(name, geom, fem, opt)] for
    tof_b200.batch.DesignSweep."""
    out = []
    for vf in vfs:
        geom, fem, opt = arm_simp(mode="mixed", vf=vf, n_modes=n_modes, tile=tile)
        out.append((f"2mm_vf{vf:.2f}", geom, fem, opt))
    if fine:
        geom, fem, opt = arm_simp(mode="mixed", nx=220, ny=28, nz=24, h=1e-3, vf=0.08, n_modes=n_modes, tile=tile)
        out.append(("1mm_vf0.08", geom, fem, opt))
    return out
