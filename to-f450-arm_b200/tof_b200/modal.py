"""Modal effective mass in the thrust direction (sims/modal_participation.py).

`effective_mass_voxel` has the reference's signature
(sims/modal_participation.py:37) and computes
(phi^T M r)^2 / (phi^T M phi) / (r^T M r) with the same consistent mass and
tip lump the eigensolve used, on the device (one block M product and one Gram
matrix).
"""
from __future__ import annotations

import numpy as np
import torch

EXCITABLE_FRAC = 0.05          # sims/modal_participation.py:34


def effective_mass_voxel(fem, geom, rho_active, mode_shapes, tip_mass_kg, direction=2):
    """Effective-mass fraction per mode (sims/modal_participation.py:37-57).
    `fem` is a tof_b200.fem.FEM3D; mode_shapes is (N, m)."""
    nodes = geom.motor_mount_top_nodes()
    ctx = fem._prepare(rho_active, tip_mass_kg, nodes)
    modes = np.asarray(mode_shapes, dtype=np.float64)
    m4 = ctx.pack(torch.from_numpy(np.ascontiguousarray(modes.T)))
    return ctx.effective_mass(m4, direction)


def first_excitable(freqs, eff, thresh=EXCITABLE_FRAC):
    """(frequency, effective-mass fraction, index) of the lowest excitable mode
    (sims/modal_participation.py:89-94)."""
    for k, (f, e) in enumerate(zip(freqs, eff)):
        if e >= thresh:
            return float(f), float(e), k
    return None, None, None


def rank_by_effective_mass(freqs, eff):
    """Mode indices ordered by effective mass, largest first."""
    return list(np.argsort(-np.asarray(eff), kind="stable"))
