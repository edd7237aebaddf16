"""Oracle restatement of modal effective mass (sims/modal_participation.py) —
test infrastructure."""
from __future__ import annotations

import numpy as np

EXCITABLE_FRAC = 0.05           # sims/modal_participation.py:34


def effective_mass(fem, rho, modes, tip_mass_kg, tip_nodes, direction=2):
    """(phi^T M r)^2 / (phi^T M phi) / (r^T M r) over free DOFs, r = unit
    translation along `direction`: sims/modal_participation.py:37-57."""
    M = fem.reduce(fem.assemble_M(rho, tip_mass_kg, tip_nodes))
    r = np.zeros(fem.geom.n_dofs)
    r[direction::3] = 1.0
    fd = fem.free_dofs
    rf = r[fd]
    Mr = M @ rf
    total = float(rf @ Mr)
    out = []
    for k in range(modes.shape[1]):
        p = modes[fd, k]
        gm = float(p @ (M @ p))
        L = float(p @ Mr)
        out.append(L * L / max(gm, 1e-30) / total)
    return np.array(out)


def first_excitable(freqs, eff, thresh=EXCITABLE_FRAC):
    """sims/modal_participation.py:89-94."""
    for k, (f, e) in enumerate(zip(freqs, eff)):
        if e >= thresh:
            return float(f), float(e), k
    return None, None, None
