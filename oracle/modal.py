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


def modal_frf_at_dof(frequencies_Hz, mode_shapes, dof_idx, freq_range_Hz=(10.0, 1500.0), n_pts=600,
                     modal_damping=0.02):
    """|H_dd(f)| = |sum_k v_k[d]^2 / ((w_k^2 - w^2) + 2 i zeta w_k w)| on a
    geometric frequency grid (src/plotting.py:378-399)."""
    f = np.geomspace(freq_range_Hz[0], freq_range_Hz[1], n_pts)
    w = 2.0 * np.pi * f
    wk = 2.0 * np.pi * np.asarray(frequencies_Hz)
    v = np.asarray(mode_shapes)[dof_idx, :]
    H = np.zeros(n_pts, dtype=complex)
    for k in range(len(wk)):
        H += v[k] ** 2 / (wk[k] ** 2 - w ** 2 + 2j * modal_damping * wk[k] * w)
    return f, np.abs(H)
