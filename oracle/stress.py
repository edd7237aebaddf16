"""Oracle (test infrastructure only): element stress and the fatigue field.

NumPy restatement of the reference's stress recovery (src/fem.py:153-176
`unit_element_B_at_centre`, src/fem.py:564-602 `compute_stress`,
`von_mises`, `principal_stress_max`) and its stress-life fatigue assessment
(src/fatigue.py:24-122).  Used only as the checker of the device kernels.
"""
from __future__ import annotations

import numpy as np

from .fem import LOCAL, shape

# PA12 SLS S-N curve at R = -1 (src/fatigue.py:20-21): cycles, alternating MPa
SN_CYCLES = np.array([1e2, 1e3, 1e4, 1e5, 1e6, 5e6, 1e7])
SN_ALT_MPA = np.array([45.0, 38.0, 28.0, 20.0, 13.0, 12.0, 12.0])


def B_centre(dx, dy, dz):
    """6 x 24 strain-displacement matrix at the element centre
    (src/fem.py:153-176); Voigt order exx, eyy, ezz, gxy, gyz, gxz."""
    _, dN = shape(0.0, 0.0, 0.0)
    dN = dN / (0.5 * np.array([dx, dy, dz]))[None, :]
    B = np.zeros((6, 24))
    for n in range(len(LOCAL)):
        i = 3 * n
        nx, ny, nz = dN[n]
        B[0, i], B[1, i + 1], B[2, i + 2] = nx, ny, nz
        B[3, i], B[3, i + 1] = ny, nx
        B[4, i + 1], B[4, i + 2] = nz, ny
        B[5, i], B[5, i + 2] = nz, nx
    return B


def compute_stress(u, elem_dof_ids, B, D, rho_active):
    """sigma_e = rho_e D B u_e, (n_active, 6) (src/fem.py:564-579)."""
    return rho_active[:, None] * ((u[elem_dof_ids] @ B.T) @ D.T)


def von_mises(s):
    """src/fem.py:582-589."""
    vm2 = 0.5 * ((s[..., 0] - s[..., 1]) ** 2 + (s[..., 1] - s[..., 2]) ** 2 + (s[..., 2] - s[..., 0]) ** 2) \
        + 3.0 * (s[..., 3] ** 2 + s[..., 4] ** 2 + s[..., 5] ** 2)
    return np.sqrt(np.maximum(vm2, 0.0))


def principal_stress_max(s):
    """Largest eigenvalue of the stress tensor per element (src/fem.py:592-602)."""
    T = np.zeros((s.shape[0], 3, 3))
    T[:, 0, 0], T[:, 1, 1], T[:, 2, 2] = s[:, 0], s[:, 1], s[:, 2]
    T[:, 0, 1] = T[:, 1, 0] = s[:, 3]
    T[:, 1, 2] = T[:, 2, 1] = s[:, 4]
    T[:, 0, 2] = T[:, 2, 0] = s[:, 5]
    return np.linalg.eigvalsh(T)[:, -1]


def sn_table():
    """(xp, fp) for the stress -> life interpolation of src/fatigue.py:38-56:
    log10 stress (MPa) increasing, ties nudged by 1e-12, and log10 cycles."""
    xp = np.log10(SN_ALT_MPA)[::-1].copy()
    fp = np.log10(SN_CYCLES)[::-1].copy()
    for i in range(1, len(xp)):
        if xp[i] <= xp[i - 1]:
            xp[i] = xp[i - 1] + 1e-12
    return xp, fp


def sn_life(s_eq_pa):
    """Cycles to failure at an equivalent fully reversed stress (src/fatigue.py:24-65)."""
    s = np.asarray(s_eq_pa, float) / 1e6
    xp, fp = sn_table()
    life = 10.0 ** np.interp(np.log10(np.where(s > 0, s, 1e-10)), xp, fp, left=fp[0], right=fp[-1])
    life = np.where(s < SN_ALT_MPA[-1] * 0.99, 1e9, life)
    return np.where(s > SN_ALT_MPA[0] * 1.5, 1.0, life)


def goodman(s_alt, s_mean, uts):
    """src/fatigue.py:68-80."""
    return s_alt / np.maximum(1.0 - np.maximum(s_mean, 0.0) / uts, 1e-6)


def sn_alt_stress_at(n):
    """Alternating stress (MPa) at n cycles (src/fatigue.py:115-121)."""
    return float(10.0 ** np.interp(np.log10(n), np.log10(SN_CYCLES), np.log10(SN_ALT_MPA)))


def fatigue_life_field(s1, s2, uts):
    """src/fatigue.py:83-112."""
    s1, s2 = np.asarray(s1, float), np.asarray(s2, float)
    peak, valley = np.maximum(s1, s2), np.minimum(s1, s2)
    mean, alt = 0.5 * (peak + valley), 0.5 * (peak - valley)
    eq = goodman(alt, mean, uts)
    life = sn_life(eq)
    return dict(sigma_mean=mean, sigma_alt=alt, sigma_alt_eq=eq, life=life,
                damage=1.0 / np.maximum(life, 1.0),
                factor_of_safety=sn_alt_stress_at(1e6) * 1e6 / np.maximum(eq, 1e-6))
