"""Stress-life fatigue with the Goodman mean-stress correction, on the GPU.

Mirrors src/fatigue.py: `sn_life`, `equivalent_alt_stress_goodman`,
`fatigue_life_field`, `sn_alt_stress_at` and the PA12 SLS S-N table.  The
element-wise arithmetic runs in libtof (`tof_fatigue`, `tof_sn_life`); the
scalar table lookup `sn_alt_stress_at` stays on the host.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from .engine import _stream

# PA12 SLS at R = -1 (src/fatigue.py:20-21): cycles, alternating stress (MPa)
SN_CYCLES = np.array([1e2, 1e3, 1e4, 1e5, 1e6, 5e6, 1e7], dtype=float)
SN_ALT_MPA = np.array([45.0, 38.0, 28.0, 20.0, 13.0, 12.0, 12.0], dtype=float)


def _dev(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64), device=torch.device("cuda", torch.cuda.current_device()))


def sn_alt_stress_at(N: float) -> float:
    """Alternating stress (MPa) at N cycles (src/fatigue.py:115-121)."""
    return float(10.0 ** np.interp(np.log10(N), np.log10(SN_CYCLES), np.log10(SN_ALT_MPA),
                                   left=np.log10(SN_ALT_MPA)[0], right=np.log10(SN_ALT_MPA)[-1]))


def sn_life(sigma_alt_eq_Pa) -> np.ndarray:
    """Cycles to failure at equivalent fully reversed stresses (src/fatigue.py:24-65)."""
    s = _dev(sigma_alt_eq_Pa).reshape(-1).contiguous()
    life = torch.empty_like(s)
    L.check("tof_sn_life", L.load().tof_sn_life(s.numel(), L.ptr(s), L.ptr(life), _stream()))
    return life.cpu().numpy().reshape(np.shape(sigma_alt_eq_Pa))


def equivalent_alt_stress_goodman(sigma_alt, sigma_mean, sigma_uts_Pa: float) -> np.ndarray:
    """sigma_a / (1 - max(sigma_m, 0) / sigma_uts), denominator floored at 1e-6
    (src/fatigue.py:68-80)."""
    sm = np.maximum(np.asarray(sigma_mean, float), 0.0)
    return np.asarray(sigma_alt, float) / np.maximum(1.0 - sm / sigma_uts_Pa, 1e-6)


def fatigue_life_field(stress_lc1, stress_lc2, sigma_uts_Pa: float) -> dict:
    """Per-element fatigue of the cycle between two von Mises stress fields
    (Pa) (src/fatigue.py:83-112); the same keys as the reference's result."""
    s1 = _dev(stress_lc1).reshape(-1).contiguous()
    s2 = _dev(stress_lc2).reshape(-1).contiguous()
    n = s1.numel()
    out = torch.empty((6, n), dtype=torch.float64, device=s1.device)
    L.check("tof_fatigue", L.load().tof_fatigue(n, L.ptr(s1), L.ptr(s2), float(sigma_uts_Pa),
                                               sn_alt_stress_at(1e6) * 1e6, L.ptr(out), _stream()))
    o = out.cpu().numpy()
    keys = ("sigma_mean", "sigma_alt", "sigma_alt_eq", "life", "damage", "factor_of_safety")
    return {k: o[i] for i, k in enumerate(keys)}
