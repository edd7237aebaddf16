"""Result payloads in the reference's pickle layout (sims/run_freq_gpu.py:224-240).

The reference's consolidation reads one pickle per (volume fraction, frequency
target) run; `result_payload` builds the same dictionary from this package's
outputs and `save_result` writes it under the reference's file name.
"""
from __future__ import annotations

import os
import pickle

import numpy as np


def payload_name(vol_frac: float, omega_target_Hz: float) -> str:
    """freq_vfXX_omegaYYYY.pkl (sims/run_freq_gpu.py:224-227)."""
    return f"freq_vf{int(vol_frac * 100):02d}_omega{int(omega_target_Hz):04d}.pkl"


def result_payload(rho, static, fatigue, frequencies_Hz, mode_shapes, omega_sq, tip_mass_kg, history,
                   record) -> dict:
    """The reference's result dictionary: rho, static, fatigue, modal
    {frequencies_Hz, mode_shapes, omega_sq, tip_mass_kg}, history, record."""
    return dict(rho=np.asarray(rho), static=static, fatigue=fatigue,
                modal=dict(frequencies_Hz=np.asarray(frequencies_Hz), mode_shapes=np.asarray(mode_shapes),
                           omega_sq=np.asarray(omega_sq), tip_mass_kg=float(tip_mass_kg)),
                history=history, record=record)


def save_result(results_dir: str, vol_frac: float, omega_target_Hz: float, **payload) -> str:
    """Write result_payload(**payload) to results_dir/payload_name(...)."""
    path = os.path.join(results_dir, payload_name(vol_frac, omega_target_Hz))
    with open(path, "wb") as f:
        pickle.dump(result_payload(**payload), f)
    return path
