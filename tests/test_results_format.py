"""Result pickles keep the reference's layout (sims/run_freq_gpu.py:224-240)."""
import os
import pickle
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "to-f450-arm_b200"))


def test_payload_layout_and_name(tmp_path):
    from tof_b200.results import payload_name, save_result
    assert payload_name(0.08, 500.0) == "freq_vf08_omega0500.pkl"
    path = save_result(str(tmp_path), 0.08, 500.0, rho=np.ones(4), static={"compliance": 1.0},
                       fatigue={"life": np.ones(4)}, frequencies_Hz=[1.0, 2.0], mode_shapes=np.zeros((6, 2)),
                       omega_sq=[39.5, 158.0], tip_mass_kg=0.06, history={"compliance": [1.0]},
                       record={"vf": 0.08})
    d = pickle.load(open(path, "rb"))
    assert set(d) == {"rho", "static", "fatigue", "modal", "history", "record"}
    assert set(d["modal"]) == {"frequencies_Hz", "mode_shapes", "omega_sq", "tip_mass_kg"}
    assert d["modal"]["tip_mass_kg"] == 0.06 and d["modal"]["mode_shapes"].shape == (6, 2)
