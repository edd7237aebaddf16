"""The production arm domain (the reference's ArmGeometry3D, src/mesh3d.py)
built with array operations reproduces the reference's masks, clamped and
tip-mass node sets (same order) and load vectors exactly
(tests/golden/arm3d.npz, written by the reference itself)."""
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "to-f450-arm_b200"))


def test_production_domain_matches_reference(golden):
    from tof_b200.geometry3d import ArmGeometry3D
    d = golden("arm3d")
    t0 = time.perf_counter()
    g = ArmGeometry3D()
    m = g.build_masks()
    fixed = g.fixed_nodes()
    motor = g.motor_mount_top_nodes()
    elapsed = time.perf_counter() - t0
    assert (g.nx, g.ny, g.nz) == (108, 21, 27)
    for k in ("in_arm", "design", "keep_solid", "keep_screw", "keep_motor"):
        assert np.array_equal(m[k], d[k]), k
    assert np.array_equal(fixed, d["fixed_nodes"])
    assert np.array_equal(motor, d["motor_nodes"])
    for tag, F in (("thrust", (0.0, 0.0, -15.0)), ("inplane", (3.0, -4.0, 2.0))):
        dofs, vals = g.load_dofs_for_force(F)
        assert np.array_equal(dofs, d[f"{tag}_dofs"]) and np.array_equal(vals, d[f"{tag}_vals"]), tag
    dofs, vals = g.load_dofs_for_moment_Mz(0.3)
    assert np.array_equal(dofs, d["mz_dofs"]) and np.array_equal(vals, d["mz_vals"])
    assert elapsed < 2.0                      # array builders; the reference's node loops take seconds


def test_load_vector_sums_to_applied_force():
    from tof_b200.geometry3d import ArmGeometry3D
    g = ArmGeometry3D()
    F = g.load_vector(F=(3.0, -4.0, 2.0))
    assert np.isclose(F[0::3].sum(), 3.0) and np.isclose(F[1::3].sum(), -4.0) and np.isclose(F[2::3].sum(), 2.0)
