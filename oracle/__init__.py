"""CPU FP64 oracle for the voxel SIMP path — TEST INFRASTRUCTURE ONLY.

A NumPy/SciPy restatement of the reference's algorithm for the static solve,
modal solve, sensitivities, density filter, OC update and effective-mass
ranking (reference files src/fem.py, src/topopt.py,
sims/modal_participation.py; each function cites the lines it follows).

Only the test suite, `__graft_entry__.smoke()` and the CPU-baseline leg of
`bench.py` may import this package, and only as the checker or the timed CPU
baseline.  The product path (the `tof_b200` package and its CUDA library)
never imports, calls or falls back to it.

Parity pin: `tests/golden/make_golden.py` runs the reference itself (imported
from its source tree) on the same synthetic inputs and stores the outputs as
fixtures under `tests/golden/`; `tests/test_oracle_golden.py` checks this
oracle against those fixtures.
"""
