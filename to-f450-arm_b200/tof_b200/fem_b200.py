"""Drop-in patch of the reference's `FEM3D` (the counterpart of
src/fem_gpu.py:176-228, `enable_gpu_solver`).

    from tof_b200.fem_b200 import enable_b200_solver
    enable_b200_solver(FEM3D_class, topopt_module)   # returns True if patched

Patches `solve`, `apply_BCs_and_solve`, `modal_analysis`,
`eigenvalue_sensitivity`, `elem_compliance` of the given class and
`filter_field` of the given topopt module, so the reference's own callers
(`SIMPOptimizer.run`, the sweep runners) run their hot path on the B200.
Each patched instance lazily builds a `tof_b200.fem.FEM3D` twin from its own
geometry, material and (possibly overwritten) Ke_solid / Me_solid.  Unlike
the reference's patch there is no silent CPU fallback: errors propagate.
"""
from __future__ import annotations

import numpy as np

from . import topopt as _topopt
from .fem import FEM3D as _DeviceFEM3D


def gpu_available() -> bool:
    try:
        import torch
        from . import _lib
        _lib.load()
        return torch.cuda.is_available()
    except Exception:
        return False


def _twin(self, mode):
    t = getattr(self, "_b200_twin", None)
    if t is None:
        t = _DeviceFEM3D(self.geom, self.mat, mode=mode)
        self._b200_twin = t
    # the reference allows overwriting the element templates (run_parallel.py)
    t.Ke_solid = np.asarray(self.Ke_solid)
    t.Me_solid = np.asarray(self.Me_solid)
    t.fixed_dofs, t.free_dofs = self.fixed_dofs, self.free_dofs
    return t


def enable_b200_solver(fem_cls=None, topopt_module=None, force: bool = False, mode: str = "fp64") -> bool:
    """Route the reference FEM3D hot path through libtof.  `fem_cls` defaults
    to `src.fem.FEM3D` when that package is importable."""
    if not (gpu_available() or force):
        return False
    if fem_cls is None:
        from src.fem import FEM3D as fem_cls          # the reference package
    if topopt_module is None:
        try:
            import src.topopt as topopt_module
        except ImportError:
            topopt_module = None

    def solve(self, rho_active, F, method="cg", x0=None):
        t = _twin(self, mode)
        u, = t.solve_block(rho_active, [F], [x0], rtol=t.LU_RTOL if method == "lu" else t.SOLVE_RTOL)[0]
        return u

    def apply_BCs_and_solve(self, K, F, method="cg", x0=None, rtol=1e-5):
        rho = getattr(K, "rho", None)
        if rho is None:
            raise TypeError("with the B200 solver enabled, pass the density through FEM3D.solve; "
                            "an assembled CSR matrix cannot be solved on this path")
        t = _twin(self, mode)
        u, = t.solve_block(rho, [F], [x0], rtol=t.LU_RTOL if method == "lu" else rtol)[0]
        return u

    def modal_analysis(self, rho_active, n_modes=6, tip_mass_kg=0.060, tip_mass_nodes=None, X0_free=None,
                       tol=1e-4, maxiter=500):
        return _twin(self, mode).modal_analysis(rho_active, n_modes, tip_mass_kg, tip_mass_nodes, X0_free, tol,
                                                maxiter)

    def eigenvalue_sensitivity(self, rho_active, omega_sq_k, v_k, tip_mass_kg=0.060, tip_mass_nodes=None):
        return _twin(self, mode).eigenvalue_sensitivity(rho_active, omega_sq_k, v_k, tip_mass_kg, tip_mass_nodes)

    def elem_compliance(self, u, rho_active=None):
        return _twin(self, mode).elem_compliance(u, rho_active)

    fem_cls.solve = solve
    fem_cls.apply_BCs_and_solve = apply_BCs_and_solve
    fem_cls.modal_analysis = modal_analysis
    fem_cls.eigenvalue_sensitivity = eigenvalue_sensitivity
    fem_cls.elem_compliance = elem_compliance
    if topopt_module is not None:
        topopt_module.filter_field = _topopt.filter_field
    return True
