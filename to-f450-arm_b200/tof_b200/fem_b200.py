"""Drop-in patch of the reference's `FEM3D` (the counterpart of
src/fem_gpu.py:176-228, `enable_gpu_solver`).

    from tof_b200.fem_b200 import enable_b200_solver
    enable_b200_solver(FEM3D_class, topopt_module)   # returns True if patched

Patches `solve`, `apply_BCs_and_solve`, `assemble_K`, `modal_analysis`,
`eigenvalue_sensitivity`, `elem_compliance` of the given class and
`filter_field` of the given topopt module, so the reference's own callers
(`SIMPOptimizer.run`, the sweep runners, the `python -m src.fem` self-test)
run their hot path on the B200.  Each patched instance lazily builds a
`tof_b200.fem.FEM3D` twin per solver form from its own geometry, material and
(possibly overwritten) Ke_solid / Me_solid.  Unlike the reference's patch
there is no silent CPU fallback: errors propagate.

The reference's plug-in point is `apply_BCs_and_solve(K, F, ...)` with an
assembled CSR K (src/fem.py:529-555, patched by src/fem_gpu.py:190-200).
Here `assemble_K` still returns the reference's own CSR (its original code),
tagged with the density it was built from and a checksum of its values; the
patched `apply_BCs_and_solve` solves that K matrix-free on the device.  A
CSR that carries no tag, or whose values changed after assembly, is
rejected with a TypeError (the matrix-free path has no way to read it).

Tolerances: `solve` uses the reference's default relative residual (1e-5,
src/fem.py:532) unless `enable_b200_solver(..., rtol=...)` sets another;
`modal_analysis` tightens the LOBPCG tolerance to at most 1e-5 and raises
its iteration cap to at least 1000 (multigrid) / 6000 (Jacobi), see
`tof_b200.fem.FEM3D.modal_analysis`: the reference's defaults (1e-4, 500)
leave f1 up to 16 % off on the production domain.
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


def _twin(self, mode, rtol=None):
    twins = self.__dict__.setdefault("_b200_twins", {})
    t = twins.get(mode)
    if t is None:
        t = twins[mode] = _DeviceFEM3D(self.geom, self.mat, mode=mode)
    if rtol is not None:
        t.SOLVE_RTOL = rtol
    # the reference allows overwriting the element templates (run_parallel.py)
    t.Ke_solid = np.asarray(self.Ke_solid)
    t.Me_solid = np.asarray(self.Me_solid)
    t.fixed_dofs, t.free_dofs = self.fixed_dofs, self.free_dofs
    return t


def _csr_tag(K):
    d = np.asarray(K.data)
    return (K.shape, int(K.nnz), float(d.sum()), float(np.abs(d).sum()))


def enable_b200_solver(fem_cls=None, topopt_module=None, force: bool = False, mode: str = "fp64",
                       rtol: float = None) -> bool:
    """Route the reference FEM3D hot path through libtof.  `fem_cls` defaults
    to `src.fem.FEM3D` when that package is importable.  `rtol` overrides
    the static-solve tolerance of `solve` (default: the reference's 1e-5).
    Returns True when patched; `disable_b200_solver` undoes it."""
    if not (gpu_available() or force):
        return False
    if fem_cls is None:
        from src.fem import FEM3D as fem_cls          # the reference package
    if topopt_module is None:
        try:
            import src.topopt as topopt_module
        except ImportError:
            topopt_module = None

    originals = {k: fem_cls.__dict__.get(k) for k in
                 ("solve", "apply_BCs_and_solve", "assemble_K", "modal_analysis", "eigenvalue_sensitivity",
                  "elem_compliance")}
    orig_assemble_K = getattr(fem_cls, "assemble_K", None)

    def solve(self, rho_active, F, method="cg", x0=None):
        t = _twin(self, mode, rtol)
        u, = t.solve_block(rho_active, [F], [x0], rtol=t.LU_RTOL if method == "lu" else t.SOLVE_RTOL)[0]
        return u

    def assemble_K(self, rho_active):
        K = orig_assemble_K(self, rho_active)               # the reference's own CSR
        K._b200_rho = np.array(rho_active, dtype=np.float64, copy=True)
        K._b200_tag = _csr_tag(K)
        return K

    def apply_BCs_and_solve(self, K, F, method="cg", x0=None, rtol=1e-5):
        rho = getattr(K, "rho", None)                       # a tof_b200 operator handle
        if rho is None and getattr(K, "_b200_rho", None) is not None:
            if _csr_tag(K) != K._b200_tag:
                raise TypeError("apply_BCs_and_solve: this CSR changed after assemble_K built it; the B200 "
                                "path solves the matrix-free operator of the density it was assembled from")
            rho = K._b200_rho
        if rho is None:
            raise TypeError("apply_BCs_and_solve: with the B200 solver enabled, K must come from "
                            "assemble_K (or pass the density to FEM3D.solve); an arbitrary assembled CSR "
                            "cannot be solved on the matrix-free path")
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

    fem_cls._b200_originals = originals
    fem_cls.solve = solve
    if orig_assemble_K is not None:
        fem_cls.assemble_K = assemble_K
    fem_cls.apply_BCs_and_solve = apply_BCs_and_solve
    fem_cls.modal_analysis = modal_analysis
    fem_cls.eigenvalue_sensitivity = eigenvalue_sensitivity
    fem_cls.elem_compliance = elem_compliance
    if topopt_module is not None:
        fem_cls._b200_topopt = (topopt_module, topopt_module.filter_field)
        topopt_module.filter_field = _topopt.filter_field
    return True


def disable_b200_solver(fem_cls) -> None:
    """Undo `enable_b200_solver` on fem_cls (and its topopt module)."""
    orig = fem_cls.__dict__.get("_b200_originals")
    if orig is None:
        return
    for k, v in orig.items():
        if v is None:
            if k in fem_cls.__dict__:
                delattr(fem_cls, k)
        else:
            setattr(fem_cls, k, v)
    del fem_cls._b200_originals
    top = fem_cls.__dict__.get("_b200_topopt")
    if top is not None:
        top[0].filter_field = top[1]
        del fem_cls._b200_topopt
