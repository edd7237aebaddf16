"""ctypes binding of libtof.so (the C ABI declared in include/tof.h).

The library is the only compute path: if it is missing or fails to load, every
call raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_longlong, c_uint8, c_void_p

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libtof.so")

TOF_OK, TOF_NOT_CONVERGED = 0, 1
TOF_ERR_ARG, TOF_ERR_CUDA, TOF_ERR_BREAKDOWN, TOF_ERR_NONFINITE, TOF_ERR_TIMEOUT = -1, -2, -3, -4, -5
OP_K, OP_M = 0, 1
F32, F64 = 0, 1
MODE_FP64, MODE_MIXED, MODE_IR = 0, 1, 2
PRECOND_JACOBI, PRECOND_PCG, PRECOND_MG = 0, 1, 2
FILTER_FORWARD, FILTER_ADJOINT, FILTER_PHYSICAL = 0, 1, 2
Q_NODES, Q_ELEMS, Q_FREE_DOFS, Q_TILE_X, Q_TILE_Y, Q_TILE_Z, Q_DEVICE_BYTES, Q_MAX_RHS, Q_MAX_MODES = range(9)

STATUS_NAMES = {0: "ok", 1: "not converged", -1: "invalid argument", -2: "CUDA error", -3: "breakdown",
                -4: "non-finite values", -5: "wait budget expired"}


class SolveStats(ctypes.Structure):
    _fields_ = [("status", c_int), ("iters", c_int), ("outer", c_int), ("relres", c_double), ("floor", c_double)]


class KernelTiming(ctypes.Structure):
    _fields_ = [("us", c_double), ("bytes", c_double), ("flops", c_double), ("units", c_longlong)]


KERNEL_MATVEC_F32, KERNEL_MG_LEVEL_OP, KERNEL_RAYLEIGH_RITZ, KERNEL_VCYCLE = range(4)


class SimpParams(ctypes.Structure):
    _fields_ = [("penal", c_double), ("emin", c_double), ("mass_threshold", c_double), ("mass_q", c_double)]


class SolverError(RuntimeError):
    """A libtof call returned an error status."""

    def __init__(self, func, code, msg=""):
        self.code = code
        super().__init__(f"{func}: {STATUS_NAMES.get(code, code)} ({code}) {msg}".strip())


P = c_void_p
# name -> (restype, argtypes); the complete list of exported entry points
SIGNATURES = {
    "tof_version": (c_int, []),
    "tof_launch_count": (c_longlong, []),
    "tof_last_error": (ctypes.c_char_p, [P]),
    "tof_ctx_create": (c_int, [c_int, c_int, c_int, POINTER(c_double), POINTER(c_double), POINTER(c_double),
                               POINTER(c_uint8), POINTER(c_uint8), POINTER(c_double), POINTER(SimpParams),
                               c_int, c_int, POINTER(c_int), POINTER(P)]),
    "tof_ctx_destroy": (None, [P]),
    "tof_ctx_query": (c_longlong, [P, c_int]),
    "tof_ctx_set_wait_limit": (c_int, [P, c_longlong]),
    "tof_wait_selftest": (c_int, [P, c_int, P]),
    "tof_set_density": (c_int, [P, P, P]),
    "tof_set_tip_lump": (c_int, [P, POINTER(c_double), P]),
    "tof_pack": (c_int, [P, P, c_longlong, P, c_int, c_int, P]),
    "tof_unpack": (c_int, [P, P, c_int, P, c_longlong, c_int, P]),
    "tof_matvec": (c_int, [P, c_int, c_int, P, P, c_int, P]),
    "tof_diag": (c_int, [P, c_int, P, P]),
    "tof_pcg": (c_int, [P, c_int, P, P, c_int, c_double, c_int, POINTER(SolveStats), P]),
    "tof_lobpcg": (c_int, [P, c_int, c_int, c_int, P, POINTER(c_double), c_double, c_int, c_int, c_int, c_double,
                           POINTER(SolveStats), POINTER(c_double), P]),
    "tof_elem_quadform": (c_int, [P, c_int, c_int, P, c_int, P, P]),
    "tof_gram": (c_int, [P, c_int, P, c_int, P, c_int, P, P]),
    "tof_gram_noalloc": (c_int, [c_longlong, c_int, P, c_int, P, c_int, P, P]),
    "tof_compliance_sens": (c_int, [P, c_int, P, P, P, P, P]),
    "tof_eig_sens": (c_int, [P, P, P, c_double, c_double, P, P]),
    "tof_effective_mass": (c_int, [P, P, c_int, c_int, POINTER(c_double), P]),
    "tof_stress": (c_int, [P, POINTER(c_double), POINTER(c_double), c_int, P, c_int, P, P, P, P, P]),
    "tof_stress_invariants": (c_int, [c_longlong, P, P, P, P]),
    "tof_fatigue": (c_int, [c_longlong, P, P, c_double, c_double, P, P]),
    "tof_sn_life": (c_int, [c_longlong, P, P, P]),
    "tof_modal_frf": (c_int, [c_longlong, c_int, P, P, c_longlong, P, c_double, P, P]),
    "tof_filter_create": (c_int, [c_int, c_int, c_int, POINTER(c_double), c_int, c_int, c_int, POINTER(c_uint8),
                                  POINTER(c_uint8), POINTER(P)]),
    "tof_filter_apply": (c_int, [P, c_int, P, P, P]),
    "tof_filter_destroy": (None, [P]),
    "tof_oc_update": (c_int, [c_int, P, P, c_double, c_double, c_double, P, P, P]),
    "tof_mg_query": (c_int, [P, c_int, POINTER(c_int), POINTER(ctypes.c_float), P]),
    "tof_mg_export": (c_int, [P, c_int, P, P]),
    "tof_mg_apply": (c_int, [P, P, P, c_int, P]),
    "tof_mg_setup": (c_int, [P, P]),
    "tof_time_kernel": (c_int, [P, c_int, c_int, c_int, c_int, POINTER(KernelTiming), P]),
}

_lib = None


def load():
    """Load libtof.so once; raises if it is absent (build it with build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libtof.so not built ({LIB_PATH}); run __graft_entry__.build() "
                           f"or python to-f450-arm_b200/build.py")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(func, code, ctx=None, allow=(TOF_OK,)):
    if code in allow:
        return code
    lib = load()
    msg = lib.tof_last_error(ctx)
    raise SolverError(func, code, msg.decode() if msg else "")


def ptr(t):
    """Raw device (or host) address of a torch tensor / numpy array."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return c_void_p(t.data_ptr())
    return t.ctypes.data_as(c_void_p)


def dptr(a):
    """POINTER(c_double) to a contiguous float64 numpy array."""
    return a.ctypes.data_as(POINTER(c_double))
