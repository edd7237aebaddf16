"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(tof_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert {"tof_ctx_create", "tof_pcg", "tof_lobpcg", "tof_matvec", "tof_filter_apply",
            "tof_oc_update", "tof_effective_mass", "tof_elem_quadform"} <= names


def test_library_exports_every_declared_symbol():
    from tof_b200 import _lib as L
    assert os.path.exists(L.LIB_PATH), "libtof.so not built"
    lib = ctypes.CDLL(L.LIB_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert declared_functions() == set(L.SIGNATURES)
    assert lib.tof_version() >= 100


def test_binding_load_sets_signatures():
    from tof_b200 import _lib as L
    lib = L.load()
    assert lib.tof_ctx_create.restype is ctypes.c_int
    assert lib.tof_last_error(None) is not None or True


def test_create_rejects_invalid_arguments_with_a_message():
    """Argument errors are reported before any CUDA call, through
    tof_last_error(NULL) (the calling thread's last create error)."""
    from tof_b200 import _lib as L
    lib = L.load()
    h = ctypes.c_void_p()
    Ke = (ctypes.c_double * 576)()
    fixed = (ctypes.c_uint8 * 8)()
    rc = lib.tof_ctx_create(0, 1, 1, None, Ke, Ke, None, fixed, None, None, 1, 1, None, ctypes.byref(h))
    assert rc == L.TOF_ERR_ARG
    msg = lib.tof_last_error(None)
    msg = msg.decode() if isinstance(msg, bytes) else msg
    assert "invalid argument" in msg
