"""The C ABI library loads without a GPU and exports every function include/thorx.h declares."""
import ctypes
import os
import re

import thor_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "thorx.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(thorx_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_python_exports():
    assert set(thor_b200.EXPORTED) <= set(declared_functions())


def test_library_exports_every_declared_function():
    lib = ctypes.CDLL(thor_b200.LIB_PATH)
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_null_arguments_are_rejected_without_a_gpu():
    L = thor_b200.lib()
    h = ctypes.c_void_p()
    assert L.thorx_create(None, None, None, ctypes.byref(h)) == -1
    assert L.thorx_field_size(None, b"Rho") == -1
    assert L.thorx_step(None, 1) == -1
    L.thorx_destroy(h.value)
