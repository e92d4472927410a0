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


def test_unsupported_sizes_and_options_are_rejected_before_device_work():
    """thorx_create checks its arguments before any CUDA call, so this runs without a GPU."""
    import pytest
    from thorx_testlib import EARTH, thorx_params
    for nv, over, code in ((129, {}, -4), (8, dict(HyDiffOrder=3), -4),
                           (8, dict(precision=5), -1), (8, dict(core_benchmark=9), -4)):
        g = thor_b200.Icogrid(4, nv)
        p = thorx_params(dict(EARTH), 600.0)
        p.update(over)
        with pytest.raises(thor_b200.ThorxError) as e:
            thor_b200.Thorx(g.as_dict(), 4, p)
        assert e.value.code == code, (nv, over, e.value)
