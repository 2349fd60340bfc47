"""The C-ABI library loads, exports every function include/mcv_gpu.h declares,
and refuses to run without a GPU (there is no CPU path).  No compute calls."""
import ctypes
import os
import re

import pytest

from mcv_sw_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(mcv_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_declares_core_api():
    names = declared_functions()
    for core in ("mcv_create", "mcv_set_geometry", "mcv_set_member", "mcv_step", "mcv_get_state",
                 "mcv_mass_energy", "mcv_destroy", "mcv_last_error"):
        assert core in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(api.lib_path())
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_argument_errors_are_reported():
    L = api.lib()
    h = ctypes.c_void_p()
    rc = L.mcv_create(5, 32, 3, 0, 100.0, 6.371e6, 1, ctypes.byref(h))
    assert rc == -1 and b"order" in L.mcv_last_error()
    assert L.mcv_footprint_bytes(4, 256, 3, 0, 1) > 0
    # checked before any device call
    for limit in (0.0, -1.0, 5000.0):
        with pytest.raises(api.MCVError) as e:
            api.selftest_wait(False, limit)
        assert e.value.code == -1
    assert L.mcv_set_geometry_equiangular(None) == -1
    assert L.mcv_set_member_balanced_flow(None, 0, 0., 0., 0., 0, None, 0., 0., 0., 0., 1.) == -1
    assert L.mcv_get_geometry(None, None, None, None, None, None, None, None) == -1


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback():
    with pytest.raises(api.MCVError) as e:
        api.Stepper(3, 8, 100.0)
    assert e.value.code == -2
