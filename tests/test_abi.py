"""The C ABI library: it loads, exports every entry point include/srk_b200.h
declares, and rejects bad arguments before touching the device.  CPU only —
no compute call is made."""
import ctypes
import os
import re

import pytest

import shrinkage_full_tests_b200 as srk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:srk_status|int|const char\*)\s+(srk_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = srk.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    assert set(declared_functions()) <= set(srk._SIGS)


def test_status_strings():
    L = srk.lib()
    assert L.srk_status_string(0) == b"SRK_OK"
    assert L.srk_status_string(1) == b"SRK_ERR_INVALID_ARG"
    assert L.srk_version() >= 100


@pytest.mark.parametrize("args", [
    (256, 200, 15, 1.0, 1, 256),     # W != N - 2e
    (256, 226, 15, 1.0, 0, 256),     # B_max < 1
    (256, 226, 15, -1.0, 1, 256),    # dx <= 0
    (256, 226, 15, 1.0, 1, 255),     # odd spectra size
    (2, 2, 0, 1.0, 1, 2),            # N too small
])
def test_plan_create_rejects_bad_sizes(args):
    with pytest.raises(srk.SrkError) as ei:
        srk.SrkPlan(*args)
    assert ei.value.status == srk.SRK_ERR_INVALID_ARG


def test_plan_create_rejects_unbuilt_tile_and_dtype():
    with pytest.raises(srk.SrkError) as ei:
        srk.SrkPlan(256, 226, 15, 1.0, 1, 256, tile_M=1024)
    assert ei.value.status == srk.SRK_ERR_INVALID_ARG
    with pytest.raises(srk.SrkError) as ei:
        srk.SrkPlan(256, 226, 15, 1.0, 1, 256, dtype=7)
    assert ei.value.status == srk.SRK_ERR_INVALID_ARG
    with pytest.raises(srk.SrkError) as ei:  # erosion too large for any tile
        srk.SrkPlan(2048, 2048 - 2 * 300, 300, 1.0, 1, 2048)
    assert ei.value.status == srk.SRK_ERR_UNSUPPORTED


def test_operators_reject_null_plan_without_device_work():
    L = srk.lib()
    st = L.srk_training_forward(None, None, None, None, 256, 226, 15, 1.0, 1, None, None, None)
    assert st == srk.SRK_ERR_INVALID_ARG
    assert b"plan" in L.srk_last_error()
    assert L.srk_vjp(None, None, None, 1, None, None, None, None) == srk.SRK_ERR_INVALID_ARG
    assert L.srk_green_tensor(None, None, 31, 0.1, 10.0, 1.0, None) == srk.SRK_ERR_INVALID_ARG
    assert L.srk_precompute_kernel_freq(None, 31, 64, None, None) == srk.SRK_ERR_INVALID_ARG
