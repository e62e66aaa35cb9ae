"""The C-ABI library loads, exports every entry point include/amls_b200.h
declares, and its host-only paths behave (no GPU work is launched here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from amls_b200 import _lib, cases, recursive_bisection

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "amls_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(amls_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = header_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(L, name), f"{name} not exported"
    assert set(names) == set(_lib.EXPORTS)


def test_options_default_match_reference():
    o = _lib.Options()
    assert _lib.lib().amls_options_default(C.byref(o)) == 0
    # AmlsOptions defaults (src/amls/solver.hpp:18-30)
    assert (o.nLevels, o.leafSize, o.thresholdFactor, o.fixedKeep, o.nev) == (6, 500, 2.0, 0, 100)
    assert (o.denseProjectedMax, o.shift, o.twoPass, o.recoverVectors) == (5000, 0.0, 1, 1)


def test_partition_error_paths():
    p = cases.path_graph(10)
    with pytest.raises(ValueError):
        recursive_bisection(p.K[:0, :0], p.M[:0, :0], 2, 4)


def test_create_without_device_reports_status():
    """On a machine without a GPU amls_create fails with a status code (no
    crash, no fallback)."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = _lib.lib().amls_create(0, C.byref(h))
    assert rc == _lib.AMLS_ERR_NO_DEVICE
    assert b"device" in _lib.lib().amls_last_error()


def test_null_arguments_rejected():
    L = _lib.lib()
    assert L.amls_solve(None, 0, None, None, None, None, None, None, None, None, None, None,
                        None) == _lib.AMLS_ERR_INVALID_ARGUMENT
    assert L.amls_info(None, None) == _lib.AMLS_ERR_INVALID_ARGUMENT
    assert L.amls_options_default(None) == _lib.AMLS_ERR_INVALID_ARGUMENT
