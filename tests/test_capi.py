"""CPU: the C-ABI library loads, exports every entry point include/xns_b200.h declares, and reports
the absence of a usable device instead of computing anything on the CPU."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "xns_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(xns_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header_symbols():
    import xns_b200
    lib = ctypes.CDLL(xns_b200.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings():
    import xns_b200
    for st in range(6):
        assert xns_b200.lib.xns_status_string(st)


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import xns_b200
    with pytest.raises(xns_b200.XnsError) as e:
        xns_b200.Context(0)
    assert e.value.status == 3  # XNS_ERR_NODEV


def test_rotation_matrix_matches_reference():
    """xns_rot_matrix (host code, no device) against calcRotMatrix's matrices for all 12 conventions."""
    import numpy as np

    import xns_b200
    from conftest import load_golden
    g = load_golden("rot__all")
    f = xns_b200.lib.xns_rot_matrix
    f.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_uint32, ctypes.POINTER(ctypes.c_double)]
    f.restype = None
    eul = (ctypes.c_double * 3)(*[float(v) for v in g["euler"]])
    for c in range(12):
        m = (ctypes.c_double * 9)()
        f(eul, c, m)
        assert np.allclose(np.array(m[:]).reshape(3, 3), np.asarray(g["m"][c]).reshape(3, 3), rtol=0, atol=1e-15), c
