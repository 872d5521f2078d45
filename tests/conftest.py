import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "softx-d-16-00083_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU; run with -m gpu")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def golden_names(prefix):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "__*.npz")))


def split_elements(xyz, n_el):
    out, o = [], 0
    for n in n_el:
        out.append(xyz[o:o + int(n)])
        o += int(n)
    return out


def rel_err(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def rel_err_floor(a, b, floor_frac):
    """Max relative error with the denominator floored at floor_frac * median|b|: near-zero points of an
    interference pattern (|A|^2 of a sum of N unit phasors that nearly cancel) carry the absolute
    error of the phasor sum, not a relative one."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    floor = floor_frac * float(np.median(np.abs(b)))
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def gpu_ctx():
    import xns_b200
    ctx = xns_b200.Context(0)
    yield ctx
    ctx.close()
