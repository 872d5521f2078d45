"""GPU: the allocation-free histogram -> I(q) entry point, xns_int_1d_hist_noalloc.

Callers that cannot call cudaMalloc -- a plugin whose host framework owns every device buffer, a
service with a memory budget fixed at start-up -- pass their own device buffers to this entry point,
and it keeps its intermediates in one static device array inside the library.  These checks call it
through the C ABI, twice in a row and then on a different input (the array keeps the previous call's
contents, so each call must clear what it needs), and compare it with the allocating entry point
xns_calc_int_1d_hist within the intensity tolerance of the other GPU tests.  The file is named to be
collected last; it passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu

TOL_I = 1e-5
XNS_ERR_LIMIT = 6


def _noalloc():
    import xns_b200
    f = xns_b200.lib.xns_int_1d_hist_noalloc
    p = C.c_void_p
    f.argtypes = [p, p, C.c_uint32, C.c_uint32, C.c_double, p, C.c_uint32, C.c_int, p, p, C.c_int, C.c_double, p, p]
    f.restype = C.c_int
    return f


def _call(f, d_hist, n_el, nhist, bin, q, source, ff, sl, polar, lam, d_out):
    import torch
    n_el = np.ascontiguousarray(n_el, dtype=np.uint32)
    q = np.ascontiguousarray(q, dtype=np.float64)
    rows = [np.ascontiguousarray(r, dtype=np.float64) for r in ff] if ff is not None else None
    table = (C.c_void_p * len(rows))(*[r.ctypes.data for r in rows]) if rows is not None else None
    sl = np.ascontiguousarray(sl, dtype=np.float64) if sl is not None else None
    st = f(C.c_void_p(d_hist.data_ptr()), n_el.ctypes.data_as(C.c_void_p), len(n_el), nhist, bin,
           q.ctypes.data_as(C.c_void_p), len(q), source, table, None if sl is None else sl.ctypes.data_as(C.c_void_p),
           int(polar), lam, C.c_void_p(d_out.data_ptr()), None)
    torch.cuda.synchronize()
    return st


def test_noalloc_matches_allocating_entry_point(gpu_ctx):
    import torch
    f = _noalloc()
    # neutron, two elements: the reference's rock-salt histogram at 0.001 A bins
    gn = load_golden("hist__rocksalt_b0.001")
    qn = np.linspace(0.1, 25.0, 4096, endpoint=False)
    sl = np.array([3.63, 9.58])
    want_n = gpu_ctx.calc_int_1d_hist(gn["hist"], gn["n_el"], int(gn["nhist"]), float(gn["bin"]), qn, 0, sl=sl)
    # X-ray with polarisation
    gx = load_golden("iqhist__rocksalt_xray")
    want_x = gpu_ctx.calc_int_1d_hist(gx["hist"], gx["n_el"], int(gx["nhist"]), float(gx["bin"]), gx["q"], 1, ff=gx["ff"],
                                      polar=True, lam=float(gx["lam"]))
    assert rel_err(want_x, gx["I"]) < TOL_I

    dev = torch.device("cuda", 0)
    hn = torch.from_numpy(gn["hist"].view(np.int64)).to(dev)
    hx = torch.from_numpy(gx["hist"].view(np.int64)).to(dev)
    out_n = torch.full((len(qn),), float("nan"), dtype=torch.float64, device=dev)
    out_x = torch.full((len(gx["q"]),), float("nan"), dtype=torch.float64, device=dev)
    for _ in range(2):  # two calls in a row on the same input
        assert _call(f, hn, gn["n_el"], int(gn["nhist"]), float(gn["bin"]), qn, 0, None, sl, False, 0.0, out_n) == 0
        assert rel_err(out_n.cpu().numpy(), want_n) < TOL_I
    # then a different input through the same static array
    assert _call(f, hx, gx["n_el"], int(gx["nhist"]), float(gx["bin"]), gx["q"], 1, gx["ff"], None, True,
                 float(gx["lam"]), out_x) == 0
    assert rel_err(out_x.cpu().numpy(), want_x) < TOL_I
    assert rel_err(out_x.cpu().numpy(), gx["I"]) < TOL_I


def test_noalloc_large_histogram_and_nonuniform_mesh(gpu_ctx, oracle):
    """A 10-cell rock-salt cube at 0.001 A (about 7200 atoms, 3 x 97,000 bins) on 4096 q: the deep
    low-q minima of I(q), where the bin sum cancels to ~1e-5 of its terms, are where an FP32 sum shows.
    The allocation-free result stays within TOL_I of the allocating entry point (FP64 angle-split
    sums) and of the oracle, on two calls in a row; then a non-uniform mesh (per-term sines) of 1500 q."""
    import torch
    from xns_b200 import synth
    f = _noalloc()
    els = synth.rocksalt_cube(cells=10, seed=21)
    nh = synth.hist_size(els, 0.001)
    h = gpu_ctx.calc_hist(els, nh, 0.001)
    n_el = np.array([len(e) for e in els], dtype=np.uint32)
    sl = np.array([3.63, 9.58])
    q = synth.q_mesh(0.1, 25.0, 4096)
    want = gpu_ctx.calc_int_1d_hist(h, n_el, nh, 0.001, q, 0, sl=sl)
    ref = oracle.int_1d_hist(h, n_el, nh, 0.001, q, 0, sl=sl)
    assert rel_err(want, ref) < TOL_I
    dev = torch.device("cuda", 0)
    dh = torch.from_numpy(h.view(np.int64)).to(dev)
    out = torch.full((len(q),), float("nan"), dtype=torch.float64, device=dev)
    for _ in range(2):
        assert _call(f, dh, n_el, nh, 0.001, q, 0, None, sl, False, 0.0, out) == 0
        got = out.cpu().numpy()
        assert rel_err(got, want) < TOL_I
        assert rel_err(got, ref) < TOL_I
    qn = np.sort(np.random.default_rng(22).uniform(0.05, 20.0, 1500))
    want_n = gpu_ctx.calc_int_1d_hist(h, n_el, nh, 0.001, qn, 0, sl=sl)
    out_n = torch.full((len(qn),), float("nan"), dtype=torch.float64, device=dev)
    assert _call(f, dh, n_el, nh, 0.001, qn, 0, None, sl, False, 0.0, out_n) == 0
    assert rel_err(out_n.cpu().numpy(), want_n) < TOL_I


def test_noalloc_rejects_sizes_beyond_its_limits(gpu_ctx):
    import torch
    f = _noalloc()
    dev = torch.device("cuda", 0)
    nel = 17  # more elements than the static array is laid out for
    n_el = np.full(nel, 2, dtype=np.uint32)
    nhist = 8
    h = torch.zeros(nel * (nel + 1) // 2 * nhist, dtype=torch.int64, device=dev)
    out = torch.zeros(16, dtype=torch.float64, device=dev)
    assert _call(f, h, n_el, nhist, 0.1, np.linspace(0.1, 5, 16), 0, None, np.ones(nel), False, 0.0, out) == XNS_ERR_LIMIT
    # a non-uniform mesh takes 16 q per lane: at most XNS_NOALLOC_MAX_Q_NONUNIFORM (2048) points
    h2 = torch.zeros(nhist, dtype=torch.int64, device=dev)
    qn = np.sort(np.random.default_rng(3).uniform(0.1, 5.0, 2049))
    out2 = torch.zeros(len(qn), dtype=torch.float64, device=dev)
    assert _call(f, h2, [2], nhist, 0.1, qn, 0, None, np.ones(1), False, 0.0, out2) == XNS_ERR_LIMIT
