"""GPU: failure paths return a status and leave the context usable -- no fault, trap or hang is made.

* non-finite coordinates: the histogram plan and the Debye sum reject them (XNS_ERR_ARG) before any
  distance is binned or summed;
* a device-memory budget: xns_set_memory_limit caps the context's scratch, a call that would need
  more returns XNS_ERR_NOMEM before it queues work;
* a pipeline wait that runs out: xns_inject_pipeline_stall makes the next tensor-core transform's copy
  warp issue nothing and bounds its waits to 5 ms; the waits give up, the kernel frees its tensor
  memory and returns, the call (the integer-digit histogram transform) reports XNS_ERR_CUDA.
After each, the same context computes the right answer again."""
import numpy as np
import pytest

from conftest import load_golden, rel_err

from xns_b200 import synth

pytestmark = pytest.mark.gpu

XNS_ERR_ARG, XNS_ERR_CUDA, XNS_ERR_NOMEM = 1, 2, 5


def test_non_finite_coordinates_are_rejected(gpu_ctx, oracle):
    import xns_b200
    els = synth.rocksalt_cube(cells=3, seed=31)
    nh = synth.hist_size(els, 0.01)
    for bad in (np.nan, np.inf, -np.inf):
        b = [e.copy() for e in els]
        b[1][4, 2] = bad
        with pytest.raises(xns_b200.XnsError) as e:
            gpu_ctx.calc_hist(b, nh, 0.01)
        assert e.value.status == XNS_ERR_ARG
        with pytest.raises(xns_b200.XnsError) as e:
            gpu_ctx.calc_int_debye(b, synth.q_mesh(0.1, 5.0, 64), 0, sl=[3.63, 9.58])
        assert e.value.status == XNS_ERR_ARG
    assert np.array_equal(gpu_ctx.calc_hist(els, nh, 0.01), oracle.hist(els, nh, 0.01))


def test_memory_limit_gives_nomem_then_recovers(oracle):
    import xns_b200
    ctx = xns_b200.Context(0)
    try:
        els = synth.rocksalt_cube(cells=5, seed=32)
        nh = synth.hist_size(els, 0.001)
        ctx.set_memory_limit(64 * 1024)
        with pytest.raises(xns_b200.XnsError) as e:
            ctx.calc_hist(els, nh, 0.001)
        assert e.value.status == XNS_ERR_NOMEM
        ctx.set_memory_limit(0)
        assert np.array_equal(ctx.calc_hist(els, nh, 0.001), oracle.hist(els, nh, 0.001))
        # a cap below what the context now holds releases it; a generous cap changes nothing
        ctx.set_memory_limit(1 << 30)
        assert np.array_equal(ctx.calc_hist(els, nh, 0.001), oracle.hist(els, nh, 0.001))
    finally:
        ctx.close()


def test_pipeline_wait_runs_out_and_context_recovers(gpu_ctx):
    import xns_b200
    g = load_golden("iqhist__rocksalt_xray")
    nh, bin, q = int(g["nhist"]), float(g["bin"]), g["q"]
    H = np.asarray(g["hist"], dtype=np.uint64).reshape(-1, nh)
    G64 = gpu_ctx.hist_transform(H, bin, q, "split")  # FP64, no tensor-core pipeline
    G0 = gpu_ctx.hist_transform(H, bin, q, "exact")
    assert np.max(np.abs(G0 - G64)) < 1e-8 * np.max(np.abs(G64))
    gpu_ctx.inject_pipeline_stall(5_000_000)  # 5 ms
    with pytest.raises(xns_b200.XnsError) as e:
        gpu_ctx.hist_transform(H, bin, q, "exact")
    assert e.value.status == XNS_ERR_CUDA and "ran out of time" in str(e.value)
    # the next call (no injection) is whole again, and so are the calc functions
    assert np.max(np.abs(gpu_ctx.hist_transform(H, bin, q, "exact") - G0)) < 1e-12 * np.max(np.abs(G0))
    args = (g["hist"], g["n_el"], nh, bin, q, 1)
    assert rel_err(gpu_ctx.calc_int_1d_hist(*args, ff=g["ff"], polar=True, lam=float(g["lam"])), g["I"]) < 1e-5
    # the limit must be positive and within the kernels' own bound
    with pytest.raises(xns_b200.XnsError) as e:
        gpu_ctx.inject_pipeline_stall(0)
    assert e.value.status == XNS_ERR_ARG
