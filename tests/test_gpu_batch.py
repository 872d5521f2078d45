"""Batched ensembles: one plan, one persistent histogram launch and one tensor-core transform for many
structures must give each structure exactly what the single-structure entry points give it
(histograms bit-identical, I(q) to FP64 rounding), and graph replays must repeat the result."""
import numpy as np
import pytest

from conftest import rel_err

from xns_b200 import synth

pytestmark = pytest.mark.gpu


def ensemble(seed=0):
    """Mixed sizes: fcc spheres (one element), rock-salt cubes (two), a 2-atom molecule, and a
    two-element cluster with an empty element."""
    rng = np.random.default_rng(seed)
    structs, sls = [], []
    for n in (1000, 300, 2500):
        structs.append(synth.fcc_sphere(n=n, sigma=float(rng.uniform(0.02, 0.1)), seed=int(rng.integers(1 << 30))))
        sls.append([7.63])
    for cells in (3, 5):
        structs.append(synth.rocksalt_cube(cells=cells, seed=int(rng.integers(1 << 30))))
        sls.append([3.63, 9.58])
    structs.append([np.array([[0.0, 0.0, 0.0], [1.1, 0.2, -0.3]])])
    sls.append([5.0])
    structs.append([rng.normal(0, 4, (200, 3)), np.zeros((0, 3))])
    sls.append([2.0, 4.0])
    return structs, sls


def common_nhist(structs, bin):
    return max(synth.hist_size(s, bin) for s in structs)


def test_batch_matches_single_structure_calls(gpu_ctx):
    structs, sls = ensemble()
    bin = 0.001
    nh = common_nhist(structs, bin)
    q = synth.q_mesh(0.1, 25.0, 1024)
    I, h = gpu_ctx.calc_batch_debye_hist(structs, nh, bin, q, 0, sl=sls, want_hist=True)
    off = 0
    for s, (els, sl) in enumerate(zip(structs, sls)):
        P = len(els) * (len(els) + 1) // 2
        hs = gpu_ctx.calc_hist(els, nh, bin)
        assert np.array_equal(h[off * nh:(off + P) * nh], hs), s
        Is = gpu_ctx.calc_int_1d_hist(hs, [len(e) for e in els], nh, bin, q, 0, sl=sl)
        # the batch transforms with the integer-digit GEMM, the single call with the FP64 angle split:
        # they agree to the digits' quantization (~1e-12 of a sinc value)
        assert rel_err(I[s], Is) < 1e-8, s
        off += P


def test_batch_xray_polar(gpu_ctx):
    structs, _ = ensemble(1)
    bin = 0.002
    nh = common_nhist(structs, bin)
    q = synth.q_mesh(0.2, 12.0, 300)
    ff = [list(synth.ff_on_mesh(synth.ff_coefficients(len(els), seed=7 * s + 1), q)) for s, els in enumerate(structs)]
    I = gpu_ctx.calc_batch_debye_hist(structs, nh, bin, q, 1, ff=ff, polar=True, lam=1.5)
    for s, els in enumerate(structs):
        hs = gpu_ctx.calc_hist(els, nh, bin)
        Is = gpu_ctx.calc_int_1d_hist(hs, [len(e) for e in els], nh, bin, q, 1, ff=ff[s], polar=True, lam=1.5)
        assert rel_err(I[s], Is) < 1e-8, s  # digit GEMM against the FP64 angle split, as above


@pytest.mark.parametrize("autotune", [False, True])
def test_batch_graph_replay(gpu_ctx, autotune):
    structs, sls = ensemble(2)
    bin = 0.001
    nh = common_nhist(structs, bin)
    q = synth.q_mesh(0.1, 20.0, 512)
    b = gpu_ctx.batch(structs, nh, bin, q, 0, sl=sls, autotune=autotune)
    I1, h1 = b.run(want_hist=True)
    I2, h2 = b.run(want_hist=True)
    assert np.array_equal(h1, h2)
    assert rel_err(I2, I1) < 1e-12
    I0 = gpu_ctx.calc_batch_debye_hist(structs, nh, bin, q, 0, sl=sls)
    assert rel_err(I1, I0) < 1e-10
    ct, wb, ms = b.tuning()
    assert (ct, wb) in {(56, 42 * 1024 + 512), (32, 42 * 1024 + 512), (96, 42 * 1024 + 512), (56, 16 * 1024)}
    assert (ms > 0) == autotune
    assert b.last_ms > 0
    b.close()


def test_batch_range_error(gpu_ctx):
    import xns_b200
    structs, sls = ensemble(3)
    with pytest.raises(xns_b200.XnsError) as e:
        gpu_ctx.calc_batch_debye_hist(structs, 100, 0.001, synth.q_mesh(0.1, 5.0, 64), 0, sl=sls)
    assert e.value.status == 4


def test_batch_too_many_structures(gpu_ctx):
    """The transform's grid has one row of CTAs per structure: 65536 structures are refused up front."""
    import xns_b200
    structs = [[np.zeros((1, 3))]] * 65536
    with pytest.raises(xns_b200.XnsError) as e:
        gpu_ctx.calc_batch_debye_hist(structs, 16, 0.01, synth.q_mesh(0.1, 5.0, 8), 0, sl=[[1.0]] * 65536)
    assert e.value.status == 1
