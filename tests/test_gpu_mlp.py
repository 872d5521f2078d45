"""The learned correction's perceptron: hand-written GPU forward / backward kernels against the FP64
numpy oracle (oracle/mlp_oracle.py), training, and what the trained network gains over the coarse
histogram alone -- with the exact Debye double sum as the arbiter and the fallback."""
import numpy as np
import pytest

from conftest import rel_err

from xns_b200 import synth

pytestmark = pytest.mark.gpu

DIMS = (10, 16, 12, 7)


def _data(seed=0, B=9):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(B, DIMS[0])).astype(np.float32), rng.normal(size=(B, DIMS[3])).astype(np.float32)


def test_forward_matches_oracle(gpu_ctx):
    import mlp_oracle
    import xns_b200
    net = xns_b200.MLP(gpu_ctx, DIMS, seed=3)
    x, _ = _data()
    y = net.forward(x)
    y_ref, _ = mlp_oracle.forward(net.get_params(), DIMS, x)
    assert np.max(np.abs(y - y_ref)) < 1e-5 * max(1.0, np.abs(y_ref).max())
    net.close()


def test_gradients_match_oracle(gpu_ctx):
    import mlp_oracle
    import xns_b200
    net = xns_b200.MLP(gpu_ctx, DIMS, seed=4)
    x, t = _data(1)
    w = np.linspace(0.5, 2.0, DIMS[3]).astype(np.float32)
    loss, g = net.gradients(x, t, w)
    loss_ref, g_ref = mlp_oracle.gradients(net.get_params(), DIMS, x, t, w)
    assert abs(loss - loss_ref) < 1e-5 * loss_ref
    assert np.max(np.abs(g - g_ref)) < 1e-4 * np.abs(g_ref).max()
    net.close()


def test_training_fits_a_smooth_map(gpu_ctx):
    import xns_b200
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, size=(1024, 4)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]) * x[:, 1], x[:, 2] ** 2 - x[:, 3]], axis=1).astype(np.float32)
    net = xns_b200.MLP(gpu_ctx, (4, 64, 64, 2), seed=1)
    first = net.train(x, t, batch=128, epochs=1, lr=3e-3)
    last = net.train(x, t, batch=128, epochs=300, lr=3e-3)
    assert last < 0.05 * first
    net.close()


def test_learned_correction_gain_and_fallback(gpu_ctx):
    """Trained on 384 small structures (fcc crystallites with substitution and displacement, 10 %
    amorphous clusters), against the exact double sum on held-out structures (median over structures
    of the max relative error over q):
      * the second-order bin correction itself works: with the exact within-bin moments (from 32x finer
        histograms) it removes more than 90 % of the coarse-bin error;
      * the network's moments, predicted from the coarse histogram alone, gain little or nothing over
        the uncorrected coarse bins (measured: 0.0216 vs 0.0214 at 0.02 A, q up to 20) -- the within-bin
        offsets are barely determined by the neighbouring coarse counts (R^2 ~ 0.1) -- so it must at
        least not make the intensity worse by more than 10 %;
      * its validated error misses 1e-4, so predict() returns the exact double sum."""
    from xns_b200 import learned
    q = synth.q_mesh(0.1, 20.0, 256)
    structs, sls = learned.training_structures(384, seed=11, nmin=80, nmax=400)
    lc = learned.LearnedCorrector(gpu_ctx, q, tol=1e-4, seed=2)
    lc.fit(structs, sls, holdout=0.125, samples=100000, epochs=30, batch=512, lr=1e-3)
    v = lc.validation
    assert v["median_exact_moments"] < 0.1 * v["median_coarse"], v
    assert v["median_learned"] < 1.1 * v["median_coarse"], v
    test_s, test_sl = learned.training_structures(4, seed=99, nmin=80, nmax=400)
    I, path = lc.predict(test_s, test_sl)
    exact = learned.exact_pass(gpu_ctx, test_s, test_sl, q)
    if path == "exact":
        assert not lc.trusted
        assert rel_err(I, exact) == 0.0
    else:
        assert lc.trusted and rel_err(I, exact) < 1e-3
    lc.close()
