"""Learned binning correction of the histogram Debye intensity (no reference counterpart).

Coarse bins (0.02 A) make the histogram -> I(q) transform 20x smaller and let the histogram window
cover every distance, but at q = 20 A^-1 a bin spans 0.4 rad of phase and I(q) is off by ~1e-2.  The
error comes from placing every pair of bin k at the bin centre.  Expanding sin(q r)/(q r) to second order
in the offset d from the centre corrects it with two moments per bin, mu1 = E[d/D] and m2 = E[(d/D)^2]
(learned.cu).  Those moments are not in the coarse histogram, but they follow from how the distance
density varies around the bin: a small perceptron (xns_b200.MLP: 3 layers, width 256, GELU, BF16
weights, FP32 accumulation, trained on the GPU by the library's own forward and backward kernels)
predicts them from the bin's neighbourhood in the coarse histogram.

Training data come from the GPU: coarse histograms for the inputs, histograms 32x finer for the exact
per-bin moments, and the exact Debye double sum (xns_calc_int_debye: no binning at all) as the arbiter.
The integer histograms are never altered.  fit() holds structures out and records the largest relative
error of the corrected I(q) against the double sum; predict() uses the network only where that
validated error is within the tolerance, and otherwise returns the exact double sum for every structure.
"""
import numpy as np

from . import MLP, NEUTRON, lib, _ptr, synth

COARSE_BIN = 0.02
SUB = 32          # fine bins per coarse bin for the training moments
NFEAT = 18        # XNS_BINNING_FEATURES
HIDDEN = 256
MOMENT_SCALE = 4.0  # targets (mu1 in [-1/2, 1/2], m2 in [0, 1/4]) are learned times this


def self_term(structure, sl):
    n = [len(e) for e in structure]
    return sum(ni * w * w for ni, w in zip(n, sl)) / max(sum(n), 1)


def weighted_hist(structure, sl, hist, nhist):
    """h = 2 sum_{a<=b} w_a w_b n_ab / (N s0): I(q) = s0 [1 + sum_k h_k sin(q r_k)/(q r_k)]."""
    nel, N = len(structure), sum(len(e) for e in structure)
    s0 = self_term(structure, sl)
    h = np.zeros(nhist)
    t = 0
    for a in range(nel):
        for b in range(a, nel):
            h += 2.0 * sl[a] * sl[b] * hist[t * nhist:(t + 1) * nhist]
            t += 1
    return h / (N * s0)


def hist_pass(ctx, structures, sls, q, bin, nh=None):
    """Batched histograms: (I (S x nq), per-structure weighted histograms h, s0, nh)."""
    nh = nh or max(synth.hist_size(s, bin) for s in structures)
    I, hc = ctx.calc_batch_debye_hist(structures, nh, bin, q, NEUTRON, sl=sls, want_hist=True)
    hs, off = [], 0
    for s, sl in zip(structures, sls):
        P = len(s) * (len(s) + 1) // 2
        hs.append(weighted_hist(s, sl, hc[off * nh:(off + P) * nh], nh))
        off += P
    return I, hs, np.array([self_term(s, sl) for s, sl in zip(structures, sls)]), nh


def exact_pass(ctx, structures, sls, q):
    """The exact Debye double sum of every structure (S x nq)."""
    return np.stack([ctx.calc_int_debye(s, q, NEUTRON, sl=sl) for s, sl in zip(structures, sls)])


def moments(h_fine, nh):
    """Per coarse bin (mu1, m2) in units of the coarse bin, from SUB fine bins per coarse bin."""
    f = h_fine[:nh * SUB].reshape(nh, SUB)
    d = (np.arange(SUB) + 0.5) / SUB - 0.5
    w = f.sum(axis=1)
    mu1 = np.where(w > 0, (f * d).sum(axis=1) / np.maximum(w, 1e-300), 0.0)
    m2 = np.where(w > 0, (f * d * d).sum(axis=1) / np.maximum(w, 1e-300), 1.0 / 12.0)
    return np.stack([mu1, m2], axis=1).astype(np.float32)


def features(ctx, h):
    X = np.zeros((len(h), NFEAT), dtype=np.float32)
    ctx._check(lib.xns_binning_features(ctx.handle, _ptr(np.ascontiguousarray(h, np.float64)), len(h), _ptr(X)))
    return X


def correction(ctx, h, mu, q, s0):
    dI = np.zeros(len(q))
    ctx._check(lib.xns_binning_correction(ctx.handle, _ptr(np.ascontiguousarray(h, np.float64)),
                                          _ptr(np.ascontiguousarray(mu, np.float32)), len(h), COARSE_BIN,
                                          _ptr(np.ascontiguousarray(q, np.float64)), len(q), s0, _ptr(dI)))
    return dI


def max_rel_err(a, b):
    return np.max(np.abs(a - b) / np.abs(b), axis=-1)


class LearnedCorrector:
    def __init__(self, ctx, q, tol=1e-4, seed=0):
        self.ctx, self.q, self.tol = ctx, np.asarray(q, dtype=np.float64), tol
        self.net = MLP(ctx, (NFEAT, HIDDEN, HIDDEN, 2), seed=seed)
        self.validated_err = None
        self.validation = None
        self.weight_power = 1.0

    def _moments_pred(self, h):
        return self.net.forward(features(self.ctx, h)) / MOMENT_SCALE

    def corrected(self, I_c, hs, s0):
        return np.stack([I_c[i] + correction(self.ctx, hs[i], self._moments_pred(hs[i]), self.q, s0[i])
                         for i in range(len(hs))])

    def fit(self, structures, sls, holdout=0.125, samples=200000, epochs=40, batch=512, lr=1e-3, seed=0):
        rng = np.random.default_rng(seed)
        I_c, hs, s0, nh = hist_pass(self.ctx, structures, sls, self.q, COARSE_BIN)
        _, hf, _, _ = hist_pass(self.ctx, structures, sls, self.q, COARSE_BIN / SUB, nh=nh * SUB)
        mus = [moments(f, nh) for f in hf]
        idx = rng.permutation(len(structures))
        nv = max(1, int(len(idx) * holdout))
        va, tr = idx[:nv], idx[nv:]
        # training bins drawn in proportion to their share of the correction's amplitude, h_k / r_k
        # (S' and S'' fall off as 1/r): the near shells that set I(q) at high q
        X = np.concatenate([features(self.ctx, hs[i]) for i in tr])
        Y = np.concatenate([mus[i] for i in tr]) * MOMENT_SCALE
        wts = np.concatenate([hs[i] / (np.arange(nh) + 0.5) ** self.weight_power for i in tr])
        p = np.clip(wts, 0, None)
        pick = rng.choice(len(p), size=min(samples, int((p > 0).sum()) * 4), p=p / p.sum())
        losses = [self.net.train(X[pick], Y[pick], batch=batch, epochs=1, lr=lr) for _ in range(epochs)]
        # the arbiter: the exact double sum on the held-out structures
        held = [structures[i] for i in va]
        I_x = exact_pass(self.ctx, held, [sls[i] for i in va], self.q)
        I_l = self.corrected(I_c[va], [hs[i] for i in va], s0[va])
        unif = np.tile(np.array([[0.0, 1.0 / 12.0]], np.float32), (nh, 1))
        I_u = np.stack([I_c[i] + correction(self.ctx, hs[i], unif, self.q, s0[i]) for i in va])
        I_m = np.stack([I_c[i] + correction(self.ctx, hs[i], mus[i], self.q, s0[i]) for i in va])
        e = {k: max_rel_err(v, I_x) for k, v in (("coarse", I_c[va]), ("uniform_bins", I_u), ("learned", I_l),
                                                 ("exact_moments", I_m))}
        self.validated_err = float(e["learned"].max())
        self.validation = {"median_" + k: float(np.median(v)) for k, v in e.items()}
        self.validation.update({"max_" + k: float(v.max()) for k, v in e.items()})
        return losses

    @property
    def trusted(self):
        return self.validated_err is not None and self.validated_err <= self.tol

    def predict(self, structures, sls):
        """(I (S x nq), path): the corrected coarse intensity where the validated error is within tol,
        else the exact double sum."""
        if self.trusted:
            I_c, hs, s0, _ = hist_pass(self.ctx, structures, sls, self.q, COARSE_BIN)
            return self.corrected(I_c, hs, s0), "learned"
        return exact_pass(self.ctx, structures, sls, self.q), "exact"

    def close(self):
        self.net.close()


def training_structures(count, seed=0, nmin=200, nmax=1500):
    """The config-3 generator at small sizes (fcc a = 3.61 A with 5 % substitution, random orientation,
    Gaussian displacement 0.02-0.1 A) plus 10 % random-packed amorphous clusters (0.085 atoms/A^3).
    Returns (structures, per-structure neutron lengths)."""
    rng = np.random.default_rng(seed)
    structs, sls = [], []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        if rng.random() < 0.1:
            structs.append(synth.random_cluster(n, density=0.085, seed=int(rng.integers(1 << 30))))
            sls.append([1.0])
        else:
            cells = max(2, int(round((n / 4) ** (1 / 3))))
            els = synth.fcc_crystallite(cells=cells, a=3.61, subst=0.05, seed=int(rng.integers(1 << 30)))
            sig = rng.uniform(0.02, 0.1)
            els = [e + rng.normal(0.0, sig, e.shape) for e in els]
            structs.append(els)
            sls.append([1.0, 0.6])
    return structs, sls
