"""The rearrangement correction (RearrangementInt, CalcFunctions.cpp:469-545).

CPU: the oracle's restatement against the reference's own RearrangementInt, bit for bit (same loops,
same grouping, no contraction).  GPU: xns_rearrangement_int against the oracle, within FP64 rounding
(its terms are summed in another order)."""
import os

import numpy as np
import pytest

from oracle import REF_SO, Oracle, Reference
from xns_b200.structure import RearrBlock

needs_reference = pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")


def molecule_block(n=60, radius=3.5, seed=0, coeff=8, rcorr=0.5, rearrangement=True):
    """n atoms on a sphere (two elements: the first 2n/3 element 0, the rest element 1); each atom lists
    its two nearest neighbours in the molecule and its nearest atom of a copy 9 A away"""
    rng = np.random.default_rng(seed)
    k = np.arange(n) + 0.5
    th, ph = np.arccos(1 - 2 * k / n), np.pi * (1 + 5 ** 0.5) * k
    r = radius * np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
    r += rng.normal(0, 0.02, r.shape)
    ne = [2 * n // 3, n - 2 * n // 3]
    el = np.repeat([0, 1], ne)
    copy = r + np.array([9.0, 0.0, 0.0])
    neigh = []
    for i in range(n):
        d = np.linalg.norm(r - r[i], axis=1)
        d[i] = np.inf
        nb = [tuple(r[j]) + (int(el[j]),) for j in np.argsort(d)[:2]]
        j = int(np.argmin(np.linalg.norm(copy - r[i], axis=1)))
        nb.append(tuple(copy[j]) + (int(el[j]),))
        neigh.append(nb)
    return RearrBlock(r, ne, [0, 1], neigh, rcorr, coeff, rearrangement)


def case(partial, source, polar, nblocks=2, ntot=5000):
    rng = np.random.default_rng(1)
    nq = 300
    q = np.linspace(0.1, 12.0, nq)
    blocks = [molecule_block(seed=0), molecule_block(n=45, seed=1, coeff=3, rearrangement=(nblocks == 3))]
    if nblocks == 3:
        blocks.append(molecule_block(n=30, seed=2, coeff=5, rcorr=0.8))
    n0 = nq * (1 + nblocks * (nblocks + 1) // 2) if partial else nq
    I0 = 1.0 + rng.random(n0)
    ff = 2.0 + rng.random((2, nq)) if source == 1 else None
    sl = np.array([6.65, 9.36]) if source == 0 else None
    return dict(I0=I0, q=q, blocks=blocks, nel=2, source=source, ff=ff, sl=sl, partial=partial, polar=polar, lam=1.54,
                ntot=ntot)


CASES = {"neutron": case(False, 0, False), "xray_polar": case(False, 1, True), "partial_neutron": case(True, 0, False, 3),
         "partial_xray_polar": case(True, 1, True, 3), "ntot_beyond_2^16": case(False, 0, False, ntot=100000)}


def _run(impl, c):
    return impl.rearrangement_int(c["I0"], c["q"], c["blocks"], c["nel"], c["source"], ff=c["ff"], sl=c["sl"],
                                  partial=c["partial"], polar=c["polar"], lam=c["lam"], ntot=c["ntot"])


@needs_reference
@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_bit_for_bit(name):
    c = CASES[name]
    a, b = _run(Oracle(), c), _run(Reference(), c)
    assert np.array_equal(a, b, equal_nan=True)
    assert not np.array_equal(a, c["I0"], equal_nan=True)  # the correction changed something


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_oracle(gpu_ctx, name):
    c = CASES[name]
    g, o = _run(gpu_ctx, c), _run(Oracle(), c)
    fin = np.isfinite(o)
    assert np.array_equal(fin, np.isfinite(g))
    # the GPU adds the terms in an order set by atomics, and the correction cancels terms some 1e4 times
    # its result: FP64 rounding leaves a few 1e-12 of relative difference
    assert np.allclose(g[fin], o[fin], rtol=1e-10, atol=0)


def random_case(seed):
    """random blocks (1-3 elements, 5-80 sites, 0-4 neighbours per site from a shifted copy and the
    block itself, random Rcorr and coeff), neutron or X-ray, polar or not, partial or not"""
    rng = np.random.default_rng(100 + seed)
    nel = int(rng.integers(1, 4))
    nb = int(rng.integers(1, 4))
    blocks = []
    for b in range(nb):
        n = int(rng.integers(5, 81))
        r = rng.uniform(-6, 6, (n, 3))
        k = int(rng.integers(1, nel + 1))
        cuts = np.sort(rng.choice(np.arange(1, n), k - 1, replace=False)) if k > 1 else np.array([], int)
        ne = np.diff(np.concatenate([[0], cuts, [n]]))
        ids = rng.choice(nel, k, replace=False)
        shift = rng.uniform(-12, 12, 3)
        neigh = []
        for i in range(n):
            m = int(rng.integers(0, 5))
            js = rng.choice(n, m)
            neigh.append([tuple(r[j] + (shift if rng.random() < 0.5 else 0.0) + rng.normal(0, 0.3, 3)) +
                          (int(rng.integers(0, nel)),) for j in js])
        blocks.append(RearrBlock(r, ne, ids, neigh, float(rng.uniform(0, 1.5)), int(rng.integers(1, 30)),
                                 bool(rng.random() < 0.8)))
    nq = 150
    q = np.linspace(0.05, 15.0, nq)
    partial = bool(rng.random() < 0.5)
    n0 = nq * (1 + nb * (nb + 1) // 2) if partial else nq
    source = int(rng.integers(0, 2))
    return dict(I0=1.0 + rng.random(n0), q=q, blocks=blocks, nel=nel, source=source,
                ff=2.0 + rng.random((nel, nq)) if source == 1 else None,
                sl=rng.uniform(-4, 10, nel) if source == 0 else None, partial=partial,
                polar=bool(rng.random() < 0.5), lam=float(rng.uniform(0.5, 2.0)), ntot=int(rng.integers(100, 20000)))


@needs_reference
@pytest.mark.parametrize("seed", range(12))
def test_random_cases_oracle_matches_reference(seed):
    c = random_case(seed)
    assert np.array_equal(_run(Oracle(), c), _run(Reference(), c), equal_nan=True)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(12))
def test_random_cases_gpu_matches_oracle(gpu_ctx, seed):
    c = random_case(seed)
    g, o = _run(gpu_ctx, c), _run(Oracle(), c)
    fin = np.isfinite(o)
    assert np.array_equal(fin, np.isfinite(g))
    # relative to the correction's scale at each q as well as to I0 itself: the correction can cancel
    scale = np.maximum(np.abs(o[fin]), 1e-3 * np.max(np.abs(o[fin])))
    assert np.max(np.abs(g[fin] - o[fin]) / scale) < 1e-10
