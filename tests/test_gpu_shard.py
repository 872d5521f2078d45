"""GPU: one structure's histogram split into shards (xns_calc_hist_shard / xns_hist_shard_device).

The shards of one GPU are computed one after another here (each launch independent, nothing waits on
another): their sum must be xns_calc_hist's histogram and the oracle's, bit for bit, and the
one-rank pipeline in xns_b200.shard must reproduce xns_calc_pdf_and_debye."""
import numpy as np
import pytest

import xns_b200
from xns_b200 import shard, synth

pytestmark = pytest.mark.gpu

BIN = 0.001


@pytest.mark.parametrize("nshard", [2, 3, 8])
def test_shards_sum_to_histogram(gpu_ctx, oracle, nshard):
    els = synth.rocksalt_cube(cells=9, seed=3)
    nh = synth.hist_size(els, BIN)
    full = gpu_ctx.calc_hist(els, nh, BIN)
    parts = [shard.hist_shard(gpu_ctx, els, nh, BIN, s, nshard) for s in range(nshard)]
    assert all(p.sum() > 0 for p in parts)  # every shard has work
    assert np.array_equal(np.sum(parts, axis=0, dtype=np.uint64), full)
    assert np.array_equal(full, oracle.hist(els, nh, BIN))
    # the shares are balanced: no shard holds more than twice its share of the pairs
    assert max(p.sum() for p in parts) < 2.0 * full.sum() / nshard


def test_shard_arguments_checked(gpu_ctx):
    els = synth.rocksalt_cube(cells=3, seed=3)
    with pytest.raises(xns_b200.XnsError):
        shard.hist_shard(gpu_ctx, els, 20000, BIN, 2, 2)


def test_one_rank_pipeline_matches_calc_pdf_and_debye(gpu_ctx):
    import torch
    els = synth.rocksalt_cube(cells=6, seed=4)
    sl = np.array([3.63, 9.58])
    nh = synth.hist_size(els, BIN)
    q = synth.q_mesh(0.1, 25.0, 512)
    n_el = np.array([len(e) for e in els], dtype=np.uint32)
    P = 3
    I_ref, pdf_ref, h_ref = gpu_ctx.calc_pdf_and_debye(els, nh, BIN, xns_b200.DEBYE_PDF, xns_b200.RPDF, 0.05, q,
                                                       xns_b200.NEUTRON, sl=sl, want_hist=True)
    xyz = torch.from_numpy(np.ascontiguousarray(np.concatenate(els))).cuda()
    hist = torch.zeros(P * nh, dtype=torch.int64, device="cuda")
    I = torch.zeros(len(q), dtype=torch.float64, device="cuda")
    pdf = torch.zeros((1 + P) * nh, dtype=torch.float64, device="cuda")
    gpu_ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        shard.pdf_and_debye(gpu_ctx, xyz, n_el, nh, BIN, xns_b200.DEBYE_PDF, xns_b200.RPDF, 0.05, q, xns_b200.NEUTRON, sl,
                            hist, I, pdf)
    finally:
        gpu_ctx.set_stream(None)
    assert np.array_equal(hist.cpu().numpy().view(np.uint64), h_ref)
    # the transform's cross-CTA FP64 sums are order-dependent: equal to the last few bits
    assert np.allclose(I.cpu().numpy(), I_ref, rtol=1e-12, atol=0)
    assert np.allclose(pdf.cpu().numpy(), pdf_ref, rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("nshard", [2, 5])
def test_debye_shards_sum_to_intensity(gpu_ctx, nshard):
    els = synth.fcc_sphere(n=1500, a=4.078, sigma=0.05, seed=2)
    q = synth.q_mesh(0.1, 10.0, 256)
    full = gpu_ctx.calc_int_debye(els, q, xns_b200.NEUTRON, sl=[7.63])
    parts = [shard.int_debye_shard(gpu_ctx, els, q, xns_b200.NEUTRON, sl=[7.63], shard=s, nshard=nshard)
             for s in range(nshard)]
    assert np.allclose(np.sum(parts, axis=0), full, rtol=1e-12, atol=0)
    assert all(np.abs(p).max() > 0 for p in parts)


def test_partial_debye_shards_sum(gpu_ctx):
    rng = np.random.default_rng(6)
    els = [rng.uniform(0, 15, (300, 3)), rng.uniform(0, 15, (200, 3))]
    n_el_block = np.array([[100, 200], [150, 50]])  # (element, block)
    q = synth.q_mesh(0.5, 8.0, 128)
    full = gpu_ctx.calc_int_partial_debye(els, n_el_block, q, xns_b200.NEUTRON, sl=[3.63, 9.58])
    parts = [shard.int_debye_shard(gpu_ctx, els, q, xns_b200.NEUTRON, sl=[3.63, 9.58], shard=s, nshard=3,
                                   n_el_block=n_el_block.ravel()) for s in range(3)]
    tot = np.sum(parts, axis=0)
    # the cross-block parts cross zero: compare against the total intensity's scale at each q
    scale = np.tile(np.abs(full[:len(q)]), len(full) // len(q))
    assert np.max(np.abs(tot - full) / scale) < 1e-12


def test_2d_q_row_shards_assemble_the_pattern(gpu_ctx):
    rng = np.random.default_rng(9)
    els = [rng.uniform(-10, 10, (400, 3)), rng.uniform(-10, 10, (100, 3))]
    q = synth.q_mesh(0.2, 6.0, 37)
    args = (6, [0.1, 0.2, 0.0], [0.5, 0.9, 0.3], [2, 1, 2], 5, 1.54, xns_b200.NEUTRON)
    I2D, I = gpu_ctx.calc_int_2d(els, q, *args, sl=[3.0, 5.0])
    rows2d, rows1d = [], []
    for r in range(4):
        lo, hi = shard.q_rows(len(q), r, 4)
        a, b = gpu_ctx.calc_int_2d(els, q[lo:hi], *args, sl=[3.0, 5.0])
        rows2d.append(a)
        rows1d.append(b)
    assert np.allclose(np.concatenate(rows2d), I2D, rtol=1e-12, atol=0)
    assert np.allclose(np.concatenate(rows1d), I, rtol=1e-12, atol=0)
    # the one-rank driver returns the whole pattern
    a, b = shard.int_2d(gpu_ctx, els, q, *args, sl=[3.0, 5.0])
    assert np.allclose(a, I2D, rtol=1e-12, atol=0) and np.allclose(b, I, rtol=1e-12, atol=0)
