"""GPU: the structure builder (xns_build_atoms) against the oracle's restatement of block::calcAtoms
(CalcFunctions.cpp:251-392), which the CPU tests pin to the reference's own calcAtoms.

Same seed, same Philox draws: the same atoms in the same order.  Without random displacements or
molecule rotations the coordinates are bit-identical; with them they differ only by the last-bit
differences of the device's log / sin / cos (below 1e-12 A here)."""
import ctypes as C

import numpy as np
import pytest

from test_builder_oracle import FCC, draw_free_cases, oracle, random_draw_free_block, rocksalt
from xns_b200.structure import Block

pytestmark = pytest.mark.gpu


def _build(ctx, blocks, nel, seed):
    dev, n_el, n_all = ctx.build_atoms(blocks, nel, seed)
    return ctx.copy_atoms(n_el), n_all, dev, n_el


@pytest.mark.parametrize("name", sorted(draw_free_cases()))
def test_draw_free_builds_bit_exact(gpu_ctx, name):
    blocks, nel = draw_free_cases()[name]
    xg, ng, _, _ = _build(gpu_ctx, blocks, nel, 11)
    xo, no = oracle().build_atoms(blocks, nel, seed=11)
    assert [len(x) for x in xg] == [len(x) for x in xo]
    assert np.array_equal(ng, no)
    for a, b in zip(xg, xo):
        assert np.array_equal(a, b)


def random_cases():
    mol = Block(np.array([[0.3, -0.2, 0.1], [0.3, -0.2, 1.6]]), [1, 1], [0, 1], e=np.eye(3) * 6.0, ncell=(6, 7, 8),
                ro_mol=True, dev_mol=0.1, dev=[0.02, 0.03])
    shared = Block(np.array([[0, 0, 0], [0, 0, 0]]), [1, 1], [0, 1], occ=[0.3, 0.7], e=np.eye(3) * 3.0, ncell=(9, 9, 9))
    return {
        "rocksalt_vacancies_displacements": ([rocksalt((10, 10, 10), occ=[0.9, 0.9], dev=[0.07, 0.07])], 2),
        "molecule_rotation_displacement": ([mol], 2),
        "shared_site": ([shared], 2),
        "two_blocks": ([rocksalt((4, 5, 6), occ=[0.8, 0.95], dev=[0.05, 0.0], r_copy=[(0, 0, 0), (40.0, 0, 0)],
                                 cf=[np.eye(3), np.eye(3)[[1, 2, 0]]]), mol], 3),
    }


@pytest.mark.parametrize("name", sorted(random_cases()))
def test_random_builds_match_oracle(gpu_ctx, name):
    blocks, nel = random_cases()[name]
    for seed in (1, 2 ** 40 + 7):
        xg, ng, _, _ = _build(gpu_ctx, blocks, nel, seed)
        xo, no = oracle().build_atoms(blocks, nel, seed=seed)
        assert [len(x) for x in xg] == [len(x) for x in xo]  # every occupancy draw identical
        assert np.array_equal(ng, no)
        for a, b in zip(xg, xo):
            assert np.max(np.abs(a - b), initial=0.0) < 1e-12


def test_large_atom_file_merge_bit_exact(gpu_ctx):
    """20,000 sites read from an atom file (one cell, no symmetry), 400 of them planted within 0.5 A of
    others, occupancies that make merged sites choose: the O(sites^2) merge on the GPU"""
    rng = np.random.default_rng(21)
    n = 20000
    pts = rng.uniform(0, 60, (n, 3))
    pts[10000:10400] = pts[:400] + rng.normal(0, 0.12, (400, 3))
    occ = np.where(np.arange(n) % 3 == 0, 0.5, 1.0)
    b = Block(pts, [12000, 8000], [0, 1], occ=occ)
    xg, ng, _, _ = _build(gpu_ctx, [b], 2, 5)
    xo, no = oracle().build_atoms([b], 2, seed=5)
    assert np.array_equal(ng, no)
    for a, c in zip(xg, xo):
        assert np.array_equal(a, c)
    assert sum(len(x) for x in xg) < n


def test_chain_of_claims(gpu_ctx):
    """sites 0.3 A apart on a line: each lists only its neighbour, so which sites draw alternates along
    the chain (the rounds of propagation, then the sequential rule beyond 64 rounds)"""
    for n in (9, 301):
        pts = np.zeros((n, 3))
        pts[:, 0] = 0.3 * np.arange(n)
        b = Block(pts, [n], [0])
        xg, _, _, _ = _build(gpu_ctx, [b], 1, 3)
        xo, _ = oracle().build_atoms([b], 1, seed=3)
        assert np.array_equal(xg[0], xo[0])
        assert len(xo[0]) == (n + 1) // 2


def test_build_then_histogram_on_device(gpu_ctx):
    """the built atoms feed the histogram without leaving the GPU: same counts as the oracle's histogram
    of the oracle's build"""
    import xns_b200
    b = rocksalt((6, 6, 6), occ=[0.9, 0.9])
    dev, n_el, _ = gpu_ctx.build_atoms([b], 2, 17)
    xo, _ = oracle().build_atoms([b], 2, seed=17)
    bin_, nh = 0.01, 0
    nh = oracle().hist_size(xo, bin_)
    P = 3
    hist = np.zeros(P * nh, dtype=np.uint64)
    I = np.zeros(8)
    q = np.linspace(0.5, 4.0, 8)
    import torch
    d_hist = torch.zeros(P * nh, dtype=torch.int64, device="cuda:0")
    d_I = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    d_pdf = torch.zeros((1 + P) * nh, dtype=torch.float64, device="cuda:0")
    sl = np.array([3.63, 9.58])
    p = C.c_void_p
    st = xns_b200.lib.xns_pdf_and_debye_device(gpu_ctx.handle, p(dev), n_el.ctypes.data_as(p), 2, nh, bin_, 2, 1, 0.0,
                                               q.ctypes.data_as(p), 8, 0, None, sl.ctypes.data_as(p), 0, 0.0,
                                               p(d_I.data_ptr()), p(d_pdf.data_ptr()), p(d_hist.data_ptr()))
    assert st == 0
    hist[:] = d_hist.cpu().numpy().view(np.uint64)
    assert np.array_equal(hist, oracle().hist(xo, nh, bin_))
    assert np.allclose(d_I.cpu().numpy(), oracle().int_1d_hist(hist, n_el, nh, bin_, q, 0, sl=sl), rtol=1e-5)


def test_bad_blocks_are_rejected(gpu_ctx):
    import xns_b200
    b = rocksalt((2, 2, 2))
    with pytest.raises(xns_b200.XnsError):
        gpu_ctx.build_atoms([b], 1, 0)  # block element id 1 >= nel
    b.natom_el = np.array([1, 0], dtype=np.uint32)
    with pytest.raises(xns_b200.XnsError):
        gpu_ctx.build_atoms([b], 2, 0)  # natom_el does not sum to natom


def test_merge_threshold_far_from_origin(gpu_ctx):
    """pairs a hair either side of 0.5 A at coordinates up to 900 A, where an FP32 ulp is 6e-5 A: the
    FP32 prefilter must pass every pair the FP64 test accepts, and nothing else gets merged"""
    rng = np.random.default_rng(8)
    base = rng.uniform(-900, 900, (600, 3))
    u = rng.normal(size=(600, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    eps = np.concatenate([-np.logspace(-15, -4, 300), np.logspace(-15, -4, 300)])
    partner = base + u * (0.5 + eps)[:, None]
    pts = np.empty((1200, 3))
    pts[0::2], pts[1::2] = base, partner
    b = Block(pts, [1200], [0], occ=np.where(np.arange(1200) % 2 == 0, 0.0, 1.0))
    xg, _, _, _ = _build(gpu_ctx, [b], 1, 2)
    xo, _ = oracle().build_atoms([b], 1, seed=2)
    assert np.array_equal(xg[0], xo[0])
    # merged pairs place the partner (occupancy 1) once; unmerged ones place it alone too, but the
    # base site (occupancy 0) then draws nothing: the count shows nothing about the merge, the order does
    assert 250 < sum(np.linalg.norm(pts[1::2] - pts[0::2], axis=1) < 0.5) < 350


def test_drop_in_builder_matches_reference_program_objects():
    """calcAtomsB200 (the drop-in for CalcAndPrintAtoms' calcAtoms loop) on the reference's own block
    objects against the reference's block::calcAtoms, in one program linked with the reference's
    compiled CalcFunctions object: same atoms, order, NatomElAll and N"""
    import os
    import subprocess
    from conftest import ROOT
    exe = os.path.join(ROOT, "softx-d-16-00083_b200", "lib", "xns_build_atoms_check")
    if not os.path.exists(exe):
        pytest.skip("drop-in check program not built (needs the reference sources at build time)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 2 and all(l.endswith("identical") for l in lines)


def test_empty_inputs(gpu_ctx):
    """no blocks, a block without sites next to a real one, a fully vacant block"""
    _, n_el, n_all = gpu_ctx.build_atoms([], 3, 1)
    assert list(n_el) == [0, 0, 0] and len(n_all) == 0
    assert [len(x) for x in gpu_ctx.copy_atoms(n_el)] == [0, 0, 0]
    empty = Block(np.zeros((0, 3)), [0], [1])
    b = rocksalt((2, 2, 2))
    xg, ng, _, _ = _build(gpu_ctx, [empty, b], 2, 4)
    xo, no = oracle().build_atoms([empty, b], 2, seed=4)
    assert np.array_equal(ng, no) and list(ng) == [0, 32, 32]
    for a, c in zip(xg, xo):
        assert np.array_equal(a, c)
    xg, ng, _, _ = _build(gpu_ctx, [rocksalt((3, 3, 3), occ=[0.0, 0.0])], 2, 4)
    assert [len(x) for x in xg] == [0, 0] and list(ng) == [0, 0]


@pytest.mark.parametrize("seed", range(40))
def test_random_draw_free_blocks_bit_exact(gpu_ctx, seed):
    b = random_draw_free_block(seed)
    xg, ng, _, _ = _build(gpu_ctx, [b], 4, seed)
    xo, no = oracle().build_atoms([b], 4, seed=seed)
    assert np.array_equal(ng, no)
    for a, c in zip(xg, xo):
        assert np.array_equal(a, c)
