"""CPU: the cross-rank step of one structure split over ranks (xns_b200.shard.reduce_histogram), with
two gloo ranks (127.0.0.1 rendezvous).  Each rank holds the histogram of its share of the atom pairs
(here: rows i with i % 2 == rank, counted with the reference's binning in numpy); the all-reduce must
give every rank the oracle's whole histogram."""
import json
import os
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT

WORLD = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _share(els, nh, bin_, rank, world):
    """counts of the pairs (i < j, element pairs a <= b in loop order) whose first atom's row in its
    element satisfies row % world == rank, binned as the reference does: (unsigned)(|ri - rj| / bin)"""
    P = len(els) * (len(els) + 1) // 2
    h = np.zeros(P * nh, dtype=np.int64)
    t = 0
    for a in range(len(els)):
        for b in range(a, len(els)):
            A, B = els[a], els[b]
            for i in range(rank, len(A), world):
                js = B[i + 1:] if a == b else B
                d = np.sqrt(((A[i] - js) ** 2).sum(axis=1))
                np.add.at(h, t * nh + (d / bin_).astype(np.int64), 1)
            t += 1
    return h


def _rank_main(rank, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(WORLD))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "softx-d-16-00083_b200"))
    import datetime

    import torch
    import torch.distributed as tdist

    from xns_b200 import synth
    from xns_b200.shard import reduce_histogram
    tdist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        els = synth.rocksalt_cube(cells=3, seed=5)
        nh = synth.hist_size(els, 0.01)
        h = torch.from_numpy(_share(els, nh, 0.01, rank, WORLD))
        reduce_histogram(h)
        np.save(os.path.join(out_dir, "rank%d.npy" % rank), h.numpy())
    finally:
        tdist.destroy_process_group()


def test_two_rank_histogram_reduce(tmp_path, oracle):
    import torch.multiprocessing as mp
    from xns_b200 import synth
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, port, str(tmp_path))) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    els = synth.rocksalt_cube(cells=3, seed=5)
    nh = synth.hist_size(els, 0.01)
    ref = oracle.hist(els, nh, 0.01)
    for r in range(WORLD):
        h = np.load(os.path.join(tmp_path, "rank%d.npy" % r))
        assert np.array_equal(h.astype(np.uint64), ref)
    # each share alone is a strict part of the whole
    assert 0 < _share(els, nh, 0.01, 0, WORLD).sum() < ref.sum()


def test_reduce_without_process_group_is_identity():
    import torch
    from xns_b200.shard import reduce_histogram
    h = torch.arange(10, dtype=torch.int64)
    assert torch.equal(reduce_histogram(h.clone()), h)


def _gather_main(rank, port, out_dir):
    """two gloo ranks run the 2D assembly of xns_b200.shard.int_2d with their rows given directly"""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(WORLD))
    sys.path.insert(0, os.path.join(ROOT, "softx-d-16-00083_b200"))
    import datetime

    import torch.distributed as tdist

    from xns_b200 import shard
    tdist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        nq, nfi = 7, 3
        full2d = np.arange(nq * nfi, dtype=np.float64).reshape(nq, nfi)
        full1d = -np.arange(nq, dtype=np.float64)

        class RowCtx:  # stands in for the library: returns the rows it is asked for
            def calc_int_2d(self, els, q, *a, **k):
                lo = int(round(q[0])) if len(q) else 0
                return full2d[lo:lo + len(q)], full1d[lo:lo + len(q)]
        a, b = shard.int_2d(RowCtx(), [], np.arange(nq, dtype=np.float64), nfi, 0, 0, 0, 0, 0, 0, rank=rank, world=WORLD)
        np.save(os.path.join(out_dir, "g%d.npy" % rank), np.concatenate([a.ravel(), b]))
    finally:
        tdist.destroy_process_group()


def test_two_rank_2d_gather(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_gather_main, args=(r, port, str(tmp_path))) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    want = np.concatenate([np.arange(21, dtype=np.float64), -np.arange(7, dtype=np.float64)])
    for r in range(WORLD):
        assert np.array_equal(np.load(os.path.join(tmp_path, "g%d.npy" % r)), want)


def _debye_main(rank, port, out_dir):
    """two gloo ranks run xns_b200.shard.int_debye with each rank's shard of the sum given directly"""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(WORLD))
    sys.path.insert(0, os.path.join(ROOT, "softx-d-16-00083_b200"))
    import datetime

    import torch.distributed as tdist

    from xns_b200 import shard
    tdist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        # stands in for the library: shard s holds (s + 1) / 3 of a pattern, so the two sum to it
        def fake_shard(ctx, elements, q, source, sl, ff, polar, lam, s_, n, neb):
            return (s_ + 1) / 3.0 * np.linspace(1.0, 2.0, len(q))
        shard.int_debye_shard = fake_shard
        I = shard.int_debye(None, [], np.arange(5, dtype=np.float64), 0, rank=rank, world=WORLD)
        np.save(os.path.join(out_dir, "d%d.npy" % rank), I)
    finally:
        tdist.destroy_process_group()


def test_two_rank_debye_all_reduce(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_debye_main, args=(r, port, str(tmp_path))) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    for r in range(WORLD):
        assert np.allclose(np.load(os.path.join(tmp_path, "d%d.npy" % r)), np.linspace(1.0, 2.0, 5), rtol=0, atol=1e-15)
