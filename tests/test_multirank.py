"""CPU: the multi-rank logic of bench.py with two gloo ranks (127.0.0.1 rendezvous).

With N ranks every rank computes its own structure (seed = rank, no collective on the data path) and
the job's time is the slowest rank's: rank_max must give every rank the same maximum, job_rate must
count all ranks' pairs in that time, and the reference arm runs on rank 0 only."""
import json
import os
import socket
import sys

import pytest

from conftest import ROOT

WORLD = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(WORLD))
    sys.path.insert(0, ROOT)
    import datetime

    import numpy as np
    import torch.distributed as tdist

    import bench
    tdist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank times its own replica: rank r "took" 10 (r + 1) ms
        mine = 10.0 * (rank + 1)
        slowest = bench.rank_max(mine)
        # replicas differ: the structure is seeded by the rank
        els = bench.workload(rank, cells=3)[0]
        digest = float(sum(float(np.abs(e).sum()) for e in els))
        digests = [None] * WORLD
        tdist.all_gather_object(digests, digest)
        # the reference arm: rank 0 alone runs it, the others return 0 at once without work
        skipped = rank != 0 and bench.reference_arm(None, rank, WORLD) == 0
        with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
            json.dump({"slowest": slowest, "rate": bench.job_rate(WORLD, 1000, slowest), "digests": digests,
                       "skipped": skipped}, f)
    finally:
        tdist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
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
    for r in range(WORLD):
        res = json.load(open(os.path.join(tmp_path, "rank%d.json" % r)))
        assert res["slowest"] == 20.0  # the slower rank's time, on every rank
        assert res["rate"] == pytest.approx(WORLD * 1000 / 20e-3)
        assert res["digests"][0] != res["digests"][1]  # two different structures
        if r == 1:
            assert res["skipped"]


def test_rank_max_without_a_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.rank_max(3.5) == 3.5
    assert bench.job_rate(1, 500, 2.0) == pytest.approx(250e3)
