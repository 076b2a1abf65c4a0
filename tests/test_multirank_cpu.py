"""The multi-rank bench path on CPU (two gloo ranks): codewords are independent, so
N ranks each decode their own seeded batch (weak scaling) and the job's time is the
slowest rank's, taken with one MAX all-reduce that every rank joins; the whole-job
throughput counts every rank's information bits over that time."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, dist, "cpu")
        gbps = bench.whole_job_gbps(16384, 10, world, ms)
        info, llr = bench.make_data(3, rank)
        q.put((rank, ms, gbps, int(info.sum()), int(np.abs(llr.astype(np.int32)).sum())))
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_and_throughput():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    (_, ms0, g0, i0, l0), (_, ms1, g1, i1, l1) = got
    assert ms0 == ms1 == 15.0  # the slowest rank's time on every rank
    want = 2 * 16384 * 10 * 8448 / 15e-3 / 1e9
    assert abs(g0 - want) < 1e-9 and g0 == g1
    assert (i0, l0) != (i1, l1)  # each rank decodes its own codewords


def test_one_rank_needs_no_collective():
    import bench

    assert bench.max_over_ranks(12.5, 1) == 12.5
    assert abs(bench.whole_job_gbps(16384, 10, 1, 100.0) - 16384 * 10 * 8448 / 0.1 / 1e9) < 1e-9
