"""The multi-GPU plumbing of bench.py on CPU: two ranks over gloo (no GPU).

bench.py runs one process per GPU (replicas: every rank runs the same MSM on its own GPU, no data
exchange); the job's time is the maximum over ranks and its rate is ranks x points / that time.
Here two CPU ranks feed different times through the same helpers and must agree on the result.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        ms = [12.5, 17.25][rank]
        ms_max = bench.max_over_ranks(torch, dist, world, ms, device="cpu")
        rate = bench.whole_job_rate(1 << 22, world, ms_max)
        q.put((rank, ms_max, rate))
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_is_the_slowest_and_rate_counts_all_ranks():
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
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [17.25, 17.25]
    want = 2 * (1 << 22) / 17.25e-3
    assert all(abs(r[2] - want) < 1e-6 * want for r in res)


def test_single_rank_helpers():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(torch, None, 1, 3.5, device="cpu") == 3.5
    assert bench.whole_job_rate(1000, 1, 2.0) == pytest.approx(5e5)
