"""The multi-GPU bench path on CPU: two gloo ranks, world size 2.

bench.py runs N independent replicas (one process per GPU, no collective on the
data path), each on its own seeded parameter rows; the step time is the largest
of the ranks' device times (one max all-reduce, taken by every rank) and the
whole-job rate counts every rank's evaluations.  These ranks run the same
helpers with CPU tensors over gloo.
"""

import os
import socket

import numpy as np
import pytest

WORLD = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out):
    import sys
    from datetime import timedelta

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=WORLD, timeout=timedelta(seconds=60))
    try:
        P = bench.replica_parameters(11, rank, 4, 6)
        # rank-dependent device times: the job step is the slowest rank's
        ms = [3.0, 5.0][rank]
        ms_all = bench.max_over_ranks(ms, WORLD, "cpu")
        ms_e2e = bench.max_over_ranks(ms + 1.0, WORLD, "cpu")
        dist.barrier()
        out.put((rank, P, ms_all, ms_e2e, bench.whole_job_rate(WORLD, 4, ms_all)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_combine_like_the_bench():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(WORLD):
        r, P, ms_all, ms_e2e, rate = q.get(timeout=120)
        got[r] = (P, ms_all, ms_e2e, rate)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(WORLD):
        P, ms_all, ms_e2e, rate = got[r]
        # every rank sees the slowest rank's step time
        assert ms_all == 5.0 and ms_e2e == 6.0
        assert rate == pytest.approx(WORLD * 4 / 5e-3)
        assert P.shape == (4, 6) and np.all(np.abs(P) <= 0.1)
    # each replica evaluates its own rows, reproducibly
    assert not np.allclose(got[0][0], got[1][0])
    import bench  # noqa: E402  (conftest puts the repository root on sys.path)
    assert np.array_equal(got[1][0], bench.replica_parameters(11, 1, 4, 6))


def test_single_rank_takes_no_collective():
    import bench
    # world size 1: no process group exists, the value passes through
    assert bench.max_over_ranks(2.5, 1, "cpu") == 2.5
    assert bench.whole_job_rate(1, 256, 2.0) == pytest.approx(128000.0)
