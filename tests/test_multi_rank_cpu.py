"""The multi-rank host logic of bench.py on CPU: two gloo ranks, no GPU.

Trees do not shard (one tree per GPU, replicas), and batched systems are
partitioned across ranks with no exchange; what crosses ranks is only the
timing reduction.  Checked here: the max-over-ranks reduction every rank
takes part in, the whole-job rate from it, and a partition of independent
systems that gives every system to exactly one rank with balanced loads.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, sizes, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank "measured" a different time; all must agree on the slowest
        slowest = bench.max_over_ranks(10.0 + 5.0 * rank, world, torch.device("cpu"))
        owner = bench.partition_by_particles(sizes, world)
        mine = [k for k in range(len(sizes)) if owner[k] == rank]
        shares = [None] * world
        dist.all_gather_object(shares, mine)
        out.put((rank, slowest, shares))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_timings_and_partition_systems():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    world = 2
    sizes = np.floor(10.0 ** np.random.default_rng(4).uniform(3.0, 6.0, 64)).astype(np.int64)
    port = _free_port()
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, shares in results:
        assert slowest == 15.0  # the max over both ranks, seen by each
        covered = sorted(k for share in shares for k in share)
        assert covered == list(range(len(sizes)))  # every system exactly once
        loads = [int(sizes[share].sum()) for share in shares]
        assert max(loads) - min(loads) <= int(sizes.max())  # greedy balance bound
    # whole-job rate: all ranks' units over the slowest rank's time
    assert bench.job_rate(2 * 1000, 15.0) == pytest.approx(2000 / 0.015)


def test_partition_is_deterministic_and_single_rank_owns_all():
    sizes = [5, 3, 3, 2, 2, 2, 1]
    assert bench.partition_by_particles(sizes, 1) == [0] * len(sizes)
    a = bench.partition_by_particles(sizes, 3)
    assert a == bench.partition_by_particles(sizes, 3)
    loads = [sum(s for s, o in zip(sizes, a) if o == r) for r in range(3)]
    assert sum(loads) == sum(sizes) and max(loads) - min(loads) <= max(sizes)
