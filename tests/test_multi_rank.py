"""The bench's multi-rank path on CPU: two gloo ranks split the roots and
combine their times and counts exactly as `bench.py --gpus N` does under
torchrun (no GPU; the enumeration itself is per rank and has no exchange)."""
from __future__ import annotations

import datetime
import multiprocessing as mp
import os
import socket

import numpy as np

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m = 1_000_003
        full = bench.rank_roots(m, rank, world, True, 0)
        sample = bench.rank_roots(m, rank, world, False, 64)
        t = bench.reduce_over_ranks(0.5 + rank, dist.ReduceOp.MAX, world, "cpu")
        c = bench.reduce_over_ranks(10 * (rank + 1), dist.ReduceOp.SUM, world, "cpu")
        q.put((rank, int(full[0]), int(full[-1]), len(full), sample.tolist(), t, c))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_roots_and_combine():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, a0, b0, n0, s0, t0, c0), (r1, a1, b1, n1, s1, t1, c1) = out
    # contiguous shares partition [0, m)
    assert (a0, b0 + 1, b1 + 1) == (0, a1, 1_000_003) and n0 + n1 == 1_000_003
    # each rank's sample: sorted, distinct, in range, seeded per rank
    for smp in (s0, s1):
        assert len(smp) == 64 and smp == sorted(set(smp)) and smp[-1] < 1_000_003
    assert s0 != s1
    # job time is the slowest rank, cliques the sum
    assert t0 == t1 == 1.5 and c0 == c1 == 30.0


def test_single_rank_is_identity():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_over_ranks(2.5, None, 1, "cpu") == 2.5
    r = bench.rank_roots(10, 0, 1, True, 0)
    assert np.array_equal(r, np.arange(10, dtype=np.uint64))
