"""The bench's multi-rank plumbing on CPU: two gloo ranks line up with the
barrier and agree on the slowest rank's time (max over ranks), as
`bench.py --gpus N` does over NCCL with one replica per GPU."""

import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench

    barrier, max_over_ranks, dist = bench.rank_sync(world, backend="gloo", device="cpu")
    barrier()
    q.put((rank, max_over_ranks(1.0 + rank)))
    barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in ps)
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2.0), (1, 2.0)]


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    barrier, max_over_ranks, dist = bench.rank_sync(1, backend="gloo", device="cpu")
    barrier()
    assert dist is None and max_over_ranks(3.5) == 3.5
