"""The multi-rank plumbing of bench.py on CPU with the gloo backend (2 ranks):
each rank simulates its own seeded scene (replicas, no data-path collective)
and the timings are reduced to the slowest rank."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(1.5 + rank, world, "cpu")
        s = bench.make_scene("config1", rank)
        out[rank] = (t, s.n, float(s.x[s.type == 2].sum()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_max_and_run_distinct_replicas():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.5  # the slowest rank's time on every rank
    assert res[0][1] == res[1][1]  # equal work per rank (weak scaling)
    assert res[0][2] != res[1][2]  # different seeds: debris placed differently


def test_single_rank_needs_no_process_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1, "cpu") == 3.25
