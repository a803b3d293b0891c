"""The multi-GPU bench path on CPU: two gloo ranks exercise the max-over-ranks timing and
the per-rank (weak scaling) populations without a GPU."""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    t = bench.reduce_max(1.0 + rank, world)
    bench.barrier(world)
    pos, _, _, _, _ = bench.workload(8, seed=21 + rank)
    out[rank] = (t, float(pos[0, 0]))
    dist.destroy_process_group()


def test_two_rank_timing_and_populations():
    import torch.multiprocessing as mp

    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0][0] == out[1][0] == 2.0  # both ranks see the slowest rank's time
    assert out[0][1] != out[1][1]  # each rank propagates its own population
