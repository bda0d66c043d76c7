"""The N > 1 path of the benchmark on CPU: two gloo ranks (replicas, no data-path
collective).  Checks the max / sum over ranks the JSON line is built from and that
each rank draws its own held-out instances (weak scaling)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        t_max = bench.max_over_ranks(10.0 + rank, world)
        solved = bench.sum_over_ranks(100.0 + rank, world)
        bench.barrier(world)

        class A:
            heldout = 8
        _, _, P = bench.learned_setup(A, rank)
        q.put((rank, t_max, solved, P[0, :4].tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [11.0, 11.0]     # max over ranks, seen by every rank
    assert [o[2] for o in out] == [201.0, 201.0]   # sum over ranks
    assert not np.allclose(out[0][3], out[1][3])   # each rank solves its own instances
