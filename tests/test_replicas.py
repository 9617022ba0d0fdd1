"""Multi-rank path on CPU (gloo, world size 2): each rank holds its own
walker population; only timing and the energy accumulators are reduced."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from qmcbeaver_b200.replicas import aggregate_timing, reduce_energy, replica_seed, trial_energy


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms, moves = aggregate_timing(10.0 + rank, 1000.0 * (rank + 1))
        e = reduce_energy(sum_w=2.0 + rank, sum_we=-2.0 * (2.0 + rank) * (1 + rank), sum_we2=8.0 + rank,
                          n_walkers=100 + rank, weight=50.0 + rank)
        q.put((rank, ms, moves, e, replica_seed(77, rank)))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, ms, moves, e, seed in res:
        assert ms == 11.0 and moves == 3000.0
        assert e["walkers"] == 201 and e["weight"] == 101.0
        # sum_we = -2*2*1 + -2*3*2 = -16, sum_w = 5
        assert abs(e["energy"] - (-16.0 / 5.0)) < 1e-12
    assert res[0][4] != res[1][4]


def test_single_process_passthrough():
    assert aggregate_timing(3.0, 7.0) == (3.0, 7.0)
    e = reduce_energy(2.0, -4.0, 9.0, 5, 2.0)
    assert e["energy"] == -2.0 and abs(e["variance"] - 0.5) < 1e-12
    assert abs(trial_energy(-2.0, 20.0, 10.0, 1.0) - (-2.0 - __import__("math").log(2.0))) < 1e-12
