"""Sharding of independent models across ranks: the partition is balanced and
complete, and a world-size-2 gloo run (CPU, the oracle as the per-rank solver)
gathers every model's solution on every rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rustyfem_b200 import shard
from rustyfem_b200 import workloads as W


def test_partition_balanced_and_complete():
    sizes = W.plate_sizes(512, seed=0)
    work = [nx ** 2.2 for nx, _ in sizes]
    for world in (1, 2, 4, 8):
        shares = shard.partition(work, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(512))
        assert shard.imbalance(work, shares) < 1.02


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    from oracle import refcpu

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    models = [W.plate(nx, ny).full() for nx, ny in W.plate_sizes(10, seed=4)]
    work = [refcpu.Symbolic(m.graph, 16).work() for m in models]
    shares = shard.partition(work, world)
    local = {}
    for i in shares[rank]:
        h, _, _ = refcpu.factor(models[i])
        local[i] = h.solve(models[i].rhs)
    merged = shard.gather_solutions(local, world, dist)
    out[rank] = {k: v.tolist() for k, v in merged.items()}
    dist.destroy_process_group()


def test_gloo_world2_gather():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        res = dict(out)
    assert set(res[0]) == set(range(10)) and res[0].keys() == res[1].keys()
    models = [W.plate(nx, ny).full() for nx, ny in W.plate_sizes(10, seed=4)]
    for i, m in enumerate(models):
        x = np.array(res[0][i])
        assert np.array_equal(x, np.array(res[1][i]))
        assert np.linalg.norm(m.matvec(x) - m.rhs) / np.linalg.norm(m.rhs) < 1e-8
