"""Ensemble sharding across ranks (host logic, CPU, gloo, world size 2):
boxes are partitioned by particle count, each rank steps only its boxes
(here with the CPU oracle standing in for the GPU engine), and rank 0
gathers per-box summaries equal to stepping every box locally."""
import copy
import os
import socket

import numpy
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from sphere_b200 import ensemble, scenes


def _boxes():
    return [scenes.lattice_pack(n, seed=k, periodic=1, nw=1, wmode=1, sid="box%d" % k)
            for k, n in enumerate([120, 300, 80, 200, 150])]


def _oracle_steps(sims, steps):
    import oracle as O
    out = []
    for s in sims:
        run = O.CpuRun(s, "oracle")
        run.step(steps)
        out.append(run.to_sim(copy.deepcopy(s)))
    return out


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = ensemble.run_rank(_boxes(), 5, rank, world, _oracle_steps)
        if rank == 0:
            q.put(res)
    finally:
        dist.destroy_process_group()


def test_partition_balances_and_covers():
    counts = [500, 20000, 7000, 300, 12000, 9000, 800]
    parts = ensemble.partition(counts, 3)
    flat = sorted(b for p in parts for b in p)
    assert flat == list(range(len(counts)))
    loads = [sum(counts[b] for b in p) for p in parts]
    assert max(loads) - min(loads) <= max(counts)
    assert ensemble.partition([5], 4)[0] == [0]


def test_gather_matches_local_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    local = [ensemble.summary(s) for s in _oracle_steps(_boxes(), 5)]
    assert res == local
