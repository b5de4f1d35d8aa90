"""Ensembles of independent boxes across GPUs.

An ensemble (many independent simulation boxes) shards without any
data-path exchange: each rank steps its own subset of boxes in one handle
(one set of kernel launches for all of its boxes) and only per-box summaries
travel, once, to rank 0.  Boxes are assigned by particle count with the
longest-processing-time rule so that ranks get near-equal work.
"""
import numpy


def partition(counts, world):
    """Assign boxes (particle counts `counts`) to `world` ranks: largest box
    first, each to the least-loaded rank.  Returns one ascending list of box
    indexes per rank."""
    counts = numpy.asarray(counts, dtype=numpy.int64)
    load = numpy.zeros(world, dtype=numpy.int64)
    parts = [[] for _ in range(world)]
    for b in numpy.argsort(-counts, kind="stable"):
        r = int(numpy.argmin(load))
        parts[r].append(int(b))
        load[r] += counts[b]
    return [sorted(p) for p in parts]


def summary(s):
    """Per-box result sent to rank 0: time, top-wall position and force,
    kinetic energy, mean position."""
    return {
        "sid": s.sid,
        "t": float(s.time_current[0]),
        "wall_x": float(s.w_x[0]) if int(s.nw[0]) > 0 else None,
        "wall_force": float(s.w_force[0]) if int(s.nw[0]) > 0 else None,
        "kinetic": float(s.totalKineticEnergy()),
        "x_mean": [float(v) for v in numpy.mean(s.x, axis=0)],
    }


def run_rank(sims, steps, rank, world, step_fn, group=None):
    """Step this rank's share of `sims` (the same list on every rank) with
    step_fn(list_of_sims, steps) -> list_of_sims, then gather the per-box
    summaries on rank 0 in box order.  Returns the gathered list on rank 0
    and None elsewhere.  Collective: every rank calls it once."""
    import torch.distributed as dist
    parts = partition([int(s.np[0]) for s in sims], world)
    mine = [sims[b] for b in parts[rank]]
    done = step_fn(mine, steps) if mine else []
    local = list(zip(parts[rank], [summary(s) for s in done]))
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(local, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(sims)
    for chunk in gathered:
        for b, summ in chunk:
            out[b] = summ
    return out
