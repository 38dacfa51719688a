"""Batched Airfoil across GPUs: one process per GPU, instances partitioned by
cell count, no collective on the data path.

Independent instances shard without any exchange: each rank solves its own
share with the batched solver (op2b.batch) and only the per-instance results
(iterations, rms, phase, optional q) travel, once, at the end.  Partitioning
is greedy longest-processing-time: instances in decreasing cell count, each to
the rank with the least cells so far (ties to the lower rank) -- within 4/3 of
the optimal makespan, deterministic, and identical on every rank.

The process group is torch.distributed (NCCL on GPUs, gloo on the host); the
gather uses gather_object on the host side, so the same code runs in the CPU
tests.
"""
from __future__ import annotations

import numpy as np


def partition(cells, world: int):
    """Greedy LPT: list of instance indices per rank."""
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(cells[i])
    return [sorted(p) for p in parts]


def instance_cells(spec):
    return int(spec["I"]) * int(spec["J"])


def solve_local(specs, tol=1e-6, promote_tol=1e-4, max_iter=2_000_000, check_every=500,
                fp32=True):
    """Solve `specs` on this process's GPU with the batched solver; per-instance
    results in the order of `specs`."""
    from . import lib as L
    from .batch import AirfoilBatch
    if not specs:
        return dict(iters=[], iters32=[], rms0=[], rms_last=[], phase=[], ms=0.0)
    L.op_init()
    try:
        b = AirfoilBatch(specs, fp32=fp32)
        b.set("tol", tol)
        b.set("promote_tol", promote_tol)
        b.set("max_iter", max_iter)
        _active, ms = b.run(max_iter, check_every=check_every)
        st = b.stats()
        b.close()
        return dict(iters=st["iters"].tolist(), iters32=st["iters32"].tolist(),
                    rms0=st["rms0"].tolist(), rms_last=st["rms_last"].tolist(),
                    phase=st["phase"].tolist(), ms=ms)
    finally:
        L.op_exit()


def run_sharded(specs, solve=solve_local, **kw):
    """Every rank solves its partition; rank 0 returns the merged results in
    the caller's instance order (other ranks return None).  `solve` is the
    per-rank solver (a stand-in in the host-only tests)."""
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_initialized() else 1
    rank = dist.get_rank() if dist.is_initialized() else 0
    parts = partition([instance_cells(s) for s in specs], world)
    mine = parts[rank]
    res = solve([specs[i] for i in mine], **kw)
    res["rank"] = rank
    res["instances"] = mine
    if world == 1:
        gathered = [res]
    else:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(res, gathered, dst=0)
    if rank != 0:
        return None
    n = len(specs)
    out = {k: [None] * n for k in ("iters", "iters32", "rms0", "rms_last", "phase")}
    out["rank_of"] = [None] * n
    out["rank_ms"] = [0.0] * world
    for r in gathered:
        out["rank_ms"][r["rank"]] = r["ms"]
        for j, i in enumerate(r["instances"]):
            for k in ("iters", "iters32", "rms0", "rms_last", "phase"):
                out[k][i] = r[k][j]
            out["rank_of"][i] = r["rank"]
    out["ms"] = max(out["rank_ms"])  # the job ends with its slowest rank
    out["loads"] = [int(np.sum([instance_cells(specs[i]) for i in p])) for p in parts]
    return out
