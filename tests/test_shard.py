"""Sharding batched instances over ranks (op2b/shard.py) on the host: the LPT
partition, and a world-size-2 gloo run whose per-rank solver is a stand-in
(each 'solve' returns values derived from the instance), checking that every
instance is solved exactly once and the results come back in order."""
import os
import socket

import numpy as np
import pytest

from op2b import shard
from op2b.batch import sample_instances


def test_partition_is_balanced_and_complete():
    rng = np.random.default_rng(0)
    cells = rng.integers(10_000, 500_000, size=64)
    for world in (1, 2, 3, 4, 8):
        parts = shard.partition(cells, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [cells[p].sum() for p in parts]
        # LPT bound: makespan <= 4/3 optimum; optimum >= max(mean load, largest item)
        lower = max(cells.sum() / world, cells.max())
        assert max(loads) <= 4 / 3 * lower + 1
    assert shard.partition([5, 5], 2) == [[0], [1]]
    with pytest.raises(ValueError):
        shard.partition([1], 0)


def _fake_solve(specs, **kw):
    return dict(iters=[s["I"] * 10 for s in specs], iters32=[s["I"] for s in specs],
                rms0=[float(s["J"]) for s in specs], rms_last=[s["mach"] for s in specs],
                phase=[2] * len(specs), ms=float(sum(s["I"] * s["J"] for s in specs)))


def _worker(rank, world, port, specs, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = shard.run_sharded(specs, solve=_fake_solve)
        if rank == 0:
            q.put(out)
        else:
            q.put(None if out is None else "rank1 returned a result")
    finally:
        dist.destroy_process_group()


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_gloo_run_gathers_every_instance_once():
    import torch.multiprocessing as mp
    specs = sample_instances(11, seed=5, cells=(100, 4000))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, specs, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out = [g for g in got if isinstance(g, dict)]
    assert len(out) == 1 and None in got
    out = out[0]
    want = _fake_solve(specs)
    for k in ("iters", "iters32", "rms0", "rms_last"):
        assert out[k] == want[k]
    assert sorted(set(out["rank_of"])) == [0, 1]
    parts = shard.partition([shard.instance_cells(s) for s in specs], 2)
    for r, p in enumerate(parts):
        assert all(out["rank_of"][i] == r for i in p)
    assert out["ms"] == max(out["rank_ms"])
