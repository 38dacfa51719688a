"""Host side of data-parallel warm-start training (no GPU): the shared
minibatch schedule (every rank draws the same permutations; ranks take
disjoint minibatches of each step, and one rank reproduces the schedule a
single process used before), the learning-rate schedule, and the gradient
average over a world-size-2 gloo group (GraphNet.average_grad on host
tensors)."""
import math
import os
import socket

import numpy as np
import pytest

from op2b import warmstart as W


def test_schedule_partitions_each_step_and_matches_the_single_process_order():
    # two ranks, each with its own copy of the schedule: over a pass (4 steps
    # of 2 minibatches) they take all 8 minibatches between them, none twice
    a, b = W.Schedule(8, seed=5), W.Schedule(8, seed=5)
    for e in range(3):
        got = [a.start(it * 2) for it in range(4 * e, 4 * e + 4)] + \
              [b.start(it * 2 + 1) for it in range(4 * e, 4 * e + 4)]
        assert sorted(got) == list(range(8))
    nb = 7
    # each pass over the data visits every minibatch once
    s = W.Schedule(nb, seed=3)
    for e in range(3):
        assert sorted(s.start(e * nb + j) for j in range(nb)) == list(range(nb))
    # one rank: the order a single process used (a fresh permutation per pass)
    rng = np.random.default_rng(3)
    ref = []
    for e in range(3):
        ref += list(rng.permutation(nb))
    s = W.Schedule(nb, seed=3)
    assert [s.start(j) for j in range(3 * nb)] == [int(v) for v in ref]


def test_learning_rate_warms_up_then_decays():
    lr = [W.lr_at(i, 100, 1e-3, 1e-5, 10) for i in range(100)]
    assert lr[0] == pytest.approx(1e-4) and lr[9] == pytest.approx(1e-3)
    assert lr[10] == pytest.approx(1e-3)
    assert all(x >= y for x, y in zip(lr[10:], lr[11:]))
    assert lr[-1] == pytest.approx(1e-5 + 0.5 * (1e-3 - 1e-5) * (1 + math.cos(math.pi * 89 / 90)))


class _Grad:
    def __init__(self, g):
        self.g = g


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from op2b import gnn as G
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        h = _Grad(torch.arange(6, dtype=torch.float32) * (rank + 1) + rank)
        G.GraphNet.average_grad(h, dist.group.WORLD)
        q.put((rank, h.g.numpy().tolist()))
    finally:
        dist.destroy_process_group()


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_gradient_average_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = ((np.arange(6) * 1 + 0) + (np.arange(6) * 2 + 1)) / 2
    assert np.array_equal(out[0], want) and np.array_equal(out[1], want)
