"""Data-parallel training of the learned warm start (op2b.warmstart.train
with a torch.distributed group, GraphNet.average_grad): two ranks, each
training on its own minibatches and averaging gradients before every AdamW
step, end with the parameters of one process that computes both ranks'
gradients per step and averages them itself.  The ranks run as two processes
on one GPU with gloo (the all-reduce goes through host memory; no kernel
waits for the other rank); NCCL between GPUs takes the same code path with an
on-device all-reduce.  The backward pass's split-K products add with atomics,
so gradients agree to rounding, not bit for bit, and AdamW magnifies that
rounding on parameters whose gradients are near zero: the emulation run twice
has differed from itself by 1.7e-5 to 2.1e-3 of the update's norm between
runs, the data-parallel parameters from it by 5e-4 to 2.1e-3.  The test
asks for at most 1e-2, and at least twenty times closer than training on
rank 0's minibatches alone (0.19 away)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS, BATCH, MP = 6, 4, 4


def _data():
    from op2b import warmstart as W
    fam = W.MeshFamily(20, 10, seed=0)
    return W.Dataset(fam, W.sample_flows(16, seed=3), None)   # seeded synthetic targets


def _worker(rank, world, init_file, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank,
                            world_size=world)
    from op2b import gnn as G, lib as L, warmstart as W
    L.load()
    data = _data()
    net = G.GraphNet(steps=MP, seed=0, norm=data.norm)
    W.train(net, data, steps=STEPS, batch=BATCH, warmup=2, log=lambda s: None,
            group=dist.group.WORLD)
    if rank == 0:
        np.save(out, net.params())
    dist.barrier()
    dist.destroy_process_group()


def _emulate(ranks):
    """One process: per step the gradients of the given ranks' minibatches,
    averaged, then the AdamW step."""
    from op2b import gnn as G, warmstart as W
    data = _data()
    net = G.GraphNet(steps=MP, seed=0, norm=data.norm)
    p0 = net.params().copy()
    dg = net.upload_graph(G.replicate_graph(data.g, BATCH))
    sched = W.Schedule(data.n // BATCH, 0)
    for it in range(STEPS):
        gs = []
        for r in ranks:
            ni, ei, tg = data.batch(sched.start(it * 2 + r) * BATCH, BATCH)
            net.loss_grad(dg, ni, ei, tg)
            gs.append(net.g.clone())
            net.zero_grad()
        net.g.copy_(sum(gs[1:], gs[0]) / len(gs))
        net.step(W.lr_at(it, STEPS, 1e-3, 1e-5, 2), weight_decay=1e-5)
    net.torch.cuda.synchronize()
    return p0, net.params()


def test_two_ranks_train_as_one_process_averaging_their_gradients(tmp_path):
    import torch.multiprocessing as mp
    from op2b import build
    build.build()
    out = str(tmp_path / "p.npy")
    mp.spawn(_worker, args=(2, str(tmp_path / "init"), out), nprocs=2, join=True)
    p_dp = np.load(out)
    p0, p_avg = _emulate([0, 1])
    _, p_avg2 = _emulate([0, 1])
    _, p_one = _emulate([0])
    upd = np.linalg.norm(p_avg - p0)
    rel = lambda p: float(np.linalg.norm(p - p_avg) / upd)
    print(f"update {upd:.3e}; relative distance: data parallel {rel(p_dp):.3e}, the same "
          f"emulation again {rel(p_avg2):.3e}, rank 0 alone {rel(p_one):.3e}")
    assert upd > 0
    assert rel(p_one) >= 0.1
    assert rel(p_dp) <= 1e-2 and rel(p_dp) <= 0.05 * rel(p_one)
