"""Learned warm start for Airfoil: training data from the solver, training,
prediction, and time-to-tolerance against the freestream start.

Pipeline (python -m op2b.warmstart --help):
  data   converged q fields of the channel-with-bump family at I x J (default
         200 x 100) over sampled flow conditions: Mach ~ U[0.3, 0.7], angle of
         attack ~ U[-4, 6] deg, bump ~ U[0, 0.1].  Every sample shares the
         mesh topology (one seed); the bump moves the nodes, and node
         coordinates are affine in the bump height, so a sample's mesh is
         x0 + bump * dx.  Solved by the batched solver (op2b.batch), FP32
         storage until rms < tol * rms0 (or a stall, then FP64).
  train  the graph network of op2b.gnn on those fields (AdamW, cosine decay),
         every forward/backward kernel the library's own.
  solve  from freestream and from the network's prediction, plain FP64 OP2
         iteration (the five op_par_loops of airfoil.cpp) until
         rms < tol * rms0_freestream -- the same absolute tolerance for both;
         the prediction is used only if its first-iteration rms is below
         freestream's (else freestream is the fallback).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import gnn as G
from . import lib as L
from .airfoil import Airfoil
from .mesh import Mesh, airfoil_constants, channel_bump

FLOW_RANGES = dict(mach=(0.3, 0.7), alpha=(-4.0, 6.0), bump=(0.0, 0.1))


def sample_flows(n, seed):
    rng = np.random.default_rng(seed)
    return [dict(mach=float(rng.uniform(*FLOW_RANGES["mach"])),
                 alpha=float(rng.uniform(*FLOW_RANGES["alpha"])),
                 bump=float(rng.uniform(*FLOW_RANGES["bump"]))) for _ in range(n)]


class MeshFamily:
    """All bump heights of one I x J mesh (seed, numbering): x(b) = x0 + b * dx."""

    def __init__(self, I, J, seed=0, permute=False):
        self.I, self.J, self.seed, self.permute = I, J, seed, permute
        self.m0 = channel_bump(I, J, seed=seed, bump=0.0, permute=permute)
        m1 = channel_bump(I, J, seed=seed, bump=0.1, permute=permute)
        if not (np.array_equal(m1.cell, self.m0.cell) and np.array_equal(m1.edge, self.m0.edge)
                and np.array_equal(m1.bedge, self.m0.bedge)):
            raise ValueError("bump changed the mesh topology")
        self.dx = (m1.x - self.m0.x) / 0.1

    def mesh(self, bump):
        m = self.m0
        return Mesh(x=m.x + bump * self.dx, cell=m.cell, edge=m.edge, ecell=m.ecell,
                    bedge=m.bedge, becell=m.becell, bound=m.bound,
                    meta=dict(m.meta, bump=bump))


def solve_family(fam: MeshFamily, flows, tol=1e-5, max_iter=80000, chunk=1000, log=print):
    """Converged q (float32, n x ncell x 4) of every flow on the family, by the
    batched solver in chunks of `chunk` instances."""
    from .batch import AirfoilBatch
    n = len(flows)
    out = np.zeros((n, fam.m0.ncell, 4), np.float32)
    iters = np.zeros(n, np.int64)
    rel = np.zeros(n)
    for c0 in range(0, n, chunk):
        fl = flows[c0:c0 + chunk]
        L.op_init()
        try:
            specs = [dict(I=fam.I, J=fam.J, seed=fam.seed, **f) for f in fl]
            b = AirfoilBatch(specs, fp32=True, renumber=False,
                             meshes=[fam.mesh(f["bump"]) for f in fl])
            b.set("tol", tol)
            b.set("promote_tol", tol)
            b.set("max_iter", max_iter)
            t0 = time.time()
            active, ms = b.run(max_iter, check_every=500)
            st = b.stats()
            qs = b.q_final()
            for k, q in enumerate(qs):
                out[c0 + k] = q
            iters[c0:c0 + len(fl)] = st["iters"]
            rel[c0:c0 + len(fl)] = st["rms_last"] / st["rms0"]
            log(f"solved {c0 + len(fl)}/{n}: {ms / 1e3:.1f} s device, {time.time() - t0:.1f} s "
                f"wall, iterations {st['iters'].min()}..{st['iters'].max()}, "
                f"unconverged {int(active)}")
            b.close()
        finally:
            L.op_exit()
    return out, iters, rel


class Dataset:
    """Device-resident features and normalised targets of n samples on one family."""

    def __init__(self, fam: MeshFamily, flows, q, norm=None):
        import torch
        self.torch = torch
        self.fam = fam
        self.flows = flows
        self.g = G.cell_graph(fam.m0)
        n, N = len(flows), fam.m0.ncell
        dq = np.empty((n, N, 4), np.float64)
        if q is None:  # synthetic targets (timing and profiling of training only)
            dq[:] = np.random.default_rng(0).standard_normal((1, N, 4))
        for i, f in enumerate(flows if q is not None else ()):
            qinf = airfoil_constants(mach=f["mach"], alpha_deg=f["alpha"])["qinf"]
            dq[i] = q[i].astype(np.float64) - qinf
        if norm is None:
            mean = dq.reshape(-1, 4).mean(axis=0)
            std = dq.reshape(-1, 4).std(axis=0) + 1e-12
            norm = np.concatenate([mean, std])
        self.norm = np.asarray(norm, np.float64)
        t = ((dq - self.norm[:4]) / self.norm[4:]).astype(np.float32)
        del dq
        self.target = torch.from_numpy(t.reshape(n * N, 4)).cuda()
        E = self.g["E"]
        self.node_in = torch.empty(n * N, G.NODE_IN, dtype=torch.bfloat16, device="cuda")
        self.edge_in = torch.empty(n * E, G.EDGE_IN, dtype=torch.bfloat16, device="cuda")
        for i, f in enumerate(flows):
            m = fam.mesh(f["bump"])
            nf = G.node_features(m, f["mach"], f["alpha"], f["bump"])
            self.node_in[i * N:(i + 1) * N] = torch.from_numpy(nf).to(torch.bfloat16)
            self.edge_in[i * E:(i + 1) * E] = torch.from_numpy(
                G.edge_features(m, self.g)).to(torch.bfloat16)
        self.n, self.N, self.E = n, N, E

    def batch(self, s, B):
        N, E = self.N, self.E
        return (self.node_in[s * N:(s + B) * N], self.edge_in[s * E:(s + B) * E],
                self.target[s * N:(s + B) * N])


def lr_at(it, steps, lr=1e-3, lr_min=1e-5, warmup=100):
    """Linear warm-up over `warmup` steps, then cosine decay to lr_min."""
    if it < warmup:
        return lr * (it + 1) / warmup
    u = (it - warmup) / max(1, steps - warmup)
    return lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * u))


class Schedule:
    """Minibatch order: minibatch j of the run (j = step * ranks + rank under
    data parallelism) is entry j % nb of a permutation of the nb minibatches,
    drawn afresh from one seeded generator for every pass over the data, so
    that every rank draws the same permutations."""

    def __init__(self, nb, seed=0):
        self.nb = nb
        self.rng = np.random.default_rng(seed)
        self.order = self.rng.permutation(nb)
        self.epoch = 0

    def start(self, j):
        while j // self.nb > self.epoch:
            self.order = self.rng.permutation(self.nb)
            self.epoch += 1
        return int(self.order[j % self.nb])


def train(net: G.GraphNet, data: Dataset, val: Dataset | None = None, steps=3000, batch=8,
          lr=1e-3, lr_min=1e-5, warmup=100, weight_decay=1e-5, seed=0, log=print,
          log_every=100, group=None):
    """AdamW with linear warm-up and cosine decay over `steps` minibatches of
    `batch` consecutive samples.  With a torch.distributed `group`, data
    parallel: each rank takes its own minibatches (step * ranks + rank of the
    shared schedule) and the gradients are averaged before every step, so all
    ranks keep the same parameters.  Returns the loss history (this rank's
    losses) and the device time."""
    torch = net.torch
    dg = net.upload_graph(G.replicate_graph(data.g, batch))
    nb = data.n // batch
    if group is not None:
        import torch.distributed as dist
        rank, world = dist.get_rank(group), dist.get_world_size(group)
    else:
        rank, world = 0, 1
    sched = Schedule(nb, seed)
    hist = []
    t0 = time.time()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    fresh = True
    for it in range(steps):
        s = sched.start(it * world + rank) * batch
        ni, ei, tg = data.batch(s, batch)
        acc = net.loss_grad(dg, ni, ei, tg, zero_loss=fresh)
        fresh = False
        if world > 1:
            net.average_grad(group)
        lr_it = lr_at(it, steps, lr, lr_min, warmup)
        net.step(lr_it, weight_decay=weight_decay)
        if (it + 1) % log_every == 0 or it + 1 == steps:
            l = float(acc.item()) / (it % log_every + 1)
            fresh = True
            rec = dict(step=it + 1, loss=l, lr=lr_it, wall=time.time() - t0)
            if val is not None:
                rec["val"] = evaluate(net, val, batch)
            hist.append(rec)
            log(json.dumps(rec))
    ev1.record()
    torch.cuda.synchronize()
    assert G._lib().op2b_gemm_error(1) == 0, "a tensor-core GEMM timed out"
    return hist, ev0.elapsed_time(ev1)


def evaluate(net, data: Dataset, batch=8):
    """Mean normalised MSE over the dataset (forward only, training workspace)."""
    dg = net.upload_graph(G.replicate_graph(data.g, batch))
    tot = 0.0
    nb = data.n // batch
    for b in range(nb):
        ni, ei, tg = data.batch(b * batch, batch)
        out = net.forward(dg, ni, ei, train=False)
        tot += float(((out[:, :4] - tg) ** 2).mean().item())
    return tot / max(nb, 1)


def predict_q(net: G.GraphNet, mesh: Mesh, mach, alpha, bump):
    """Predicted q (ncell x 4, float64, declared cell order): qinf + mean + std * net."""
    torch = net.torch
    g = G.cell_graph(mesh)
    dg = net.upload_graph(g)
    ni = torch.from_numpy(G.node_features(mesh, mach, alpha, bump)).to(torch.bfloat16).cuda()
    ei = torch.from_numpy(G.edge_features(mesh, g)).to(torch.bfloat16).cuda()
    out = net.forward(dg, ni, ei, train=False)
    qinf = airfoil_constants(mach=mach, alpha_deg=alpha)["qinf"]
    ms = torch.from_numpy(net.norm).cuda()
    qi = torch.from_numpy(np.asarray(qinf, np.float64)).cuda()
    q = torch.empty(mesh.ncell, 4, dtype=torch.float64, device="cuda")
    G._call("op2b_gnn_decode_q", mesh.ncell, out.data_ptr(), G.OUT, ms.data_ptr(),
            qi.data_ptr(), q.data_ptr(), net.stream)
    res = q.cpu().numpy()
    net.release()
    return res


def solve(mesh: Mesh, consts, q0=None, tol_abs=None, tol_rel=None, max_iter=400000,
          renumber=True, dtype=np.float64, abort_above=None):
    """Plain OP2 iteration from q0 (freestream if None) until rms < tol_abs
    (or tol_rel * the first iteration's rms).  Returns a dict with the
    iterations, device-timed loop milliseconds, the rms history's first and
    last values, and the final q (declared order).  With abort_above, stops
    after the first iteration if its rms exceeds that value (aborted=True).
    Runs inside its own op_init / op_exit."""
    import torch
    L.op_init()
    try:
        app = Airfoil(mesh, consts, dtype=dtype, rms_only=True, q0=q0)
        if renumber:
            app.renumber()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        L.synchronize()
        t0 = time.time()
        e0.record()
        h = app.iterate(1)
        rms0 = h[0][0]
        tol = tol_abs if tol_abs is not None else tol_rel * rms0
        it, rms = 1, rms0
        aborted = abort_above is not None and not (rms0 <= abort_above)   # NaN aborts too
        while not aborted and rms >= tol and it < max_iter:
            rms = app.iterate(1)[0][0]
            it += 1
        e1.record()
        L.synchronize()
        torch.cuda.synchronize()
        wall = time.time() - t0
        q = app.fetch_original().astype(np.float64)
        return dict(iterations=it, ms=e0.elapsed_time(e1), wall_s=wall, rms0=rms0, rms=rms,
                    converged=bool(rms < tol), aborted=bool(aborted), q=q)
    finally:
        L.op_exit()


def warm_vs_freestream(net, mesh, flow, tol_rel=1e-5, max_iter=400000, renumber=True, log=print):
    """Time-to-tolerance from freestream and from the network's prediction, at
    the same absolute tolerance tol_rel * rms0(freestream)."""
    import torch
    c = airfoil_constants(mach=flow["mach"], alpha_deg=flow["alpha"])
    free = solve(mesh, c, None, tol_rel=tol_rel, max_iter=max_iter, renumber=renumber)
    log(f"freestream: {free['iterations']} iterations, {free['ms']:.0f} ms")
    tol_abs = tol_rel * free["rms0"]
    t0 = time.time()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    q0 = predict_q(net, mesh, flow["mach"], flow["alpha"], flow["bump"])
    e1.record()
    torch.cuda.synchronize()
    infer_ms = e0.elapsed_time(e1)
    infer_wall = time.time() - t0
    warm = solve(mesh, c, q0, tol_abs=tol_abs, max_iter=max_iter, renumber=renumber,
                 abort_above=free["rms0"])
    fallback = warm["aborted"]
    if fallback:
        # the prediction's first residual is above freestream's: the solve falls
        # back to freestream (whose run above is that answer), after one wasted
        # iteration
        warm = dict(free, iterations=free["iterations"] + 1, ms=free["ms"] + warm["ms"])
    log(f"warm: {warm['iterations']} iterations, {warm['ms']:.0f} ms (+{infer_ms:.0f} ms "
        f"inference), first rms {warm['rms0']:.3e} vs freestream {free['rms0']:.3e}")
    qerr = np.abs(q0 - free["q"]).max(axis=0) / np.abs(free["q"]).max(axis=0)
    return dict(free={k: v for k, v in free.items() if k != "q"},
                warm={k: v for k, v in warm.items() if k != "q"},
                inference_ms=infer_ms, inference_wall_s=infer_wall, fallback=bool(fallback),
                pred_max_rel_err=qerr.tolist(), tol_abs=tol_abs,
                iteration_ratio=warm["iterations"] / free["iterations"],
                time_ratio=(warm["ms"] + infer_ms) / free["ms"])


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--samples", type=int, default=2000)
    ap.add_argument("--I", type=int, default=200)
    ap.add_argument("--J", type=int, default=100)
    ap.add_argument("--tol", type=float, default=1e-5)
    ap.add_argument("--max-iter", type=int, default=80000)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--mp-steps", type=int, default=8)
    ap.add_argument("--val", type=int, default=64)
    ap.add_argument("--data", default=None, help="npz of solved fields (reuse or write)")
    ap.add_argument("--out", default=None, help="npz for the trained network")
    ap.add_argument("--eval", nargs="*", default=[],
                    help="meshes to evaluate: IxJ[:flows[:tol]], e.g. 480x240:2:1e-5")
    ap.add_argument("--eval-tol", type=float, default=1e-5)
    ap.add_argument("--eval-flows", type=int, default=1)
    ap.add_argument("--eval-max-iter", type=int, default=600000)
    ap.add_argument("--load", default=None, help="trained network npz (skip training)")
    ap.add_argument("--report", default=None, help="json report path")
    ap.add_argument("--synthetic", action="store_true",
                    help="random targets instead of solved fields (timing/profiling of training)")
    ap.add_argument("--log-every", type=int, default=100)
    ap.add_argument("--dp-backend", default="nccl", choices=["nccl", "gloo"],
                    help="under torchrun (WORLD_SIZE > 1) training is data parallel; the "
                         "gradient all-reduce's backend (gloo: ranks may share a GPU)")
    ap.add_argument("--gemm-tma", type=int, default=1,
                    help="1: forward products on the TMA-fed tensor-core GEMM; 0: all on the "
                         "register-staged one")
    a = ap.parse_args(argv)
    G.GEMM_TMA = bool(a.gemm_tma)
    log = lambda s: print(s, flush=True)
    report = dict(args=vars(a))
    group, rank = None, 0
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")) % torch.cuda.device_count())
        dist.init_process_group(a.dp_backend, timeout=datetime.timedelta(seconds=300))
        group, rank = dist.group.WORLD, dist.get_rank()
        report["ranks"] = dist.get_world_size()
        if rank:  # rank 0 reports and writes; every rank trains
            log = lambda s: None
            a.out = a.report = None
            a.eval = []
    if a.load:
        net = G.GraphNet.load(a.load)
    else:
        fam = MeshFamily(a.I, a.J, seed=0, permute=False)
        flows = sample_flows(a.samples + a.val, seed=1)
        if a.synthetic:
            q = None
        elif a.data and os.path.exists(a.data):
            z = np.load(a.data)
            q, iters = z["q"], z["iters"]
        else:
            t0 = time.time()
            q, iters, rel = solve_family(fam, flows, tol=a.tol, max_iter=a.max_iter, log=log)
            report["data_s"] = time.time() - t0
            report["data_iters"] = [int(iters.min()), int(np.median(iters)), int(iters.max())]
            if a.data:
                np.savez(a.data, q=q, iters=iters)
        tr = Dataset(fam, flows[:a.samples], None if q is None else q[:a.samples])
        va = Dataset(fam, flows[a.samples:], None if q is None else q[a.samples:],
                     norm=tr.norm) if a.val else None
        net = G.GraphNet(steps=a.mp_steps, seed=0, norm=tr.norm)
        hist, ms = train(net, tr, va, steps=a.steps, batch=a.batch, lr=a.lr, log=log,
                         log_every=a.log_every, group=group)
        report["train"] = dict(ms=ms, ms_per_step=ms / max(a.steps, 1), history=hist,
                               launches=net.launches)
        if a.out:
            net.save(a.out)
        if a.report:
            with open(a.report, "w") as fh:
                json.dump(report, fh, indent=1, default=float)
        del tr, va
    ev = []
    for spec in a.eval:
        # IxJ[:flows[:tol]]
        parts = spec.split(":")
        I, J = (int(v) for v in parts[0].split("x"))
        nflow = int(parts[1]) if len(parts) > 1 else a.eval_flows
        tol = float(parts[2]) if len(parts) > 2 else a.eval_tol
        for k, f in enumerate(sample_flows(nflow, seed=100 + I)):
            mesh = channel_bump(I, J, seed=7 + k, bump=f["bump"])
            r = warm_vs_freestream(net, mesh, f, tol_rel=tol, max_iter=a.eval_max_iter, log=log)
            r.update(mesh=parts[0], flow=f, tol_rel=tol)
            ev.append(r)
            log(json.dumps({k2: v for k2, v in r.items() if k2 not in ("free", "warm")}))
            if a.report:
                with open(a.report, "w") as fh:
                    json.dump(dict(report, eval=ev), fh, indent=1, default=float)
    report["eval"] = ev
    if a.report:
        with open(a.report, "w") as fh:
            json.dump(report, fh, indent=1, default=float)
    if group is not None:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
