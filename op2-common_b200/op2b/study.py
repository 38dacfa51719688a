"""Forms study: the mixed-precision and batched forms against plain FP64.

  python -m op2b.study mixed-error [--I 2400 --J 1200 --iters 2000]
  python -m op2b.study mixed-ttt   [--I 480 --J 240 --tol 1e-5]
  python -m op2b.study batch       [--n 64 --tol 1e-6 --plain api|graph|none
                                    --plain-subset K --subset-seed S]

Each prints one JSON object per line.

* mixed-error: the same renumbered mesh iterated `iters` times in plain FP64
  and in the mixed form (q, x, adt, res stored and fluxes computed in FP32;
  the update's arithmetic, rms and the convergence test in FP64); per field
  of q the relative L2 and max errors of the mixed q against the FP64 q, and
  the rms history's relative error.  The FP64 path stands in for the FP64
  oracle at this size: in its default owner-computes mode it reproduces the
  reference's sequential build bit for bit (tests/test_airfoil_gpu.py).
* mixed-ttt: time to an rms tolerance on one mesh, plain FP64 from freestream
  against the mixed form followed by FP64 (FP32 storage until rms falls below
  promote * rms1 or stops falling, then FP64 from that state) to the same
  absolute tolerance tol * rms1, rms1 being plain FP64's first-iteration rms.
* batch: many instances of uneven size and flow condition (cells log-uniform
  in [10K, 500K], Mach in [0.3, 0.7], alpha in [-4, 6] degrees, bump in
  [0, 0.1]) to rms < tol * rms0 each: the batched form (one persistent launch
  per loop stage over all instances, a CUDA graph per iteration, autotuned,
  FP32 then FP64 storage) against solving the instances one after another
  with plain FP64 through the OP2 API.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import lib as L
from .airfoil import Airfoil
from .mesh import airfoil_constants, channel_bump


def _torch():
    import torch
    return torch


def _emit(obj):
    print(json.dumps(obj), flush=True)


def _field_errors(q, ref):
    d = q - ref
    l2 = np.sqrt((d * d).sum(axis=0)) / np.maximum(np.sqrt((ref * ref).sum(axis=0)), 1e-300)
    mx = np.abs(d).max(axis=0) / np.maximum(np.abs(ref).max(axis=0), 1e-300)
    names = ("rho", "rho_u", "rho_v", "rho_E")
    return {n: {"rel_l2": float(a), "rel_max": float(b)} for n, a, b in zip(names, l2, mx)}


def _run_fixed(mesh, consts, dtype, iters):
    """iters iterations from freestream on the renumbered mesh; rms history,
    device ms per iteration, final q in declared order (float64)."""
    torch = _torch()
    L.op_init()
    try:
        app = Airfoil(mesh, consts, dtype=dtype, rms_only=True)
        app.renumber()
        L.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.ExternalStream(L.load().op2b_get_stream())
        e0.record(stream)
        hist = app.iterate(iters)
        e1.record(stream)
        L.synchronize()
        ms = e0.elapsed_time(e1)
        q = app.fetch_original().astype(np.float64)
        return np.array([h[0] for h in hist]), ms / iters, q
    finally:
        L.op_exit()


def mixed_error(a):
    mesh = channel_bump(a.I, a.J, seed=a.seed)
    c = airfoil_constants()
    r64, ms64, q64 = _run_fixed(mesh, c, np.float64, a.iters)
    r32, ms32, q32 = _run_fixed(mesh, c, np.float32, a.iters)
    rel = np.abs(r32 / r64 - 1)
    _emit({"study": "mixed-error", "mesh": f"{a.I}x{a.J}", "cells": mesh.ncell,
           "iterations": a.iters, "ms_per_iter_fp64": ms64, "ms_per_iter_mixed": ms32,
           "speedup_per_iter": ms64 / ms32,
           "q_error_vs_fp64": _field_errors(q32, q64),
           "rms_rel_error": {"max": float(rel.max()), "final": float(rel[-1]),
                             "at_100": float(rel[min(99, len(rel) - 1)])},
           "rms_final": {"fp64": float(r64[-1]), "mixed": float(r32[-1])}})


def _solve_phase(mesh, consts, dtype, q0, tol_abs, max_iter, stall_every=0, promote_abs=None):
    """Iterate until rms < tol_abs (or, in the FP32 phase, rms < promote_abs or
    no 1 % progress over stall_every iterations).  Returns iterations, device
    ms, wall s, first and last rms, final q (declared order, float64)."""
    torch = _torch()
    L.op_init()
    try:
        t0 = time.perf_counter()
        app = Airfoil(mesh, consts, dtype=dtype, rms_only=True, q0=q0)
        app.renumber()
        L.synchronize()
        stream = torch.cuda.ExternalStream(L.load().op2b_get_stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rms = rms1 = app.iterate(1)[0][0]
        it, ref = 1, rms
        stop = promote_abs if promote_abs is not None else tol_abs
        while rms >= stop and it < max_iter:
            rms = app.iterate(1)[0][0]
            it += 1
            if stall_every and it % stall_every == 0:
                if rms > 0.99 * ref:
                    break
                ref = rms
        e1.record(stream)
        L.synchronize()
        q = app.fetch_original().astype(np.float64)
        return dict(iterations=it, ms=e0.elapsed_time(e1), wall_s=time.perf_counter() - t0,
                    rms1=rms1, rms=rms), q
    finally:
        L.op_exit()


def _graph_engine_solve(spec, fp32, tol, promote, max_iter, check_every):
    """One instance on the batched engine (CUDA-graph iterations, no per-loop
    host round trip): FP64 storage throughout, or FP32 storage then FP64."""
    from .batch import AirfoilBatch
    L.op_init()
    try:
        b = AirfoilBatch([spec], fp32=fp32)
        b.set("tol", tol)
        b.set("promote_tol", promote)
        active, ms = b.run(max_iter, check_every=check_every)
        st = b.stats()
        q = b.q_final()[0]
        b.close()
        return dict(device_ms=ms, unconverged=int(active), iterations=int(st["iters"][0]),
                    iterations_fp32=int(st["iters32"][0]), rms0=float(st["rms0"][0]),
                    rms=float(st["rms_last"][0])), q
    finally:
        L.op_exit()


def mixed_ttt(a):
    if a.engine == "graph":
        spec = dict(I=a.I, J=a.J, mach=0.4, alpha=0.0, bump=0.05, seed=a.seed)
        r64, q64 = _graph_engine_solve(spec, False, a.tol, a.promote, a.max_iter, a.check_every)
        r32, q32 = _graph_engine_solve(spec, True, a.tol, a.promote, a.max_iter, a.check_every)
        _emit({"study": "mixed-ttt", "engine": "graph", "mesh": f"{a.I}x{a.J}",
               "cells": a.I * a.J, "tol": a.tol, "promote": a.promote, "plain_fp64": r64,
               "mixed_then_fp64": r32, "time_ratio": r32["device_ms"] / r64["device_ms"],
               "final_q_vs_plain": _field_errors(q32, q64)})
        return
    mesh = channel_bump(a.I, a.J, seed=a.seed)
    c = airfoil_constants()
    # plain FP64 from freestream; its first rms fixes the absolute tolerance
    probe, _ = _solve_phase(mesh, c, np.float64, None, 0.0, 1)
    tol_abs = a.tol * probe["rms1"]
    plain, q_plain = _solve_phase(mesh, c, np.float64, None, tol_abs, a.max_iter)
    p32, q32 = _solve_phase(mesh, c, np.float32, None, tol_abs, a.max_iter,
                            stall_every=a.stall_every, promote_abs=a.promote * probe["rms1"])
    p64, q_mixed = _solve_phase(mesh, c, np.float64, q32, tol_abs, a.max_iter)
    mixed_ms = p32["ms"] + p64["ms"]
    _emit({"study": "mixed-ttt", "engine": "api", "mesh": f"{a.I}x{a.J}", "cells": mesh.ncell,
           "tol": a.tol,
           "tol_abs": tol_abs, "promote": a.promote,
           "plain_fp64": plain, "mixed_fp32_phase": p32, "mixed_fp64_phase": p64,
           "mixed_total_iterations": p32["iterations"] + p64["iterations"],
           "mixed_total_ms": mixed_ms, "time_ratio": mixed_ms / plain["ms"],
           "wall_ratio": (p32["wall_s"] + p64["wall_s"]) / plain["wall_s"],
           "final_q_vs_plain": _field_errors(q_mixed, q_plain)})


def batch(a):
    from .batch import AirfoilBatch, sample_instances
    specs = sample_instances(a.n, seed=a.seed, cells=(a.cells_min, a.cells_max))
    L.op_init()
    try:
        t0 = time.perf_counter()
        b = AirfoilBatch(specs, fp32=True)
        setup_s = time.perf_counter() - t0
        tune = b.tune(iters=a.tune_iters)
        b.set("tol", a.tol)
        b.set("promote_tol", a.promote)
        t1 = time.perf_counter()
        active, ms = b.run(a.max_iter, check_every=a.check_every)
        run_s = time.perf_counter() - t1
        st = b.stats()
        b.close()
    finally:
        L.op_exit()
    cells = [s["I"] * s["J"] for s in specs]
    out = {"study": "batch", "instances": a.n, "cells_total": int(sum(cells)),
           "cells_min": int(min(cells)), "cells_max": int(max(cells)), "tol": a.tol,
           "batched": {"device_ms": ms, "run_wall_s": run_s, "setup_wall_s": setup_s,
                       "unconverged": int(active), "iterations": st["iters"].tolist(),
                       "iterations_fp32": st["iters32"].tolist(),
                       "tuner": tune.strip().splitlines()[-1]}}
    _emit(out)
    if a.plain == "none":
        return
    batched_ms, batched_wall, subset = ms, run_s, list(range(len(specs)))
    if a.plain_subset and a.plain_subset < len(specs):
        # plain FP64 on a seeded random subset of the same instances, against
        # the batched form on that subset alone (same tolerance)
        rng = np.random.default_rng(a.subset_seed)
        subset = sorted(int(i) for i in rng.choice(len(specs), a.plain_subset, replace=False))
        sub = [specs[i] for i in subset]
        L.op_init()
        try:
            b = AirfoilBatch(sub, fp32=True)
            tune_sub = b.tune(iters=a.tune_iters)
            b.set("tol", a.tol)
            b.set("promote_tol", a.promote)
            t1 = time.perf_counter()
            active_sub, batched_ms = b.run(a.max_iter, check_every=a.check_every)
            batched_wall = time.perf_counter() - t1
            st_sub = b.stats()
            b.close()
        finally:
            L.op_exit()
        _emit({"study": "batch-subset", "subset": subset,
               "cells": [int(specs[i]["I"] * specs[i]["J"]) for i in subset],
               "batched": {"device_ms": batched_ms, "run_wall_s": batched_wall,
                           "unconverged": int(active_sub),
                           "iterations": st_sub["iters"].tolist(),
                           "tuner": tune_sub.strip().splitlines()[-1]}})
        specs = sub
    # the same instances one after another in plain FP64: through the OP2 API
    # (op_par_loop calls from the host), or on the same engine one instance at
    # a time (CUDA-graph iterations, no batching)
    seq_ms, seq_wall, seq_it, worst = 0.0, 0.0, [], 0.0
    for s in specs:
        t0 = time.perf_counter()
        if a.plain == "graph":
            r, _ = _graph_engine_solve(s, False, a.tol, a.promote, a.max_iter, a.check_every)
            seq_ms += r["device_ms"]
            worst = max(worst, r["rms"] / (a.tol * r["rms0"]))
        else:
            mesh = channel_bump(s["I"], s["J"], seed=s["seed"], bump=s["bump"])
            c = airfoil_constants(mach=s["mach"], alpha_deg=s["alpha"])
            probe, _ = _solve_phase(mesh, c, np.float64, None, 0.0, 1)
            r, _ = _solve_phase(mesh, c, np.float64, None, a.tol * probe["rms1"], a.max_iter)
            seq_ms += r["ms"]
            worst = max(worst, r["rms"] / (a.tol * probe["rms1"]))
        seq_wall += time.perf_counter() - t0
        seq_it.append(r["iterations"])
    _emit({"study": "batch-vs-plain", "plain": a.plain, "instances": a.n,
           "compared_instances": subset, "tol": a.tol,
           "plain_sequential": {"device_ms": seq_ms, "wall_s": seq_wall, "iterations": seq_it,
                                "max_final_rms_over_tol": worst},
           "batched_device_ms": batched_ms, "time_ratio": batched_ms / seq_ms,
           "wall_ratio": batched_wall / seq_wall})


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("mixed-error")
    p.add_argument("--I", type=int, default=2400)
    p.add_argument("--J", type=int, default=1200)
    p.add_argument("--iters", type=int, default=2000)
    p.add_argument("--seed", type=int, default=1)
    p = sub.add_parser("mixed-ttt")
    p.add_argument("--I", type=int, default=480)
    p.add_argument("--J", type=int, default=240)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--tol", type=float, default=1e-5)
    p.add_argument("--promote", type=float, default=1e-4)
    p.add_argument("--stall-every", type=int, default=500)
    p.add_argument("--max-iter", type=int, default=400000)
    p.add_argument("--engine", default="api", choices=["api", "graph"],
                   help="api: op_par_loop calls from the host; graph: the batched engine "
                        "with one instance (CUDA-graph iterations)")
    p.add_argument("--check-every", type=int, default=200)
    p = sub.add_parser("batch")
    p.add_argument("--n", type=int, default=64)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--tol", type=float, default=1e-6)
    p.add_argument("--promote", type=float, default=1e-4)
    p.add_argument("--max-iter", type=int, default=400000)
    p.add_argument("--check-every", type=int, default=200)
    p.add_argument("--tune-iters", type=int, default=10)
    p.add_argument("--cells-min", type=int, default=10_000)
    p.add_argument("--cells-max", type=int, default=500_000)
    p.add_argument("--plain", default="api", choices=["api", "graph", "none"],
                   help="sequential plain FP64 baseline: through the OP2 API, on the engine "
                        "one instance at a time, or none")
    p.add_argument("--plain-subset", type=int, default=0,
                   help="compare on a seeded random subset of this many instances (the "
                        "batched form re-run on the subset alone); 0 = all")
    p.add_argument("--subset-seed", type=int, default=0)
    a = ap.parse_args(argv)
    from . import build
    build.build()
    L.load()
    {"mixed-error": mixed_error, "mixed-ttt": mixed_ttt, "batch": batch}[a.cmd](a)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
