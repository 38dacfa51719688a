"""Benchmark: Airfoil ms/iteration on the 2400x1200 (2.88M-cell) mesh, plain FP64.

One step = one Airfoil outer iteration through the OP2 API on libop2b
(save_soln + 2 x {adt_calc, res_calc, bres_calc, update}, rms read back after
each update, as apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:221-297 does).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl op2b|reference]

N > 1 runs under torchrun: every rank solves its own replica (the single-mesh
path does not shard; there is no collective on the data path), timing is the
max over ranks.  Prints one JSON line on rank 0.

* value      device-timed ms/iteration, inputs resident in HBM (CUDA events on
             the library's stream, K iterations between a barrier and a
             synchronize on both sides).  The working set (~0.7 GB) is larger
             than the 126 MB L2, so no flush is needed between iterations.
             Default configuration: the mesh renumbered on the GPU
             (op_renumber, reverse Cuthill-McKee), owner-computes increments
             over corner records, the runtime's loop fusion (res_calc with
             bres_calc), its speculative adt_calc (computed by the update
             before it), save_soln by renaming (the update after it
             writes the new q into qold's array and the two dats swap
             arrays, so no copy is made), and the res_calc + bres_calc pair
             launched by each update's call before it waits for the rms.
* loops      per loop (or fused loop pair) device time, algorithmic bytes per
             call and GB/s.
* e2e        the whole 1000-iteration job (the configuration's length) through
             the public API from host buffers, per iteration: op_decl_*
             uploads from pinned mesh arrays, op_renumber, the iterations,
             op_fetch_data of q.
* roofline   the dominant loop's algorithmic bytes per call / its mean
             CUDA-event duration, against MEASURED_PEAKS.json hbm_gbs; traffic
             = ncu DRAM bytes per launch (profiles/traffic.json).
* variants   the same timing for random/RCM numbering x increment strategies,
             gather kernels, and fusion off (per-loop figures).
* cpu_baseline  the reference's own OpenMP build (oracle/_ref, compiled from the
             reference sources) on a bounded sample of the same mesh.
* --impl reference   times that reference build alone (rank 0; others exit).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "op2-common_b200"))
sys.path.insert(0, REPO)

FALLBACK_HBM_GBS = 6650.0
LOOPS = ("save_soln", "adt_calc", "res_calc", "bres_calc", "update",
         # the runtime's fused launches: loop pairs, update computing the next
         # adt_calc ahead (and putting adt back when another call came first)
         "save_soln+adt_calc", "res_calc+bres_calc", "update+adt_calc", "adt restore")
METRIC = "Airfoil ms/iter (2400x1200 FP64)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="op2b", choices=["op2b", "reference"])
    p.add_argument("--mesh", type=int, nargs=2, default=[2400, 1200])
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--numbering", default="rcm", choices=["rcm", "random"])
    p.add_argument("--inc-mode", type=int, default=3,
                   help="0 atomics, 1 block/thread colouring, 2 staged hybrid, 3 gather")
    p.add_argument("--part-size", type=int, default=0)
    p.add_argument("--gather-kernel", type=int, default=6,
                   help="inc_mode 3 kernel: 1 csr, 2 lanes, 3 cell4, 4 shared-memory pipeline, "
                        "5 register pipeline, 6 register pipeline over corner records")
    p.add_argument("--pipe-block", type=int, default=256)
    p.add_argument("--e2e-iters", type=int, default=1000,
                   help="length of the end-to-end job (the 2400x1200 configuration runs 1000 "
                        "iterations)")
    p.add_argument("--precision", default="f64", choices=["f64", "mixed"])
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-variants", action="store_true")
    p.add_argument("--cpu-iters", type=int, default=4)
    p.add_argument("--ref-trajectory", type=int, default=1,
                   help="1: the CPU baseline runs the reference's OpenMP build for the whole "
                        "end-to-end job's iterations on the same mesh (timing and rms "
                        "trajectory); 0: a bounded sample of --cpu-iters iterations")
    p.add_argument("--option", action="append", default=[], metavar="KEY=VALUE",
                   help="a library option (op2b_set_option) for the timed runs and the "
                        "end-to-end job; repeatable")
    return p.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return ws, rank, local


def mesh_file(I, J, seed):
    from op2b import mesh as M
    path = os.path.join(tempfile.gettempdir(), f"op2b_mesh_{I}x{J}_s{seed}.bin")
    if not os.path.exists(path):
        m = M.channel_bump(I, J, seed=seed)
        tmp = path + f".{os.getpid()}"
        M.write_grid_bin(m, tmp)
        os.replace(tmp, path)
        return m, path
    return M.read_grid_bin(path), path


def rcm_mesh_file(I, J, seed, m):
    """The same mesh in the numbering the GPU arm solves on: renumbered by the
    oracle's restatement of op_renumber (reverse Cuthill-McKee; the library's
    GPU permutations equal it bit for bit).  For the reference legs only."""
    from op2b import mesh as M
    from oracle import oracle as O
    path = os.path.join(tempfile.gettempdir(), f"op2b_mesh_{I}x{J}_s{seed}_rcm.bin")
    if not os.path.exists(path):
        mr, _ = O.rcm_mesh(m)
        tmp = path + f".{os.getpid()}"
        M.write_grid_bin(mr, tmp)
        os.replace(tmp, path)
    return path


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def algorithmic_bytes(loop, C, N, E, B, es=8):
    """Compulsory bytes of one call of `loop` (each array element moved once;
    es-byte reals, int32 maps): save_soln 64 C; adt_calc 16 C + 16 N + 40 C;
    res_calc 16 E + 16 N + 104 C; bres_calc 12 B + 120 B; update 136 C -- for
    es = 8.  A fused launch counts the loops it stands for."""
    r = es / 8.0
    one = {"save_soln": 64 * r * C,
           "adt_calc": 16 * C + 16 * r * N + 40 * r * C,
           "res_calc": 16 * E + 16 * r * N + 104 * r * C,
           "bres_calc": 12 * B + 120 * r * B,
           "update": 136 * r * C}
    parts = loop.split("+")
    if not all(p in one for p in parts):
        return None
    return sum(one[p] for p in parts)


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def traffic_from_profiles(key, loop):
    """dram bytes per launch of `loop` from the committed ncu summary, if any."""
    p = os.path.join(REPO, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(key, {}).get(loop)


class Clocks:
    """SM clock and throttle reasons sampled during the timed region (start
    before, stop after): NVML every 2 ms from a thread, or nvidia-smi every
    200 ms where NVML cannot be loaded."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.thread = None
        self.path = os.path.join(tempfile.gettempdir(), f"op2b_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            import threading
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.samples, self.mask = [], 0
            self.done = threading.Event()

            def poll():
                while True:
                    self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                    self.mask |= int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))
                    if self.done.wait(0.002):
                        return

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index),
                                          f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.done.set()
            self.thread.join()
            reasons = sorted(n for b, n in self.REASONS.items() if self.mask & b)
            sm = self.samples
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(sm), "source": "nvml, every 2 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for ln in f:
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, every 200 ms"}


def run_reference(args, m_path, ncell, iters, skip, threads, numbering):
    """The reference's OpenMP build on a mesh file; returns (baseline dict, rms history)."""
    from oracle import oracle as O
    binary = O.ref_binary("ref_airfoil_openmp")
    if binary is None:
        return None, None
    summary, rms = O.run_reference_airfoil_timed(binary, m_path, iters, skip,
                                                 env={"OMP_NUM_THREADS": str(threads)})
    label = ("RCM-renumbered as the GPU arm solves it" if numbering == "rcm"
             else "random numbering")
    return dict(value=summary["ms_per_iter"], unit="ms/iter",
                cores=summary.get("threads", threads), cpu=cpu_model(), kind="reference",
                numbering=numbering,
                sample=f"{summary['timed_iters']} iterations of the {args.mesh[0]}x{args.mesh[1]} "
                       f"mesh ({ncell} cells, {label}) after {skip} untimed, the "
                       "reference's OpenMP build (v1 translator output), "
                       f"OMP_NUM_THREADS={threads}"), rms


def impl_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    m, path = mesh_file(*args.mesh, args.seed)
    threads = os.cpu_count() or 1
    # one step = one iteration of the reference's OpenMP build on the mesh the
    # GPU arm solves (same numbering); warm-up iterations (its plan
    # construction included) run but are not timed
    main_path = rcm_mesh_file(*args.mesh, args.seed, m) if args.numbering == "rcm" else path
    res, _ = run_reference(args, main_path, m.ncell, args.warmup + args.steps, args.warmup,
                           threads, args.numbering)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/ref_airfoil_openmp not built (make -C oracle)"}))
        return 0
    # the other numbering, as a second, labelled sample (block colouring
    # collapses on random order: a few iterations suffice)
    other = None
    if args.numbering == "rcm":
        other, _ = run_reference(args, path, m.ncell, 1 + args.cpu_iters, 1, threads, "random")
    v = res["value"]
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": "ms/iter", "impl": "reference", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"airfoil {args.mesh[0]}x{args.mesh[1]} plain FP64",
                   "cells": m.ncell, "edges": m.nedge, "numbering": args.numbering},
        "cpu_baseline": res,
        "other_numbering": other,
        "e2e": {"value": v, "unit": "ms/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def trajectory_parity(args, rms, q, ref_rms):
    """The end-to-end job's rms history and final q against the reference on
    the same mesh and numbering: the reference's sequential build (committed
    fixture: rms of every iteration and a digest of q after 1000) and, when it
    ran, the reference's OpenMP build timed beside (its rms history)."""
    import hashlib
    out = {"iterations": int(rms.size)}
    fx = os.path.join(REPO, "tests", "golden",
                      f"airfoil_{args.mesh[0]}x{args.mesh[1]}_s{args.seed}_rcm.npz")
    if (args.numbering == "rcm" and args.precision == "f64" and os.path.exists(fx)):
        gd = np.load(fx)
        n = int(gd["niter_traj"])
        if rms.size == n:
            out["vs_reference_seq"] = {
                "rms_traj_max_rel": float(np.max(np.abs(rms / gd["rms_traj"] - 1))),
                "q_bit_exact": hashlib.sha256(np.ascontiguousarray(q, dtype="<f8").tobytes())
                .hexdigest() == str(gd["q_digest_traj"]),
                "source": os.path.relpath(fx, REPO)}
    if ref_rms is not None and ref_rms.size == rms.size:
        out["vs_reference_openmp"] = {"rms_traj_max_rel":
                                      float(np.max(np.abs(rms / ref_rms - 1)))}
    return out


def timed_run(L, Airfoil, mesh, dtype, numbering, inc_mode, part, steps, warmup, torch,
              barrier=None, clocks=None, opts=None):
    """Declare, optionally renumber, warm up, then time `steps` iterations."""
    L.op_init()
    L.set_option("inc_mode", inc_mode)
    L.set_option("part_size", part)
    for k, v in (opts or {}).items():
        L.set_option(k, v)
    app = Airfoil(mesh, dtype=dtype)
    ren = None
    if numbering == "rcm":
        t0 = time.perf_counter()
        ren = app.renumber()
        ren["ms"] = 1e3 * (time.perf_counter() - t0)
    stream = torch.cuda.ExternalStream(L.load().op2b_get_stream())
    app.iterate(warmup, history=False)
    L.synchronize()
    L.load().op2b_reset_stats()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if barrier:
        barrier()
    L.synchronize()
    launches0 = L.load().op2b_kernel_launches()
    if clocks:
        clocks.start()
    e0.record(stream)
    hist = app.iterate(steps)
    e1.record(stream)
    L.synchronize()
    if barrier:
        barrier()
    clk = clocks.stop() if clocks else None
    launches = L.load().op2b_kernel_launches() - launches0
    ms = e0.elapsed_time(e1) / max(steps, 1)
    stats = {n: L.loop_stats(n) for n in LOOPS}
    L.op_exit()
    loops = {}
    for n, s in stats.items():
        if s and s["calls"]:
            avg = s["total_ms"] / s["calls"]
            loops[n] = {"calls": s["calls"], "avg_ms": avg, "alg_bytes": s["bytes_per_call"],
                        "gbs": s["bytes_per_call"] / (avg * 1e-3) / 1e9 if avg > 0 else None}
    return dict(ms=ms, loops=loops, launches=launches, clocks=clk, renumber=ren,
                rms=hist[-1][0] if hist else None)


def main():
    args = parse()
    if args.impl == "reference":
        return impl_reference(args)
    ws, rank, local = dist_env()
    os.environ["OP2B_DEVICE"] = str(local)
    import torch
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    from op2b import build, lib as L
    from op2b.airfoil import Airfoil
    build.build()
    L.load()
    m, m_path = mesh_file(*args.mesh, args.seed)
    dtype = np.float64 if args.precision == "f64" else np.float32

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---------------------------------------------------------- device-resident timing
    gopts = {"gather_kernel": args.gather_kernel, "pipe_block": args.pipe_block}
    for kv in args.option:
        k, _, v = kv.partition("=")
        gopts[k] = int(v)
    main_run = timed_run(L, Airfoil, m, dtype, args.numbering, args.inc_mode, args.part_size,
                         args.steps, args.warmup, torch, barrier, Clocks(local), opts=gopts)
    ms = max_over_ranks(main_run["ms"])

    # ---------------------------------------------------------- variants (same rank-local work)
    variants = []
    if not args.no_variants:
        for numbering in ("random", "rcm"):
            for mode in (0, 1, 2, 3):
                if numbering == "random" and mode == 1:
                    continue  # hundreds of block colours: one launch each
                v = timed_run(L, Airfoil, m, dtype, numbering, mode, args.part_size, 20, 3, torch,
                              barrier)
                variants.append({"numbering": numbering, "inc_mode": mode,
                                 "ms_per_iter": max_over_ranks(v["ms"]),
                                 "res_calc_gbs": v["loops"].get("res_calc", {}).get("gbs"),
                                 "launches_per_iter": v["launches"] / 20})
        # per-edge atomics beside the default segmented ones, and the plan-driven
        # strategies on the parallel (Jones-Plassmann) colouring
        for numbering, mode, o in (("random", 0, {"atomic_segmented": 0}),
                                   ("rcm", 0, {"atomic_segmented": 0}),
                                   ("rcm", 1, {"plan_mode": 1}), ("rcm", 2, {"plan_mode": 1}),
                                   ("random", 2, {"plan_mode": 1})):
            v = timed_run(L, Airfoil, m, dtype, numbering, mode, args.part_size, 20, 3, torch,
                          barrier, opts=o)
            variants.append({"numbering": numbering, "inc_mode": mode, **o,
                             "ms_per_iter": max_over_ranks(v["ms"]),
                             "res_calc_gbs": v["loops"].get("res_calc", {}).get("gbs"),
                             "launches_per_iter": v["launches"] / 20})
        # gather kernels of inc_mode 3, and the pipelined direct loop's switches
        for o in ({"gather_kernel": 1}, {"gather_kernel": 3}, {"gather_kernel": 4},
                  {"gather_kernel": 5, "pipe_block": 128}, {"gather_kernel": 5, "pipe_block": 256},
                  {"gather_kernel": 6, "pipe_block": 128}, {"gather_kernel": 6, "pipe_block": 256},
                  {"gather_kernel": 7}, {"gather_kernel": 7, "fuse": 0},
                  {"gather_kernel": 6, "pipe_block": 256, "bres_kernel": 0},
                  {"lazy_res": 0}, {"speculate_res": 0, "lazy_res": 0},
                  {"rename_save": 0, "speculate_res": 0, "lazy_res": 0},
                  {"speculate_adt": 0, "rename_save": 0, "speculate_res": 0, "lazy_res": 0},
                  {"fuse": 0, "speculate_adt": 0, "rename_save": 0, "speculate_res": 0,
                   "lazy_res": 0}):
            v = timed_run(L, Airfoil, m, dtype, "rcm", 3, args.part_size, 20, 3, torch, barrier,
                          opts=o)
            lp = v["loops"]
            variants.append({"numbering": "rcm", "inc_mode": 3, **o,
                             "ms_per_iter": max_over_ranks(v["ms"]),
                             "loops": {n: {"us": round(1e3 * x["avg_ms"], 2),
                                           "gbs": round(x["gbs"])}
                                       for n, x in lp.items()}})

    # ---------------------------------------------------------- plan construction
    plans = []
    if not args.no_variants:
        for numbering in ("rcm", "random"):
            for mode, label in ((2, "greedy (reference order)"), (1, "jones-plassmann")):
                L.op_init()
                L.set_option("plan_mode", mode)
                app = Airfoil(m, dtype=dtype)
                if numbering == "rcm":
                    app.renumber()
                p = L.op_plan_get_stage("res_calc", app.edges, args.part_size, app.a_res,
                                        [0, 0, 1, 1, 2, 2, 3, 3], 2)
                n_bad, _ = L.plan_validate(p)
                plans.append({"loop": "res_calc", "numbering": numbering, "colouring": label,
                              "build_ms": round(L.load().op2b_plan_build_ms(p), 2),
                              "blocks": p.contents.nblocks, "block_colours": p.contents.ncolors,
                              "conflicts": n_bad})
                L.op_exit()

    # ---------------------------------------------------------- end to end through the API
    e2e = None
    if not args.no_e2e:
        keep = []

        def pin(a):
            t = torch.empty(a.shape, dtype={np.float64: torch.float64, np.float32: torch.float32,
                                            np.int32: torch.int32}[a.dtype.type],
                            pin_memory=True)
            arr = t.numpy()
            arr[...] = a
            keep.append(t)
            return arr

        from op2b.mesh import Mesh, airfoil_constants
        hm = Mesh(x=pin(m.x.astype(dtype)), cell=pin(m.cell), edge=pin(m.edge),
                  ecell=pin(m.ecell), bedge=pin(m.bedge), becell=pin(m.becell),
                  bound=pin(m.bound))
        # the initial field (freestream), a host input like the mesh
        q0 = pin(np.tile(np.asarray(airfoil_constants()["qinf"], dtype), (m.ncell, 1)))
        L.op_init()
        L.set_option("inc_mode", args.inc_mode)
        L.set_option("part_size", args.part_size)
        for k, v in gopts.items():
            L.set_option(k, v)
        barrier()
        K = max(args.e2e_iters, 1)
        t0 = time.perf_counter()
        app2 = Airfoil(hm, dtype=dtype, q0=q0)
        ta = time.perf_counter()
        if args.numbering == "rcm":
            app2.renumber(stats=False)  # as airfoil.cpp's op_renumber: no bandwidth report
        tb = time.perf_counter()
        e2e_hist = app2.iterate(K)
        tc = time.perf_counter()
        q = L.op_fetch_data(app2.p_q, out=q0)  # into the pinned array the initial q came from
        t1 = time.perf_counter()
        barrier()
        ms_e2e = max_over_ranks(1e3 * (t1 - t0) / K)
        # (outside the timed region) q back in the declared cell order
        e2e_q = q[L.set_permutation(app2.cells)] if args.numbering == "rcm" else q
        e2e_rms = np.array([h[0] for h in e2e_hist])
        es = np.dtype(dtype).itemsize
        # x, the maps, the bound flags and q are uploaded; qold/adt/res are
        # declared without data (zeroed on the device)
        h2d = (m.x.size * es + (m.cell.size + m.edge.size + m.ecell.size + m.bedge.size
                                + m.becell.size + m.bound.size) * 4
               + m.ncell * 4 * es)
        d2h = q.nbytes + K * 2 * 32  # q, and the update's reduction read back per call
        e2e = {"value": ms_e2e, "unit": "ms/iter", "iterations": K,
               "phases_ms": {"declare": round(1e3 * (ta - t0), 1),
                             "renumber": round(1e3 * (tb - ta), 1),
                             "iterate": round(1e3 * (tc - tb), 1),
                             "fetch": round(1e3 * (t1 - tc), 1)},
               "h2d_bytes_per_step": int(h2d / K),
               "d2h_bytes_per_step": int(d2h / K),
               "note": f"per iteration of a whole {K}-iteration job through the API: "
                       "op_decl_* uploads (mesh arrays and the initial q pinned), op_renumber, "
                       "the iterations (rms read back after every update), op_fetch_data(q) "
                       "into the pinned array the initial q came from"}
        L.op_exit()

    # ---------------------------------------------------------- CPU baseline (rank 0, N=1)
    cpu = cpu_other = ref_rms = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        # on the mesh the GPU arm solves: the whole job's iterations (first one
        # untimed) when the configuration is the 1000-iteration one, for the
        # rms trajectory; a bounded sample of the other numbering beside it
        if args.numbering == "rcm":
            K_ref = max(args.e2e_iters, 1) if args.ref_trajectory else 1 + args.cpu_iters
            cpu, ref_rms = run_reference(args, rcm_mesh_file(*args.mesh, args.seed, m), m.ncell,
                                         K_ref, 1, threads, "rcm")
            cpu_other, _ = run_reference(args, m_path, m.ncell, 1 + args.cpu_iters, 1, threads,
                                         "random")
        else:
            cpu, _ = run_reference(args, m_path, m.ncell, 1 + args.cpu_iters, 1, threads,
                                   "random")
        if cpu is None:
            from oracle import oracle as O
            from op2b.mesh import airfoil_constants
            t0 = time.perf_counter()
            O.airfoil_run(m, airfoil_constants(), 2)
            cpu = dict(value=1e3 * (time.perf_counter() - t0) / 2, unit="ms/iter", cores=1,
                       kind="port", sample="2 iterations of the C restatement (oracle)")

    if rank == 0:
        peak, peak_src = peaks()
        work = f"{args.mesh[0]}x{args.mesh[1]}"
        loops = main_run["loops"]
        es = np.dtype(dtype).itemsize
        sizes = (m.ncell, m.nnode, m.nedge, m.nbedge)
        for n, x in loops.items():
            sb = algorithmic_bytes(n, *sizes, es=es)
            x["moved_bytes"] = x.pop("alg_bytes")       # what the runtime's launch must move
            x["alg_bytes"] = sb                          # the loops' compulsory bytes
            x["moved_gbs"] = x.pop("gbs")
            x["gbs"] = sb / (x["avg_ms"] * 1e-3) / 1e9 if sb and x["avg_ms"] > 0 else None
        dom = max(loops, key=lambda n: loops[n]["avg_ms"] * loops[n]["calls"])
        d = loops[dom]
        key = f"{work}_{args.precision}_{args.numbering}_mode{args.inc_mode}"
        # the iteration: save_soln + 2 x (adt_calc, res_calc, bres_calc, update)
        it_bytes = (algorithmic_bytes("save_soln", *sizes, es=es) + 2 * algorithmic_bytes(
            "adt_calc+res_calc+bres_calc+update", *sizes, es=es))
        it_gbs = it_bytes / (ms * 1e-3) / 1e9 if ms > 0 else None
        parity = None
        if e2e is not None:
            parity = trajectory_parity(args, e2e_rms, e2e_q, ref_rms)
        line = {
            "metric": METRIC, "value": ms, "unit": "ms/iter", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "f64" else "f32-storage/f64-update",
            "data": "synthetic (seeded channel-with-bump mesh)",
            "config": {"workload": f"airfoil {work} plain "
                                   f"{'FP64' if args.precision == 'f64' else 'mixed'}, "
                                   f"{args.numbering} numbering, inc_mode {args.inc_mode}",
                       "cells": m.ncell, "edges": m.nedge, "nodes": m.nnode,
                       "bedges": m.nbedge, "numbering": args.numbering,
                       "inc_mode": args.inc_mode, "part_size": args.part_size,
                       "gather_kernel": args.gather_kernel if args.inc_mode == 3 else None,
                       "parallelism": "replicas" if ws > 1 else "single",
                       "l2": "inputs larger than L2 (working set ~0.7 GB > 126 MB), no flush"},
            "roofline": {"bound": "hbm", "loop": dom, "achieved": d["gbs"], "peak": peak,
                         "unit": "GB/s", "frac": d["gbs"] / peak if d["gbs"] else None,
                         "traffic": traffic_from_profiles(key, dom),
                         "alg_bytes_per_launch": d["alg_bytes"],
                         "launch_us": 1e3 * d["avg_ms"],
                         "moved_bytes_per_launch": d["moved_bytes"],
                         "peak_source": peak_src,
                         # the whole iteration: the five loops' compulsory bytes
                         # (save_soln + 2 x the other four) over the measured
                         # time per iteration
                         "iteration_alg_bytes": it_bytes,
                         "iteration_achieved": it_gbs,
                         "iteration_frac": it_gbs / peak if it_gbs else None},
            "loops": loops,
            "renumber": main_run["renumber"],
            "rms_final": main_run["rms"],
            "variants": variants,
            "plans": plans,
            "cpu_baseline": cpu,
            "cpu_other_numbering": cpu_other,
            "parity": parity,
            "e2e": e2e,
            "gpu_launches": int(main_run["launches"]),
            "clocks": main_run["clocks"],
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
