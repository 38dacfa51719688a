"""The run-time compiled loop path on the Airfoil workload: the five Airfoil
loops written as OP2 user kernels (this module's own restatement, registered
under other names, so no hand-written kernel matches them) run through
libop2b's generated loops, beside the hand-written kernels on the same mesh.

    python -m op2b.jit_bench [--mesh 2400 1200] [--iters 20] [--renumber 1] [--soa 1]

Prints one JSON line: per loop, the mean device time per call (CUDA events,
every call timed) and GB/s on the loop's algorithmic bytes (the same bytes as
bench.py's), for the generated loops and for the hand-written ones run alone
(no fusion or speculation); with --soa 1 also the generated loops on
structure-of-arrays copies (one one-component dat per component of x, q, qold
and res)."""
import argparse
import json

import numpy as np

from . import lib as L
from . import mesh as M
from .airfoil import Airfoil

KERNELS = r"""
inline void jsave(const double *q, double *qold) {
  for (int n = 0; n < 4; n++) qold[n] = q[n];
}
inline void jadt(const double *x1, const double *x2, const double *x3, const double *x4,
                 const double *q, double *adt) {
  double dx, dy, ri, u, v, c;
  ri = 1.0f / q[0];
  u = ri * q[1];
  v = ri * q[2];
  c = sqrt(gam * gm1 * (ri * q[3] - 0.5f * (u * u + v * v)));
  dx = x2[0] - x1[0]; dy = x2[1] - x1[1];
  *adt = fabs(u * dy - v * dx) + c * sqrt(dx * dx + dy * dy);
  dx = x3[0] - x2[0]; dy = x3[1] - x2[1];
  *adt += fabs(u * dy - v * dx) + c * sqrt(dx * dx + dy * dy);
  dx = x4[0] - x3[0]; dy = x4[1] - x3[1];
  *adt += fabs(u * dy - v * dx) + c * sqrt(dx * dx + dy * dy);
  dx = x1[0] - x4[0]; dy = x1[1] - x4[1];
  *adt += fabs(u * dy - v * dx) + c * sqrt(dx * dx + dy * dy);
  *adt = (*adt) / cfl;
}
inline void jres(const double *x1, const double *x2, const double *q1, const double *q2,
                 const double *adt1, const double *adt2, double *res1, double *res2) {
  double dx, dy, mu, ri, p1, vol1, p2, vol2, f;
  dx = x1[0] - x2[0]; dy = x1[1] - x2[1];
  ri = 1.0f / q1[0];
  p1 = gm1 * (q1[3] - 0.5f * ri * (q1[1] * q1[1] + q1[2] * q1[2]));
  vol1 = ri * (q1[1] * dy - q1[2] * dx);
  ri = 1.0f / q2[0];
  p2 = gm1 * (q2[3] - 0.5f * ri * (q2[1] * q2[1] + q2[2] * q2[2]));
  vol2 = ri * (q2[1] * dy - q2[2] * dx);
  mu = 0.5f * ((*adt1) + (*adt2)) * eps;
  f = 0.5f * (vol1 * q1[0] + vol2 * q2[0]) + mu * (q1[0] - q2[0]);
  res1[0] += f; res2[0] -= f;
  f = 0.5f * (vol1 * q1[1] + p1 * dy + vol2 * q2[1] + p2 * dy) + mu * (q1[1] - q2[1]);
  res1[1] += f; res2[1] -= f;
  f = 0.5f * (vol1 * q1[2] - p1 * dx + vol2 * q2[2] - p2 * dx) + mu * (q1[2] - q2[2]);
  res1[2] += f; res2[2] -= f;
  f = 0.5f * (vol1 * (q1[3] + p1) + vol2 * (q2[3] + p2)) + mu * (q1[3] - q2[3]);
  res1[3] += f; res2[3] -= f;
}
inline void jbres(const double *x1, const double *x2, const double *q1, const double *adt1,
                  double *res1, const int *bound) {
  double dx, dy, mu, ri, p1, vol1, p2, vol2, f;
  dx = x1[0] - x2[0]; dy = x1[1] - x2[1];
  ri = 1.0f / q1[0];
  p1 = gm1 * (q1[3] - 0.5f * ri * (q1[1] * q1[1] + q1[2] * q1[2]));
  if (*bound == 1) {
    res1[1] += +p1 * dy;
    res1[2] += -p1 * dx;
  } else {
    vol1 = ri * (q1[1] * dy - q1[2] * dx);
    ri = 1.0f / qinf[0];
    p2 = gm1 * (qinf[3] - 0.5f * ri * (qinf[1] * qinf[1] + qinf[2] * qinf[2]));
    vol2 = ri * (qinf[1] * dy - qinf[2] * dx);
    mu = (*adt1) * eps;
    f = 0.5f * (vol1 * q1[0] + vol2 * qinf[0]) + mu * (q1[0] - qinf[0]);
    res1[0] += f;
    f = 0.5f * (vol1 * q1[1] + p1 * dy + vol2 * qinf[1] + p2 * dy) + mu * (q1[1] - qinf[1]);
    res1[1] += f;
    f = 0.5f * (vol1 * q1[2] - p1 * dx + vol2 * qinf[2] - p2 * dx) + mu * (q1[2] - qinf[2]);
    res1[2] += f;
    f = 0.5f * (vol1 * (q1[3] + p1) + vol2 * (qinf[3] + p2)) + mu * (q1[3] - qinf[3]);
    res1[3] += f;
  }
}
inline void jupdate(const double *qold, double *q, double *res, const double *adt,
                    double *rms) {
  double del, adti;
  adti = 1.0f / (*adt);
  for (int n = 0; n < 4; n++) {
    del = adti * res[n];
    q[n] = qold[n] - del;
    res[n] = 0.0f;
    *rms += del * del;
  }
}
"""

# the same loops on structure-of-arrays dats: every component of x, q, qold
# and res its own one-component dat
KERNELS_SOA = r"""
inline void ssave(const double *q0, const double *q1, const double *q2, const double *q3,
                  double *o0, double *o1, double *o2, double *o3) {
  *o0 = *q0; *o1 = *q1; *o2 = *q2; *o3 = *q3;
}
inline void sadt(const double *x1a, const double *x1b, const double *x2a, const double *x2b,
                 const double *x3a, const double *x3b, const double *x4a, const double *x4b,
                 const double *q0, const double *q1, const double *q2, const double *q3,
                 double *adt) {
  const double x1[2] = {*x1a, *x1b}, x2[2] = {*x2a, *x2b}, x3[2] = {*x3a, *x3b},
               x4[2] = {*x4a, *x4b}, q[4] = {*q0, *q1, *q2, *q3};
  jadt(x1, x2, x3, x4, q, adt);
}
inline void sres(const double *x1a, const double *x1b, const double *x2a, const double *x2b,
                 const double *a0, const double *a1, const double *a2, const double *a3,
                 const double *b0, const double *b1, const double *b2, const double *b3,
                 const double *adt1, const double *adt2, double *r0, double *r1, double *r2,
                 double *r3, double *s0, double *s1, double *s2, double *s3) {
  const double x1[2] = {*x1a, *x1b}, x2[2] = {*x2a, *x2b}, q1[4] = {*a0, *a1, *a2, *a3},
               q2[4] = {*b0, *b1, *b2, *b3};
  double res1[4] = {0, 0, 0, 0}, res2[4] = {0, 0, 0, 0};
  jres(x1, x2, q1, q2, adt1, adt2, res1, res2);
  *r0 += res1[0]; *r1 += res1[1]; *r2 += res1[2]; *r3 += res1[3];
  *s0 += res2[0]; *s1 += res2[1]; *s2 += res2[2]; *s3 += res2[3];
}
inline void supdate(const double *o0, const double *o1, const double *o2, const double *o3,
                    double *q0, double *q1, double *q2, double *q3, double *r0, double *r1,
                    double *r2, double *r3, const double *adt, double *rms) {
  const double qold[4] = {*o0, *o1, *o2, *o3};
  double q[4], res[4] = {*r0, *r1, *r2, *r3};
  jupdate(qold, q, res, adt, rms);
  *q0 = q[0]; *q1 = q[1]; *q2 = q[2]; *q3 = q[3];
  *r0 = res[0]; *r1 = res[1]; *r2 = res[2]; *r3 = res[3];
}
"""


def soa_loops(app, rms):
    """The structure-of-arrays loops over copies of the Airfoil dats."""
    t, R, W, RW, INC = "double", L.OP_READ, L.OP_WRITE, L.OP_RW, L.OP_INC
    A = L.op_arg_dat
    x = L.op_fetch_data(app.p_x)
    q = L.op_fetch_data(app.p_q)
    dx = [L.op_decl_dat(app.nodes, 1, t, np.ascontiguousarray(x[:, k]), f"sx{k}") for k in range(2)]
    dq = [L.op_decl_dat(app.cells, 1, t, np.ascontiguousarray(q[:, k]), f"sq{k}") for k in range(4)]
    do = [L.op_decl_dat(app.cells, 1, t, None, f"so{k}") for k in range(4)]
    dr = [L.op_decl_dat(app.cells, 1, t, None, f"sr{k}") for k in range(4)]
    xs = lambda i, m: [A(d, i, m, 1, t, R) for d in dx]
    return [
        ("ssave", app.cells, [A(d, -1, L.OP_ID, 1, t, R) for d in dq] +
         [A(d, -1, L.OP_ID, 1, t, W) for d in do]),
        ("sadt", app.cells, sum((xs(i, app.pcell) for i in range(4)), []) +
         [A(d, -1, L.OP_ID, 1, t, R) for d in dq] + [A(app.p_adt, -1, L.OP_ID, 1, t, W)]),
        ("sres", app.edges, xs(0, app.pedge) + xs(1, app.pedge) +
         [A(d, 0, app.pecell, 1, t, R) for d in dq] + [A(d, 1, app.pecell, 1, t, R) for d in dq] +
         [A(app.p_adt, 0, app.pecell, 1, t, R), A(app.p_adt, 1, app.pecell, 1, t, R)] +
         [A(d, 0, app.pecell, 1, t, INC) for d in dr] + [A(d, 1, app.pecell, 1, t, INC) for d in dr]),
        ("supdate", app.cells, [A(d, -1, L.OP_ID, 1, t, R) for d in do] +
         [A(d, -1, L.OP_ID, 1, t, W) for d in dq] + [A(d, -1, L.OP_ID, 1, t, RW) for d in dr] +
         [A(app.p_adt, -1, L.OP_ID, 1, t, R), L.op_arg_gbl(rms, 1, "double", L.OP_INC)])]


# algorithmic bytes per call (C cells, N nodes, E edges, B boundary edges):
# the figures bench.py's roofline uses
def alg_bytes(m):
    C, N, E, B = m.ncell, m.nnode, m.nedge, m.nbedge
    return {"save_soln": 64 * C, "adt_calc": 16 * C + 16 * N + 40 * C,
            "res_calc": 16 * E + 16 * N + 104 * C, "bres_calc": 136 * B,
            "update": 136 * C}


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--mesh", type=int, nargs=2, default=[2400, 1200])
    p.add_argument("--iters", type=int, default=20)
    p.add_argument("--renumber", type=int, default=1)
    p.add_argument("--option", action="append", default=[], metavar="KEY=VALUE")
    p.add_argument("--soa", type=int, default=0,
                   help="also time the loops on structure-of-arrays copies of the dats")
    a = p.parse_args(argv)
    m = M.channel_bump(a.mesh[0], a.mesh[1], seed=1)
    L.op_init()
    for kv in a.option:
        k, v = kv.split("=")
        L.set_option(k, int(v))
    app = Airfoil(m)
    if a.renumber:
        app.renumber(stats=False)
    for k in ("jsave", "jadt", "jres", "jbres", "jupdate"):
        L.register_kernel(k, KERNELS)
    t, R, W, RW, INC = "double", L.OP_READ, L.OP_WRITE, L.OP_RW, L.OP_INC
    A = L.op_arg_dat
    rms = np.zeros(1)
    loops = [
        ("jsave", app.cells, [A(app.p_q, -1, L.OP_ID, 4, t, R),
                              A(app.p_qold, -1, L.OP_ID, 4, t, W)]),
        ("jadt", app.cells, [A(app.p_x, i, app.pcell, 2, t, R) for i in range(4)] +
         [A(app.p_q, -1, L.OP_ID, 4, t, R), A(app.p_adt, -1, L.OP_ID, 1, t, W)]),
        ("jres", app.edges, [A(app.p_x, 0, app.pedge, 2, t, R), A(app.p_x, 1, app.pedge, 2, t, R),
                             A(app.p_q, 0, app.pecell, 4, t, R), A(app.p_q, 1, app.pecell, 4, t, R),
                             A(app.p_adt, 0, app.pecell, 1, t, R),
                             A(app.p_adt, 1, app.pecell, 1, t, R),
                             A(app.p_res, 0, app.pecell, 4, t, INC),
                             A(app.p_res, 1, app.pecell, 4, t, INC)]),
        ("jbres", app.bedges, [A(app.p_x, 0, app.pbedge, 2, t, R),
                               A(app.p_x, 1, app.pbedge, 2, t, R),
                               A(app.p_q, 0, app.pbecell, 4, t, R),
                               A(app.p_adt, 0, app.pbecell, 1, t, R),
                               A(app.p_res, 0, app.pbecell, 4, t, INC),
                               A(app.p_bound, -1, L.OP_ID, 1, "int", R)]),
        ("jupdate", app.cells, [A(app.p_qold, -1, L.OP_ID, 4, t, R),
                                A(app.p_q, -1, L.OP_ID, 4, t, W),
                                A(app.p_res, -1, L.OP_ID, 4, t, RW),
                                A(app.p_adt, -1, L.OP_ID, 1, t, R),
                                L.op_arg_gbl(rms, 1, "double", L.OP_INC)])]

    def run_generated(n):
        for _ in range(n):
            L.op_par_loop(*loops[0][:2], *loops[0][2])
            for _k in range(2):
                for i in (1, 2, 3):
                    L.op_par_loop(loops[i][0], loops[i][1], *loops[i][2])
                rms[0] = 0.0
                L.op_par_loop(loops[4][0], loops[4][1], *loops[4][2])

    L.set_option("timing_stride", 1)
    run_generated(2)  # compile and warm up
    L.load().op2b_reset_stats()
    run_generated(a.iters)
    bytes_ = alg_bytes(m)
    names = {"jsave": "save_soln", "jadt": "adt_calc", "jres": "res_calc", "jbres": "bres_calc",
             "jupdate": "update"}
    out = {"mesh": f"{a.mesh[0]}x{a.mesh[1]}", "cells": m.ncell, "renumbered": bool(a.renumber),
           "generated": {}, "hand_written": {}}
    for j, n in names.items():
        st = L.loop_stats(j)
        ms = st["total_ms"] / st["calls"]
        out["generated"][n] = {"us": round(ms * 1000, 2),
                               "gbs": round(bytes_[n] / (ms * 1e-3) / 1e9, 1)}
    rms_gen = float(rms[0])
    # the hand-written kernels alone, on the same mesh and options
    for k, v in (("fuse", 0), ("speculate_adt", 0), ("rename_save", 0), ("speculate_res", 0),
                 ("lazy_res", 0)):
        L.set_option(k, v)
    app.iterate(2, history=False)
    L.load().op2b_reset_stats()
    app.iterate(a.iters, history=False)
    for n in names.values():
        st = L.loop_stats(n)
        ms = st["total_ms"] / st["calls"]
        out["hand_written"][n] = {"us": round(ms * 1000, 2),
                                  "gbs": round(bytes_[n] / (ms * 1e-3) / 1e9, 1)}
    out["last_rms_sum_generated"] = rms_gen
    if a.soa:
        for k in ("ssave", "sadt", "sres", "supdate"):
            L.register_kernel(k, KERNELS + KERNELS_SOA)
        sl = soa_loops(app, rms)
        for _ in range(2):
            for nm, st_, args in sl:
                L.op_par_loop(nm, st_, *args)
        L.load().op2b_reset_stats()
        for _ in range(a.iters):
            for nm, st_, args in sl:
                L.op_par_loop(nm, st_, *args)
        out["generated_soa"] = {}
        for j, n in (("ssave", "save_soln"), ("sadt", "adt_calc"), ("sres", "res_calc"),
                     ("supdate", "update")):
            st = L.loop_stats(j)
            ms = st["total_ms"] / st["calls"]
            out["generated_soa"][n] = {"us": round(ms * 1000, 2),
                                       "gbs": round(bytes_[n] / (ms * 1e-3) / 1e9, 1)}
    print(json.dumps(out))
    L.op_exit()


if __name__ == "__main__":
    main()
