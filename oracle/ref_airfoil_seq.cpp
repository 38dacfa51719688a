/*
 * Oracle harness (test infrastructure only; never linked into the product).
 *
 * Runs the reference's Airfoil time loop through the reference's own
 * sequential op_par_loop (op2/include/op_seq.h) and the unmodified reference
 * kernels (apps/c/airfoil/airfoil_plain/dp/{save_soln,adt_calc,res_calc,
 * bres_calc,update}.h, found on the include path set by oracle/Makefile).
 * The loop calls are those of apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:
 * 221-297; only the mesh source (a binary file from op2b.mesh), the iteration
 * count and the outputs differ from that driver.
 *
 * usage: ref_airfoil_seq MESH.bin NITER OUT_PREFIX [SKIP] [OP2 argv tokens...]
 * SKIP (default 0) leading iterations are run but left out of the timing.
 * writes OUT_PREFIX.{rms,maxerr,errloc,q,res,adt} and prints one JSON line.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

double gam, gm1, cfl, eps, mach, alpha, qinf[4];

#include "op_seq.h"
#include "ref_harness_io.h"

#include "adt_calc.h"
#include "bres_calc.h"
#include "res_calc.h"
#include "save_soln.h"
#include "update.h"

int main(int argc, char **argv) {
  if (argc < 4)
    harness_die("usage: ref_airfoil_seq MESH.bin NITER OUT_PREFIX", NULL);
  op_init(argc, argv, 0);
  harness_mesh m = harness_read_mesh(argv[1]);
  int niter = atoi(argv[2]);
  const char *out = argv[3];
  int skip = (argc > 4 && argv[4][0] >= '0' && argv[4][0] <= '9') ? atoi(argv[4]) : 0;
  if (skip > niter)
    skip = niter;

  gam = 1.4f;
  gm1 = gam - 1.0f;
  cfl = 0.9f;
  eps = 0.05f;
  mach = 0.4f;
  alpha = 3.0f * atan(1.0f) / 45.0f;
  double p = 1.0f, r = 1.0f;
  double u = sqrt(gam * p / r) * mach;
  double e = p / (r * gm1) + 0.5f * u * u;
  qinf[0] = r;
  qinf[1] = r * u;
  qinf[2] = 0.0f;
  qinf[3] = r * e;

  double *q = (double *)malloc(sizeof(double) * 4 * (size_t)m.ncell);
  double *res = (double *)malloc(sizeof(double) * 4 * (size_t)m.ncell);
  double *qold = (double *)calloc(4 * (size_t)m.ncell, sizeof(double));
  double *adt = (double *)calloc((size_t)m.ncell, sizeof(double));
  for (int n = 0; n < m.ncell; n++)
    for (int k = 0; k < 4; k++) {
      q[4 * n + k] = qinf[k];
      res[4 * n + k] = 0.0;
    }

  op_set nodes = op_decl_set(m.nnode, "nodes");
  op_set edges = op_decl_set(m.nedge, "edges");
  op_set bedges = op_decl_set(m.nbedge, "bedges");
  op_set cells = op_decl_set(m.ncell, "cells");
  op_map pedge = op_decl_map(edges, nodes, 2, m.edge, "pedge");
  op_map pecell = op_decl_map(edges, cells, 2, m.ecell, "pecell");
  op_map pbedge = op_decl_map(bedges, nodes, 2, m.bedge, "pbedge");
  op_map pbecell = op_decl_map(bedges, cells, 1, m.becell, "pbecell");
  op_map pcell = op_decl_map(cells, nodes, 4, m.cell, "pcell");
  op_dat p_bound = op_decl_dat(bedges, 1, "int", m.bound, "p_bound");
  op_dat p_x = op_decl_dat(nodes, 2, "double", m.x, "p_x");
  op_dat p_q = op_decl_dat(cells, 4, "double", q, "p_q");
  op_dat p_qold = op_decl_dat(cells, 4, "double", qold, "p_qold");
  op_dat p_adt = op_decl_dat(cells, 1, "double", adt, "p_adt");
  op_dat p_res = op_decl_dat(cells, 4, "double", res, "p_res");

  double *rms_hist = (double *)calloc((size_t)niter + 1, sizeof(double));
  double *maxerr_hist = (double *)calloc((size_t)niter + 1, sizeof(double));
  int *errloc_hist = (int *)calloc((size_t)niter + 1, sizeof(int));
  double rms = 0.0, maxerr = 0.0;
  int errloc = 0;

  double c1, c2, t1, t2;
  op_timers(&c1, &t1);
  for (int iter = 1; iter <= niter; iter++) {
    if (iter == skip + 1)
      op_timers(&c1, &t1);
    op_par_loop(save_soln, "save_soln", cells,
                op_arg_dat(p_q, -1, OP_ID, 4, "double", OP_READ),
                op_arg_dat(p_qold, -1, OP_ID, 4, "double", OP_WRITE));
    for (int k = 0; k < 2; k++) {
      op_par_loop(adt_calc, "adt_calc", cells,
                  op_arg_dat(p_x, 0, pcell, 2, "double", OP_READ),
                  op_arg_dat(p_x, 1, pcell, 2, "double", OP_READ),
                  op_arg_dat(p_x, 2, pcell, 2, "double", OP_READ),
                  op_arg_dat(p_x, 3, pcell, 2, "double", OP_READ),
                  op_arg_dat(p_q, -1, OP_ID, 4, "double", OP_READ),
                  op_arg_dat(p_adt, -1, OP_ID, 1, "double", OP_WRITE));
      op_par_loop(res_calc, "res_calc", edges,
                  op_arg_dat(p_x, 0, pedge, 2, "double", OP_READ),
                  op_arg_dat(p_x, 1, pedge, 2, "double", OP_READ),
                  op_arg_dat(p_q, 0, pecell, 4, "double", OP_READ),
                  op_arg_dat(p_q, 1, pecell, 4, "double", OP_READ),
                  op_arg_dat(p_adt, 0, pecell, 1, "double", OP_READ),
                  op_arg_dat(p_adt, 1, pecell, 1, "double", OP_READ),
                  op_arg_dat(p_res, 0, pecell, 4, "double", OP_INC),
                  op_arg_dat(p_res, 1, pecell, 4, "double", OP_INC));
      op_par_loop(bres_calc, "bres_calc", bedges,
                  op_arg_dat(p_x, 0, pbedge, 2, "double", OP_READ),
                  op_arg_dat(p_x, 1, pbedge, 2, "double", OP_READ),
                  op_arg_dat(p_q, 0, pbecell, 4, "double", OP_READ),
                  op_arg_dat(p_adt, 0, pbecell, 1, "double", OP_READ),
                  op_arg_dat(p_res, 0, pbecell, 4, "double", OP_INC),
                  op_arg_dat(p_bound, -1, OP_ID, 1, "int", OP_READ));
      rms = 0.0;
      maxerr = 0.0;
      errloc = 0;
      op_par_loop(update, "update", cells,
                  op_arg_dat(p_qold, -1, OP_ID, 4, "double", OP_READ),
                  op_arg_dat(p_q, -1, OP_ID, 4, "double", OP_WRITE),
                  op_arg_dat(p_res, -1, OP_ID, 4, "double", OP_RW),
                  op_arg_dat(p_adt, -1, OP_ID, 1, "double", OP_READ),
                  op_arg_gbl(&rms, 1, "double", OP_INC),
                  op_arg_gbl(&maxerr, 1, "double", OP_MAX),
                  op_arg_idx(-1, OP_ID),
                  op_arg_info(&errloc, 1, "int", 5));
    }
    rms = sqrt(rms / (double)op_get_size(cells));
    rms_hist[iter] = rms;
    maxerr_hist[iter] = maxerr;
    errloc_hist[iter] = errloc;
  }
  op_timers(&c2, &t2);

  size_t nc = (size_t)m.ncell;
  harness_write(out, "rms", rms_hist + 1, sizeof(double) * (size_t)niter);
  harness_write(out, "maxerr", maxerr_hist + 1, sizeof(double) * (size_t)niter);
  harness_write(out, "errloc", errloc_hist + 1, sizeof(int) * (size_t)niter);
  harness_write(out, "q", p_q->data, sizeof(double) * 4 * nc);
  harness_write(out, "qold", p_qold->data, sizeof(double) * 4 * nc);
  harness_write(out, "res", p_res->data, sizeof(double) * 4 * nc);
  harness_write(out, "adt", p_adt->data, sizeof(double) * nc);
  printf("{\"build\": \"seq\", \"ncell\": %d, \"niter\": %d, \"wall_s\": %.6f, "
         "\"ms_per_iter\": %.6f, \"timed_iters\": %d, \"rms\": %.17g}\n",
         m.ncell, niter, t2 - t1, niter > skip ? 1e3 * (t2 - t1) / (niter - skip) : 0.0,
         niter - skip, niter ? rms_hist[niter] : 0.0);
  op_exit();
  return 0;
}
