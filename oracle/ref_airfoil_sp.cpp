/*
 * Oracle harness (test infrastructure only; never linked into the product).
 *
 * The single-precision Airfoil of the reference
 * (apps/c/airfoil/airfoil_plain/sp/airfoil.cpp:148-300): float dats and
 * constants, the unmodified sp kernels (save_soln, adt_calc, res_calc,
 * bres_calc, update with a float rms; found on the include path set by
 * oracle/Makefile), the same loop calls.  Only the mesh source (a binary
 * file from op2b.mesh, coordinates rounded to float as the reference's
 * fscanf("%f") reads them), the iteration count and the outputs differ: it
 * writes q after the last iteration (op_fetch_data) and the float rms of
 * every iteration.
 *
 * Built twice by oracle/Makefile: against the reference's sequential library
 * (ref_airfoil_sp_harness) and against include/op_seq.h + libop2b.so
 * (airfoil_sp_harness_dropin), so the two q fields can be compared bit for
 * bit.
 *
 * usage: ref_airfoil_sp MESH.bin NITER OUT_PREFIX
 * writes OUT_PREFIX.{q,rms} (float32) and prints one JSON line.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

float gam, gm1, cfl, eps, mach, alpha, qinf[4];

#include "op_seq.h"
#include "ref_harness_io.h"

#include "adt_calc.h"
#include "bres_calc.h"
#include "res_calc.h"
#include "save_soln.h"
#include "update.h"

int main(int argc, char **argv) {
  if (argc < 4)
    harness_die("usage: ref_airfoil_sp MESH.bin NITER OUT_PREFIX", NULL);
  op_init(argc, argv, 0);
  harness_mesh m = harness_read_mesh(argv[1]);
  int niter = atoi(argv[2]);
  const char *out = argv[3];

  gam = 1.4f;
  gm1 = gam - 1.0f;
  cfl = 0.9f;
  eps = 0.05f;
  mach = 0.4f;
  alpha = 3.0f * atan(1.0f) / 45.0f;
  float p = 1.0f, r = 1.0f;
  float u = sqrt(gam * p / r) * mach;
  float e = p / (r * gm1) + 0.5f * u * u;
  qinf[0] = r;
  qinf[1] = r * u;
  qinf[2] = 0.0f;
  qinf[3] = r * e;

  size_t nc = (size_t)m.ncell;
  float *x = (float *)malloc(sizeof(float) * 2 * (size_t)m.nnode + 8);
  for (size_t i = 0; i < 2 * (size_t)m.nnode; i++) x[i] = (float)m.x[i];
  float *q = (float *)malloc(sizeof(float) * 4 * nc);
  float *res = (float *)calloc(4 * nc, sizeof(float));
  float *qold = (float *)calloc(4 * nc, sizeof(float));
  float *adt = (float *)calloc(nc, sizeof(float));
  for (size_t n = 0; n < nc; n++)
    for (int k = 0; k < 4; k++) q[4 * n + k] = qinf[k];

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
  op_dat p_x = op_decl_dat(nodes, 2, "float", x, "p_x");
  op_dat p_q = op_decl_dat(cells, 4, "float", q, "p_q");
  op_dat p_qold = op_decl_dat(cells, 4, "float", qold, "p_qold");
  op_dat p_adt = op_decl_dat(cells, 1, "float", adt, "p_adt");
  op_dat p_res = op_decl_dat(cells, 4, "float", res, "p_res");
  op_decl_const(1, "float", &gam);
  op_decl_const(1, "float", &gm1);
  op_decl_const(1, "float", &cfl);
  op_decl_const(1, "float", &eps);
  op_decl_const(1, "float", &mach);
  op_decl_const(1, "float", &alpha);
  op_decl_const(4, "float", qinf);

  float *rms_hist = (float *)calloc((size_t)niter + 1, sizeof(float));
  float rms = 0.0f;
  double c1, c2, t1, t2;
  op_timers(&c1, &t1);
  for (int iter = 1; iter <= niter; iter++) {
    op_par_loop(save_soln, "save_soln", cells,
                op_arg_dat(p_q, -1, OP_ID, 4, "float", OP_READ),
                op_arg_dat(p_qold, -1, OP_ID, 4, "float", OP_WRITE));
    for (int k = 0; k < 2; k++) {
      op_par_loop(adt_calc, "adt_calc", cells,
                  op_arg_dat(p_x, 0, pcell, 2, "float", OP_READ),
                  op_arg_dat(p_x, 1, pcell, 2, "float", OP_READ),
                  op_arg_dat(p_x, 2, pcell, 2, "float", OP_READ),
                  op_arg_dat(p_x, 3, pcell, 2, "float", OP_READ),
                  op_arg_dat(p_q, -1, OP_ID, 4, "float", OP_READ),
                  op_arg_dat(p_adt, -1, OP_ID, 1, "float", OP_WRITE));
      op_par_loop(res_calc, "res_calc", edges,
                  op_arg_dat(p_x, 0, pedge, 2, "float", OP_READ),
                  op_arg_dat(p_x, 1, pedge, 2, "float", OP_READ),
                  op_arg_dat(p_q, 0, pecell, 4, "float", OP_READ),
                  op_arg_dat(p_q, 1, pecell, 4, "float", OP_READ),
                  op_arg_dat(p_adt, 0, pecell, 1, "float", OP_READ),
                  op_arg_dat(p_adt, 1, pecell, 1, "float", OP_READ),
                  op_arg_dat(p_res, 0, pecell, 4, "float", OP_INC),
                  op_arg_dat(p_res, 1, pecell, 4, "float", OP_INC));
      op_par_loop(bres_calc, "bres_calc", bedges,
                  op_arg_dat(p_x, 0, pbedge, 2, "float", OP_READ),
                  op_arg_dat(p_x, 1, pbedge, 2, "float", OP_READ),
                  op_arg_dat(p_q, 0, pbecell, 4, "float", OP_READ),
                  op_arg_dat(p_adt, 0, pbecell, 1, "float", OP_READ),
                  op_arg_dat(p_res, 0, pbecell, 4, "float", OP_INC),
                  op_arg_dat(p_bound, -1, OP_ID, 1, "int", OP_READ));
      rms = 0.0f;
      op_par_loop(update, "update", cells,
                  op_arg_dat(p_qold, -1, OP_ID, 4, "float", OP_READ),
                  op_arg_dat(p_q, -1, OP_ID, 4, "float", OP_WRITE),
                  op_arg_dat(p_res, -1, OP_ID, 4, "float", OP_RW),
                  op_arg_dat(p_adt, -1, OP_ID, 1, "float", OP_READ),
                  op_arg_gbl(&rms, 1, "float", OP_INC));
    }
    rms = sqrtf(rms / (float)op_get_size(cells));
    rms_hist[iter] = rms;
  }
  op_timers(&c2, &t2);
  float *qout = (float *)malloc(sizeof(float) * 4 * nc);
  op_fetch_data(p_q, qout);
  harness_write(out, "q", qout, sizeof(float) * 4 * nc);
  harness_write(out, "rms", rms_hist + 1, sizeof(float) * (size_t)niter);
  printf("{\"build\": \"sp\", \"ncell\": %d, \"niter\": %d, \"wall_s\": %.6f, \"rms\": %.9g}\n",
         m.ncell, niter, t2 - t1, niter ? rms_hist[niter] : 0.0f);
  op_exit();
  return 0;
}
