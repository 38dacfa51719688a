/*
 * Oracle harness (test infrastructure only; never linked into the product).
 *
 * Builds the reference's execution plans (op_plan_get_stage ->
 * op_plan_core, op2/src/core/op_rt_support.cpp:301-1126) for the three
 * indirect Airfoil loops on a mesh file from op2b.mesh, with the argument
 * lists of apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:235-261 and the `inds`
 * arrays the reference v1 translator emits for them, and dumps every plan
 * array so the product's GPU plan builder can be compared with it.
 *
 * usage: ref_plan_dump MESH.bin STAGING PART_SIZE OUT_PREFIX
 *   STAGING: 1 = OP_STAGE_INC, 2 = OP_STAGE_ALL, 3 = OP_STAGE_PERMUTE,
 *            4 = OP_COLOR2 (op2/include/op_lib_core.h:121-125)
 * writes OUT_PREFIX.<loop>.plan, a list of records
 *   int32 name_len, name, int32 kind (0 int32, 1 int16, 2 float32), int64 n, data
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

double gam, gm1, cfl, eps, mach, alpha, qinf[4];

#include "op_seq.h"
#include "ref_harness_io.h"

static void rec(FILE *f, const char *name, int kind, long long n,
                const void *data) {
  int len = (int)strlen(name);
  size_t esz = kind == 1 ? 2 : 4;
  fwrite(&len, 4, 1, f);
  fwrite(name, 1, len, f);
  fwrite(&kind, 4, 1, f);
  fwrite(&n, 8, 1, f);
  if (n > 0)
    fwrite(data, esz, (size_t)n, f);
}

static void dump_plan(const char *prefix, const char *loop, op_plan *p,
                      int nargs, int ninds, int staging) {
  char path[4096];
  snprintf(path, sizeof(path), "%s.%s.plan", prefix, loop);
  FILE *f = fopen(path, "wb");
  if (!f)
    harness_die("cannot write", path);
  int exec_length = p->set->size;
  int nb = p->nblocks;
  int nst = p->ninds_staged;
  int scalars[6] = {nb, p->ncolors, nst, exec_length, p->nshared, staging};
  rec(f, "scalars", 0, 6, scalars);
  rec(f, "nthrcol", 0, nb, p->nthrcol);
  rec(f, "thrcol", 0, exec_length, p->thrcol);
  rec(f, "offset", 0, nb, p->offset);
  rec(f, "nelems", 0, nb, p->nelems);
  rec(f, "ind_offs", 0, (long long)nb * nst, p->ind_offs);
  rec(f, "ind_sizes", 0, (long long)nb * nst, p->ind_sizes);
  rec(f, "nindirect", 0, ninds, p->nindirect);
  rec(f, "inds_staged", 0, nargs, p->inds_staged);
  for (int m = 0; m < nst; m++) {
    long long used = 0;
    for (int b = 0; b < nb; b++)
      used += p->ind_sizes[m + b * nst];
    char nm[64];
    snprintf(nm, sizeof(nm), "ind_map%d", m);
    rec(f, nm, 0, used, p->ind_maps[m]);
  }
  for (int a = 0; a < nargs; a++) {
    if (p->loc_maps[a] == NULL)
      continue;
    char nm[64];
    snprintf(nm, sizeof(nm), "loc_map%d", a);
    rec(f, nm, 1, exec_length, p->loc_maps[a]);
  }
  rec(f, "ncolblk", 0, p->ncolors, p->ncolblk);
  rec(f, "blkmap", 0, nb, p->blkmap);
  rec(f, "nsharedCol", 0, p->ncolors, p->nsharedCol);
  float tr[2] = {p->transfer, p->transfer2};
  rec(f, "transfer", 2, 2, tr);
  if (staging == OP_STAGE_PERMUTE || staging == OP_COLOR2) {
    rec(f, "col_reord", 0, exec_length, p->col_reord);
    long long ncoloff = 0;
    for (int b = 0; b < nb; b++)
      ncoloff += p->nthrcol[b] + 1;
    rec(f, "col_offsets", 0, ncoloff, p->col_offsets[0]);
  }
  fclose(f);
}

int main(int argc, char **argv) {
  if (argc < 5)
    harness_die("usage: ref_plan_dump MESH.bin STAGING PART_SIZE OUT_PREFIX", NULL);
  op_init(argc, argv, 0);
  harness_mesh m = harness_read_mesh(argv[1]);
  int staging = atoi(argv[2]);
  int part_size = atoi(argv[3]);
  const char *out = argv[4];

  double *zero4 = (double *)calloc(4 * (size_t)m.ncell, sizeof(double));
  double *zero1 = (double *)calloc((size_t)m.ncell, sizeof(double));
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
  op_dat p_q = op_decl_dat(cells, 4, "double", zero4, "p_q");
  op_dat p_adt = op_decl_dat(cells, 1, "double", zero1, "p_adt");
  op_dat p_res = op_decl_dat(cells, 4, "double", zero4, "p_res");

  {
    op_arg args[6] = {op_arg_dat(p_x, 0, pcell, 2, "double", OP_READ),
                      op_arg_dat(p_x, 1, pcell, 2, "double", OP_READ),
                      op_arg_dat(p_x, 2, pcell, 2, "double", OP_READ),
                      op_arg_dat(p_x, 3, pcell, 2, "double", OP_READ),
                      op_arg_dat(p_q, -1, OP_ID, 4, "double", OP_READ),
                      op_arg_dat(p_adt, -1, OP_ID, 1, "double", OP_WRITE)};
    int inds[6] = {0, 0, 0, 0, -1, -1};
    op_plan *p = op_plan_get_stage("adt_calc", cells, part_size, 6, args, 1,
                                   inds, staging);
    dump_plan(out, "adt_calc", p, 6, 1, staging);
  }
  {
    op_arg args[8] = {op_arg_dat(p_x, 0, pedge, 2, "double", OP_READ),
                      op_arg_dat(p_x, 1, pedge, 2, "double", OP_READ),
                      op_arg_dat(p_q, 0, pecell, 4, "double", OP_READ),
                      op_arg_dat(p_q, 1, pecell, 4, "double", OP_READ),
                      op_arg_dat(p_adt, 0, pecell, 1, "double", OP_READ),
                      op_arg_dat(p_adt, 1, pecell, 1, "double", OP_READ),
                      op_arg_dat(p_res, 0, pecell, 4, "double", OP_INC),
                      op_arg_dat(p_res, 1, pecell, 4, "double", OP_INC)};
    int inds[8] = {0, 0, 1, 1, 2, 2, 3, 3};
    op_plan *p = op_plan_get_stage("res_calc", edges, part_size, 8, args, 4,
                                   inds, staging);
    dump_plan(out, "res_calc", p, 8, 4, staging);
  }
  {
    op_arg args[6] = {op_arg_dat(p_x, 0, pbedge, 2, "double", OP_READ),
                      op_arg_dat(p_x, 1, pbedge, 2, "double", OP_READ),
                      op_arg_dat(p_q, 0, pbecell, 4, "double", OP_READ),
                      op_arg_dat(p_adt, 0, pbecell, 1, "double", OP_READ),
                      op_arg_dat(p_res, 0, pbecell, 4, "double", OP_INC),
                      op_arg_dat(p_bound, -1, OP_ID, 1, "int", OP_READ)};
    int inds[6] = {0, 0, 1, 2, 3, -1};
    op_plan *p = op_plan_get_stage("bres_calc", bedges, part_size, 6, args, 4,
                                   inds, staging);
    dump_plan(out, "bres_calc", p, 6, 4, staging);
  }
  op_exit();
  return 0;
}
