/*
 * op2b_plan.h -- execution plans (block partition, local renumbering, thread
 * and block colouring) built on the GPU.
 *
 * Replaces the reference's plan interface, op2/include/op_rt_support.h:46-120
 * (struct op_plan, op_plan_get, op_plan_get_stage, op_plan_get_stage_upload,
 * op_plan_check), built by op_plan_core in op2/src/core/op_rt_support.cpp:
 * 301-1126.  The struct keeps the reference's field names, types and
 * meaning; its arrays are host copies of the plan the GPU built (the device
 * copies are reachable through op2b_plan_device_*).
 *
 * Integer outputs follow op_plan_core bit for bit: offset, nelems, ind_maps,
 * ind_offs, ind_sizes, nindirect, loc_maps, thrcol, nthrcol, ncolors,
 * ncolblk, blkmap, nsharedCol, nshared (with plan_mode 0, the default, which
 * runs the block colouring's greedy sequence on the device).  col_reord orders
 * elements of equal thread colour by position (the reference's qsort leaves
 * that order to the C library).  transfer/transfer2 are diagnostics.
 * Single rank: core_size = size, no exec halo.
 */
#ifndef OP2B_PLAN_H
#define OP2B_PLAN_H

#include "op2b.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  /* input arguments */
  char const *name;
  op_set set;
  int nargs, ninds, ninds_staged, part_size;
  op_map *maps;
  op_dat *dats;
  int *idxs;
  int *optflags;
  op_access *accs;
  int *inds_staged;

  /* execution plan (host copies) */
  int *nthrcol;        /* number of thread colours for each block */
  int *thrcol;         /* thread colours */
  int *col_reord;      /* permutation of elements by thread colour (PERMUTE/COLOR2) */
  int **col_offsets;   /* offsets to the start of each colour, per block */
  int *color2_offsets; /* colour offsets of the flat colouring (COLOR2) */
  int *offset;         /* first element of each block */
  int *offset_d;       /* unused (Fortran in the reference) */
  int *ind_map;        /* concatenated lists of indirectly referenced elements */
  int **ind_maps;      /* per staged indirection: pointer into ind_map */
  int *ind_offs;       /* block offsets into ind_maps [b * ninds_staged + m] */
  int *ind_sizes;      /* block sizes of ind_maps [b * ninds_staged + m] */
  int *nindirect;      /* total size of each indirection's list */
  short *loc_map;      /* concatenated maps to local (staged) indices */
  short **loc_maps;    /* per argument: pointer into loc_map, NULL if not staged */
  int nblocks;         /* number of blocks */
  int *nelems;         /* elements in each block */
  int *nelems_d;       /* unused (Fortran in the reference) */
  int ncolors_core;
  int ncolors_owned;
  int ncolors;         /* number of block colours */
  int *ncolblk;        /* blocks of each colour */
  int *blkmap;         /* blocks ordered by colour */
  int *blkmap_d;       /* unused (Fortran in the reference) */
  int *nsharedCol;     /* bytes of shared memory per block colour */
  int nshared;         /* bytes of shared memory */
  float transfer;      /* bytes moved per call (diagnostic) */
  float transfer2;     /* bytes moved per call in cache lines (diagnostic) */
  int count;           /* times the plan was requested */
} op_plan;

/* op_plan_get_stage (op_rt_support.h:108-110): build (first call) or fetch
 * the cached plan for this loop.  staging: OP_STAGE_INC, OP_STAGE_ALL,
 * OP_STAGE_PERMUTE or OP_COLOR2.  inds[arg] = indirection number or -1. */
op_plan *op_plan_get_stage(char const *name, op_set set, int part_size, int nargs,
                           op_arg *args, int ninds, int *inds, int staging);
/* op_plan_get_stage_upload (op_rt_support.h:112-114): `upload` is accepted
 * for compatibility; the plan always lives on the device. */
op_plan *op_plan_get_stage_upload(char const *name, op_set set, int part_size, int nargs,
                                  op_arg *args, int ninds, int *inds, int staging,
                                  int upload);
/* op_plan_get (op_rt_support.h:116-117): OP_STAGE_ALL. */
op_plan *op_plan_get(char const *name, op_set set, int part_size, int nargs, op_arg *args,
                     int ninds, int *inds);
/* op_plan_check (op_rt_support.h:119, op_rt_support.cpp:129-295): the
 * reference's structural checks, run on the device, plus the colouring
 * checks the reference leaves empty (:290-294).  Prints what fails. */
void op_plan_check(op_plan OP_plan, int ninds, int *inds);

/* ---- op2b extensions (no reference counterpart) ------------------------ */

/* Structural + conflict-free checks of a plan on the device.  Returns the
 * number of violations (0 = valid); `detail` (may be NULL) receives
 * [nelems, offset, blkmap, ind_offs, ind_maps, loc_maps, thread-colour
 * conflicts, block-colour conflicts]. */
int op2b_plan_validate(const op_plan *plan, long detail[8]);
/* Device time (ms) the last plan construction took. */
double op2b_plan_build_ms(const op_plan *plan);
/* Device copies of the plan arrays (plain device addresses). */
const int *op2b_plan_device_blkmap(const op_plan *plan);
const int *op2b_plan_device_thrcol(const op_plan *plan);
/* Drop every cached plan (they are rebuilt on next use). */
void op2b_plan_release_all(void);

#ifdef __cplusplus
}
#endif

#endif /* OP2B_PLAN_H */
