/*
 * op2b_batch.h -- batched Airfoil: many instances of uneven mesh size and
 * flow condition solved together on one GPU.  No counterpart in the
 * reference (OP2 solves one mesh per process).
 *
 * The caller declares all instances as ONE OP2 mesh through op2b.h
 * (concatenated sets, block-diagonal maps), renumbers it so each instance
 * owns contiguous ranges of cells and edges, declares the Airfoil dats twice
 * (float for the FP32-storage phase, double for the FP64 phase) on the same
 * sets and maps, and passes the per-instance ranges and freestream states.
 * Each loop stage then runs as one persistent launch over the still-active
 * instances; one iteration is a CUDA graph.  Instances start in FP32 storage
 * (FP64 update and rms), move to FP64 storage when their rms falls below
 * promote_tol * rms0 or stalls, and stop at rms < tol * rms0 (rms0 = rms after
 * the first iteration).
 */
#ifndef OP2B_BATCH_H
#define OP2B_BATCH_H

#include "op2b.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The maps and dats of the Airfoil loops, as declared for
 * apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:180-202. */
typedef struct {
  op_map pcell, pedge, pecell, pbedge, pbecell;
  op_dat p_x, p_q, p_qold, p_adt, p_res, p_bound;
} op2b_airfoil_dats;

typedef struct op2b_batch_s *op2b_batch;

#define OP2B_BATCH_RES_GATHER 0 /* owner computes over cells (no conflicts) */
#define OP2B_BATCH_RES_ATOMIC 1 /* one thread an edge, atomic increments */
#define OP2B_BATCH_RES_COLOUR 2 /* edges by colour (parallel OP_COLOR2 plan), no atomics */

/* fp32 may be NULL (FP64 only).  cell_off / edge_off: ninst + 1 offsets of
 * each instance's cells and edges; qinf: 4 doubles per instance.  The
 * constants gam, gm1, cfl, eps must be declared (op_decl_const). */
op2b_batch op2b_batch_create(const op2b_airfoil_dats *fp32, const op2b_airfoil_dats *fp64,
                             int ninst, const int *cell_off, const int *edge_off,
                             const double *qinf);
/* keys: "tol", "promote_tol", "max_iter", "stall_window", "block" (128, 256,
 * 512), "blocks_per_sm", "res_kernel" (OP2B_BATCH_RES_*), "part_size"
 * (elements per work item, >= 256; the reference's OP_PART_SIZE,
 * op_lib_core.cpp:205-220). */
int op2b_batch_set(op2b_batch b, const char *key, double value);
/* Time every (res_calc strategy: gather, atomics or colouring) x (block size:
 * 128, 256, 512) x (partition size: 512, 2048, 8192) candidate for `iters`
 * iterations, keep the fastest; the solve's state is left untouched. */
int op2b_batch_tune(op2b_batch b, int iters, char *report, int report_len);
/* Run up to max_iterations iterations (graphs when use_graph), checking for
 * completion every check_every; returns the number of instances still active,
 * -1 on error.  elapsed_ms: device time of the run. */
int op2b_batch_run(op2b_batch b, int max_iterations, int check_every, int use_graph,
                   double *elapsed_ms);
/* Per-instance iterations (total and with FP32 storage), rms0, last rms and
 * phase (0 FP32, 1 FP64, 2 done, 3 promotion pending). */
int op2b_batch_stats(op2b_batch b, int *iters, int *iters32, double *rms0, double *rms_last,
                     int *phase);
void op2b_batch_destroy(op2b_batch b);

#ifdef __cplusplus
}
#endif

#endif /* OP2B_BATCH_H */
