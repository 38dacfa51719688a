// Batched Airfoil: many instances in one mesh, one persistent launch per loop
// stage, the iteration captured in a CUDA graph.  Internal to libop2b; the C
// API is in include/op2b_batch.h.
#pragma once

#include <cuda_runtime.h>

#include "airfoil_math.cuh"

namespace op2b {

// A contiguous range [begin, end) of elements of one instance.
struct WorkItem {
  int inst, begin, end, pad;
};

// Work lists of one precision phase: cells (direct loops and the gather
// res_calc), boundary rows (cells with boundary edges) and edges.
struct WorkLists {
  WorkItem *cells, *brows, *edges;
  int *count;  // [0] cells, [1] brows, [2] edges
};

struct BatchDev {
  int ninst;
  const int *cell_off, *edge_off, *brow_off;  // per instance ranges (ninst + 1)
  int *phase;        // 0 = FP32 storage, 1 = FP64, 2 = converged, 3 = promote pending
  double *rms_sum;   // per instance, summed by the update kernels
  double *rms0;      // per instance rms after the first iteration
  double *rms_last;  // per instance rms of the last iteration
  double *rms_prev;  // per instance rms at the last stall check
  int *iters;        // per instance iterations run
  int *iters32;      // per instance iterations run with FP32 storage
  int *stall;        // per instance iterations since the rms last fell by 1 %
  const double *qinf;  // per instance freestream (4 doubles)
  WorkLists w32, w64;  // FP32-phase and FP64-phase work
  WorkItem *promote;   // cells of instances moving from FP32 to FP64
  int *npromote;
  int *mapped;       // mapped host page: [0] active instances, [1] iteration
  int chunk;         // elements per work item
  double tol, promote_tol;
  int max_iter, stall_window;
};

}  // namespace op2b
