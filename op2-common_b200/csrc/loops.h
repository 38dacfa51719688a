// Launch interface between the host runtime (op2b_core.cpp) and the device
// loops (*.cu).  Internal to libop2b.
#pragma once

#include <cuda_runtime.h>

#include "airfoil_math.cuh"

namespace op2b {

// Where and how a launcher issues its kernels.
struct LaunchCtx {
  cudaStream_t stream;
  int nsm;                 // SMs on the device (148 on B200)
  long *launch_counter;    // incremented once per kernel launch
  bool pdl = false;        // programmatic dependent launch for the kernels that wait for it
  void count() const {
    if (launch_counter) ++*launch_counter;
  }
};

// Launch `kern` on ctx's stream, with programmatic dependent launch when
// ctx.pdl: the kernel's CTAs may start as the previous kernel's finish, and
// the kernel itself waits (griddepcontrol.wait, grid_dependency_wait below)
// for the previous grid to complete before it touches memory.  Only kernels
// that make that wait their first step may be launched this way.
template <typename... KArgs, typename... Args>
cudaError_t launch_dependent(const LaunchCtx &ctx, void (*kern)(KArgs...), dim3 grid, dim3 block,
                             size_t smem, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx.stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = ctx.pdl ? at : nullptr;
  cfg.numAttrs = ctx.pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// First step of a kernel launched by launch_dependent: let the next kernel in
// the stream be launched (its CTAs still wait for this grid to complete),
// then wait for the previous grid's completion and memory.  Without
// programmatic launch both are no-ops.
__device__ __forceinline__ void grid_dependency_wait() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// One partial of the fused update reduction (32 bytes).
struct RedSlot {
  double sum;
  double maxv;
  long long idx;
  long long pad;
};

// Device scratch of the update reduction: `capacity` partial slots, a ticket
// counter (zero between launches) and the final slot.
struct RedScratch {
  RedSlot *parts;
  unsigned *counter;
  RedSlot *out;
  int capacity;
  // mapped pinned host copy of the result; `pad` receives `seq` after the
  // values, so the host can poll it instead of copying and synchronising
  RedSlot *host_out;
  long long seq;
};

cudaError_t launch_copy(const LaunchCtx &c, const void *src, void *dst, size_t bytes);

// map_check.cu: *first_bad = lowest i with map[i] outside [0, nto); the
// caller initialises it to ~0ull
cudaError_t launch_map_check(const LaunchCtx &c, const int *map, long long n, int nto,
                             unsigned long long *first_bad);

// minb: __launch_bounds__ minimum CTAs of 256 threads per SM (0 or 1 = no
// register cap; 6 caps registers at 40, 8 at 32)
template <typename T>
cudaError_t launch_adt_calc(const LaunchCtx &c, int ncell, const int *pcell, const T *x,
                            const T *q, T *adt, const AirConst<T> &k, int minb = 0);
// save_soln (q -> qold) fused into adt_calc: one pass over q
template <typename T>
cudaError_t launch_adt_save(const LaunchCtx &c, int ncell, const int *pcell, const T *x,
                            const T *q, T *adt, T *qold, const AirConst<T> &k);
// segmented: a warp's increments to one cell are combined before the atomics;
// blocks_per_sm: the grid's 256-thread CTAs per SM, up to one edge a thread
template <typename T>
cudaError_t launch_res_calc_atomic(const LaunchCtx &c, int nedge, const int *pedge,
                                   const int *pecell, const T *x, const T *q, const T *adt,
                                   T *res, const AirConst<T> &k, bool segmented = true,
                                   int blocks_per_sm = 4096);
template <typename T>
cudaError_t launch_bres_calc_atomic(const LaunchCtx &c, int nbedge, const int *pbedge,
                                    const int *pbecell, const int *bound, const T *x,
                                    const T *q, const T *adt, T *res, const AirConst<T> &k);
// adt_next (optional): also each cell's time step from its new q, pcell and
// x with constants k, as adt_calc computes it, written into adt_next (adt is
// only read).  keep_res: res is read but not zeroed (the
// runtime records that it is zero and zeroes it only if something reads it
// before a res_calc rewrites it).  reverse: the cells are taken from the last
// down (the loop before walked them upwards, so the rows it touched last are
// the ones still in L2); the result is the same but for rms's summation order
template <typename T>
cudaError_t launch_update(const LaunchCtx &c, int ncell, const T *qold, T *q, T *res,
                          const T *adt, const RedScratch &s, const int *pcell = nullptr,
                          const T *x = nullptr, T *adt_next = nullptr,
                          const AirConst<T> *k = nullptr, bool keep_res = false,
                          bool reverse = false);

}  // namespace op2b
