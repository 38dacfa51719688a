// Batched Airfoil on the GPU (the batching form): many instances of uneven
// mesh size and flow condition solved together.
//
//  * The instances are one OP2 mesh (concatenated, then renumbered so every
//    instance owns a contiguous range of cells, edges and boundary cells).
//  * Each loop stage is ONE persistent launch over a device-side list of work
//    items (instance, [begin, end) chunk); only unconverged instances are
//    listed, so finished instances cost nothing and launch shapes never change.
//  * Instances start with FP32 storage (fluxes in FP32, update and rms in
//    FP64 -- the mixed form) and are promoted to FP64 storage when their rms
//    falls below promote_tol * rms0 or stops falling (FP32 rounding floors
//    the residual near 1e-5 of its start); they finish in FP64 at
//    rms < tol * rms0.  rms0 is an instance's rms after its first iteration.
//  * A single-CTA convergence kernel ends each iteration: per-instance rms,
//    phase changes, and the rebuilt work lists; it publishes the number of
//    active instances to mapped host memory.  The whole iteration (promote,
//    save_soln, 2 x {adt_calc, res_calc, bres_calc, update} for both
//    precisions, convergence) is captured once in a CUDA graph and replayed.
//  * The res_calc strategy and the block size are chosen by a project-written
//    autotuner (op2b_batch_tune) that times each candidate on the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "airfoil_math.cuh"
#include "batch.h"
#include "gather.h"
#include "op2b_batch.h"
#include "op2b_runtime.h"
#include "plan.h"
#include "vec.cuh"

namespace op2b {

constexpr int kMinChunk = 256;  // smallest partition size (elements per work item)

// ------------------------------------------------------------------ stage kernels

#define FOR_ITEMS(list, count)                                   \
  const int nitems = *(count);                                   \
  for (int w = blockIdx.x; w < nitems; w += gridDim.x)

template <typename T>
__global__ void k_b_save(const WorkItem *items, const int *count, const T *q, T *qold) {
  FOR_ITEMS(items, count) {
    WorkItem it = items[w];
    for (int c = it.begin + threadIdx.x; c < it.end; c += blockDim.x) {
      T v[4];
      Vec<T>::ld4(q + 4 * (size_t)c, v);
      Vec<T>::st4(qold + 4 * (size_t)c, v);
    }
  }
}

template <typename T>
__global__ void k_b_adt(const WorkItem *items, const int *count, const int4 *pcell, const T *x,
                        const T *q, T *adt, AirConst<T> k) {
  FOR_ITEMS(items, count) {
    WorkItem it = items[w];
    for (int c = it.begin + threadIdx.x; c < it.end; c += blockDim.x) {
      int4 p = __ldg(pcell + c);
      T a[8], qq[4];
      Vec<T>::ld2(x + 2 * (size_t)p.x, a[0], a[1]);
      Vec<T>::ld2(x + 2 * (size_t)p.y, a[2], a[3]);
      Vec<T>::ld2(x + 2 * (size_t)p.z, a[4], a[5]);
      Vec<T>::ld2(x + 2 * (size_t)p.w, a[6], a[7]);
      Vec<T>::ld4(q + 4 * (size_t)c, qq);
      adt[c] = air_adt<T>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], qq[0], qq[1], qq[2],
                          qq[3], k);
    }
  }
}

constexpr unsigned kRole = 1u << 30;
constexpr unsigned kValid = 1u << 31;

// owner-computes res_calc over the cell items (slot records, see airfoil_gather.cu)
template <typename T>
__global__ void k_b_res_gather(const WorkItem *items, const int *count, const int4 *rec_o,
                               const int4 *rec_n1, const uint4 *rec_n2, const T *x, const T *q,
                               const T *adt, T *res, AirConst<T> k) {
  FOR_ITEMS(items, count) {
    WorkItem it = items[w];
    for (int c = it.begin + threadIdx.x; c < it.end; c += blockDim.x) {
      const int4 o4 = __ldg(rec_o + c), a4 = __ldg(rec_n1 + c);
      const uint4 b4 = __ldg(rec_n2 + c);
      const int o[4] = {o4.x, o4.y, o4.z, o4.w}, n1[4] = {a4.x, a4.y, a4.z, a4.w};
      const unsigned r2[4] = {b4.x, b4.y, b4.z, b4.w};
      T qc[4], acc[4];
      Vec<T>::ld4(q + 4 * (size_t)c, qc);
      T ac = __ldg(adt + c);
      Vec<T>::ld4_rw(res + 4 * (size_t)c, acc);
#pragma unroll
      for (int s = 0; s < 4; s++) {
        if (!(r2[s] & kValid)) continue;
        T qo[4], x1x, x1y, x2x, x2y, f[4];
        Vec<T>::ld4(q + 4 * (size_t)o[s], qo);
        T ao = __ldg(adt + o[s]);
        Vec<T>::ld2(x + 2 * (size_t)n1[s], x1x, x1y);
        Vec<T>::ld2(x + 2 * (size_t)(r2[s] & (kRole - 1)), x2x, x2y);
        if (r2[s] & kRole) {
          air_flux<T>(x1x, x1y, x2x, x2y, qo, qc, ao, ac, k, f);
#pragma unroll
          for (int m = 0; m < 4; m++) acc[m] -= f[m];
        } else {
          air_flux<T>(x1x, x1y, x2x, x2y, qc, qo, ac, ao, k, f);
#pragma unroll
          for (int m = 0; m < 4; m++) acc[m] += f[m];
        }
      }
      Vec<T>::st4(res + 4 * (size_t)c, acc);
    }
  }
}

// atomic res_calc over the edge items
template <typename T>
__global__ void k_b_res_atomic(const WorkItem *items, const int *count, const int2 *pedge,
                               const int2 *pecell, const T *x, const T *q, const T *adt, T *res,
                               AirConst<T> k) {
  FOR_ITEMS(items, count) {
    WorkItem it = items[w];
    for (int e = it.begin + threadIdx.x; e < it.end; e += blockDim.x) {
      int2 nn = __ldg(pedge + e), cc = __ldg(pecell + e);
      T x1x, x1y, x2x, x2y, q1[4], q2[4], f[4];
      Vec<T>::ld2(x + 2 * (size_t)nn.x, x1x, x1y);
      Vec<T>::ld2(x + 2 * (size_t)nn.y, x2x, x2y);
      Vec<T>::ld4(q + 4 * (size_t)cc.x, q1);
      Vec<T>::ld4(q + 4 * (size_t)cc.y, q2);
      air_flux<T>(x1x, x1y, x2x, x2y, q1, q2, __ldg(adt + cc.x), __ldg(adt + cc.y), k, f);
#pragma unroll
      for (int m = 0; m < 4; m++) {
        atomicAdd(res + 4 * (size_t)cc.x + m, f[m]);
        atomicAdd(res + 4 * (size_t)cc.y + m, -f[m]);
      }
    }
  }
}

// coloured res_calc: the edges of one colour (elems[0..n) of the batch's
// OP_COLOR2 plan) share no cell, so each adds its flux to both cells without
// atomics; an edge whose instance is not in this precision's phase is skipped
template <typename T>
__global__ void k_b_res_colour(const int *elems, int n, const int *edge_off, int ninst,
                               const int *phase, int fp64, const int2 *pedge, const int2 *pecell,
                               const T *x, const T *q, const T *adt, T *res, AirConst<T> k) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int e = __ldg(elems + i);
    int lo = 0, hi = ninst - 1;  // the instance owning edge e: edge_off[lo] <= e < edge_off[lo+1]
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(edge_off + mid) <= e) lo = mid;
      else hi = mid - 1;
    }
    const int p = __ldg(phase + lo);
    if (fp64 ? !(p == 1 || p == 3) : p != 0) continue;
    int2 nn = __ldg(pedge + e), cc = __ldg(pecell + e);
    T x1x, x1y, x2x, x2y, q1[4], q2[4], f[4], r1[4], r2[4];
    Vec<T>::ld2(x + 2 * (size_t)nn.x, x1x, x1y);
    Vec<T>::ld2(x + 2 * (size_t)nn.y, x2x, x2y);
    Vec<T>::ld4(q + 4 * (size_t)cc.x, q1);
    Vec<T>::ld4(q + 4 * (size_t)cc.y, q2);
    air_flux<T>(x1x, x1y, x2x, x2y, q1, q2, __ldg(adt + cc.x), __ldg(adt + cc.y), k, f);
    Vec<T>::ld4_rw(res + 4 * (size_t)cc.x, r1);
    Vec<T>::ld4_rw(res + 4 * (size_t)cc.y, r2);
#pragma unroll
    for (int m = 0; m < 4; m++) {
      r1[m] += f[m];
      r2[m] -= f[m];
    }
    Vec<T>::st4(res + 4 * (size_t)cc.x, r1);
    Vec<T>::st4(res + 4 * (size_t)cc.y, r2);
  }
}

// boundary fluxes over the boundary-row items, with each instance's freestream
template <typename T>
__global__ void k_b_bres(const WorkItem *items, const int *count, InvMap inv,
                         const int2 *pbedge, const int *bound, const T *x, const T *q,
                         const T *adt, T *res, const double *qinf, AirConst<T> k) {
  FOR_ITEMS(items, count) {
    WorkItem it = items[w];
    AirConst<T> kk = k;
#pragma unroll
    for (int m = 0; m < 4; m++) kk.qinf[m] = (T)qinf[4 * it.inst + m];
    for (int r = it.begin + threadIdx.x; r < it.end; r += blockDim.x) {
      int c = inv.rows[r];
      long long b = inv.off[c], e = inv.off[c + 1];
      T qc[4], acc[4];
      Vec<T>::ld4(q + 4 * (size_t)c, qc);
      Vec<T>::ld4_rw(res + 4 * (size_t)c, acc);
      T ac = __ldg(adt + c);
      for (long long i = b; i < e; i++) {
        int be = inv.ent[i];
        int2 nn = __ldg(pbedge + be);
        int bnd = __ldg(bound + be);
        T x1x, x1y, x2x, x2y, rr[4];
        Vec<T>::ld2(x + 2 * (size_t)nn.x, x1x, x1y);
        Vec<T>::ld2(x + 2 * (size_t)nn.y, x2x, x2y);
        air_bflux<T>(x1x, x1y, x2x, x2y, qc, ac, bnd, kk, rr);
        if (bnd == 1) {
          acc[1] += rr[1];
          acc[2] += rr[2];
        } else {
#pragma unroll
          for (int m = 0; m < 4; m++) acc[m] += rr[m];
        }
      }
      Vec<T>::st4(res + 4 * (size_t)c, acc);
    }
  }
}

// update (q = qold - res/adt in FP64, res = 0) and the instance's sum of del^2
template <typename T>
__global__ void k_b_update(const WorkItem *items, const int *count, const T *qold, T *q, T *res,
                           const T *adt, double *rms_sum) {
  __shared__ double s_part[32];
  FOR_ITEMS(items, count) {
    WorkItem it = items[w];
    double sum = 0.0;
    for (int c = it.begin + threadIdx.x; c < it.end; c += blockDim.x) {
      T qo[4], r[4], qn[4];
      Vec<T>::ld4(qold + 4 * (size_t)c, qo);
      Vec<T>::ld4_rw(res + 4 * (size_t)c, r);
      double adti = 1.0f / (double)__ldg(adt + c);
#pragma unroll
      for (int m = 0; m < 4; m++) {
        double del = adti * (double)r[m];
        qn[m] = (T)((double)qo[m] - del);
        sum += del * del;
      }
      Vec<T>::st4(q + 4 * (size_t)c, qn);
      T z[4] = {(T)0, (T)0, (T)0, (T)0};
      Vec<T>::st4(res + 4 * (size_t)c, z);
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0 && rms_sum) {  // only the second update of an iteration counts
      double t = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += s_part[i];
      atomicAdd(rms_sum + it.inst, t);
    }
    __syncthreads();
  }
}

// FP32 -> FP64 storage for instances entering the FP64 phase
__global__ void k_b_promote(const WorkItem *items, const int *count, const float *q32,
                            double *q64) {
  FOR_ITEMS(items, count) {
    WorkItem it = items[w];
    for (int c = it.begin + threadIdx.x; c < it.end; c += blockDim.x)
      for (int m = 0; m < 4; m++) q64[4 * (size_t)c + m] = (double)q32[4 * (size_t)c + m];
  }
}

// ------------------------------------------------------------------ convergence + lists

__device__ void build_list(const BatchDev &b, const int *off, int ninst, const int *sel,
                           WorkItem *out, int *count, int *s_scan) {
  // sel[i] != 0: instance i belongs to this list; items of b.chunk elements
  int i = threadIdx.x;
  int n = 0;
  if (i < ninst && sel[i]) n = (off[i + 1] - off[i] + b.chunk - 1) / b.chunk;
  s_scan[i] = n;
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int j = 0; j < ninst; j++) {
      int t = s_scan[j];
      s_scan[j] = acc;
      acc += t;
    }
    *count = acc;
  }
  __syncthreads();
  if (i < ninst && sel[i]) {
    int base = s_scan[i];
    for (int k = 0; k < n; k++) {
      int beg = off[i] + k * b.chunk;
      out[base + k] = WorkItem{i, beg, min(beg + b.chunk, off[i + 1]), 0};
    }
  }
  __syncthreads();
}

__global__ void k_b_converge(BatchDev b, int init) {
  __shared__ int s_sel32[1024], s_sel64[1024], s_selp[1024], s_scan[1024];
  __shared__ int s_active, s_iter;
  int i = threadIdx.x;
  if (i == 0) {
    s_active = 0;
    s_iter = 0;
  }
  __syncthreads();
  if (i < b.ninst) {
    int p = b.phase[i];
    if (!init) {
      if (p == 3) p = 1;  // promoted during the iteration just finished
      if (p == 0 || p == 1) {
        int it = ++b.iters[i];
        if (p == 0) b.iters32[i]++;
        double nc = (double)(b.cell_off[i + 1] - b.cell_off[i]);
        double rms = sqrt(b.rms_sum[i] / (nc > 0 ? nc : 1.0));
        b.rms_sum[i] = 0.0;
        if (it == 1) {
          b.rms0[i] = rms;
          b.rms_prev[i] = rms;
        }
        b.rms_last[i] = rms;
        if (++b.stall[i] >= b.stall_window) {
          bool stalled = rms > 0.99 * b.rms_prev[i];
          b.rms_prev[i] = rms;
          b.stall[i] = stalled ? -1 : 0;  // -1 marks a stall
        }
        bool stalled = b.stall[i] == -1;
        if (stalled) b.stall[i] = 0;
        if (rms < b.tol * b.rms0[i] || it >= b.max_iter || !(rms == rms)) {
          p = 2;
        } else if (p == 0 && (rms < b.promote_tol * b.rms0[i] || stalled)) {
          p = 3;
        }
      }
      b.phase[i] = p;
      atomicMax(&s_iter, b.iters[i]);
    }
    s_sel32[i] = p == 0;
    s_sel64[i] = p == 1 || p == 3;
    s_selp[i] = p == 3;
    if (p != 2) atomicAdd(&s_active, 1);
  } else if (i < 1024) {
    s_sel32[i] = s_sel64[i] = s_selp[i] = 0;
  }
  __syncthreads();
  build_list(b, b.cell_off, b.ninst, s_sel32, b.w32.cells, b.w32.count + 0, s_scan);
  build_list(b, b.brow_off, b.ninst, s_sel32, b.w32.brows, b.w32.count + 1, s_scan);
  build_list(b, b.edge_off, b.ninst, s_sel32, b.w32.edges, b.w32.count + 2, s_scan);
  build_list(b, b.cell_off, b.ninst, s_sel64, b.w64.cells, b.w64.count + 0, s_scan);
  build_list(b, b.brow_off, b.ninst, s_sel64, b.w64.brows, b.w64.count + 1, s_scan);
  build_list(b, b.edge_off, b.ninst, s_sel64, b.w64.edges, b.w64.count + 2, s_scan);
  build_list(b, b.cell_off, b.ninst, s_selp, b.promote, b.npromote, s_scan);
  if (threadIdx.x == 0) {
    volatile int *m = b.mapped;
    m[1] = s_iter;
    __threadfence_system();
    m[0] = s_active;
  }
}

}  // namespace op2b

// ====================================================================== host

using namespace op2b;

struct PrecisionDats {
  int bytes = 0;  // 4 or 8; 0 = absent
  const int *pcell = nullptr, *pedge = nullptr, *pecell = nullptr, *pbedge = nullptr,
            *bound = nullptr;
  void *x = nullptr, *q = nullptr, *qold = nullptr, *adt = nullptr, *res = nullptr;
};

struct op2b_batch_s {
  BatchDev dev{};
  std::vector<void *> owned;
  PrecisionDats p32, p64;
  const SlotRecords *slots = nullptr;
  const InvMap *inv_cells = nullptr, *inv_bound = nullptr;
  op2b_airfoil_dats h32{}, h64{};
  int ninst = 0, ncells = 0;
  int block = 256, blocks_per_sm = 4;
  int res_kernel = OP2B_BATCH_RES_GATHER;
  // OP2B_BATCH_RES_COLOUR: the edges grouped by colour (device) and each
  // colour's first element (host, ncolours + 1 entries), from a parallel
  // OP_COLOR2 colouring of the batch's edges
  const int *colour_elems = nullptr;
  std::vector<int> colour_off;
  cudaGraphExec_t graph = nullptr;
  bool graph_dirty = true;
  std::string tune_report;
  double last_ms = 0.0;
  int graph_iters = 0;
};

template <typename T> static AirConst<T> consts_or(bool &ok) {
  AirConst<T> k{};
  Runtime &r = rt();
  const double *gam = r.const_ptr("gam", 1), *gm1 = r.const_ptr("gm1", 1),
               *cfl = r.const_ptr("cfl", 1), *eps = r.const_ptr("eps", 1);
  ok = gam && gm1 && cfl && eps;
  if (!ok) return k;
  k.gam = (T)*gam;
  k.gm1 = (T)*gm1;
  k.cfl = (T)*cfl;
  k.eps = (T)*eps;
  return k;
}

template <typename T>
static void enqueue_stage(op2b_batch_s *b, const PrecisionDats &d, const WorkLists &w,
                          cudaStream_t s, bool second_half_only) {
  (void)second_half_only;
  bool ok;
  AirConst<T> k = consts_or<T>(ok);
  int grid = rt().nsm * b->blocks_per_sm, th = b->block;
  const T *x = (const T *)d.x;
  T *q = (T *)d.q, *qold = (T *)d.qold, *adt = (T *)d.adt, *res = (T *)d.res;
  k_b_save<T><<<grid, th, 0, s>>>(w.cells, w.count, q, qold);
  for (int step = 0; step < 2; step++) {
    k_b_adt<T><<<grid, th, 0, s>>>(w.cells, w.count, reinterpret_cast<const int4 *>(d.pcell), x,
                                   q, adt, k);
    if (b->res_kernel == OP2B_BATCH_RES_ATOMIC)
      k_b_res_atomic<T><<<grid, th, 0, s>>>(w.edges, w.count + 2,
                                            reinterpret_cast<const int2 *>(d.pedge),
                                            reinterpret_cast<const int2 *>(d.pecell), x, q, adt,
                                            res, k);
    else if (b->res_kernel == OP2B_BATCH_RES_COLOUR)
      for (size_t c = 0; c + 1 < b->colour_off.size(); c++) {
        const int n = b->colour_off[c + 1] - b->colour_off[c];
        if (n <= 0) continue;
        k_b_res_colour<T><<<std::min(grid, (n + th - 1) / th), th, 0, s>>>(
            b->colour_elems + b->colour_off[c], n, b->dev.edge_off, b->ninst, b->dev.phase,
            sizeof(T) == 8, reinterpret_cast<const int2 *>(d.pedge),
            reinterpret_cast<const int2 *>(d.pecell), x, q, adt, res, k);
      }
    else
      k_b_res_gather<T><<<grid, th, 0, s>>>(w.cells, w.count,
                                            reinterpret_cast<const int4 *>(b->slots->o),
                                            reinterpret_cast<const int4 *>(b->slots->n1),
                                            reinterpret_cast<const uint4 *>(b->slots->n2), x, q,
                                            adt, res, k);
    k_b_bres<T><<<grid, th, 0, s>>>(w.brows, w.count + 1, *b->inv_bound,
                                    reinterpret_cast<const int2 *>(d.pbedge), d.bound, x, q, adt,
                                    res, b->dev.qinf, k);
    // rms is that of the second update (airfoil.cpp:265, :281)
    k_b_update<T><<<grid, th, 0, s>>>(w.cells, w.count, qold, q, res, adt,
                                      step == 1 ? b->dev.rms_sum : nullptr);
  }
}

static void enqueue_iteration(op2b_batch_s *b, cudaStream_t s) {
  int grid = rt().nsm * b->blocks_per_sm;
  if (b->p32.bytes && b->p64.bytes)
    k_b_promote<<<grid, b->block, 0, s>>>(b->dev.promote, b->dev.npromote,
                                          (const float *)b->p32.q, (double *)b->p64.q);
  if (b->p32.bytes) enqueue_stage<float>(b, b->p32, b->dev.w32, s, false);
  if (b->p64.bytes) enqueue_stage<double>(b, b->p64, b->dev.w64, s, false);
  k_b_converge<<<1, 1024, 0, s>>>(b->dev, 0);
}

static bool fill_dats(const op2b_airfoil_dats *h, PrecisionDats &d, int want_bytes) {
  if (!h || !h->p_q) return true;
  int tb = type_bytes(h->p_q->type);
  if (tb != want_bytes) {
    set_error("op2b_batch_create: %s dats must be of %s", want_bytes == 4 ? "fp32" : "fp64",
              want_bytes == 4 ? "float" : "double");
    return false;
  }
  d.bytes = tb;
  d.pcell = h->pcell->map_d;
  d.pedge = h->pedge->map_d;
  d.pecell = h->pecell->map_d;
  d.pbedge = h->pbedge->map_d;
  d.bound = (const int *)h->p_bound->data_d;
  d.x = h->p_x->data_d;
  d.q = h->p_q->data_d;
  d.qold = h->p_qold->data_d;
  d.adt = h->p_adt->data_d;
  d.res = h->p_res->data_d;
  return true;
}

// the colours of the batch's edges for OP2B_BATCH_RES_COLOUR: a parallel
// (Jones-Plassmann) OP_COLOR2 plan of res_calc's two increments over pecell,
// built once (before any capture) and kept in the plan cache
static bool build_colouring(op2b_batch_s *b) {
  op_arg args[2] = {op_arg_dat(b->h64.p_res, 0, b->h64.pecell, 4, "double", OP_INC),
                    op_arg_dat(b->h64.p_res, 1, b->h64.pecell, 4, "double", OP_INC)};
  int inds[2] = {0, 0};
  Plan *pl = build_plan("batch res_calc#coloured", b->h64.pecell->from, 0, 2, args, 1, inds,
                        OP_COLOR2, OP2B_COLOUR_JP);
  if (!pl || !pl->col_reord_d || !pl->pub.color2_offsets) {
    if (!op2b_last_error()[0]) set_error("op2b_batch: colouring the edges failed");
    return false;
  }
  b->colour_elems = pl->col_reord_d;
  b->colour_off.assign(pl->pub.color2_offsets, pl->pub.color2_offsets + pl->pub.ncolors + 1);
  return true;
}

extern "C" {

op2b_batch op2b_batch_create(const op2b_airfoil_dats *fp32, const op2b_airfoil_dats *fp64,
                             int ninst, const int *cell_off, const int *edge_off,
                             const double *qinf) {
  Runtime &r = rt();
  if (!r.ready()) return nullptr;
  if (ninst <= 0 || ninst > 1024 || !cell_off || !edge_off || !qinf) {
    set_error("op2b_batch_create: 1..1024 instances with cell/edge offsets and qinf");
    return nullptr;
  }
  if (!fp64 || !fp64->p_q) {
    set_error("op2b_batch_create: the fp64 dats are required (the finishing phase)");
    return nullptr;
  }
  auto *b = new op2b_batch_s();
  b->ninst = ninst;
  if (!fill_dats(fp32, b->p32, 4) || !fill_dats(fp64, b->p64, 8)) {
    delete b;
    return nullptr;
  }
  b->h64 = *fp64;
  if (fp32) b->h32 = *fp32;
  op_map pecell = fp64->pecell, pedge = fp64->pedge, pbecell = fp64->pbecell;
  b->ncells = pecell->to->size;
  if (cell_off[0] != 0 || cell_off[ninst] != b->ncells || edge_off[0] != 0 ||
      edge_off[ninst] != pecell->from->size) {
    set_error("op2b_batch_create: offsets must start at 0 and end at the set sizes");
    delete b;
    return nullptr;
  }
  b->slots = get_slot_records(pecell, pedge);
  b->inv_bound = get_inverse_map(pbecell);
  if (!b->slots || !b->inv_bound || !b->slots->usable) {
    if (b->slots && !b->slots->usable)
      set_error("op2b_batch_create: a cell has more than four edges");
    delete b;
    return nullptr;
  }
  // boundary-row ranges: rows are sorted cells, instances own contiguous cell ranges
  std::vector<int> rows(b->inv_bound->nrows);
  if (!rows.empty())
    cudaMemcpy(rows.data(), b->inv_bound->rows, sizeof(int) * rows.size(), cudaMemcpyDeviceToHost);
  std::vector<int> brow_off(ninst + 1);
  for (int i = 0; i <= ninst; i++)
    brow_off[i] = (int)(std::lower_bound(rows.begin(), rows.end(), cell_off[i]) - rows.begin());
  auto A = [&](size_t bytes) -> void * {
    void *p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, bytes ? bytes : 1);
    b->owned.push_back(p);
    return p;
  };
  BatchDev &d = b->dev;
  d.ninst = ninst;
  d.chunk = 2048;
  d.tol = 1e-6;
  d.promote_tol = 1e-4;
  d.max_iter = 1000000;
  d.stall_window = 2000;
  int *co = (int *)A(sizeof(int) * (ninst + 1)), *eo = (int *)A(sizeof(int) * (ninst + 1)),
      *bo = (int *)A(sizeof(int) * (ninst + 1));
  cudaMemcpy(co, cell_off, sizeof(int) * (ninst + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(eo, edge_off, sizeof(int) * (ninst + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(bo, brow_off.data(), sizeof(int) * (ninst + 1), cudaMemcpyHostToDevice);
  d.cell_off = co;
  d.edge_off = eo;
  d.brow_off = bo;
  d.phase = (int *)A(sizeof(int) * ninst);
  d.rms_sum = (double *)A(sizeof(double) * ninst);
  d.rms0 = (double *)A(sizeof(double) * ninst);
  d.rms_last = (double *)A(sizeof(double) * ninst);
  d.rms_prev = (double *)A(sizeof(double) * ninst);
  d.iters = (int *)A(sizeof(int) * ninst);
  d.iters32 = (int *)A(sizeof(int) * ninst);
  d.stall = (int *)A(sizeof(int) * ninst);
  double *qi = (double *)A(sizeof(double) * 4 * ninst);
  cudaMemcpy(qi, qinf, sizeof(double) * 4 * ninst, cudaMemcpyHostToDevice);
  d.qinf = qi;
  // list capacities: every instance active, at the smallest partition size
  size_t cap_c = 0, cap_b = 0, cap_e = 0;
  const int cmin = kMinChunk;
  for (int i = 0; i < ninst; i++) {
    cap_c += (cell_off[i + 1] - cell_off[i] + cmin - 1) / cmin;
    cap_b += (brow_off[i + 1] - brow_off[i] + cmin - 1) / cmin;
    cap_e += (edge_off[i + 1] - edge_off[i] + cmin - 1) / cmin;
  }
  for (WorkLists *w : {&d.w32, &d.w64}) {
    w->cells = (WorkItem *)A(sizeof(WorkItem) * (cap_c + 1));
    w->brows = (WorkItem *)A(sizeof(WorkItem) * (cap_b + 1));
    w->edges = (WorkItem *)A(sizeof(WorkItem) * (cap_e + 1));
    w->count = (int *)A(sizeof(int) * 4);
  }
  d.promote = (WorkItem *)A(sizeof(WorkItem) * (cap_c + 1));
  d.npromote = (int *)A(sizeof(int));
  void *mh = nullptr, *md = nullptr;
  if (cudaHostAlloc(&mh, 4096, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(&md, mh, 0) != cudaSuccess) {
    set_error("op2b_batch_create: mapped host page");
    delete b;
    return nullptr;
  }
  memset(mh, 0, 4096);
  b->owned.push_back(nullptr);  // marker: mapped page freed separately
  d.mapped = (int *)md;
  // start phase: FP32 storage when fp32 dats exist
  std::vector<int> ph(ninst, b->p32.bytes ? 0 : 1);
  cudaMemcpy(d.phase, ph.data(), sizeof(int) * ninst, cudaMemcpyHostToDevice);
  b->owned.push_back(mh);  // host page pointer kept last (freed with cudaFreeHost)
  k_b_converge<<<1, 1024, 0, r.stream>>>(d, 1);
  if (!cuda_ok(cudaStreamSynchronize(r.stream), "op2b_batch_create")) {
    op2b_batch_destroy(b);
    return nullptr;
  }
  return b;
}

static volatile int *mapped_host(op2b_batch b) { return (volatile int *)b->owned.back(); }

int op2b_batch_set(op2b_batch b, const char *key, double value) {
  if (!b || !key) return -1;
  std::string k(key);
  BatchDev &d = b->dev;
  if (k == "tol") d.tol = value;
  else if (k == "promote_tol") d.promote_tol = value;
  else if (k == "max_iter") d.max_iter = (int)value;
  else if (k == "stall_window") d.stall_window = std::max(1, (int)value);
  else if (k == "block") b->block = (int)value;
  else if (k == "blocks_per_sm") b->blocks_per_sm = std::max(1, (int)value);
  else if (k == "res_kernel") {
    if (value < OP2B_BATCH_RES_GATHER || value > OP2B_BATCH_RES_COLOUR) {
      set_error("op2b_batch_set: res_kernel must be OP2B_BATCH_RES_GATHER, _ATOMIC or _COLOUR");
      return -1;
    }
    b->res_kernel = (int)value;
  } else if (k == "part_size") {
    if (value < kMinChunk || value > (1 << 24)) {
      set_error("op2b_batch_set: part_size must be in [%d, %d]", kMinChunk, 1 << 24);
      return -1;
    }
    d.chunk = (int)value;  // the work lists of the next iteration use it
  } else {
    set_error("op2b_batch_set: unknown key '%s'", key);
    return -1;
  }
  if (b->block != 128 && b->block != 256 && b->block != 512) {
    set_error("op2b_batch_set: block must be 128, 256 or 512");
    b->block = 256;
    return -1;
  }
  b->graph_dirty = true;
  return 0;
}

int op2b_batch_run(op2b_batch b, int max_iterations, int check_every, int use_graph,
                   double *elapsed_ms) {
  Runtime &r = rt();
  if (!b || !r.ready()) return -1;
  cudaStream_t s = r.stream;
  if (check_every < 1) check_every = 1;
  if (b->res_kernel == OP2B_BATCH_RES_COLOUR && !b->colour_elems && !build_colouring(b))
    return -1;
  if (use_graph && b->graph_dirty) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    cudaGraph_t g;
    cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    enqueue_iteration(b, s);
    if (!cuda_ok(cudaStreamEndCapture(s, &g), "op2b_batch_run: capture")) return -1;
    if (!cuda_ok(cudaGraphInstantiate(&b->graph, g, 0), "op2b_batch_run: instantiate")) {
      cudaGraphDestroy(g);
      return -1;
    }
    cudaGraphDestroy(g);
    b->graph_dirty = false;
  }
  volatile int *m = mapped_host(b);
  auto t0 = std::chrono::steady_clock::now();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  int done = 0;
  while (done < max_iterations) {
    int n = std::min(check_every, max_iterations - done);
    for (int i = 0; i < n; i++) {
      if (use_graph) {
        if (!cuda_ok(cudaGraphLaunch(b->graph, s), "op2b_batch_run: graph launch")) return -1;
      } else {
        enqueue_iteration(b, s);
        r.launches += 20;
      }
    }
    if (use_graph) r.launches += 20L * n;
    done += n;
    if (!cuda_ok(cudaStreamSynchronize(s), "op2b_batch_run")) return -1;
    if (m[0] == 0) break;
  }
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  (void)t0;
  b->last_ms = ms;
  if (elapsed_ms) *elapsed_ms = ms;
  return m[0];  // instances still active
}

int op2b_batch_stats(op2b_batch b, int *iters, int *iters32, double *rms0, double *rms_last,
                     int *phase) {
  if (!b) return -1;
  int n = b->ninst;
  BatchDev &d = b->dev;
  cudaStreamSynchronize(rt().stream);
  if (iters) cudaMemcpy(iters, d.iters, sizeof(int) * n, cudaMemcpyDeviceToHost);
  if (iters32) cudaMemcpy(iters32, d.iters32, sizeof(int) * n, cudaMemcpyDeviceToHost);
  if (rms0) cudaMemcpy(rms0, d.rms0, sizeof(double) * n, cudaMemcpyDeviceToHost);
  if (rms_last) cudaMemcpy(rms_last, d.rms_last, sizeof(double) * n, cudaMemcpyDeviceToHost);
  if (phase) cudaMemcpy(phase, d.phase, sizeof(int) * n, cudaMemcpyDeviceToHost);
  return cuda_ok(cudaGetLastError(), "op2b_batch_stats") ? 0 : -1;
}

// Autotuner: time `iters` iterations of every candidate (res_calc strategy x
// block size) on the batch as it stands, keep the fastest.  The batch state is
// restored afterwards (q, phases and counters), so tuning does not advance the
// solve.
int op2b_batch_tune(op2b_batch b, int iters, char *report, int report_len) {
  Runtime &r = rt();
  if (!b || !r.ready()) return -1;
  cudaStream_t s = r.stream;
  BatchDev &d = b->dev;
  int n = b->ninst;
  // snapshot
  std::vector<void *> snap;
  auto save = [&](const void *src, size_t bytes) {
    void *p = nullptr;
    cudaMalloc(&p, bytes ? bytes : 1);
    cudaMemcpyAsync(p, src, bytes, cudaMemcpyDeviceToDevice, s);
    snap.push_back(p);
    return p;
  };
  auto restore = [&](void *dst, const void *src, size_t bytes) {
    cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s);
  };
  size_t qb32 = b->p32.bytes ? (size_t)b->ncells * 16 : 0, qb64 = (size_t)b->ncells * 32;
  void *sq32 = qb32 ? save(b->p32.q, qb32) : nullptr;
  void *sq64 = save(b->p64.q, qb64);
  void *sph = save(d.phase, sizeof(int) * n);
  struct Cand {
    int res_kernel, block, part;
  };
  std::vector<Cand> cands;
  for (int rk : {OP2B_BATCH_RES_GATHER, OP2B_BATCH_RES_ATOMIC, OP2B_BATCH_RES_COLOUR})
    for (int blk : {128, 256, 512})
      for (int part : {512, 2048, 8192}) cands.push_back({rk, blk, part});
  double best = 1e30;
  Cand bestc = {b->res_kernel, b->block, d.chunk};
  std::string rep;
  static const char *kRes[] = {"gather", "atomic", "colour"};
  for (const Cand &c : cands) {
    b->res_kernel = c.res_kernel;
    b->block = c.block;
    d.chunk = c.part;
    b->graph_dirty = true;
    // reset state before each candidate
    if (sq32) restore(b->p32.q, sq32, qb32);
    restore(b->p64.q, sq64, qb64);
    restore(d.phase, sph, sizeof(int) * n);
    cudaMemsetAsync(d.iters, 0, sizeof(int) * n, s);
    cudaMemsetAsync(d.iters32, 0, sizeof(int) * n, s);
    cudaMemsetAsync(d.rms_sum, 0, sizeof(double) * n, s);
    cudaMemsetAsync(d.stall, 0, sizeof(int) * n, s);
    k_b_converge<<<1, 1024, 0, s>>>(d, 1);
    double ms = 0.0;
    op2b_batch_run(b, 2, 2, 1, &ms);  // warm up (builds the graph)
    if (op2b_batch_run(b, iters, iters, 1, &ms) < 0) return -1;
    double per = ms / std::max(iters, 1);
    char line[160];
    snprintf(line, sizeof(line), "res_kernel=%s block=%d part_size=%d: %.4f ms/iter\n",
             kRes[c.res_kernel], c.block, c.part, per);
    rep += line;
    if (per < best) {
      best = per;
      bestc = c;
    }
  }
  b->res_kernel = bestc.res_kernel;
  b->block = bestc.block;
  d.chunk = bestc.part;
  b->graph_dirty = true;
  if (sq32) restore(b->p32.q, sq32, qb32);
  restore(b->p64.q, sq64, qb64);
  restore(d.phase, sph, sizeof(int) * n);
  cudaMemsetAsync(d.iters, 0, sizeof(int) * n, s);
  cudaMemsetAsync(d.iters32, 0, sizeof(int) * n, s);
  cudaMemsetAsync(d.rms_sum, 0, sizeof(double) * n, s);
  cudaMemsetAsync(d.stall, 0, sizeof(int) * n, s);
  if (b->p32.bytes) cudaMemsetAsync(b->p32.res, 0, qb32, s);
  cudaMemsetAsync(b->p64.res, 0, qb64, s);
  k_b_converge<<<1, 1024, 0, s>>>(d, 1);
  bool ok = cuda_ok(cudaStreamSynchronize(s), "op2b_batch_tune");
  for (void *p : snap) cudaFree(p);
  char line[160];
  snprintf(line, sizeof(line), "chosen: res_kernel=%s block=%d part_size=%d\n",
           kRes[bestc.res_kernel], bestc.block, bestc.part);
  rep += line;
  b->tune_report = rep;
  if (report && report_len > 0) {
    strncpy(report, rep.c_str(), (size_t)report_len - 1);
    report[report_len - 1] = 0;
  }
  return ok ? 0 : -1;
}

void op2b_batch_destroy(op2b_batch b) {
  if (!b) return;
  cudaStreamSynchronize(rt().stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  void *mh = b->owned.back();
  b->owned.pop_back();
  cudaFreeHost(mh);
  for (void *p : b->owned)
    if (p) cudaFree(p);
  delete b;
}

}  // extern "C"
