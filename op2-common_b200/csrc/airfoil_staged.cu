// Plan-driven indirect-increment loops: res_calc and bres_calc with block and
// thread colouring, and the staged hybrid.
//
// res_calc, staged (one CTA per plan block of `bsize` edges):
//   1. stage the block's distinct cells (q, adt; res accumulators zeroed) and
//      nodes (x) into shared memory through the plan's ind_maps -- each
//      gathered record is read from HBM once per block, not once per edge;
//   2. every thread computes its edges' fluxes from shared memory through the
//      plan's loc_maps (16-bit local indices);
//   3. increments are applied to the shared accumulators one thread colour at
//      a time (the plan guarantees that no two edges of a colour share a cell),
//      with a barrier between colours;
//   4. the block's accumulators are added to res in HBM:
//      * colouring (inc_mode 1): one launch per block colour; blocks of a
//        colour share no cell, so a plain read-modify-write is race free;
//      * hybrid (inc_mode 2): one launch over all blocks; cells that only this
//        block touches take a plain read-modify-write, cells shared with
//        another block an FP64 atomicAdd (flags built once per plan).
// The colouring variant is deterministic: a cell's increments arrive in
// thread-colour order within a block and in block-colour order across blocks.
//
// bres_calc, colouring: thread colours within a block and block colours
// across launches, applying each boundary edge's increment to res in HBM
// directly (7,200 edges at 2.88M cells: staging would not pay).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "airfoil_math.cuh"
#include "op2b_runtime.h"
#include "plan.h"
#include "staged.h"
#include "vec.cuh"

namespace op2b {

struct ResPlanDev {
  int bsize, nst;
  const int *nodes_map, *cells_map;  // ind_map of staged slots 0 (x) and 1 (q; adt, res identical)
  const int *ind_offs, *ind_sizes;
  const short *ln1, *ln2, *lc1, *lc2;
  const int *thrcol, *nthrcol, *blkmap;
  const unsigned char *cell_shared;
};

constexpr int kStagedThreads = 256;

template <typename T, int EPT, bool HYBRID>
__global__ void __launch_bounds__(kStagedThreads)
k_res_staged(ResPlanDev P, int blk_first, int nedge, const T *__restrict__ x,
             const T *__restrict__ q, const T *__restrict__ adt, T *__restrict__ res,
             AirConst<T> k) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int b = HYBRID ? (int)blockIdx.x : P.blkmap[blk_first + blockIdx.x];
  const int beg = b * P.bsize;
  const int n = min(P.bsize, nedge - beg);
  const int on = P.ind_offs[(size_t)b * P.nst], nn = P.ind_sizes[(size_t)b * P.nst];
  const int oc = P.ind_offs[(size_t)b * P.nst + 1], nc = P.ind_sizes[(size_t)b * P.nst + 1];
  T *q_s = reinterpret_cast<T *>(smraw);
  T *r_s = q_s + 4 * nc;
  T *x_s = r_s + 4 * nc;
  T *a_s = x_s + 2 * nn;

  // 1. stage
  for (int i = threadIdx.x; i < nc; i += kStagedThreads) {
    int c = __ldg(P.cells_map + oc + i);
    T v[4];
    Vec<T>::ld4(q + 4 * (size_t)c, v);
    Vec<T>::st4(q_s + 4 * i, v);
    T z[4] = {(T)0, (T)0, (T)0, (T)0};
    Vec<T>::st4(r_s + 4 * i, z);
    a_s[i] = __ldg(adt + c);
  }
  for (int i = threadIdx.x; i < nn; i += kStagedThreads) {
    int nd = __ldg(P.nodes_map + on + i);
    T a0, a1;
    Vec<T>::ld2(x + 2 * (size_t)nd, a0, a1);
    x_s[2 * i] = a0;
    x_s[2 * i + 1] = a1;
  }
  __syncthreads();

  // 2. fluxes of this thread's edges
  T f[EPT][4];
  int col[EPT], l1[EPT], l2[EPT];
#pragma unroll
  for (int j = 0; j < EPT; j++) {
    int e = threadIdx.x + j * kStagedThreads;
    col[j] = -1;
    if (e < n) {
      int g = beg + e;
      int n1 = P.ln1[g], n2 = P.ln2[g];
      l1[j] = P.lc1[g];
      l2[j] = P.lc2[g];
      col[j] = P.thrcol[g];
      air_flux<T>(x_s[2 * n1], x_s[2 * n1 + 1], x_s[2 * n2], x_s[2 * n2 + 1], q_s + 4 * l1[j],
                  q_s + 4 * l2[j], a_s[l1[j]], a_s[l2[j]], k, f[j]);
    }
  }

  // 3. increments, one thread colour at a time
  const int ncol = P.nthrcol[b];
  for (int cc = 0; cc < ncol; cc++) {
#pragma unroll
    for (int j = 0; j < EPT; j++) {
      if (col[j] == cc) {
        T *r1 = r_s + 4 * l1[j], *r2 = r_s + 4 * l2[j];
#pragma unroll
        for (int m = 0; m < 4; m++) {
          r1[m] += f[j][m];
          r2[m] -= f[j][m];
        }
      }
    }
    __syncthreads();
  }
  if (ncol == 0) __syncthreads();

  // 4. accumulate into res
  for (int i = threadIdx.x; i < nc; i += kStagedThreads) {
    int c = __ldg(P.cells_map + oc + i);
    T *dst = res + 4 * (size_t)c;
    const T *src = r_s + 4 * i;
    if (HYBRID && P.cell_shared[oc + i]) {
#pragma unroll
      for (int m = 0; m < 4; m++) atomicAdd(dst + m, src[m]);
    } else {
      T v[4];
      Vec<T>::ld4_rw(dst, v);
#pragma unroll
      for (int m = 0; m < 4; m++) v[m] += src[m];
      Vec<T>::st4(dst, v);
    }
  }
}

struct BresPlanDev {
  int bsize;
  const int *thrcol, *nthrcol, *blkmap;
};

template <typename T>
__global__ void __launch_bounds__(kStagedThreads)
k_bres_colour(BresPlanDev P, int blk_first, int nbedge, const int2 *__restrict__ pbedge,
              const int *__restrict__ pbecell, const int *__restrict__ bound,
              const T *__restrict__ x, const T *__restrict__ q, const T *__restrict__ adt,
              T *__restrict__ res, AirConst<T> k) {
  const int b = P.blkmap[blk_first + blockIdx.x];
  const int beg = b * P.bsize;
  const int n = min(P.bsize, nbedge - beg);
  const int ncol = P.nthrcol[b];
  for (int e0 = 0; e0 < n; e0 += kStagedThreads) {
    int e = e0 + threadIdx.x;
    int col = -1, c1 = 0, bnd = 0;
    T r[4];
    if (e < n) {
      int g = beg + e;
      int2 nd = __ldg(pbedge + g);
      c1 = __ldg(pbecell + g);
      bnd = __ldg(bound + g);
      col = P.thrcol[g];
      T x1x, x1y, x2x, x2y, q1[4];
      Vec<T>::ld2(x + 2 * (size_t)nd.x, x1x, x1y);
      Vec<T>::ld2(x + 2 * (size_t)nd.y, x2x, x2y);
      Vec<T>::ld4(q + 4 * (size_t)c1, q1);
      air_bflux<T>(x1x, x1y, x2x, x2y, q1, __ldg(adt + c1), bnd, k, r);
    }
    for (int cc = 0; cc < ncol; cc++) {
      if (col == cc) {
        T *d = res + 4 * (size_t)c1;
        if (bnd == 1) {  // a wall edge leaves components 0 and 3 untouched
          d[1] += r[1];
          d[2] += r[2];
        } else {
#pragma unroll
          for (int m = 0; m < 4; m++) d[m] += r[m];
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------------ host side

Plan *get_res_plan(const char *name, op_set set, int nargs, op_arg *args) {
  int inds[8] = {0, 0, 1, 1, 2, 2, 3, 3};
  return build_plan(name, set, rt().opt_part_size, nargs, args, 4, inds, OP_STAGE_ALL,
                    rt().opt_plan_mode == 1 ? OP2B_COLOUR_JP : OP2B_COLOUR_GREEDY);
}

Plan *get_bres_plan(const char *name, op_set set, int nargs, op_arg *args) {
  int inds[6] = {0, 0, 1, 2, 3, -1};
  return build_plan(name, set, rt().opt_part_size, nargs, args, 4, inds, OP_STAGE_ALL,
                    rt().opt_plan_mode == 1 ? OP2B_COLOUR_JP : OP2B_COLOUR_GREEDY);
}

template <typename T, int EPT, bool HYBRID>
static cudaError_t launch_staged(const LaunchCtx &c, const ResCalcArgs<T> &a, const ResPlanDev &d,
                                 const Plan &pl, size_t smem) {
  auto kern = k_res_staged<T, EPT, HYBRID>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
  }
  if (HYBRID) {
    kern<<<pl.pub.nblocks, kStagedThreads, smem, c.stream>>>(d, 0, a.nedge, a.x, a.q, a.adt,
                                                             a.res, a.k);
    c.count();
  } else {
    int first = 0;
    for (int col = 0; col < pl.pub.ncolors; col++) {
      int nb = pl.pub.ncolblk[col];
      if (nb > 0) {
        kern<<<nb, kStagedThreads, smem, c.stream>>>(d, first, a.nedge, a.x, a.q, a.adt, a.res,
                                                     a.k);
        c.count();
      }
      first += nb;
    }
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t run_res_calc(const LaunchCtx &c, const ResCalcArgs<T> &a, Plan *plan, int mode) {
  if (a.nedge <= 0) return cudaSuccess;
  if (mode == OP2B_INC_ATOMIC || !plan)
    return launch_res_calc_atomic<T>(c, a.nedge, a.pedge, a.pecell, a.x, a.q, a.adt, a.res, a.k,
                                     rt().opt_atomic_seg != 0, rt().opt_atomic_blocks);
  const Plan &pl = *plan;
  ResPlanDev d{};
  d.bsize = pl.bsize;
  d.nst = pl.pub.ninds_staged;
  d.nodes_map = plan_ind_map_slot(pl, 0);
  d.cells_map = plan_ind_map_slot(pl, 1);
  d.ind_offs = pl.ind_offs_d;
  d.ind_sizes = pl.ind_sizes_d;
  const size_t E = (size_t)pl.set->size;
  d.ln1 = pl.loc_map_d;
  d.ln2 = pl.loc_map_d + E;
  d.lc1 = pl.loc_map_d + 2 * E;
  d.lc2 = pl.loc_map_d + 3 * E;
  d.thrcol = pl.thrcol_d;
  d.nthrcol = pl.nthrcol_d;
  d.blkmap = pl.blkmap_d;
  d.cell_shared = nullptr;
  if (mode == OP2B_INC_HYBRID) {
    d.cell_shared = plan_shared_flags(const_cast<Plan &>(pl), 1);
    if (!d.cell_shared) return cudaErrorMemoryAllocation;
  }
  size_t smem = sizeof(T) * (9 * (size_t)pl.max_ind_size[1] + 2 * (size_t)pl.max_ind_size[0]);
  int ept = (pl.bsize + kStagedThreads - 1) / kStagedThreads;
  bool hyb = mode == OP2B_INC_HYBRID;
#define OP2B_STAGED(E)                                                                  \
  return hyb ? launch_staged<T, E, true>(c, a, d, pl, smem)                             \
             : launch_staged<T, E, false>(c, a, d, pl, smem);
  if (ept <= 1) OP2B_STAGED(1)
  if (ept <= 2) OP2B_STAGED(2)
  if (ept <= 4) OP2B_STAGED(4)
  if (ept <= 8) OP2B_STAGED(8)
#undef OP2B_STAGED
  return cudaErrorInvalidConfiguration;
}

template <typename T>
cudaError_t run_bres_calc(const LaunchCtx &c, const BresCalcArgs<T> &a, Plan *plan, int mode) {
  if (a.nbedge <= 0) return cudaSuccess;
  if (mode != OP2B_INC_COLOR || !plan)
    return launch_bres_calc_atomic<T>(c, a.nbedge, a.pbedge, a.pbecell, a.bound, a.x, a.q, a.adt,
                                      a.res, a.k);
  const Plan &pl = *plan;
  BresPlanDev d{pl.bsize, pl.thrcol_d, pl.nthrcol_d, pl.blkmap_d};
  int first = 0;
  for (int col = 0; col < pl.pub.ncolors; col++) {
    int nb = pl.pub.ncolblk[col];
    if (nb > 0) {
      k_bres_colour<T><<<nb, kStagedThreads, 0, c.stream>>>(
          d, first, a.nbedge, reinterpret_cast<const int2 *>(a.pbedge), a.pbecell, a.bound, a.x,
          a.q, a.adt, a.res, a.k);
      c.count();
    }
    first += nb;
  }
  return cudaGetLastError();
}

template cudaError_t run_res_calc<double>(const LaunchCtx &, const ResCalcArgs<double> &, Plan *,
                                          int);
template cudaError_t run_res_calc<float>(const LaunchCtx &, const ResCalcArgs<float> &, Plan *,
                                         int);
template cudaError_t run_bres_calc<double>(const LaunchCtx &, const BresCalcArgs<double> &,
                                           Plan *, int);
template cudaError_t run_bres_calc<float>(const LaunchCtx &, const BresCalcArgs<float> &, Plan *,
                                          int);

}  // namespace op2b
