// Device loops for the five Airfoil kernels (save_soln, adt_calc, res_calc,
// bres_calc, update) on sm_100a.
//
// Layout: every dat is AoS in HBM (element = dim contiguous values), maps
// are AoS int32 [from][dim].  A cell's q is one aligned 32-byte (FP64) or
// 16-byte (FP32) record, so a gathered q costs one DRAM sector, and direct
// loops read it with 16-byte vector loads that coalesce across a warp.
//
// Direct loops (save_soln, update, adt_calc's cell-side streams) run a
// persistent grid (a multiple of the SM count) with grid-stride loops.
// update fuses the rms sum and the maxerr max/argmax (op_arg_gbl OP_INC,
// OP_MAX and op_arg_info of update.h) into one pass: warp shuffles, one shared
// memory round per block, and the last block to finish reduces the per-block
// partials in a fixed order, so the result is deterministic run to run and
// needs no second launch.
//
// Indirect increments (res_calc, bres_calc) have three variants, selected by
// the runtime: plain FP64/FP32 atomics (this file), and the plan-driven
// staged variants in airfoil_staged.cu.
#include <mutex>
#include <unordered_map>

#include "airfoil_math.cuh"
#include "loops.h"
#include "vec.cuh"

#include <stdint.h>

namespace op2b {

static inline int grid_for(const LaunchCtx &c, long long n, int threads, int per_sm) {
  long long want = (n + threads - 1) / threads;
  long long cap = (long long)c.nsm * per_sm;
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

// grid_for with per_sm capped at the CTAs an SM can actually hold of `kern`
// (its registers or shared memory may allow fewer than asked): a grid-stride
// kernel then runs as one wave, every CTA resident, instead of a wave and a
// partial second one.  adt_calc gains (45.6 against 49.7 us at 2400x1200);
// the atomic res_calc loses (its late CTAs even out the scattered atomics),
// so it keeps grid_for.
template <typename K>
static int grid_resident(const LaunchCtx &c, K kern, long long n, int threads, int per_sm) {
  static std::mutex mu;
  static std::unordered_map<const void *, int> fit;  // kernel -> resident CTAs per SM
  int r = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = fit.find((const void *)kern);
    if (it != fit.end()) r = it->second;
  }
  if (r == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, kern, threads, 0) != cudaSuccess ||
        r < 1) {
      cudaGetLastError();
      r = 1;
    }
    std::lock_guard<std::mutex> lock(mu);
    fit[(const void *)kern] = r;
  }
  return grid_for(c, n, threads, per_sm < r ? per_sm : r);
}

// ---------------------------------------------------------------- save_soln

// save_soln.h:1-4 is a copy of q into qold: 16-byte vector copy, 4 loads in
// flight per thread before the stores.
__global__ void __launch_bounds__(256) k_copy16(const uint4 *__restrict__ src,
                                                uint4 *__restrict__ dst, long long n16) {
  long long stride = (long long)gridDim.x * blockDim.x;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n16; i += 4 * stride) {
    uint4 a = __ldcs(src + i), b = __ldcs(src + i + stride);
    uint4 c = __ldcs(src + i + 2 * stride), d = __ldcs(src + i + 3 * stride);
    __stcs(dst + i, a);
    __stcs(dst + i + stride, b);
    __stcs(dst + i + 2 * stride, c);
    __stcs(dst + i + 3 * stride, d);
  }
  for (; i < n16; i += stride)
    __stcs(dst + i, __ldcs(src + i));
}

__global__ void k_copy_tail(const unsigned char *src, unsigned char *dst, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i];
}

cudaError_t launch_copy(const LaunchCtx &c, const void *src, void *dst, size_t bytes) {
  long long n16 = (long long)(bytes / 16);
  if (n16 > 0) {
    k_copy16<<<grid_for(c, n16, 256, 8), 256, 0, c.stream>>>(
        static_cast<const uint4 *>(src), static_cast<uint4 *>(dst), n16);
    c.count();
  }
  long long tail = (long long)(bytes - 16 * (size_t)n16);
  if (tail > 0) {
    k_copy_tail<<<1, 32, 0, c.stream>>>(static_cast<const unsigned char *>(src) + 16 * n16,
                                        static_cast<unsigned char *>(dst) + 16 * n16, tail);
    c.count();
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------- adt_calc

template <typename T>
__device__ __forceinline__ void adt_calc_cells(int ncell, const int4 *__restrict__ pcell,
                                               const T *__restrict__ x, const T *__restrict__ q,
                                               T *__restrict__ adt, const AirConst<T> &k) {
  int stride = gridDim.x * blockDim.x;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < ncell; n += stride) {
    int4 c = __ldg(pcell + n);
    T x1x, x1y, x2x, x2y, x3x, x3y, x4x, x4y, qq[4];
    Vec<T>::ld2(x + 2 * (size_t)c.x, x1x, x1y);
    Vec<T>::ld2(x + 2 * (size_t)c.y, x2x, x2y);
    Vec<T>::ld2(x + 2 * (size_t)c.z, x3x, x3y);
    Vec<T>::ld2(x + 2 * (size_t)c.w, x4x, x4y);
    Vec<T>::ld4(q + 4 * (size_t)n, qq);
    adt[n] = air_adt<T>(x1x, x1y, x2x, x2y, x3x, x3y, x4x, x4y, qq[0], qq[1],
                        qq[2], qq[3], k);
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
k_adt_calc(int ncell, const int4 *__restrict__ pcell, const T *__restrict__ x,
           const T *__restrict__ q, T *__restrict__ adt, AirConst<T> k) {
  adt_calc_cells<T>(ncell, pcell, x, q, adt, k);
}

// save_soln fused into the adt_calc that follows it (the runtime defers a
// save_soln until the next loop call and, when that is adt_calc over the same
// q, launches this instead of both): q is read once, copied to qold and used
// for the time step.  Same values as the two loops run one after the other.
template <typename T>
__global__ void __launch_bounds__(256)
k_adt_save(int ncell, const int4 *__restrict__ pcell, const T *__restrict__ x,
           const T *__restrict__ q, T *__restrict__ adt, T *__restrict__ qold, AirConst<T> k) {
  int stride = gridDim.x * blockDim.x;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < ncell; n += stride) {
    int4 c = __ldg(pcell + n);
    T x1x, x1y, x2x, x2y, x3x, x3y, x4x, x4y, qq[4];
    Vec<T>::ld2(x + 2 * (size_t)c.x, x1x, x1y);
    Vec<T>::ld2(x + 2 * (size_t)c.y, x2x, x2y);
    Vec<T>::ld2(x + 2 * (size_t)c.z, x3x, x3y);
    Vec<T>::ld2(x + 2 * (size_t)c.w, x4x, x4y);
    Vec<T>::ld4(q + 4 * (size_t)n, qq);
    Vec<T>::st4_cs(qold + 4 * (size_t)n, qq);  // read again only by update
    adt[n] = air_adt<T>(x1x, x1y, x2x, x2y, x3x, x3y, x4x, x4y, qq[0], qq[1],
                        qq[2], qq[3], k);
  }
}

template <typename T>
cudaError_t launch_adt_save(const LaunchCtx &c, int ncell, const int *pcell, const T *x,
                            const T *q, T *adt, T *qold, const AirConst<T> &k) {
  if (ncell <= 0) return cudaSuccess;
  k_adt_save<T><<<grid_for(c, ncell, 256, 8), 256, 0, c.stream>>>(
      ncell, reinterpret_cast<const int4 *>(pcell), x, q, adt, qold, k);
  c.count();
  return cudaGetLastError();
}

// the same loop with a register cap (MINB CTAs of 256 threads per SM)
template <typename T, int MINB>
__global__ void __launch_bounds__(256, MINB)
k_adt_calc_mb(int ncell, const int4 *__restrict__ pcell, const T *__restrict__ x,
              const T *__restrict__ q, T *__restrict__ adt, AirConst<T> k) {
  adt_calc_cells<T>(ncell, pcell, x, q, adt, k);
}

// (A register-pipelined persistent form of this loop -- the next cell's node
// gathers in flight during the current cell's square roots -- needs 92
// registers instead of 54 and measured 3.93 TB/s against this kernel's 4.14 TB/s
// at 2400x1200: for adt_calc the occupancy is worth more than the prefetch.)
template <typename T>
cudaError_t launch_adt_calc(const LaunchCtx &c, int ncell, const int *pcell, const T *x,
                            const T *q, T *adt, const AirConst<T> &k, int minb) {
  if (ncell <= 0) return cudaSuccess;
  const int4 *pc = reinterpret_cast<const int4 *>(pcell);
  if (minb >= 8)
    k_adt_calc_mb<T, 8><<<grid_resident(c, k_adt_calc_mb<T, 8>, ncell, 256, 8), 256, 0,
                          c.stream>>>(ncell, pc, x, q, adt, k);
  else if (minb >= 6)
    k_adt_calc_mb<T, 6><<<grid_resident(c, k_adt_calc_mb<T, 6>, ncell, 256, 8), 256, 0,
                          c.stream>>>(ncell, pc, x, q, adt, k);
  else
    k_adt_calc<T><<<grid_resident(c, k_adt_calc<T>, ncell, 256, 8), 256, 0, c.stream>>>(
        ncell, pc, x, q, adt, k);
  c.count();
  return cudaGetLastError();
}

// ---------------------------------------------------------------- res_calc (atomics)

template <typename T> __device__ __forceinline__ void red_add(T *p, T v) { atomicAdd(p, v); }

template <typename T>
__global__ void __launch_bounds__(256)
k_res_calc_atomic(int nedge, const int2 *__restrict__ pedge, const int2 *__restrict__ pecell,
                  const T *__restrict__ x, const T *__restrict__ q,
                  const T *__restrict__ adt, T *__restrict__ res, AirConst<T> k) {
  int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nedge; e += stride) {
    int2 nn = __ldg(pedge + e);
    int2 cc = __ldg(pecell + e);
    T x1x, x1y, x2x, x2y, q1[4], q2[4], f[4];
    Vec<T>::ld2(x + 2 * (size_t)nn.x, x1x, x1y);
    Vec<T>::ld2(x + 2 * (size_t)nn.y, x2x, x2y);
    Vec<T>::ld4(q + 4 * (size_t)cc.x, q1);
    Vec<T>::ld4(q + 4 * (size_t)cc.y, q2);
    T a1 = __ldg(adt + cc.x), a2 = __ldg(adt + cc.y);
    air_flux<T>(x1x, x1y, x2x, x2y, q1, q2, a1, a2, k, f);
    T *r1 = res + 4 * (size_t)cc.x, *r2 = res + 4 * (size_t)cc.y;
#pragma unroll
    for (int m = 0; m < 4; m++) {
      red_add(r1 + m, f[m]);
      red_add(r2 + m, -f[m]);
    }
  }
}

// Segmented atomics: a warp's 32 edges first combine their increments to the
// same cell, then one lane of each group issues the atomics.  Each side (the
// +f into c1 and the -f into c2) is grouped by __match_any_sync on the cell
// index; the group's lowest lane sums the members' fluxes from shared memory
// in lane (edge) order and adds the sum with one atomic per component.  On a
// renumbered mesh edges are sorted by their first cell, so most cells are c1
// of two edges of one warp, and the two edges that reach a cell as c2 lie in
// neighbouring segments: the atomics roughly halve.  Results differ from the
// per-edge atomics only by rounding (the increments are grouped differently).
template <typename T, int NT>
__global__ void __launch_bounds__(NT)
k_res_calc_atomic_seg(int nedge, const int2 *__restrict__ pedge, const int2 *__restrict__ pecell,
                      const T *__restrict__ x, const T *__restrict__ q,
                      const T *__restrict__ adt, T *__restrict__ res, AirConst<T> k) {
  __shared__ T sf[NT / 32][4][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int stride = gridDim.x * NT;
  // the loop bound is the same for the 32 lanes (warps start at multiples of
  // 32 and the stride is one), so every lane reaches each __match_any_sync
  for (int base = blockIdx.x * NT + w * 32; base < nedge; base += stride) {
    const int e = base + lane;
    const bool valid = e < nedge;
    int2 cc = make_int2(-1 - lane, -33 - lane);  // distinct keys: no group for idle lanes
    T f[4] = {(T)0, (T)0, (T)0, (T)0};
    if (valid) {
      int2 nn = __ldg(pedge + e);
      cc = __ldg(pecell + e);
      T x1x, x1y, x2x, x2y, q1[4], q2[4];
      Vec<T>::ld2(x + 2 * (size_t)nn.x, x1x, x1y);
      Vec<T>::ld2(x + 2 * (size_t)nn.y, x2x, x2y);
      Vec<T>::ld4(q + 4 * (size_t)cc.x, q1);
      Vec<T>::ld4(q + 4 * (size_t)cc.y, q2);
      air_flux<T>(x1x, x1y, x2x, x2y, q1, q2, __ldg(adt + cc.x), __ldg(adt + cc.y), k, f);
    }
#pragma unroll
    for (int m = 0; m < 4; m++) sf[w][m][lane] = f[m];
    __syncwarp();
#pragma unroll
    for (int side = 0; side < 2; side++) {
      const int cell = side == 0 ? cc.x : cc.y;
      const unsigned g = __match_any_sync(0xffffffffu, cell);
      if (valid && lane == __ffs(g) - 1) {
        T acc[4] = {sf[w][0][lane], sf[w][1][lane], sf[w][2][lane], sf[w][3][lane]};
        for (unsigned rest = g & (g - 1); rest; rest &= rest - 1) {
          const int src = __ffs(rest) - 1;
#pragma unroll
          for (int m = 0; m < 4; m++) acc[m] += sf[w][m][src];
        }
        T *r = res + 4 * (size_t)cell;
#pragma unroll
        for (int m = 0; m < 4; m++) red_add(r + m, side == 0 ? acc[m] : -acc[m]);
      }
    }
    __syncwarp();
  }
}

template <typename T>
cudaError_t launch_res_calc_atomic(const LaunchCtx &c, int nedge, const int *pedge,
                                   const int *pecell, const T *x, const T *q, const T *adt,
                                   T *res, const AirConst<T> &k, bool segmented,
                                   int blocks_per_sm) {
  if (nedge <= 0) return cudaSuccess;
  if (segmented)
    k_res_calc_atomic_seg<T, 256><<<grid_for(c, nedge, 256, blocks_per_sm), 256, 0, c.stream>>>(
        nedge, reinterpret_cast<const int2 *>(pedge), reinterpret_cast<const int2 *>(pecell), x,
        q, adt, res, k);
  else
    k_res_calc_atomic<T><<<grid_for(c, nedge, 256, blocks_per_sm), 256, 0, c.stream>>>(
        nedge, reinterpret_cast<const int2 *>(pedge), reinterpret_cast<const int2 *>(pecell), x,
        q, adt, res, k);
  c.count();
  return cudaGetLastError();
}

// ---------------------------------------------------------------- bres_calc (atomics)

template <typename T>
__global__ void __launch_bounds__(128)
k_bres_calc_atomic(int nbedge, const int2 *__restrict__ pbedge, const int *__restrict__ pbecell,
                   const int *__restrict__ bound, const T *__restrict__ x,
                   const T *__restrict__ q, const T *__restrict__ adt, T *__restrict__ res,
                   AirConst<T> k) {
  int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nbedge; e += stride) {
    int2 nn = __ldg(pbedge + e);
    int c1 = __ldg(pbecell + e);
    int b = __ldg(bound + e);
    T x1x, x1y, x2x, x2y, q1[4], r[4];
    Vec<T>::ld2(x + 2 * (size_t)nn.x, x1x, x1y);
    Vec<T>::ld2(x + 2 * (size_t)nn.y, x2x, x2y);
    Vec<T>::ld4(q + 4 * (size_t)c1, q1);
    air_bflux<T>(x1x, x1y, x2x, x2y, q1, __ldg(adt + c1), b, k, r);
    T *r1 = res + 4 * (size_t)c1;
    if (b == 1) {  // a wall edge leaves components 0 and 3 untouched
      red_add(r1 + 1, r[1]);
      red_add(r1 + 2, r[2]);
    } else {
#pragma unroll
      for (int m = 0; m < 4; m++) red_add(r1 + m, r[m]);
    }
  }
}

template <typename T>
cudaError_t launch_bres_calc_atomic(const LaunchCtx &c, int nbedge, const int *pbedge,
                                    const int *pbecell, const int *bound, const T *x,
                                    const T *q, const T *adt, T *res, const AirConst<T> &k) {
  if (nbedge <= 0) return cudaSuccess;
  k_bres_calc_atomic<T><<<grid_for(c, nbedge, 128, 8), 128, 0, c.stream>>>(
      nbedge, reinterpret_cast<const int2 *>(pbedge), pbecell, bound, x, q, adt, res, k);
  c.count();
  return cudaGetLastError();
}

// ---------------------------------------------------------------- update

// (sum, max, argmax) triple; argmax keeps the lowest index among equal
// maxima, which is the index op_seq.h's in-order "sqdel > maxerr" test
// (update.h:13-16) ends with.
struct RedTriple {
  double sum, maxv;
  long long idx;
};

__device__ __forceinline__ void red_merge(RedTriple &a, double s, double m, long long i) {
  a.sum += s;
  if (m > a.maxv || (m == a.maxv && i < a.idx)) {
    a.maxv = m;
    a.idx = i;
  }
}

template <int THREADS>
__device__ __forceinline__ RedTriple block_reduce(RedTriple t) {
  __shared__ double s_sum[THREADS / 32], s_max[THREADS / 32];
  __shared__ long long s_idx[THREADS / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    double s = __shfl_down_sync(0xffffffffu, t.sum, off);
    double m = __shfl_down_sync(0xffffffffu, t.maxv, off);
    long long i = __shfl_down_sync(0xffffffffu, t.idx, off);
    red_merge(t, s, m, i);
  }
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    s_sum[warp] = t.sum;
    s_max[warp] = t.maxv;
    s_idx[warp] = t.idx;
  }
  __syncthreads();
  if (warp == 0) {
    RedTriple w{0.0, -INFINITY, LLONG_MAX};
    if (lane < THREADS / 32) w = RedTriple{s_sum[lane], s_max[lane], s_idx[lane]};
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      double s = __shfl_down_sync(0xffffffffu, w.sum, off);
      double m = __shfl_down_sync(0xffffffffu, w.maxv, off);
      long long i = __shfl_down_sync(0xffffffffu, w.idx, off);
      red_merge(w, s, m, i);
    }
    t = w;
  }
  return t;  // valid in thread 0
}

// One pass over the cells: q = qold - res/adt, res = 0, and the block's
// partial (sum del^2, max del^2, first index of the max).  The last block to
// arrive reduces all partials in block order and writes `out`.
// With ADT the kernel also computes, from each cell's new q, the time step
// that the following adt_calc computes (same arithmetic on the same stored q
// values) and writes it into `next`, a second array of the runtime's (option
// speculate_adt); the adt dat itself is only read.
template <typename T> struct AdtNext {
  const int4 *pcell;
  const T *x;
  T *next;     // receives the next adt_calc's result
  AirConst<T> k;
};

template <typename T, int THREADS, bool ADT, bool KEEP_RES = false>
__global__ void __launch_bounds__(THREADS)
k_update(int ncell, const T *__restrict__ qold, T *__restrict__ q, T *__restrict__ res,
         const T *adt, RedSlot *__restrict__ parts, unsigned *__restrict__ counter,
         RedSlot *__restrict__ out, RedSlot *host_out, long long seq, AdtNext<T> an, int rev) {
  grid_dependency_wait();
  RedTriple t{0.0, -INFINITY, LLONG_MAX};
  int stride = gridDim.x * THREADS;
  for (int i = blockIdx.x * THREADS + threadIdx.x; i < ncell; i += stride) {
    const int n = rev ? ncell - 1 - i : i;
    T qo[4], r[4], qn[4];
    T x1x, x1y, x2x, x2y, x3x, x3y, x4x, x4y;
    if constexpr (ADT) {  // the node gathers first: they do not depend on the update
      const int4 c = __ldg(an.pcell + n);
      Vec<T>::ld2(an.x + 2 * (size_t)c.x, x1x, x1y);
      Vec<T>::ld2(an.x + 2 * (size_t)c.y, x2x, x2y);
      Vec<T>::ld2(an.x + 2 * (size_t)c.z, x3x, x3y);
      Vec<T>::ld2(an.x + 2 * (size_t)c.w, x4x, x4y);
    }
    Vec<T>::ld4(qold + 4 * (size_t)n, qo);
    Vec<T>::ld4_rw(res + 4 * (size_t)n, r);
    const T a_old = __ldg(adt + n);
    double adti = 1.0f / (double)a_old;
#pragma unroll
    for (int m = 0; m < 4; m++) {
      double del = adti * (double)r[m];
      qn[m] = (T)((double)qo[m] - del);
      double sq = del * del;
      t.sum += sq;
      if (sq > t.maxv || (sq == t.maxv && n < t.idx)) {  // the lowest cell on ties
        t.maxv = sq;
        t.idx = n;
      }
    }
    Vec<T>::st4(q + 4 * (size_t)n, qn);
    if constexpr (!KEEP_RES) {
      T z[4] = {(T)0, (T)0, (T)0, (T)0};
      Vec<T>::st4(res + 4 * (size_t)n, z);
    }
    if constexpr (ADT)
      an.next[n] = air_adt<T>(x1x, x1y, x2x, x2y, x3x, x3y, x4x, x4y, qn[0], qn[1], qn[2],
                              qn[3], an.k);
  }
  t = block_reduce<THREADS>(t);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    parts[blockIdx.x] = RedSlot{t.sum, t.maxv, t.idx, 0};
    __threadfence();
    unsigned ticket = atomicAdd(counter, 1u);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  RedTriple a{0.0, -INFINITY, LLONG_MAX};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += THREADS) {
    const volatile RedSlot *p = parts + b;
    red_merge(a, p->sum, p->maxv, p->idx);
  }
  a = block_reduce<THREADS>(a);
  if (threadIdx.x == 0) {
    *out = RedSlot{a.sum, a.maxv, a.idx, 0};
    if (host_out) {
      volatile RedSlot *h = host_out;
      h->sum = a.sum;
      h->maxv = a.maxv;
      h->idx = a.idx;
      __threadfence_system();
      h->pad = seq;  // published last
    }
    *counter = 0u;  // ready for the next launch (same stream, so ordered)
  }
}

template <typename T>
cudaError_t launch_update(const LaunchCtx &c, int ncell, const T *qold, T *q, T *res,
                          const T *adt, const RedScratch &s, const int *pcell, const T *x,
                          T *adt_next, const AirConst<T> *k, bool keep_res, bool reverse) {
  constexpr int TH = 256;
  int grid = grid_for(c, ncell, TH, 4);
  if (grid > s.capacity) grid = s.capacity;
  const int rev = reverse ? 1 : 0;
  cudaError_t e;
  if (adt_next) {
    const AdtNext<T> an{reinterpret_cast<const int4 *>(pcell), x, adt_next, *k};
    e = keep_res ? launch_dependent(c, k_update<T, TH, true, true>, grid, TH, 0, ncell, qold, q,
                                    res, adt, s.parts, s.counter, s.out, s.host_out, s.seq, an, rev)
                 : launch_dependent(c, k_update<T, TH, true>, grid, TH, 0, ncell, qold, q, res,
                                    adt, s.parts, s.counter, s.out, s.host_out, s.seq, an, rev);
  } else {
    e = keep_res ? launch_dependent(c, k_update<T, TH, false, true>, grid, TH, 0, ncell, qold, q,
                                    res, adt, s.parts, s.counter, s.out, s.host_out, s.seq,
                                    AdtNext<T>{}, rev)
                 : launch_dependent(c, k_update<T, TH, false>, grid, TH, 0, ncell, qold, q, res,
                                    adt, s.parts, s.counter, s.out, s.host_out, s.seq,
                                    AdtNext<T>{}, rev);
  }
  c.count();
  return e != cudaSuccess ? e : cudaGetLastError();
}

// ---------------------------------------------------------------- instantiations

template cudaError_t launch_adt_calc<double>(const LaunchCtx &, int, const int *, const double *,
                                             const double *, double *, const AirConst<double> &,
                                             int);
template cudaError_t launch_adt_calc<float>(const LaunchCtx &, int, const int *, const float *,
                                            const float *, float *, const AirConst<float> &, int);
template cudaError_t launch_adt_save<double>(const LaunchCtx &, int, const int *, const double *,
                                             const double *, double *, double *,
                                             const AirConst<double> &);
template cudaError_t launch_adt_save<float>(const LaunchCtx &, int, const int *, const float *,
                                            const float *, float *, float *,
                                            const AirConst<float> &);
template cudaError_t launch_res_calc_atomic<double>(const LaunchCtx &, int, const int *,
                                                    const int *, const double *, const double *,
                                                    const double *, double *,
                                                    const AirConst<double> &, bool, int);
template cudaError_t launch_res_calc_atomic<float>(const LaunchCtx &, int, const int *,
                                                   const int *, const float *, const float *,
                                                   const float *, float *,
                                                   const AirConst<float> &, bool, int);
template cudaError_t launch_bres_calc_atomic<double>(const LaunchCtx &, int, const int *,
                                                     const int *, const int *, const double *,
                                                     const double *, const double *, double *,
                                                     const AirConst<double> &);
template cudaError_t launch_bres_calc_atomic<float>(const LaunchCtx &, int, const int *,
                                                    const int *, const int *, const float *,
                                                    const float *, const float *, float *,
                                                    const AirConst<float> &);
template cudaError_t launch_update<double>(const LaunchCtx &, int, const double *, double *,
                                           double *, const double *, const RedScratch &,
                                           const int *, const double *, double *,
                                           const AirConst<double> *, bool, bool);
template cudaError_t launch_update<float>(const LaunchCtx &, int, const float *, float *,
                                          float *, const float *, const RedScratch &,
                                          const int *, const float *, float *,
                                          const AirConst<float> *, bool, bool);

} // namespace op2b
