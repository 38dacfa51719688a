// res_calc (and the fused res_calc + bres_calc) with each interior flux
// computed once: the flux ring.
//
// The owner-computes kernels (airfoil_pipe.cu) keep the reference's
// increment order -- each cell sums the fluxes of its <= 4 interior edges in
// increasing edge order -- by computing every interior edge's flux twice,
// once from each side.  That doubles the FP64 work (res_calc.h:1-33, about
// 60 operations and a division per side), and at the register budget the
// corner kernel needs, the doubled dependency chains, not HBM, bound it.
//
// Here each CTA owns a contiguous range of cells (ring_span of them; with the
// mesh renumbered, a cell's neighbours are close in the numbering) and sweeps
// it in tiles of NT cells, one cell per thread:
//
//   phase A  every cell computes the flux of each of its edges whose other
//            cell comes later in the range, and puts the flux (in the edge's
//            own orientation) into a ring of OP2B_RING_ENTRIES fluxes in
//            shared memory; the flux of an edge to a cell outside the range
//            it computes for itself into its own scratch entries (kept out of
//            the ring, whose entries then live at most ~3000 fluxes on a
//            renumbered mesh);
//   phase B  every cell adds the fluxes of its edges from the ring in slot
//            order (its edges in increasing edge order) -- its own, and those
//            an earlier cell of the range computed -- starting from res[c]
//            (or 0 when res is known to be zero), then its boundary edges'
//            increments (bres_calc, in edge order), and writes res[c] once.
//
// A flux is the same double whichever cell computes it (the same operands
// through the same expression), and each cell's sum runs in the same order,
// so res is bit-identical to the corner kernels' and to the reference's
// sequential build.  Only edges between ranges are computed twice (a few
// per cent).  The ring entries are assigned when the records are built
// (build_ring_records), which also checks that no entry is reused before the
// tile that reads it has done so.  Two barriers per tile: phase A's writes
// before phase B's reads, and phase B's reads before the next tile's writes.
// The next tile's operands are loaded into registers while the current tile
// is computed (as in the corner kernel), and a cell whose flux comes from the
// ring loads no operands for that edge.
#include <cuda_runtime.h>
#include <stdint.h>

#include "airfoil_math.cuh"
#include "gather.h"
#include "op2b_runtime.h"
#include "vec.cuh"

namespace op2b {
namespace {

template <typename T> struct RingOps {
  T qc[4], rs[4], qo[4][4], ao[4], xn[4][2], ac;
  unsigned meta;
  uint2 ring;
  int bnd[4];  // boundary flag of each boundary slot (fused bres_calc)
};

// coordinate `comp` of corner i (0..3), by selects
template <typename T>
__device__ __forceinline__ T ring_corner(const T (&xn)[4][2], unsigned i, int comp) {
  const T lo = (i & 1u) ? xn[1][comp] : xn[0][comp];
  const T hi = (i & 1u) ? xn[3][comp] : xn[2][comp];
  return (i & 2u) ? hi : lo;
}

__device__ __forceinline__ unsigned ring_field(const uint2 &r, int s) {
  const unsigned w = s < 2 ? r.x : r.y;
  return (s & 1) ? (w >> 16) : (w & 0xffffu);
}

// a cell's records, loaded a tile before its operands (two tiles ahead of
// its arithmetic), so one level of gather latency is left in a tile
struct RingRec {
  int4 o, cn;
  unsigned meta;
  uint2 ring;
};

__device__ __forceinline__ void ring_rec(RingRec &r, int c, int re, const int4 *__restrict__ rec_o,
                                         const int4 *__restrict__ rec_cn,
                                         const unsigned *__restrict__ rec_meta,
                                         const uint2 *__restrict__ rec_ring) {
  if (c < re) {
    r.o = __ldg(rec_o + c);
    r.cn = __ldg(rec_cn + c);
    r.meta = __ldg(rec_meta + c);
    r.ring = __ldg(rec_ring + c);
  } else {
    r.o = r.cn = make_int4(0, 0, 0, 0);
    r.meta = 0u;
    r.ring = make_uint2(0u, 0u);
  }
}

template <typename T, bool BRES, bool ZERO>
__device__ __forceinline__ void ring_load(RingOps<T> &d, int c, const RingRec &rr,
                                          const T *__restrict__ x, const T *__restrict__ q,
                                          const T *__restrict__ adt, const T *__restrict__ res,
                                          const int *__restrict__ bound) {
  const int4 o4 = rr.o;
  const int4 cn = rr.cn;
  d.meta = rr.meta;
  d.ring = rr.ring;
  Vec<T>::ld4(q + 4 * (size_t)c, d.qc);
  if constexpr (ZERO) {
#pragma unroll
    for (int j = 0; j < 4; j++) d.rs[j] = (T)0;
  } else {
    Vec<T>::ld4_rw(res + 4 * (size_t)c, d.rs);
  }
  d.ac = __ldg(adt + c);
  const int nd[4] = {cn.x, cn.y, cn.z, cn.w};
#pragma unroll
  for (int j = 0; j < 4; j++) Vec<T>::ld2(x + 2 * (size_t)nd[j], d.xn[j][0], d.xn[j][1]);
  const int o[4] = {o4.x, o4.y, o4.z, o4.w};
#pragma unroll
  for (int s = 0; s < 4; s++) {
    // the other cell's operands only for a flux this cell computes
    const bool mine = ((d.meta >> (8 * s)) & 1u) && !(ring_field(d.ring, s) & 0x8000u);
    const int oo = mine ? o[s] : c;
    Vec<T>::ld4(q + 4 * (size_t)oo, d.qo[s]);
    d.ao[s] = __ldg(adt + oo);
  }
  if constexpr (BRES) {
    if (d.meta & 0x40404040u) {
#pragma unroll
      for (int s = 0; s < 4; s++)
        d.bnd[s] = ((d.meta >> (8 * s + 6)) & 1u) ? __ldg(bound + o[s]) : 0;
    }
  }
}

// The tile scratch for fluxes to cells outside the range: value j of slot s
// of thread t at local[(4 s + j) * NT + t] (consecutive threads, consecutive
// words: no bank conflicts); ring_produce writes it, ring_sum reads it
template <typename T, int NT>
__device__ __forceinline__ void local_ld(const T *local, int s, T *f) {
#pragma unroll
  for (int j = 0; j < 4; j++) f[j] = local[(4 * s + j) * NT + threadIdx.x];
}

// v[s] for a slot index s known only at run time, by selects (no
// local-memory indexing)
template <typename V>
__device__ __forceinline__ V sel4(unsigned s, V v0, V v1, V v2, V v3) {
  const V lo = (s & 1u) ? v1 : v0;
  const V hi = (s & 1u) ? v3 : v2;
  return (s & 2u) ? hi : lo;
}

// phase A: the fluxes this cell computes (edge orientation): into the ring,
// or, for an edge to a cell outside the range, into the tile scratch.  The
// loop runs over this cell's own computed slots, in slot order, their
// operands picked by selects: a warp issues as many fluxes as its busiest
// lane computes (two for most cells of a renumbered mesh), where a loop over
// the four slot positions would issue four whenever the lanes' computed slots
// sit at different positions.
template <typename T, int NT>
__device__ __forceinline__ void ring_produce(const RingOps<T> &d, T ric, T pc, T *ring, T *local,
                                             const AirConst<T> &k) {
  unsigned todo = 0;
#pragma unroll
  for (int s = 0; s < 4; s++)
    if (((d.meta >> (8 * s)) & 1u) && !(ring_field(d.ring, s) & 0x8000u)) todo |= 1u << s;
  while (todo) {
    const unsigned s = (unsigned)__ffs(todo) - 1u;
    todo &= todo - 1u;
    const unsigned m = (d.meta >> (8 * s)) & 0xffu;
    const unsigned f16 = ((s < 2u ? d.ring.x : d.ring.y) >> (16 * (s & 1u))) & 0xffffu;
    const unsigned a = (m >> 2) & 3u, b = (m >> 4) & 3u;
    const T x1x = ring_corner<T>(d.xn, a, 0), x1y = ring_corner<T>(d.xn, a, 1);
    const T x2x = ring_corner<T>(d.xn, b, 0), x2y = ring_corner<T>(d.xn, b, 1);
    T qo[4];
#pragma unroll
    for (int j = 0; j < 4; j++) qo[j] = sel4<T>(s, d.qo[0][j], d.qo[1][j], d.qo[2][j], d.qo[3][j]);
    const T ao = sel4<T>(s, d.ao[0], d.ao[1], d.ao[2], d.ao[3]);
    T f[4], rio, po;
    air_prim<T>(qo, k, rio, po);
    if (m & 2u)  // this cell is the edge's second cell
      air_flux_prim<T>(x1x, x1y, x2x, x2y, qo, d.qc, rio, po, ric, pc, ao, d.ac, k, f);
    else
      air_flux_prim<T>(x1x, x1y, x2x, x2y, d.qc, qo, ric, pc, rio, po, d.ac, ao, k, f);
    if (f16 & 0x4000u) {
#pragma unroll
      for (int j = 0; j < 4; j++) local[(4 * s + j) * NT + threadIdx.x] = f[j];
    } else {
      Vec<T>::st4_shared(ring + 4 * (f16 & (OP2B_RING_ENTRIES - 1)), f);
    }
  }
}

// phase B: this cell's sums in slot order, then its boundary increments
template <typename T, int NT, bool BRES>
__device__ __forceinline__ void ring_sum(const RingOps<T> &d, int c, T ric, T pc,
                                         const T *ring, const T *local, T *__restrict__ res,
                                         const AirConst<T> &k) {
  T acc[4] = {d.rs[0], d.rs[1], d.rs[2], d.rs[3]};
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const unsigned m = (d.meta >> (8 * s)) & 0xffu;
    if (!(m & 1u)) continue;
    T f[4];
    const unsigned f16 = ring_field(d.ring, s);
    if (f16 & 0x4000u)
      local_ld<T, NT>(local, s, f);
    else
      Vec<T>::ld4_shared(ring + 4 * (f16 & (OP2B_RING_ENTRIES - 1)), f);
    if (m & 2u) {
#pragma unroll
      for (int j = 0; j < 4; j++) acc[j] -= f[j];
    } else {
#pragma unroll
      for (int j = 0; j < 4; j++) acc[j] += f[j];
    }
  }
  if constexpr (BRES) {
    if (d.meta & 0x40404040u) {
#pragma unroll
      for (int s = 0; s < 4; s++) {
        const unsigned m = (d.meta >> (8 * s)) & 0xffu;
        if (!(m & 0x40u)) continue;
        const unsigned a = (m >> 2) & 3u, b = (m >> 4) & 3u;
        T rr[4];
        air_bflux_prim<T>(ring_corner<T>(d.xn, a, 0), ring_corner<T>(d.xn, a, 1),
                          ring_corner<T>(d.xn, b, 0), ring_corner<T>(d.xn, b, 1), d.qc, ric, pc,
                          d.ac, d.bnd[s], k, rr);
        if (d.bnd[s] == 1) {  // a wall edge leaves components 0 and 3 untouched
          acc[1] += rr[1];
          acc[2] += rr[2];
        } else {
#pragma unroll
          for (int j = 0; j < 4; j++) acc[j] += rr[j];
        }
      }
    }
  }
  Vec<T>::st4(res + 4 * (size_t)c, acc);
}

template <typename T, int NT, bool BRES, bool ZERO>
__global__ void __launch_bounds__(NT, 1)
k_res_ring(int ncell, int span, const int4 *__restrict__ rec_o, const int4 *__restrict__ rec_cn,
           const unsigned *__restrict__ rec_meta, const uint2 *__restrict__ rec_ring,
           const T *__restrict__ x, const T *__restrict__ q, const T *__restrict__ adt,
           T *__restrict__ res, AirConst<T> k, const int *__restrict__ bound) {
  extern __shared__ __align__(16) unsigned char ring_smem[];
  T *ring = reinterpret_cast<T *>(ring_smem);
  T *local = ring + 4 * OP2B_RING_ENTRIES;  // the tile scratch (local_st / local_ld)
  const int rs = blockIdx.x * span;
  const int re = min(rs + span, ncell);
  if (rs >= re) return;  // the whole CTA
  RingOps<T> cur, nxt;
  RingRec r1, r2;
  {
    RingRec r0;
    ring_rec(r0, rs + threadIdx.x, re, rec_o, rec_cn, rec_meta, rec_ring);
    ring_rec(r1, rs + NT + threadIdx.x, re, rec_o, rec_cn, rec_meta, rec_ring);
    if (rs + (int)threadIdx.x < re)
      ring_load<T, BRES, ZERO>(cur, rs + threadIdx.x, r0, x, q, adt, res, bound);
  }
  for (int t0 = rs; t0 < re; t0 += NT) {  // the same trip count for every thread
    const int c = t0 + threadIdx.x;
    const bool valid = c < re;
    ring_rec(r2, c + 2 * NT, re, rec_o, rec_cn, rec_meta, rec_ring);
    if (c + NT < re) ring_load<T, BRES, ZERO>(nxt, c + NT, r1, x, q, adt, res, bound);
    T ric = (T)0, pc = (T)0;
    if (valid) {
      air_prim<T>(cur.qc, k, ric, pc);
      ring_produce<T, NT>(cur, ric, pc, ring, local, k);
    }
    __syncthreads();
    if (valid) ring_sum<T, NT, BRES>(cur, c, ric, pc, ring, local, res, k);
    __syncthreads();
    cur = nxt;
    r1 = r2;
  }
}

template <typename T, bool BRES, bool ZERO>
cudaError_t launch_ring(const LaunchCtx &ctx, const SlotRecords &s, const int *bound, const T *x,
                        const T *q, const T *adt, T *res, const AirConst<T> &k) {
  constexpr int NT = 256;
  // the ring, then 4 slots of 4 values a thread for fluxes to cells outside the range
  const size_t smem = sizeof(T) * 4 * ((size_t)OP2B_RING_ENTRIES + 4 * NT);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_res_ring<T, NT, BRES, ZERO>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_res_ring<T, NT, BRES, ZERO><<<(unsigned)s.ring_ctas, NT, smem, ctx.stream>>>(
      s.ncell, s.ring_span, reinterpret_cast<const int4 *>(s.o),
      reinterpret_cast<const int4 *>(s.cn), s.meta, s.ring, x, q, adt, res, k, bound);
  ctx.count();
  return cudaGetLastError();
}

}  // namespace

template <typename T>
cudaError_t launch_res_ring(const LaunchCtx &c, const SlotRecords &s, const int *bound,
                            const T *x, const T *q, const T *adt, T *res, const AirConst<T> &k,
                            bool zero_res) {
  if (s.ncell <= 0) return cudaSuccess;
  if (!s.ring || s.ring_nt != 256) return cudaErrorInvalidValue;
  if (bound)
    return zero_res ? launch_ring<T, true, true>(c, s, bound, x, q, adt, res, k)
                    : launch_ring<T, true, false>(c, s, bound, x, q, adt, res, k);
  return zero_res ? launch_ring<T, false, true>(c, s, bound, x, q, adt, res, k)
                  : launch_ring<T, false, false>(c, s, bound, x, q, adt, res, k);
}

template cudaError_t launch_res_ring<double>(const LaunchCtx &, const SlotRecords &, const int *,
                                             const double *, const double *, const double *,
                                             double *, const AirConst<double> &, bool);
template cudaError_t launch_res_ring<float>(const LaunchCtx &, const SlotRecords &, const int *,
                                            const float *, const float *, const float *, float *,
                                            const AirConst<float> &, bool);

}  // namespace op2b
