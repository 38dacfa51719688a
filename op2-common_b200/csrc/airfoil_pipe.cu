// res_calc by cell ownership with software pipelines: two variants of the
// slot-record gather (k_res_gather_cell4) that overlap the next cell's loads
// with the current cell's arithmetic.
//
// Both keep its arithmetic and increment order -- each cell sums the fluxes of
// its <= 4 interior edges in increasing edge order, starting from res[c], so q
// stays bit-identical to the reference's sequential build -- and both run a
// persistent grid: thread t of G handles cells t, t+G, t+2G, ...; slot records
// (which other cell, which nodes, role, valid) are prefetched into registers
// two cells ahead.
//
// * k_res_gather_regpipe (option gather_kernel 5, the default): the operands
//   of cell k+1 -- its own q, adt and res, and per edge the other cell's q and
//   adt and the edge's two node coordinates -- are loaded into a second set of
//   registers while cell k is computed.  222 registers, one 256-thread or two
//   128-thread CTAs per SM, L1 left at its full size for the neighbour reuse
//   that the RCM numbering creates.
// * k_res_gather_pipe (gather_kernel 4): the same operands copied into shared
//   memory by cp.async one cell ahead (368 bytes a stage for double, 208 for
//   float, strides chosen so 16-byte accesses of consecutive threads fall on
//   distinct banks).  Fewer registers, but the staging takes most of the
//   SM's L1/shared capacity and the gathers lose their L1 hits: measured
//   slower than the one-pass kernel, kept as the record of that trade-off.
#include <cuda_runtime.h>
#include <stdint.h>

#include "airfoil_math.cuh"
#include "gather.h"
#include "op2b_runtime.h"
#include "vec.cuh"

namespace op2b {
namespace {

constexpr unsigned kRole = 1u << 30;   // the slot-record bits of airfoil_gather.cu
constexpr unsigned kValid = 1u << 31;

// layout of one stage, in elements of T
constexpr int kQC = 0, kRES = 4, kQO = 8, kX = 24, kAC = 40, kAO = 41, kFLAGS = 45;
template <typename T> struct PipeLayout;
template <> struct PipeLayout<double> { static constexpr int bytes = 368; };
template <> struct PipeLayout<float> { static constexpr int bytes = 208; };

__device__ __forceinline__ uint32_t saddr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

template <int B>
__device__ __forceinline__ void cp_ca(uint32_t dst, const void *src) {
  if constexpr (B == 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
  else if constexpr (B == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_cg16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

struct Rec {
  int4 o, n1;
  uint4 n2;
};

template <bool CS = false>
__device__ __forceinline__ Rec load_rec(const int4 *ro, const int4 *rn1, const uint4 *rn2, int c,
                                        int ncell) {
  Rec r;
  if (c < ncell) {
    if (CS) {  // read once per launch: evict first, keep L1/L2 for the gathers
      r.o = __ldcs(ro + c);
      r.n1 = __ldcs(rn1 + c);
      r.n2 = __ldcs(rn2 + c);
    } else {
      r.o = __ldg(ro + c);
      r.n1 = __ldg(rn1 + c);
      r.n2 = __ldg(rn2 + c);
    }
  } else {
    r.o = r.n1 = make_int4(0, 0, 0, 0);
    r.n2 = make_uint4(0, 0, 0, 0);
  }
  return r;
}

// copy a 4-vector of T (one q or res record) into shared memory
template <typename T, bool STREAM>
__device__ __forceinline__ void cp_vec4(uint32_t dst, const T *src) {
  if constexpr (sizeof(T) == 8) {
    if (STREAM) {
      cp_cg16(dst, src);
      cp_cg16(dst + 16, src + 2);
    } else {
      cp_ca<16>(dst, src);
      cp_ca<16>(dst + 16, src + 2);
    }
  } else {
    if (STREAM)
      cp_cg16(dst, src);
    else
      cp_ca<16>(dst, src);
  }
}

template <typename T>
__device__ __forceinline__ void issue_cell(uint8_t *stage, int c, int ncell, const Rec &r,
                                           const T *__restrict__ x, const T *__restrict__ q,
                                           const T *__restrict__ adt, const T *__restrict__ res) {
  if (c < ncell) {
    const uint32_t s = saddr(stage);
    constexpr int E = sizeof(T);
    cp_vec4<T, true>(s + kQC * E, q + 4 * (size_t)c);
    cp_vec4<T, true>(s + kRES * E, res + 4 * (size_t)c);
    cp_ca<E>(s + kAC * E, adt + c);
    const int o[4] = {r.o.x, r.o.y, r.o.z, r.o.w};
    const int na[4] = {r.n1.x, r.n1.y, r.n1.z, r.n1.w};
    const unsigned nb[4] = {r.n2.x, r.n2.y, r.n2.z, r.n2.w};
    unsigned flags = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if (!(nb[k] & kValid)) continue;
      flags |= (1u << k) | ((nb[k] & kRole) ? (16u << k) : 0u);
      cp_vec4<T, false>(s + (kQO + 4 * k) * E, q + 4 * (size_t)o[k]);
      cp_ca<E>(s + (kAO + k) * E, adt + o[k]);
      cp_ca<2 * E>(s + (kX + 4 * k) * E, x + 2 * (size_t)na[k]);
      cp_ca<2 * E>(s + (kX + 4 * k + 2) * E, x + 2 * (size_t)(nb[k] & (kRole - 1)));
    }
    *reinterpret_cast<unsigned *>(stage + kFLAGS * E) = flags;
  }
  cp_commit();
}

template <typename T>
__device__ __forceinline__ void compute_cell(const uint8_t *stage, int c, T *__restrict__ res,
                                             const AirConst<T> &k) {
  const T *v = reinterpret_cast<const T *>(stage);
  const unsigned flags = *reinterpret_cast<const unsigned *>(stage + kFLAGS * sizeof(T));
  T qc[4], acc[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    qc[m] = v[kQC + m];
    acc[m] = v[kRES + m];
  }
  const T ac = v[kAC];
#pragma unroll
  for (int s = 0; s < 4; s++) {
    if (!(flags & (1u << s))) continue;
    T qo[4], f[4];
#pragma unroll
    for (int m = 0; m < 4; m++) qo[m] = v[kQO + 4 * s + m];
    const T ao = v[kAO + s];
    const T x1x = v[kX + 4 * s], x1y = v[kX + 4 * s + 1];
    const T x2x = v[kX + 4 * s + 2], x2y = v[kX + 4 * s + 3];
    if (flags & (16u << s)) {
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

template <typename T, int NT>
__global__ void __launch_bounds__(NT)
k_res_gather_pipe(int ncell, const int4 *__restrict__ rec_o, const int4 *__restrict__ rec_n1,
                  const uint4 *__restrict__ rec_n2, const T *__restrict__ x,
                  const T *__restrict__ q, const T *__restrict__ adt, T *__restrict__ res,
                  AirConst<T> k) {
  extern __shared__ __align__(16) uint8_t smem[];
  constexpr int SB = PipeLayout<T>::bytes;
  uint8_t *st[2] = {smem + threadIdx.x * SB, smem + (NT + threadIdx.x) * SB};
  const int G = gridDim.x * NT;
  int c = blockIdx.x * NT + threadIdx.x;
  if (c >= ncell) return;
  Rec cur = load_rec(rec_o, rec_n1, rec_n2, c, ncell);
  Rec nxt = load_rec(rec_o, rec_n1, rec_n2, c + G, ncell);
  issue_cell<T>(st[0], c, ncell, cur, x, q, adt, res);
  for (int it = 0; c < ncell; it++, c += G) {
    const Rec nn = load_rec(rec_o, rec_n1, rec_n2, c + 2 * G, ncell);
    issue_cell<T>(st[(it + 1) & 1], c + G, ncell, nxt, x, q, adt, res);
    cp_wait<1>();  // cell c's copies have landed
    compute_cell<T>(st[it & 1], c, res, k);
    nxt = nn;
  }
  cp_wait<0>();
}

template <typename T, int NT>
cudaError_t launch_pipe(const LaunchCtx &ctx, const SlotRecords &s, const T *x, const T *q,
                        const T *adt, T *res, const AirConst<T> &k) {
  const size_t smem = 2 * (size_t)NT * PipeLayout<T>::bytes;
  static int per_sm = -1;
  if (per_sm < 0) {
    cudaError_t e = cudaFuncSetAttribute(k_res_gather_pipe<T, NT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_res_gather_pipe<T, NT>, NT,
                                                      smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
  }
  long long blocks = (long long)ctx.nsm * per_sm;
  const long long need = (s.ncell + NT - 1) / NT;
  if (blocks > need) blocks = need;
  k_res_gather_pipe<T, NT><<<(unsigned)blocks, NT, smem, ctx.stream>>>(
      s.ncell, reinterpret_cast<const int4 *>(s.o), reinterpret_cast<const int4 *>(s.n1),
      reinterpret_cast<const uint4 *>(s.n2), x, q, adt, res, k);
  ctx.count();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The register-pipelined variant: the same per-cell arithmetic and order, with
// the operands of cell k+1 loaded into registers while cell k is computed
// (records two cells ahead).  L1 keeps its full size (no shared memory), at
// the price of ~2x the registers of k_res_gather_cell4 (one CTA of 256
// threads per SM).

template <typename T> struct CellOps {
  T qc[4], rs[4], qo[4][4], ao[4], xa[4][2], xb[4][2], ac;
  unsigned flags;
};

template <typename T, bool CS>
__device__ __forceinline__ void load_cell(CellOps<T> &d, int c, const Rec &r,
                                          const T *__restrict__ x, const T *__restrict__ q,
                                          const T *__restrict__ adt, const T *__restrict__ res) {
  Vec<T>::ld4(q + 4 * (size_t)c, d.qc);
  if (CS)
    Vec<T>::ld4_cs(res + 4 * (size_t)c, d.rs);
  else
    Vec<T>::ld4_rw(res + 4 * (size_t)c, d.rs);
  d.ac = __ldg(adt + c);
  const int o[4] = {r.o.x, r.o.y, r.o.z, r.o.w};
  const int na[4] = {r.n1.x, r.n1.y, r.n1.z, r.n1.w};
  const unsigned nb[4] = {r.n2.x, r.n2.y, r.n2.z, r.n2.w};
  unsigned flags = 0;
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const bool v = (nb[s] & kValid) != 0;
    flags |= v ? ((1u << s) | ((nb[s] & kRole) ? (16u << s) : 0u)) : 0u;
    const int oo = v ? o[s] : c;
    const int a = v ? na[s] : 0, b = v ? (int)(nb[s] & (kRole - 1)) : 0;
    Vec<T>::ld4(q + 4 * (size_t)oo, d.qo[s]);
    d.ao[s] = __ldg(adt + oo);
    Vec<T>::ld2(x + 2 * (size_t)a, d.xa[s][0], d.xa[s][1]);
    Vec<T>::ld2(x + 2 * (size_t)b, d.xb[s][0], d.xb[s][1]);
  }
  d.flags = flags;
}

template <typename T, bool CS>
__device__ __forceinline__ void compute_regs(const CellOps<T> &d, int c, T *__restrict__ res,
                                             const AirConst<T> &k) {
  T acc[4] = {d.rs[0], d.rs[1], d.rs[2], d.rs[3]};
  T ric, pc;  // the cell's own terms, once for its <= 4 edges
  air_prim<T>(d.qc, k, ric, pc);
#pragma unroll
  for (int s = 0; s < 4; s++) {
    if (!(d.flags & (1u << s))) continue;
    T f[4], rio, po;
    air_prim<T>(d.qo[s], k, rio, po);
    if (d.flags & (16u << s)) {
      air_flux_prim<T>(d.xa[s][0], d.xa[s][1], d.xb[s][0], d.xb[s][1], d.qo[s], d.qc, rio, po,
                       ric, pc, d.ao[s], d.ac, k, f);
#pragma unroll
      for (int m = 0; m < 4; m++) acc[m] -= f[m];
    } else {
      air_flux_prim<T>(d.xa[s][0], d.xa[s][1], d.xb[s][0], d.xb[s][1], d.qc, d.qo[s], ric, pc,
                       rio, po, d.ac, d.ao[s], k, f);
#pragma unroll
      for (int m = 0; m < 4; m++) acc[m] += f[m];
    }
  }
  if (CS)
    Vec<T>::st4_cs(res + 4 * (size_t)c, acc);
  else
    Vec<T>::st4(res + 4 * (size_t)c, acc);
}

// cur holds the cell being computed, nxt receives the next cell's loads.  (A
// two-way unrolled form that swaps the buffers instead of copying nxt into
// cur needs 244 registers instead of 222 and measured 126 us instead of 107 us
// per call at 2400x1200: the copy is the cheaper schedule.)
template <typename T, int NT, bool CS>
__global__ void __launch_bounds__(NT, 1)
k_res_gather_regpipe(int ncell, const int4 *__restrict__ rec_o, const int4 *__restrict__ rec_n1,
                     const uint4 *__restrict__ rec_n2, const T *__restrict__ x,
                     const T *__restrict__ q, const T *__restrict__ adt, T *__restrict__ res,
                     AirConst<T> k) {
  const int G = gridDim.x * NT;
  int c = blockIdx.x * NT + threadIdx.x;
  if (c >= ncell) return;
  CellOps<T> cur, nxt;
  Rec r1 = load_rec<CS>(rec_o, rec_n1, rec_n2, c + G, ncell);
  {
    const Rec r0 = load_rec<CS>(rec_o, rec_n1, rec_n2, c, ncell);
    load_cell<T, CS>(cur, c, r0, x, q, adt, res);
  }
  for (; c < ncell; c += G) {
    const Rec r2 = load_rec<CS>(rec_o, rec_n1, rec_n2, c + 2 * G, ncell);
    if (c + G < ncell) load_cell<T, CS>(nxt, c + G, r1, x, q, adt, res);
    compute_regs<T, CS>(cur, c, res, k);
    cur = nxt;
    r1 = r2;
  }
}

// persistent grid: as many CTAs as fit on the GPU at once, at most one cell per thread
template <typename T, typename K>
cudaError_t launch_regpipe(K kern, int nt, const LaunchCtx &ctx, const SlotRecords &s, const T *x,
                           const T *q, const T *adt, T *res, const AirConst<T> &k) {
  int per_sm = 1;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, 0);
  if (e != cudaSuccess) return e;
  long long blocks = (long long)ctx.nsm * (per_sm < 1 ? 1 : per_sm);
  const long long need = (s.ncell + nt - 1) / nt;
  if (blocks > need) blocks = need;
  kern<<<(unsigned)blocks, nt, 0, ctx.stream>>>(
      s.ncell, reinterpret_cast<const int4 *>(s.o), reinterpret_cast<const int4 *>(s.n1),
      reinterpret_cast<const uint4 *>(s.n2), x, q, adt, res, k);
  ctx.count();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The register pipeline over corner records (option gather_kernel 6): a
// cell's four corner nodes are gathered once (four 16-byte loads for FP64
// instead of eight) and each slot picks its edge's two nodes from them by the
// 2-bit corner indices of meta; the record is 36 bytes a cell instead of 48.
// The picked coordinates are the same doubles, so fluxes and sums are
// bit-identical to the slot-record kernels.

struct CornerRec {
  int4 o, cn;
  unsigned meta;
};

__device__ __forceinline__ CornerRec load_crec(const int4 *ro, const int4 *rcn,
                                               const unsigned *rmeta, int c, int ncell) {
  CornerRec r;
  if (c < ncell) {
    r.o = __ldg(ro + c);
    r.cn = __ldg(rcn + c);
    r.meta = __ldg(rmeta + c);
  } else {
    r.o = r.cn = make_int4(0, 0, 0, 0);
    r.meta = 0u;
  }
  return r;
}

template <typename T> struct CornerOps {
  T qc[4], rs[4], qo[4][4], ao[4], xn[4][2], ac;
  unsigned meta;
  int bnd[4];  // fused bres_calc: boundary flag of each boundary slot
};

// The fused res_calc + bres_calc keeps a boundary cell's boundary edges in the
// unused slots of its corner record (after its interior slots, in edge order):
// meta bit 6 marks such a slot, bits 2-5 give the edge's nodes as corners and
// o holds the boundary edge, whose flag is read from the bound dat.
struct BresLink {
  const int *bound;
};

template <typename T, bool BRES = false, bool ZERO = false>
__device__ __forceinline__ void load_corner_cell(CornerOps<T> &d, int c, const CornerRec &r,
                                                 const T *__restrict__ x,
                                                 const T *__restrict__ q,
                                                 const T *__restrict__ adt,
                                                 const T *__restrict__ res,
                                                 const BresLink &bl = BresLink{}) {
  Vec<T>::ld4(q + 4 * (size_t)c, d.qc);
  if constexpr (ZERO) {  // res known to be zero: the sums start from +0, as from the array
#pragma unroll
    for (int j = 0; j < 4; j++) d.rs[j] = (T)0;
  } else {
    Vec<T>::ld4_rw(res + 4 * (size_t)c, d.rs);
  }
  d.ac = __ldg(adt + c);
  const int nd[4] = {r.cn.x, r.cn.y, r.cn.z, r.cn.w};
#pragma unroll
  for (int j = 0; j < 4; j++) Vec<T>::ld2(x + 2 * (size_t)nd[j], d.xn[j][0], d.xn[j][1]);
  const int o[4] = {r.o.x, r.o.y, r.o.z, r.o.w};
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const int oo = ((r.meta >> (8 * s)) & 1u) ? o[s] : c;
    Vec<T>::ld4(q + 4 * (size_t)oo, d.qo[s]);
    d.ao[s] = __ldg(adt + oo);
  }
  d.meta = r.meta;
  if constexpr (BRES) {
    if (r.meta & 0x40404040u) {  // a boundary cell: its boundary edges' flags
#pragma unroll
      for (int s = 0; s < 4; s++)
        d.bnd[s] = ((r.meta >> (8 * s + 6)) & 1u) ? __ldg(bl.bound + o[s]) : 0;
    }
  }
}

// coordinate `comp` of corner i (0..3), by selects (no local-memory indexing)
template <typename T>
__device__ __forceinline__ T corner(const T (&xn)[4][2], unsigned i, int comp) {
  const T lo = (i & 1u) ? xn[1][comp] : xn[0][comp];
  const T hi = (i & 1u) ? xn[3][comp] : xn[2][comp];
  return (i & 2u) ? hi : lo;
}

template <typename T, bool BRES = false>
__device__ __forceinline__ void compute_corner(const CornerOps<T> &d, int c, T *__restrict__ res,
                                               const AirConst<T> &k) {
  T acc[4] = {d.rs[0], d.rs[1], d.rs[2], d.rs[3]};
  T ric, pc;  // the cell's own terms, once for its <= 4 edges
  air_prim<T>(d.qc, k, ric, pc);
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const unsigned m = (d.meta >> (8 * s)) & 0xffu;
    if (!(m & 1u)) continue;
    const unsigned a = (m >> 2) & 3u, b = (m >> 4) & 3u;
    const T x1x = corner<T>(d.xn, a, 0), x1y = corner<T>(d.xn, a, 1);
    const T x2x = corner<T>(d.xn, b, 0), x2y = corner<T>(d.xn, b, 1);
    T f[4], rio, po;
    air_prim<T>(d.qo[s], k, rio, po);
    if (m & 2u) {
      air_flux_prim<T>(x1x, x1y, x2x, x2y, d.qo[s], d.qc, rio, po, ric, pc, d.ao[s], d.ac, k, f);
#pragma unroll
      for (int j = 0; j < 4; j++) acc[j] -= f[j];
    } else {
      air_flux_prim<T>(x1x, x1y, x2x, x2y, d.qc, d.qo[s], ric, pc, rio, po, d.ac, d.ao[s], k, f);
#pragma unroll
      for (int j = 0; j < 4; j++) acc[j] += f[j];
    }
  }
  if constexpr (BRES) {
    // then bres_calc's increments: the boundary slots follow every interior
    // slot, in boundary-edge order (the two loops' order)
    if (d.meta & 0x40404040u) {
#pragma unroll
      for (int s = 0; s < 4; s++) {
        const unsigned m = (d.meta >> (8 * s)) & 0xffu;
        if (!(m & 0x40u)) continue;
        const unsigned a = (m >> 2) & 3u, b = (m >> 4) & 3u;
        T rr[4];
        air_bflux_prim<T>(corner<T>(d.xn, a, 0), corner<T>(d.xn, a, 1), corner<T>(d.xn, b, 0),
                          corner<T>(d.xn, b, 1), d.qc, ric, pc, d.ac, d.bnd[s], k, rr);
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

template <typename T, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
k_res_gather_corner(int ncell, const int4 *__restrict__ rec_o, const int4 *__restrict__ rec_cn,
                    const unsigned *__restrict__ rec_meta, const T *__restrict__ x,
                    const T *__restrict__ q, const T *__restrict__ adt, T *__restrict__ res,
                    AirConst<T> k) {
  const int G = gridDim.x * NT;
  int c = blockIdx.x * NT + threadIdx.x;
  if (c >= ncell) return;
  CornerOps<T> cur, nxt;
  CornerRec r1 = load_crec(rec_o, rec_cn, rec_meta, c + G, ncell);
  {
    const CornerRec r0 = load_crec(rec_o, rec_cn, rec_meta, c, ncell);
    load_corner_cell<T>(cur, c, r0, x, q, adt, res);
  }
  for (; c < ncell; c += G) {
    const CornerRec r2 = load_crec(rec_o, rec_cn, rec_meta, c + 2 * G, ncell);
    if (c + G < ncell) load_corner_cell<T>(nxt, c + G, r1, x, q, adt, res);
    compute_corner<T>(cur, c, res, k);
    cur = nxt;
    r1 = r2;
  }
}

// res_calc and the bres_calc that follows it in one launch (the runtime
// defers res_calc until the next loop call; when that is bres_calc on the
// same res, q, adt and x, this kernel runs instead of both)
template <typename T, int NT, bool ZERO = false>
__global__ void __launch_bounds__(NT, 1)
k_res_bres_corner(int ncell, const int4 *__restrict__ rec_o, const int4 *__restrict__ rec_cn,
                  const unsigned *__restrict__ rec_meta, const T *__restrict__ x,
                  const T *__restrict__ q, const T *__restrict__ adt, T *__restrict__ res,
                  AirConst<T> k, BresLink bl) {
  const int G = gridDim.x * NT;
  int c = blockIdx.x * NT + threadIdx.x;
  grid_dependency_wait();
  if (c >= ncell) return;
  CornerOps<T> cur, nxt;
  CornerRec r1 = load_crec(rec_o, rec_cn, rec_meta, c + G, ncell);
  {
    const CornerRec r0 = load_crec(rec_o, rec_cn, rec_meta, c, ncell);
    load_corner_cell<T, true, ZERO>(cur, c, r0, x, q, adt, res, bl);
  }
  for (; c < ncell; c += G) {
    const CornerRec r2 = load_crec(rec_o, rec_cn, rec_meta, c + 2 * G, ncell);
    if (c + G < ncell) load_corner_cell<T, true, ZERO>(nxt, c + G, r1, x, q, adt, res, bl);
    compute_corner<T, true>(cur, c, res, k);
    cur = nxt;
    r1 = r2;
  }
}

template <typename T, typename K>
cudaError_t launch_corner(K kern, int nt, const LaunchCtx &ctx, const SlotRecords &s,
                          const T *x, const T *q, const T *adt, T *res, const AirConst<T> &k) {
  int per_sm = 1;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, 0);
  if (e != cudaSuccess) return e;
  long long blocks = (long long)ctx.nsm * (per_sm < 1 ? 1 : per_sm);
  const long long need = (s.ncell + nt - 1) / nt;
  if (blocks > need) blocks = need;
  kern<<<(unsigned)blocks, nt, 0, ctx.stream>>>(
      s.ncell, reinterpret_cast<const int4 *>(s.o), reinterpret_cast<const int4 *>(s.cn),
      s.meta, x, q, adt, res, k);
  ctx.count();
  return cudaGetLastError();
}

}  // namespace

template <typename T>
cudaError_t launch_res_calc_gather_corner(const LaunchCtx &ctx, const SlotRecords &s, const T *x,
                                          const T *q, const T *adt, T *res,
                                          const AirConst<T> &k, int block, int minb) {
  if (s.ncell <= 0) return cudaSuccess;
  if (block == 64)
    return minb >= 6 ? launch_corner(k_res_gather_corner<T, 64, 6>, 64, ctx, s, x, q, adt, res, k)
                     : launch_corner(k_res_gather_corner<T, 64, 5>, 64, ctx, s, x, q, adt, res, k);
  if (block == 256)
    return launch_corner(k_res_gather_corner<T, 256, 1>, 256, ctx, s, x, q, adt, res, k);
  return minb >= 3 ? launch_corner(k_res_gather_corner<T, 128, 3>, 128, ctx, s, x, q, adt, res, k)
                   : launch_corner(k_res_gather_corner<T, 128, 1>, 128, ctx, s, x, q, adt, res, k);
}

template <typename T>
cudaError_t launch_res_bres_corner(const LaunchCtx &ctx, const SlotRecords &s,
                                   const BresRecords &b, const int *bound, const T *x,
                                   const T *q, const T *adt, T *res, const AirConst<T> &k,
                                   int block, bool zero_res) {
  if (s.ncell <= 0) return cudaSuccess;
  (void)b;
  const BresLink bl{bound};
  auto run = [&](auto kern, int nt) -> cudaError_t {
    int per_sm = 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, 0);
    if (e != cudaSuccess) return e;
    long long blocks = (long long)ctx.nsm * (per_sm < 1 ? 1 : per_sm);
    const long long need = (s.ncell + nt - 1) / nt;
    if (blocks > need) blocks = need;
    e = launch_dependent(ctx, kern, dim3((unsigned)blocks), dim3(nt), 0, s.ncell,
                         reinterpret_cast<const int4 *>(s.o), reinterpret_cast<const int4 *>(s.cn),
                         s.meta, x, q, adt, res, k, bl);
    ctx.count();
    return e != cudaSuccess ? e : cudaGetLastError();
  };
  if (zero_res)
    return block == 128 ? run(k_res_bres_corner<T, 128, true>, 128)
                        : run(k_res_bres_corner<T, 256, true>, 256);
  return block == 128 ? run(k_res_bres_corner<T, 128>, 128) : run(k_res_bres_corner<T, 256>, 256);
}

template cudaError_t launch_res_bres_corner<double>(const LaunchCtx &, const SlotRecords &,
                                                    const BresRecords &, const int *,
                                                    const double *, const double *,
                                                    const double *, double *,
                                                    const AirConst<double> &, int, bool);
template cudaError_t launch_res_bres_corner<float>(const LaunchCtx &, const SlotRecords &,
                                                   const BresRecords &, const int *, const float *,
                                                   const float *, const float *, float *,
                                                   const AirConst<float> &, int, bool);

template cudaError_t launch_res_calc_gather_corner<double>(const LaunchCtx &, const SlotRecords &,
                                                           const double *, const double *,
                                                           const double *, double *,
                                                           const AirConst<double> &, int, int);
template cudaError_t launch_res_calc_gather_corner<float>(const LaunchCtx &, const SlotRecords &,
                                                          const float *, const float *,
                                                          const float *, float *,
                                                          const AirConst<float> &, int, int);

template <typename T>
cudaError_t launch_res_calc_gather_regpipe(const LaunchCtx &ctx, const SlotRecords &s,
                                           const T *x, const T *q, const T *adt, T *res,
                                           const AirConst<T> &k, int block) {
  if (s.ncell <= 0) return cudaSuccess;
  const bool cs = rt().opt_pipe_hints != 0;
  if (cs) {
    switch (block) {
      case 64: return launch_regpipe(k_res_gather_regpipe<T, 64, true>, 64, ctx, s, x, q, adt, res, k);
      case 256: return launch_regpipe(k_res_gather_regpipe<T, 256, true>, 256, ctx, s, x, q, adt, res, k);
      default: return launch_regpipe(k_res_gather_regpipe<T, 128, true>, 128, ctx, s, x, q, adt, res, k);
    }
  }
  switch (block) {
    case 64: return launch_regpipe(k_res_gather_regpipe<T, 64, false>, 64, ctx, s, x, q, adt, res, k);
    case 256: return launch_regpipe(k_res_gather_regpipe<T, 256, false>, 256, ctx, s, x, q, adt, res, k);
    default: return launch_regpipe(k_res_gather_regpipe<T, 128, false>, 128, ctx, s, x, q, adt, res, k);
  }
}

template cudaError_t launch_res_calc_gather_regpipe<double>(const LaunchCtx &,
                                                            const SlotRecords &, const double *,
                                                            const double *, const double *,
                                                            double *, const AirConst<double> &,
                                                            int);
template cudaError_t launch_res_calc_gather_regpipe<float>(const LaunchCtx &, const SlotRecords &,
                                                           const float *, const float *,
                                                           const float *, float *,
                                                           const AirConst<float> &, int);

template <typename T>
cudaError_t launch_res_calc_gather_pipe(const LaunchCtx &c, const SlotRecords &s, const T *x,
                                        const T *q, const T *adt, T *res, const AirConst<T> &k,
                                        int block) {
  if (s.ncell <= 0) return cudaSuccess;
  switch (block) {
    case 64: return launch_pipe<T, 64>(c, s, x, q, adt, res, k);
    case 96: return launch_pipe<T, 96>(c, s, x, q, adt, res, k);
    case 256: return launch_pipe<T, 256>(c, s, x, q, adt, res, k);
    default: return launch_pipe<T, 128>(c, s, x, q, adt, res, k);
  }
}

template cudaError_t launch_res_calc_gather_pipe<double>(const LaunchCtx &, const SlotRecords &,
                                                         const double *, const double *,
                                                         const double *, double *,
                                                         const AirConst<double> &, int);
template cudaError_t launch_res_calc_gather_pipe<float>(const LaunchCtx &, const SlotRecords &,
                                                        const float *, const float *,
                                                        const float *, float *,
                                                        const AirConst<float> &, int);

}  // namespace op2b
