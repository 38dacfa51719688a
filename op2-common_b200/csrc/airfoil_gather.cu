// Owner-computes ("gather") indirect increments for res_calc and bres_calc.
//
// Instead of every edge scattering +f into cell 1 and -f into cell 2 (atomics
// or colouring), every cell gathers: one thread per target cell walks the
// elements that increment it -- listed by an inverse map, sorted by element
// index -- recomputes each element's flux and adds it into a register that
// starts from the cell's current res.  Consequences:
//   * no atomics, no colours, one launch, res written once per cell with a
//     coalesced store;
//   * the additions into res[c] happen in ascending element order, starting
//     from res[c] -- exactly the order of the reference's sequential loop
//     (op2/include/op_seq.h), and each flux is the same expression
//     (airfoil_math.cuh, compiled without FMA contraction): res_calc and
//     bres_calc are bit-exact with the sequential reference on the same
//     numbering;
//   * each interior edge's flux is computed twice (once per adjacent cell):
//     ~60 extra FP64 flops per edge, hidden under the memory time.
// The inverse maps (target -> sorted list of (element, slot)) are built on the
// device on first use, like a plan, and cached until the mesh is renumbered.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "airfoil_math.cuh"
#include "gather.h"
#include "op2b_runtime.h"
#include "scan.h"
#include "vec.cuh"

namespace op2b {

// ------------------------------------------------------------------ inverse maps

__global__ void k_inv_count(int n, int dim, const int *map, int *cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int d = 0; d < dim; d++) atomicAdd(&cnt[map[(size_t)i * dim + d]], 1);
}

__global__ void k_inv_fill(int n, int dim, const int *map, const long long *off, int *fill,
                           int *ent) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int d = 0; d < dim; d++) {
    int t = map[(size_t)i * dim + d];
    ent[off[t] + atomicAdd(&fill[t], 1)] = i * dim + d;
  }
}

// sort each target's entries (element*dim + slot) ascending
__global__ void k_inv_sort(int nto, const long long *off, int *ent) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nto) return;
  long long b = off[t], e = off[t + 1];
  for (long long i = b + 1; i < e; i++) {
    int v = ent[i];
    long long j = i - 1;
    while (j >= b && ent[j] > v) {
      ent[j + 1] = ent[j];
      j--;
    }
    ent[j + 1] = v;
  }
}

struct InvMapCache {
  op_map map = nullptr;
  InvMap inv;
  std::vector<void *> owned;
  ~InvMapCache() {
    for (void *p : owned) cudaFree(p);
  }
};

static std::vector<std::unique_ptr<InvMapCache>> &inv_cache() {
  static std::vector<std::unique_ptr<InvMapCache>> v;
  return v;
}

void release_inverse_maps() {
  release_slot_records();
  inv_cache().clear();
}

const InvMap *get_inverse_map(op_map map) {
  for (auto &c : inv_cache())
    if (c->map == map) return &c->inv;
  Runtime &r = rt();
  cudaStream_t s = r.stream;
  auto c = std::make_unique<InvMapCache>();
  c->map = map;
  int n = map->from->size, nto = map->to->size, dim = map->dim;
  auto A = [&](size_t bytes) -> void * {
    void *p = nullptr;
    if (cudaMallocAsync(&p, bytes ? bytes : 1, s) != cudaSuccess) return nullptr;
    c->owned.push_back(p);
    return p;
  };
  int *cnt = (int *)A(sizeof(int) * ((size_t)nto + 1));
  int *fill = (int *)A(sizeof(int) * ((size_t)nto + 1));
  long long *off = (long long *)A(sizeof(long long) * ((size_t)nto + 1));
  int *ent = (int *)A(sizeof(int) * ((size_t)n * dim + 1));
  if (!cnt || !fill || !off || !ent) {
    set_error("inverse map of %s: out of device memory", map->name);
    return nullptr;
  }
  if ((long long)n * dim >= (1LL << 31)) {
    set_error("inverse map of %s: too many entries", map->name);
    return nullptr;
  }
  cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)nto + 1), s);
  cudaMemsetAsync(fill, 0, sizeof(int) * ((size_t)nto + 1), s);
  unsigned g = (unsigned)((n + 255) / 256);
  if (n > 0) k_inv_count<<<g, 256, 0, s>>>(n, dim, map->map_d, cnt);
  if (!scan_exclusive(cnt, off, nto, s)) {
    set_error("inverse map of %s: scan failed", map->name);
    return nullptr;
  }
  if (n > 0) k_inv_fill<<<g, 256, 0, s>>>(n, dim, map->map_d, off, fill, ent);
  if (nto > 0) k_inv_sort<<<(unsigned)((nto + 255) / 256), 256, 0, s>>>(nto, off, ent);
  r.launches += 6;
  // the targets that have entries (rows), compacted on the device
  int *rows_d = (int *)A(sizeof(int) * ((size_t)nto + 1));
  long long *pos = (long long *)A(sizeof(long long) * ((size_t)nto + 1));
  int nrows = 0;
  if (!rows_d || !pos || !compact_nonzero(cnt, nto, rows_d, pos, &nrows, s)) {
    set_error("inverse map of %s: row compaction failed", map->name);
    return nullptr;
  }
  r.launches += 5;
  c->inv = InvMap{off, ent, rows_d, nrows, nto, dim, nrows == nto};
  inv_cache().push_back(std::move(c));
  return &inv_cache().back()->inv;
}

// ------------------------------------------------------------------ res_calc

template <typename T, int MINB>
__global__ void __launch_bounds__(256, MINB)
k_res_gather(InvMap inv, const int2 *__restrict__ pedge, const int2 *__restrict__ pecell,
             const T *__restrict__ x, const T *__restrict__ q, const T *__restrict__ adt,
             T *__restrict__ res, AirConst<T> k) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= inv.nrows) return;
  int c = inv.all_rows ? r : inv.rows[r];
  long long b = inv.off[c], e = inv.off[c + 1];
  T qc[4], acc[4];
  Vec<T>::ld4(q + 4 * (size_t)c, qc);
  Vec<T>::ld4_rw(res + 4 * (size_t)c, acc);
  T ac = __ldg(adt + c);
  for (long long i = b; i < e; i++) {
    int en = __ldg(inv.ent + i);
    int ed = en >> 1, slot = en & 1;
    int2 nn = __ldg(pedge + ed);
    int2 cc = __ldg(pecell + ed);
    int o = slot ? cc.x : cc.y;
    T qo[4], x1x, x1y, x2x, x2y, f[4];
    Vec<T>::ld4(q + 4 * (size_t)o, qo);
    T ao = __ldg(adt + o);
    Vec<T>::ld2(x + 2 * (size_t)nn.x, x1x, x1y);
    Vec<T>::ld2(x + 2 * (size_t)nn.y, x2x, x2y);
    if (slot == 0) {
      air_flux<T>(x1x, x1y, x2x, x2y, qc, qo, ac, ao, k, f);
#pragma unroll
      for (int m = 0; m < 4; m++) acc[m] += f[m];
    } else {
      air_flux<T>(x1x, x1y, x2x, x2y, qo, qc, ao, ac, k, f);
#pragma unroll
      for (int m = 0; m < 4; m++) acc[m] -= f[m];
    }
  }
  Vec<T>::st4(res + 4 * (size_t)c, acc);
}

template <typename T>
cudaError_t launch_res_calc_gather(const LaunchCtx &c, const InvMap &inv, const int *pedge,
                                   const int *pecell, const T *x, const T *q, const T *adt,
                                   T *res, const AirConst<T> &k) {
  if (inv.nrows <= 0) return cudaSuccess;
  unsigned g = (inv.nrows + 255) / 256;
  const int2 *pe = reinterpret_cast<const int2 *>(pedge);
  const int2 *pc = reinterpret_cast<const int2 *>(pecell);
  switch (rt().opt_gather_minb) {  // occupancy / register trade-off (tuning)
    case 4: k_res_gather<T, 4><<<g, 256, 0, c.stream>>>(inv, pe, pc, x, q, adt, res, k); break;
    case 5: k_res_gather<T, 5><<<g, 256, 0, c.stream>>>(inv, pe, pc, x, q, adt, res, k); break;
    case 6: k_res_gather<T, 6><<<g, 256, 0, c.stream>>>(inv, pe, pc, x, q, adt, res, k); break;
    default: k_res_gather<T, 1><<<g, 256, 0, c.stream>>>(inv, pe, pc, x, q, adt, res, k);
  }
  c.count();
  return cudaGetLastError();
}

// ------------------------------------------------------------------ res_calc, 4 lanes per cell
//
// One thread per (cell, incident edge) slot, four slots per cell (quad
// meshes; cells with fewer edges leave slots empty).  Slot records hold what
// the thread needs directly -- the other cell and the edge's two nodes, with
// the cell's role (first or second cell of the edge) and a valid bit in the
// top bits of n2 -- in three coalesced int arrays, so every load of a thread
// is independent of the others (two dependent steps instead of four).  Each
// lane computes its edge's flux, negated when the cell is the edge's second
// cell; lane 0 of the cell then adds the four lanes' increments to res[c] in
// slot order, i.e. ascending edge order -- the sequential reference's order.

constexpr unsigned kRoleBit = 1u << 30;
constexpr unsigned kValidBit = 1u << 31;

__global__ void k_build_slots(int ncell, const long long *off, const int *ent,
                              const int2 *pedge, const int2 *pecell, int *rec_o, int *rec_n1,
                              unsigned *rec_n2) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  long long b = off[c], e = off[c + 1];
  for (int k = 0; k < 4; k++) {
    size_t s = (size_t)c * 4 + k;
    if (b + k < e) {
      int en = ent[b + k];
      int ed = en >> 1, slot = en & 1;
      int2 cc = pecell[ed], nn = pedge[ed];
      rec_o[s] = slot ? cc.x : cc.y;
      rec_n1[s] = nn.x;
      rec_n2[s] = (unsigned)nn.y | (slot ? kRoleBit : 0u) | kValidBit;
    } else {
      rec_o[s] = c;
      rec_n1[s] = 0;
      rec_n2[s] = 0u;
    }
  }
}

__global__ void k_max_degree(int ncell, const long long *off, int *mx) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncell) atomicMax(mx, (int)(off[c + 1] - off[c]));
}

template <typename T>
__global__ void __launch_bounds__(256)
k_res_gather4(int ncell, const int *__restrict__ rec_o, const int *__restrict__ rec_n1,
              const unsigned *__restrict__ rec_n2, const T *__restrict__ x,
              const T *__restrict__ q, const T *__restrict__ adt, T *__restrict__ res,
              AirConst<T> k) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = t >> 2, slot = t & 3;
  const bool in = c < ncell;
  unsigned r2 = in ? __ldg(rec_n2 + t) : 0u;
  const bool valid = (r2 & kValidBit) != 0;
  T g[4] = {(T)0, (T)0, (T)0, (T)0};
  if (valid) {
    int o = __ldg(rec_o + t), n1 = __ldg(rec_n1 + t), n2 = (int)(r2 & (kRoleBit - 1));
    T qc[4], qo[4], x1x, x1y, x2x, x2y;
    Vec<T>::ld4(q + 4 * (size_t)c, qc);
    Vec<T>::ld4(q + 4 * (size_t)o, qo);
    T ac = __ldg(adt + c), ao = __ldg(adt + o);
    Vec<T>::ld2(x + 2 * (size_t)n1, x1x, x1y);
    Vec<T>::ld2(x + 2 * (size_t)n2, x2x, x2y);
    if (r2 & kRoleBit) {
      air_flux<T>(x1x, x1y, x2x, x2y, qo, qc, ao, ac, k, g);
#pragma unroll
      for (int m = 0; m < 4; m++) g[m] = -g[m];  // acc - f == acc + (-f) exactly
    } else {
      air_flux<T>(x1x, x1y, x2x, x2y, qc, qo, ac, ao, k, g);
    }
  }
  // lane 0 of each cell gathers its slots in order
  T h[3][4];
  bool v[3];
#pragma unroll
  for (int j = 1; j <= 3; j++) {
#pragma unroll
    for (int m = 0; m < 4; m++) h[j - 1][m] = __shfl_down_sync(0xffffffffu, g[m], j, 4);
    v[j - 1] = __shfl_down_sync(0xffffffffu, (int)valid, j, 4);
  }
  if (in && slot == 0) {
    T acc[4];
    Vec<T>::ld4_rw(res + 4 * (size_t)c, acc);
    if (valid) {
#pragma unroll
      for (int m = 0; m < 4; m++) acc[m] += g[m];
    }
#pragma unroll
    for (int j = 0; j < 3; j++)
      if (v[j]) {
#pragma unroll
        for (int m = 0; m < 4; m++) acc[m] += h[j][m];
      }
    Vec<T>::st4(res + 4 * (size_t)c, acc);
  }
}

// One thread per cell over the same slot records: the four records arrive as
// three int4 loads, the loop over the slots is unrolled so every gather of the
// cell is issued before the first flux, and the cell's own terms are computed
// once.  Increments are added in slot order, starting from res[c].
template <typename T, int MINB>
__global__ void __launch_bounds__(256, MINB)
k_res_gather_cell4(int ncell, const int4 *__restrict__ rec_o, const int4 *__restrict__ rec_n1,
                   const uint4 *__restrict__ rec_n2, const T *__restrict__ x,
                   const T *__restrict__ q, const T *__restrict__ adt, T *__restrict__ res,
                   AirConst<T> k) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int4 o4 = __ldg(rec_o + c), a4 = __ldg(rec_n1 + c);
  const uint4 b4 = __ldg(rec_n2 + c);
  const int o[4] = {o4.x, o4.y, o4.z, o4.w}, n1[4] = {a4.x, a4.y, a4.z, a4.w};
  const unsigned r2[4] = {b4.x, b4.y, b4.z, b4.w};
  T qc[4], acc[4];
  Vec<T>::ld4(q + 4 * (size_t)c, qc);
  T ac = __ldg(adt + c);
  T qo[4][4], ao[4], xa[4][2], xb[4][2];
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const bool v = (r2[s] & kValidBit) != 0;
    const int oo = v ? o[s] : c;
    const int na = v ? n1[s] : 0, nb = v ? (int)(r2[s] & (kRoleBit - 1)) : 0;
    Vec<T>::ld4(q + 4 * (size_t)oo, qo[s]);
    ao[s] = __ldg(adt + oo);
    Vec<T>::ld2(x + 2 * (size_t)na, xa[s][0], xa[s][1]);
    Vec<T>::ld2(x + 2 * (size_t)nb, xb[s][0], xb[s][1]);
  }
  Vec<T>::ld4_rw(res + 4 * (size_t)c, acc);
  T ric, pc;  // the cell's own terms, once for its edges (bit-identical)
  air_prim<T>(qc, k, ric, pc);
#pragma unroll
  for (int s = 0; s < 4; s++) {
    if (!(r2[s] & kValidBit)) continue;
    T f[4], rio, po;
    air_prim<T>(qo[s], k, rio, po);
    if (r2[s] & kRoleBit) {
      air_flux_prim<T>(xa[s][0], xa[s][1], xb[s][0], xb[s][1], qo[s], qc, rio, po, ric, pc,
                       ao[s], ac, k, f);
#pragma unroll
      for (int m = 0; m < 4; m++) acc[m] -= f[m];
    } else {
      air_flux_prim<T>(xa[s][0], xa[s][1], xb[s][0], xb[s][1], qc, qo[s], ric, pc, rio, po,
                       ac, ao[s], k, f);
#pragma unroll
      for (int m = 0; m < 4; m++) acc[m] += f[m];
    }
  }
  Vec<T>::st4(res + 4 * (size_t)c, acc);
}

template <typename T>
cudaError_t launch_res_calc_gather_cell4(const LaunchCtx &c, const SlotRecords &s, const T *x,
                                         const T *q, const T *adt, T *res,
                                         const AirConst<T> &k) {
  if (s.ncell <= 0) return cudaSuccess;
  unsigned g = (s.ncell + 255) / 256;
  const int4 *o = reinterpret_cast<const int4 *>(s.o), *n1 = reinterpret_cast<const int4 *>(s.n1);
  const uint4 *n2 = reinterpret_cast<const uint4 *>(s.n2);
  switch (rt().opt_gather_minb) {  // occupancy / register trade-off (tuning)
    case 2: k_res_gather_cell4<T, 2><<<g, 256, 0, c.stream>>>(s.ncell, o, n1, n2, x, q, adt, res, k); break;
    case 3: k_res_gather_cell4<T, 3><<<g, 256, 0, c.stream>>>(s.ncell, o, n1, n2, x, q, adt, res, k); break;
    case 4: k_res_gather_cell4<T, 4><<<g, 256, 0, c.stream>>>(s.ncell, o, n1, n2, x, q, adt, res, k); break;
    default: k_res_gather_cell4<T, 1><<<g, 256, 0, c.stream>>>(s.ncell, o, n1, n2, x, q, adt, res, k);
  }
  c.count();
  return cudaGetLastError();
}

template cudaError_t launch_res_calc_gather_cell4<double>(const LaunchCtx &,
                                                          const SlotRecords &, const double *,
                                                          const double *, const double *,
                                                          double *, const AirConst<double> &);
template cudaError_t launch_res_calc_gather_cell4<float>(const LaunchCtx &, const SlotRecords &,
                                                         const float *, const float *,
                                                         const float *, float *,
                                                         const AirConst<float> &);

struct SlotCache {
  op_map inc = nullptr, nodes = nullptr;
  SlotRecords rec{};
  bool corners_tried = false;
  int ring_state = 0;       // flux-ring records: 0 not tried, 1 built, -1 not possible
  int ring_ctas = 0, ring_nt = 0;
  uint2 *ring_buf = nullptr;
  op_map linked = nullptr;  // pbecell whose boundary records are linked in (fused bres_calc)
  int link_state = 0;       // 0 not tried, 1 linked, -1 not linkable
  std::vector<void *> owned;
  ~SlotCache() {
    for (void *p : owned) cudaFree(p);
    cudaFree(ring_buf);
  }
};

static std::vector<std::unique_ptr<SlotCache>> &slot_cache() {
  static std::vector<std::unique_ptr<SlotCache>> v;
  return v;
}

const SlotRecords *get_slot_records(op_map pecell, op_map pedge) {
  for (auto &s : slot_cache())
    if (s->inc == pecell && s->nodes == pedge) return &s->rec;
  const InvMap *inv = get_inverse_map(pecell);
  if (!inv) return nullptr;
  Runtime &r = rt();
  cudaStream_t s = r.stream;
  auto sc = std::make_unique<SlotCache>();
  sc->inc = pecell;
  sc->nodes = pedge;
  int n = pecell->to->size;
  int *mx = nullptr;
  cudaMallocAsync(&mx, sizeof(int), s);
  cudaMemsetAsync(mx, 0, sizeof(int), s);
  unsigned g = (unsigned)((n + 255) / 256);
  if (n > 0) k_max_degree<<<g, 256, 0, s>>>(n, inv->off, mx);
  int h_mx = 0;
  cudaMemcpyAsync(&h_mx, mx, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(mx, s);
  bool ok = cuda_ok(cudaStreamSynchronize(s), "slot records");
  if (!ok) return nullptr;
  sc->rec.ncell = n;
  sc->rec.usable = h_mx <= 4 && (long long)n * 4 < (1LL << 31) && pedge->to->size < (int)kRoleBit;
  if (sc->rec.usable && n > 0) {
    size_t cnt = (size_t)n * 4;
    int *o = nullptr, *n1 = nullptr;
    unsigned *n2 = nullptr;
    if (cudaMallocAsync(&o, cnt * 4, s) != cudaSuccess ||
        cudaMallocAsync(&n1, cnt * 4, s) != cudaSuccess ||
        cudaMallocAsync(&n2, cnt * 4, s) != cudaSuccess) {
      cudaFree(o);
      cudaFree(n1);
      set_error("slot records: out of device memory");
      return nullptr;
    }
    sc->owned = {o, n1, n2};
    k_build_slots<<<g, 256, 0, s>>>(n, inv->off, inv->ent,
                                    reinterpret_cast<const int2 *>(pedge->map_d),
                                    reinterpret_cast<const int2 *>(pecell->map_d), o, n1, n2);
    r.launches += 2;
    if (!cuda_ok(cudaStreamSynchronize(s), "slot records")) return nullptr;
    sc->rec.o = o;
    sc->rec.n1 = n1;
    sc->rec.n2 = n2;
  }
  slot_cache().push_back(std::move(sc));
  return &slot_cache().back()->rec;
}

// corner records of every cell from its slot records (see gather.h); *bad is
// set when a cell's valid slots touch more than four distinct nodes
__global__ void k_build_corners(int ncell, const int4 *rec_o, const int4 *rec_n1,
                                const uint4 *rec_n2, int4 *cn, unsigned *meta, int *bad) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int4 a4 = rec_n1[c];
  const uint4 b4 = rec_n2[c];
  const int na[4] = {a4.x, a4.y, a4.z, a4.w};
  const unsigned nb[4] = {b4.x, b4.y, b4.z, b4.w};
  int node[4] = {0, 0, 0, 0};
  int cnt = 0;
  unsigned m = 0;
  bool over = false;
  for (int s = 0; s < 4; s++) {
    if (!(nb[s] & kValidBit)) continue;
    const int ends[2] = {na[s], (int)(nb[s] & (kRoleBit - 1))};
    unsigned idx[2];
    for (int e = 0; e < 2; e++) {
      int j = 0;
      while (j < cnt && node[j] != ends[e]) j++;
      if (j == cnt) {
        if (cnt == 4) {
          over = true;
          j = 0;
        } else {
          node[cnt++] = ends[e];
        }
      }
      idx[e] = (unsigned)j;
    }
    m |= (1u | ((nb[s] & kRoleBit) ? 2u : 0u) | (idx[0] << 2) | (idx[1] << 4)) << (8 * s);
  }
  for (int j = cnt; j < 4; j++) node[j] = node[0];
  cn[c] = make_int4(node[0], node[1], node[2], node[3]);
  meta[c] = m;
  if (over) atomicOr(bad, 1);
}

const SlotRecords *get_corner_records(op_map pecell, op_map pedge) {
  const SlotRecords *base = get_slot_records(pecell, pedge);
  if (!base) return nullptr;
  SlotCache *sc = nullptr;
  for (auto &p : slot_cache())
    if (&p->rec == base) sc = p.get();
  if (!sc || sc->corners_tried) return base;
  sc->corners_tried = true;
  int n = base->ncell;
  // an isolated cell's unused corners read node 0: there must be one
  if (!base->usable || n <= 0 || pedge->to->size <= 0) return base;
  Runtime &r = rt();
  cudaStream_t s = r.stream;
  int4 *cn = nullptr;
  unsigned *meta = nullptr;
  int *bad = nullptr;
  if (cudaMallocAsync(&cn, sizeof(int4) * (size_t)n, s) != cudaSuccess ||
      cudaMallocAsync(&meta, sizeof(unsigned) * (size_t)n, s) != cudaSuccess ||
      cudaMallocAsync(&bad, sizeof(int), s) != cudaSuccess) {
    cudaFree(cn);
    cudaFree(meta);
    set_error("corner records: out of device memory");
    return nullptr;
  }
  cudaMemsetAsync(bad, 0, sizeof(int), s);
  k_build_corners<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      n, reinterpret_cast<const int4 *>(base->o), reinterpret_cast<const int4 *>(base->n1),
      reinterpret_cast<const uint4 *>(base->n2), cn, meta, bad);
  r.launches += 1;
  int h_bad = 1;
  cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(bad, s);
  bool ok = cuda_ok(cudaStreamSynchronize(s), "corner records");
  if (!ok) {
    cudaFree(cn);
    cudaFree(meta);
    return nullptr;
  }
  if (h_bad) {  // not a quadrilateral-style mesh: the slot-record kernels serve it
    cudaFree(cn);
    cudaFree(meta);
    return base;
  }
  sc->owned.push_back(cn);
  sc->owned.push_back(meta);
  sc->rec.cn = reinterpret_cast<const int *>(cn);
  sc->rec.meta = meta;
  sc->rec.corners = true;
  return base;
}

// ------------------------------------------------------------------ fused res_calc + bres_calc

// Place every boundary edge of a cell into the cell's corner record, after
// its interior slots and in edge order: the slot's o becomes the boundary
// edge, its meta byte 0x40 | corner of node 1 << 2 | corner of node 2 << 4.
// A node that is not yet a corner takes a free corner entry (a corner cell's
// outer node lies on its boundary edges only).  One thread per cell, on its
// first record.  With write == false only *bad is set (an edge without a free
// slot, or more than four nodes).
__global__ void k_link(int n, const int4 *__restrict__ rec, int4 *cn, int *o, unsigned *meta,
                       int *bad, bool write) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 r0 = rec[i];
  if (r0.x < 0) return;  // a continuation: handled with the cell's first record
  const int c = r0.x;
  unsigned m = meta[c];
  int nvalid = 0;
  for (int s = 0; s < 4; s++) nvalid += (int)((m >> (8 * s)) & 1u);
  const int4 k4 = cn[c];
  int corners[4] = {k4.x, k4.y, k4.z, k4.w};
  int cnt = 1;  // unused entries repeat the first corner
  for (int j = 1; j < 4; j++) cnt += corners[j] != corners[0] ? 1 : 0;
  int oo[4];
  for (int s = 0; s < 4; s++) oo[s] = o[(size_t)c * 4 + s];
  bool ok = true;
  for (int j = i, ord = 0; j < n; j++, ord++) {
    const int4 r = rec[j];
    if (j > i && r.x >= 0) break;  // the next cell's first record
    int ab[2];
    const int nodes[2] = {r.y, r.z};
    for (int e = 0; e < 2; e++) {
      int f = -1;
      for (int q = 0; q < cnt; q++)
        if (corners[q] == nodes[e]) f = q;
      if (f < 0 && cnt < 4) {
        f = cnt;
        corners[cnt++] = nodes[e];
      }
      ab[e] = f;
    }
    const int s = nvalid + ord;
    if (s >= 4 || ab[0] < 0 || ab[1] < 0) {
      ok = false;
      break;
    }
    oo[s] = r.w;
    m |= (0x40u | ((unsigned)ab[0] << 2) | ((unsigned)ab[1] << 4)) << (8 * s);
  }
  if (!ok) {
    atomicOr(bad, 1);
    return;
  }
  if (!write) return;
  for (int j = cnt; j < 4; j++) corners[j] = corners[0];
  cn[c] = make_int4(corners[0], corners[1], corners[2], corners[3]);
  for (int s = 0; s < 4; s++) o[(size_t)c * 4 + s] = oo[s];
  meta[c] = m;
}

bool link_boundary_records(const SlotRecords *rec, const BresRecords *b, op_map pbecell) {
  SlotCache *sc = nullptr;
  for (auto &p : slot_cache())
    if (&p->rec == rec) sc = p.get();
  if (!sc || !rec->corners) return false;
  if (sc->link_state != 0) return sc->link_state == 1 && sc->linked == pbecell;
  sc->link_state = -1;
  if (pbecell->to != sc->inc->to) return false;  // boundary cells must be the same set
  Runtime &r = rt();
  cudaStream_t s = r.stream;
  unsigned *meta = const_cast<unsigned *>(rec->meta);
  int *o = const_cast<int *>(rec->o);
  int4 *cn = reinterpret_cast<int4 *>(const_cast<int *>(rec->cn));
  int *bad = reinterpret_cast<int *>(r.check_d + 3);  // a word of the runtime's check scratch
  int h_bad = 1;
  const unsigned g = (unsigned)((b->n + 255) / 256);
  cudaMemsetAsync(bad, 0, sizeof(int), s);
  if (b->n > 0) {
    k_link<<<g, 256, 0, s>>>(b->n, b->rec, cn, o, meta, bad, false);
    r.launches += 1;
  }
  cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (!cuda_ok(cudaStreamSynchronize(s), "boundary link") || h_bad) return false;
  if (b->n > 0) {
    k_link<<<g, 256, 0, s>>>(b->n, b->rec, cn, o, meta, bad, true);
    r.launches += 1;
  }
  if (!cuda_ok(cudaStreamSynchronize(s), "boundary link")) return false;
  sc->link_state = 1;
  sc->linked = pbecell;
  return true;
}

// ------------------------------------------------------------------ flux-ring records

// the range [rs, re) of cell c: ranges of `span` cells
__device__ __forceinline__ void ring_range(int c, int span, int ncell, int &rs, int &re) {
  rs = (c / span) * span;
  re = min(rs + span, ncell);
}

// a slot's flux is read from the ring when the other cell is earlier in the
// same range (that cell computed it), and put into the ring when the other
// cell is later in the range; with the other cell outside the range, the
// cell computes it for itself alone (kept in its tile's scratch, not the ring)
__device__ __forceinline__ bool ring_consumes(int c, int nb, int rs, int re) {
  return nb >= rs && nb < re && nb < c;
}
__device__ __forceinline__ bool ring_produces(int c, int nb, int rs, int re) {
  return nb >= rs && nb < re && nb > c;
}

// fluxes each cell puts into the ring
__global__ void k_ring_count(int ncell, int span, const int4 *rec_o, const unsigned *meta,
                             int *cnt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int rs, re;
  ring_range(c, span, ncell, rs, re);
  const int4 o4 = rec_o[c];
  const int o[4] = {o4.x, o4.y, o4.z, o4.w};
  const unsigned m = meta[c];
  int n = 0;
  for (int s = 0; s < 4; s++)
    if ((m >> (8 * s)) & 1u) n += ring_produces(c, o[s], rs, re) ? 1 : 0;
  cnt[c] = n;
}

// ring entries: the k-th flux computed in a range (in cell order, slot order
// within a cell) goes to entry k mod OP2B_RING_ENTRIES; a consumer finds the
// entry of the producer's slot that names it.  *bad: a consumed flux whose
// entry is reused before the consumer's tile has read it, or an edge shared
// twice by one pair of cells.
__global__ void k_ring_fill(int ncell, int span, int nt, const int4 *rec_o, const unsigned *meta,
                            const long long *pre, uint2 *ring, int *bad) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int rs, re;
  ring_range(c, span, ncell, rs, re);
  const long long base = pre[rs];
  const int4 o4 = rec_o[c];
  const int o[4] = {o4.x, o4.y, o4.z, o4.w};
  const unsigned m = meta[c];
  unsigned f[4] = {0u, 0u, 0u, 0u};
  int rank = 0;
  for (int s = 0; s < 4; s++) {
    if (!((m >> (8 * s)) & 1u)) continue;
    const int nb = o[s];
    if (ring_produces(c, nb, rs, re)) {
      const long long k = pre[c] - base + rank++;
      f[s] = (unsigned)(k & (OP2B_RING_ENTRIES - 1));
      continue;
    }
    if (!ring_consumes(c, nb, rs, re)) {  // the other cell outside the range
      f[s] = 0x4000u;
      continue;
    }
    const int4 p4 = rec_o[nb];
    const int po[4] = {p4.x, p4.y, p4.z, p4.w};
    const unsigned pm = meta[nb];
    int prank = 0, found = -1, hits = 0;
    for (int t = 0; t < 4; t++) {
      if (!((pm >> (8 * t)) & 1u)) continue;
      if (po[t] == c) {
        hits++;
        found = prank;
      }
      if (ring_produces(nb, po[t], rs, re)) prank++;
    }
    const long long k = pre[nb] - base + found;
    const int tile = (c - rs) / nt;
    const int tend = min(rs + (tile + 1) * nt, re);
    const long long pend = pre[tend] - base;  // fluxes computed up to the end of c's tile
    if (hits != 1 || pend - k > OP2B_RING_ENTRIES) atomicOr(bad, 1);
    f[s] = 0x8000u | (unsigned)(k & (OP2B_RING_ENTRIES - 1));
  }
  ring[c] = make_uint2(f[0] | (f[1] << 16), f[2] | (f[3] << 16));
}

bool build_ring_records(const SlotRecords *rec, int nctas, int nt) {
  SlotCache *sc = nullptr;
  for (auto &p : slot_cache())
    if (&p->rec == rec) sc = p.get();
  if (!sc || !rec->corners || nctas <= 0 || nt <= 0) return false;
  if (sc->ring_state != 0 && sc->ring_ctas == nctas && sc->ring_nt == nt)
    return sc->ring_state == 1;
  sc->ring_state = -1;
  sc->ring_ctas = nctas;
  sc->ring_nt = nt;
  sc->rec.ring = nullptr;
  const int n = rec->ncell;
  if (n <= 0) return false;
  Runtime &r = rt();
  cudaStream_t s = r.stream;
  const int span = (int)(((long long)n + nctas - 1) / nctas);
  int *cnt = nullptr, *bad = nullptr;
  long long *pre = nullptr;
  if (!sc->ring_buf && cudaMalloc(&sc->ring_buf, sizeof(uint2) * (size_t)n) != cudaSuccess) {
    sc->ring_buf = nullptr;
    cudaGetLastError();
    return false;
  }
  if (cudaMallocAsync(&cnt, sizeof(int) * (size_t)n, s) != cudaSuccess ||
      cudaMallocAsync(&pre, sizeof(long long) * ((size_t)n + 1), s) != cudaSuccess ||
      cudaMallocAsync(&bad, sizeof(int), s) != cudaSuccess) {
    cudaGetLastError();
    if (cnt) cudaFreeAsync(cnt, s);
    if (pre) cudaFreeAsync(pre, s);
    return false;
  }
  const unsigned g = (unsigned)((n + 255) / 256);
  cudaMemsetAsync(bad, 0, sizeof(int), s);
  k_ring_count<<<g, 256, 0, s>>>(n, span, reinterpret_cast<const int4 *>(rec->o), rec->meta, cnt);
  r.launches++;
  bool ok = scan_exclusive(cnt, pre, n, s);
  if (ok) {
    k_ring_fill<<<g, 256, 0, s>>>(n, span, nt, reinterpret_cast<const int4 *>(rec->o), rec->meta,
                                  pre, sc->ring_buf, bad);
    r.launches++;
  }
  int h_bad = 1;
  cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(cnt, s);
  cudaFreeAsync(pre, s);
  cudaFreeAsync(bad, s);
  ok = cuda_ok(cudaStreamSynchronize(s), "flux-ring records") && ok;
  if (!ok || h_bad) return false;
  sc->ring_state = 1;
  sc->rec.ring = sc->ring_buf;
  sc->rec.ring_ctas = nctas;
  sc->rec.ring_span = span;
  sc->rec.ring_nt = nt;
  return true;
}

// ------------------------------------------------------------------ bres_calc records

__global__ void k_build_bres_records(int nrows, const int *rows, const long long *off,
                                     const int *ent, const int2 *pbedge, int4 *rec) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  const int c = rows[r];
  for (long long i = off[c]; i < off[c + 1]; i++) {
    const int be = ent[i];  // dim-1 map: entry = boundary edge
    const int2 nn = pbedge[be];
    rec[i] = make_int4(i == off[c] ? c : -1 - c, nn.x, nn.y, be);
  }
}

struct BresCache {
  op_map inc = nullptr, nodes = nullptr;
  BresRecords rec{};
  int4 *buf = nullptr;
  ~BresCache() { cudaFree(buf); }
};

static std::vector<std::unique_ptr<BresCache>> &bres_cache() {
  static std::vector<std::unique_ptr<BresCache>> v;
  return v;
}

const BresRecords *get_bres_records(op_map pbecell, op_map pbedge) {
  for (auto &b : bres_cache())
    if (b->inc == pbecell && b->nodes == pbedge) return &b->rec;
  if (pbecell->dim != 1) {
    set_error("bres_calc records: expected a dim-1 map (bedges -> cells)");
    return nullptr;
  }
  const InvMap *inv = get_inverse_map(pbecell);
  if (!inv) return nullptr;
  Runtime &r = rt();
  auto bc = std::make_unique<BresCache>();
  bc->inc = pbecell;
  bc->nodes = pbedge;
  const int n = pbecell->from->size;
  if (n > 0) {
    if (cudaMallocAsync(&bc->buf, sizeof(int4) * (size_t)n, r.stream) != cudaSuccess) {
      set_error("bres_calc records: out of device memory");
      return nullptr;
    }
    if (inv->nrows > 0) {
      k_build_bres_records<<<(unsigned)((inv->nrows + 255) / 256), 256, 0, r.stream>>>(
          inv->nrows, inv->rows, inv->off, inv->ent,
          reinterpret_cast<const int2 *>(pbedge->map_d), bc->buf);
      r.launches += 1;
    }
    if (!cuda_ok(cudaStreamSynchronize(r.stream), "bres_calc records")) return nullptr;
  }
  bc->rec = BresRecords{bc->buf, n};
  bres_cache().push_back(std::move(bc));
  return &bres_cache().back()->rec;
}

// One thread per record; the thread of a cell's first record adds all of the
// cell's boundary increments in ascending edge order, starting from res[c]
// (the sequential reference's order).  Two dependent load levels: the record,
// then the nodes, the flag and the cell's q, adt and res.
template <typename T>
__global__ void __launch_bounds__(128)
k_bres_records(int n, const int4 *__restrict__ rec, const int *__restrict__ bound,
               const T *__restrict__ x, const T *__restrict__ q, const T *__restrict__ adt,
               T *__restrict__ res, AirConst<T> k) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int4 r = __ldg(rec + i);
  if (r.x < 0) return;  // continuation: handled by the cell's first record
  const int c = r.x;
  T qc[4], acc[4];
  Vec<T>::ld4(q + 4 * (size_t)c, qc);
  Vec<T>::ld4_rw(res + 4 * (size_t)c, acc);
  const T ac = __ldg(adt + c);
  for (int j = i;;) {
    T x1x, x1y, x2x, x2y, rr[4];
    Vec<T>::ld2(x + 2 * (size_t)r.y, x1x, x1y);
    Vec<T>::ld2(x + 2 * (size_t)r.z, x2x, x2y);
    const int bnd = __ldg(bound + r.w);
    air_bflux<T>(x1x, x1y, x2x, x2y, qc, ac, bnd, k, rr);
    if (bnd == 1) {  // a wall edge leaves components 0 and 3 untouched
      acc[1] += rr[1];
      acc[2] += rr[2];
    } else {
#pragma unroll
      for (int m = 0; m < 4; m++) acc[m] += rr[m];
    }
    if (++j >= n) break;
    r = __ldg(rec + j);
    if (r.x >= 0) break;
  }
  Vec<T>::st4(res + 4 * (size_t)c, acc);
}

template <typename T>
cudaError_t launch_bres_calc_records(const LaunchCtx &c, const BresRecords &b, const int *bound,
                                     const T *x, const T *q, const T *adt, T *res,
                                     const AirConst<T> &k) {
  if (b.n <= 0) return cudaSuccess;
  k_bres_records<T><<<(unsigned)((b.n + 127) / 128), 128, 0, c.stream>>>(b.n, b.rec, bound, x, q,
                                                                        adt, res, k);
  c.count();
  return cudaGetLastError();
}

template cudaError_t launch_bres_calc_records<double>(const LaunchCtx &, const BresRecords &,
                                                      const int *, const double *,
                                                      const double *, const double *, double *,
                                                      const AirConst<double> &);
template cudaError_t launch_bres_calc_records<float>(const LaunchCtx &, const BresRecords &,
                                                     const int *, const float *, const float *,
                                                     const float *, float *,
                                                     const AirConst<float> &);

void release_slot_records() {
  slot_cache().clear();
  bres_cache().clear();
}

template <typename T>
cudaError_t launch_res_calc_gather4(const LaunchCtx &c, const SlotRecords &s, const T *x,
                                    const T *q, const T *adt, T *res, const AirConst<T> &k) {
  if (s.ncell <= 0) return cudaSuccess;
  long long threads = 4LL * s.ncell;
  k_res_gather4<T><<<(unsigned)((threads + 255) / 256), 256, 0, c.stream>>>(
      s.ncell, s.o, s.n1, s.n2, x, q, adt, res, k);
  c.count();
  return cudaGetLastError();
}

template cudaError_t launch_res_calc_gather4<double>(const LaunchCtx &, const SlotRecords &,
                                                     const double *, const double *,
                                                     const double *, double *,
                                                     const AirConst<double> &);
template cudaError_t launch_res_calc_gather4<float>(const LaunchCtx &, const SlotRecords &,
                                                    const float *, const float *, const float *,
                                                    float *, const AirConst<float> &);

// ------------------------------------------------------------------ bres_calc

template <typename T>
__global__ void __launch_bounds__(128)
k_bres_gather(InvMap inv, const int2 *__restrict__ pbedge, const int *__restrict__ bound,
              const T *__restrict__ x, const T *__restrict__ q, const T *__restrict__ adt,
              T *__restrict__ res, AirConst<T> k) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= inv.nrows) return;
  int c = inv.all_rows ? r : inv.rows[r];
  long long b = inv.off[c], e = inv.off[c + 1];
  T qc[4], acc[4];
  Vec<T>::ld4(q + 4 * (size_t)c, qc);
  Vec<T>::ld4_rw(res + 4 * (size_t)c, acc);
  T ac = __ldg(adt + c);
  for (long long i = b; i < e; i++) {
    int be = __ldg(inv.ent + i);  // dim 1: entry = boundary edge
    int2 nn = __ldg(pbedge + be);
    int bnd = __ldg(bound + be);
    T x1x, x1y, x2x, x2y, rr[4];
    Vec<T>::ld2(x + 2 * (size_t)nn.x, x1x, x1y);
    Vec<T>::ld2(x + 2 * (size_t)nn.y, x2x, x2y);
    air_bflux<T>(x1x, x1y, x2x, x2y, qc, ac, bnd, k, rr);
    if (bnd == 1) {  // a wall edge leaves components 0 and 3 untouched
      acc[1] += rr[1];
      acc[2] += rr[2];
    } else {
#pragma unroll
      for (int m = 0; m < 4; m++) acc[m] += rr[m];
    }
  }
  Vec<T>::st4(res + 4 * (size_t)c, acc);
}

template <typename T>
cudaError_t launch_bres_calc_gather(const LaunchCtx &c, const InvMap &inv, const int *pbedge,
                                    const int *bound, const T *x, const T *q, const T *adt,
                                    T *res, const AirConst<T> &k) {
  if (inv.nrows <= 0) return cudaSuccess;
  k_bres_gather<T><<<(inv.nrows + 127) / 128, 128, 0, c.stream>>>(
      inv, reinterpret_cast<const int2 *>(pbedge), bound, x, q, adt, res, k);
  c.count();
  return cudaGetLastError();
}

template cudaError_t launch_res_calc_gather<double>(const LaunchCtx &, const InvMap &,
                                                    const int *, const int *, const double *,
                                                    const double *, const double *, double *,
                                                    const AirConst<double> &);
template cudaError_t launch_res_calc_gather<float>(const LaunchCtx &, const InvMap &, const int *,
                                                   const int *, const float *, const float *,
                                                   const float *, float *,
                                                   const AirConst<float> &);
template cudaError_t launch_bres_calc_gather<double>(const LaunchCtx &, const InvMap &,
                                                     const int *, const int *, const double *,
                                                     const double *, const double *, double *,
                                                     const AirConst<double> &);
template cudaError_t launch_bres_calc_gather<float>(const LaunchCtx &, const InvMap &,
                                                    const int *, const int *, const float *,
                                                    const float *, const float *, float *,
                                                    const AirConst<float> &);

}  // namespace op2b
