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

__global__ void k_scan_serial_ll(const int *cnt, long long *off, int n) {
  // small-to-medium scans: one CTA, chunked (n up to a few million)
  __shared__ long long part[1024];
  int T = blockDim.x;
  long long chunk = (n + T - 1) / T;
  long long b = threadIdx.x * chunk, e = min((long long)n, b + chunk);
  long long s = 0;
  for (long long i = b; i < e; i++) s += cnt[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long acc = 0;
    for (int k = 0; k < T; k++) {
      long long t = part[k];
      part[k] = acc;
      acc += t;
    }
    off[n] = acc;
  }
  __syncthreads();
  long long acc = part[threadIdx.x];
  for (long long i = b; i < e; i++) {
    off[i] = acc;
    acc += cnt[i];
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

void release_inverse_maps() { inv_cache().clear(); }

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
    if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
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
  k_scan_serial_ll<<<1, 1024, 0, s>>>(cnt, off, nto);
  if (n > 0) k_inv_fill<<<g, 256, 0, s>>>(n, dim, map->map_d, off, fill, ent);
  if (nto > 0) k_inv_sort<<<(unsigned)((nto + 255) / 256), 256, 0, s>>>(nto, off, ent);
  r.launches += 4;
  if (!cuda_ok(cudaStreamSynchronize(s), "inverse map")) return nullptr;
  // compact list of targets that have entries (rows)
  std::vector<long long> h_off((size_t)nto + 1);
  cudaMemcpy(h_off.data(), off, sizeof(long long) * h_off.size(), cudaMemcpyDeviceToHost);
  std::vector<int> rows;
  rows.reserve(nto);
  for (int t = 0; t < nto; t++)
    if (h_off[t + 1] > h_off[t]) rows.push_back(t);
  int *rows_d = (int *)A(sizeof(int) * (rows.size() + 1));
  if (!rows.empty())
    cudaMemcpy(rows_d, rows.data(), sizeof(int) * rows.size(), cudaMemcpyHostToDevice);
  c->inv = InvMap{off, ent, rows_d, (int)rows.size(), nto, dim, rows.size() == (size_t)nto};
  inv_cache().push_back(std::move(c));
  return &inv_cache().back()->inv;
}

// ------------------------------------------------------------------ res_calc

template <typename T>
__global__ void __launch_bounds__(256)
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
  k_res_gather<T><<<(inv.nrows + 255) / 256, 256, 0, c.stream>>>(
      inv, reinterpret_cast<const int2 *>(pedge), reinterpret_cast<const int2 *>(pecell), x, q,
      adt, res, k);
  c.count();
  return cudaGetLastError();
}

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
