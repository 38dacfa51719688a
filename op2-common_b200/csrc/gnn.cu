// Graph kernels of the learned warm start (include/op2b_gnn.h): the gathers,
// aggregations and gradient combinations around the tensor-core MLPs.
//
// Rows are 128-wide feature vectors (D a multiple of 8), so every kernel moves
// 16-byte chunks: one thread per (row, 8-feature chunk), consecutive threads
// on consecutive chunks of the same row, which coalesces each row into whole
// sectors.  Aggregations walk a CSR of incoming edges per node in a fixed order
// (no atomics: deterministic sums).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "op2b_gnn.h"
#include "op2b_runtime.h"

namespace op2b {
namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ void bf16x8_to_f32(const uint4 &w, float *f) {
  const __nv_bfloat162 *p = reinterpret_cast<const __nv_bfloat162 *>(&w);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    float2 t = __bfloat1622float2(p[i]);
    f[2 * i] = t.x;
    f[2 * i + 1] = t.y;
  }
}

__device__ __forceinline__ uint4 f32_to_bf16x8(const float *f) {
  uint4 w;
  __nv_bfloat162 *p = reinterpret_cast<__nv_bfloat162 *>(&w);
#pragma unroll
  for (int i = 0; i < 4; i++) p[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
  return w;
}

__device__ __forceinline__ void ld8(const float *p, float *f) {
  float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
  f[0] = a.x, f[1] = a.y, f[2] = a.z, f[3] = a.w, f[4] = b.x, f[5] = b.y, f[6] = b.z, f[7] = b.w;
}

__device__ __forceinline__ void st8(float *p, const float *f) {
  reinterpret_cast<float4 *>(p)[0] = make_float4(f[0], f[1], f[2], f[3]);
  reinterpret_cast<float4 *>(p)[1] = make_float4(f[4], f[5], f[6], f[7]);
}

__global__ void k_gather_pair(long E, int D, const int *__restrict__ src,
                              const int *__restrict__ dst, const __nv_bfloat16 *__restrict__ h,
                              long ldh, __nv_bfloat16 *__restrict__ cat, long ldcat, int col0) {
  const int chunks = D / 8;
  const long total = E * 2 * chunks;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long k = t / (2 * chunks);
    const int r = (int)(t - k * 2 * chunks);
    const int side = r >= chunks, c = r - side * chunks;
    const int node = side ? __ldg(dst + k) : __ldg(src + k);
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(h + (long)node * ldh) + c);
    reinterpret_cast<uint4 *>(cat + k * ldcat + col0 + side * D)[c] = v;
  }
}

__global__ void k_aggregate(long N, int D, const int *__restrict__ off,
                            const int *__restrict__ idx, const __nv_bfloat16 *__restrict__ e,
                            long lde, __nv_bfloat16 *__restrict__ out, long ldo) {
  const int chunks = D / 8;
  const long total = N * chunks;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long n = t / chunks;
    const int c = (int)(t - n * chunks);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int j1 = __ldg(off + n + 1);
    for (int j = __ldg(off + n); j < j1; j++) {
      const long k = __ldg(idx + j);
      float f[8];
      bf16x8_to_f32(__ldg(reinterpret_cast<const uint4 *>(e + k * lde) + c), f);
#pragma unroll
      for (int i = 0; i < 8; i++) acc[i] += f[i];
    }
    reinterpret_cast<uint4 *>(out + n * ldo)[c] = f32_to_bf16x8(acc);
  }
}

__global__ void k_to_bf16(long M, int D, const float *__restrict__ x, long ldx,
                          __nv_bfloat16 *__restrict__ y, long ldy) {
  const int chunks = D / 8;
  const long total = M * chunks;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long m = t / chunks;
    const int c = (int)(t - m * chunks);
    float f[8];
    ld8(x + m * ldx + c * 8, f);
    reinterpret_cast<uint4 *>(y + m * ldy)[c] = f32_to_bf16x8(f);
  }
}

__global__ void k_add_f32(long M, int D, float *__restrict__ acc, const float *__restrict__ x,
                          long ldx) {
  const int chunks = D / 8;
  const long total = M * chunks;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long m = t / chunks;
    const int c = (int)(t - m * chunks);
    float a[8], f[8];
    ld8(acc + m * D + c * 8, a);
    ld8(x + m * ldx + c * 8, f);
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] += f[i];
    st8(acc + m * D + c * 8, a);
  }
}

__global__ void k_edge_grad(long E, int D, const int *__restrict__ dst, float *__restrict__ dE,
                            const float *__restrict__ dAgg, long ldagg,
                            __nv_bfloat16 *__restrict__ dy) {
  const int chunks = D / 8;
  const long total = E * chunks;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long k = t / chunks;
    const int c = (int)(t - k * chunks);
    const long n = __ldg(dst + k);
    float a[8], f[8];
    ld8(dE + k * D + c * 8, a);
    ld8(dAgg + n * ldagg + c * 8, f);
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] += f[i];
    st8(dE + k * D + c * 8, a);
    reinterpret_cast<uint4 *>(dy + k * D)[c] = f32_to_bf16x8(a);
  }
}

__global__ void k_cat_grad_edges(long E, int D, const float *__restrict__ dCat, long ldcat,
                                 float *__restrict__ dE) {
  const int chunks = D / 8;
  const long total = E * chunks;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long k = t / chunks;
    const int c = (int)(t - k * chunks);
    float a[8], f[8];
    ld8(dE + k * D + c * 8, a);
    ld8(dCat + k * ldcat + c * 8, f);
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] += f[i];
    st8(dE + k * D + c * 8, a);
  }
}

__global__ void k_cat_grad_nodes(long N, int D, const float *__restrict__ dCat, long ldcat,
                                 const int *__restrict__ off, const int *__restrict__ idx,
                                 const int *__restrict__ rev, float *__restrict__ dH) {
  const int chunks = D / 8;
  const long total = N * chunks;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long n = t / chunks;
    const int c = (int)(t - n * chunks);
    float a[8];
    ld8(dH + n * D + c * 8, a);
    const int j1 = __ldg(off + n + 1);
    for (int j = __ldg(off + n); j < j1; j++) {
      const long k = __ldg(idx + j), kr = __ldg(rev + k);
      float f[8], g[8];
      ld8(dCat + k * ldcat + 2 * D + c * 8, f);
      ld8(dCat + kr * ldcat + D + c * 8, g);
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] += f[i] + g[i];
    }
    st8(dH + n * D + c * 8, a);
  }
}

// column sums: a CTA of 256 threads covers 32 columns x 8 row lanes of a
// chunk of rows, reduces in shared memory and adds once per column
__global__ void k_colsum(long M, int N, const __nv_bfloat16 *__restrict__ dz, long ld,
                         float *__restrict__ db, long rows_per_cta) {
  __shared__ float s[8][33];
  const int cx = threadIdx.x & 31, ry = threadIdx.x >> 5;
  const int col = blockIdx.y * 32 + cx;
  const long r0 = blockIdx.x * rows_per_cta, r1 = min(M, r0 + rows_per_cta);
  float acc = 0.f;
  if (col < N)
    for (long r = r0 + ry; r < r1; r += 8) acc += __bfloat162float(dz[r * ld + col]);
  s[ry][cx] = acc;
  __syncthreads();
  if (ry == 0 && col < N) {
    float t = 0.f;
#pragma unroll
    for (int i = 0; i < 8; i++) t += s[i][cx];
    atomicAdd(db + col, t);
  }
}

__global__ void k_mse(long M, int D, const float *__restrict__ out, long ldo,
                      const float *__restrict__ target, __nv_bfloat16 *__restrict__ dy,
                      float *__restrict__ loss, float scale) {
  __shared__ float s[kBlock / 32];
  float acc = 0.f;
  const long total = M * ldo;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long m = t / ldo;
    const int c = (int)(t - m * ldo);
    float g = 0.f;
    if (c < D) {
      const float d = out[t] - target[m * D + c];
      acc += d * d;
      g = 2.f * scale * d;
    }
    dy[t] = __float2bfloat16(g);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int i = 0; i < kBlock / 32; i++) t += s[i];
    atomicAdd(loss, t * scale);
  }
}

__global__ void k_adam(long n, float *__restrict__ p, float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v,
                       __nv_bfloat16 *__restrict__ pb, float lr_t, float b1, float b2, float eps,
                       float wd_lr) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] * (1.f - wd_lr);
    pi -= lr_t * mi / (sqrtf(vi) + eps);
    p[i] = pi;
    g[i] = 0.f;
    if (pb) pb[i] = __float2bfloat16(pi);
  }
}

__global__ void k_decode_q(long ncell, const float *__restrict__ out, long ldo,
                           const double *__restrict__ ms, const double *__restrict__ qinf,
                           double *__restrict__ q) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ncell * 4;
       i += (long)gridDim.x * blockDim.x) {
    const long c = i >> 2;
    const int k = (int)(i & 3);
    q[i] = qinf[k] + ms[k] + ms[4 + k] * (double)out[c * ldo + k];
  }
}

int grid_for(long work) {
  const long g = (work + kBlock - 1) / kBlock;
  const long cap = (long)rt().nsm * 16;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

bool launched(const char *what) {
  if (rt().initialised) rt().launches++;
  return cuda_ok(cudaGetLastError(), what);
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace
}  // namespace op2b

using namespace op2b;

#define S_ static_cast<cudaStream_t>(stream)

extern "C" {

int op2b_gnn_gather_pair(int E, int D, const int *src, const int *dst, const void *h, long ldh,
                         void *cat, long ldcat, int col0, void *stream) {
  if (E < 0 || D <= 0 || D % 8 || ldh % 8 || ldcat % 8 || col0 % 8 || !aligned16(h) ||
      !aligned16(cat)) {
    set_error("op2b_gnn_gather_pair: D, leading dims and col0 must be multiples of 8 and the "
              "arrays 16-byte aligned");
    return -1;
  }
  if (E == 0) return 0;
  const long work = (long)E * 2 * (D / 8);
  k_gather_pair<<<grid_for(work), kBlock, 0, S_>>>(E, D, src, dst, (const __nv_bfloat16 *)h, ldh,
                                                  (__nv_bfloat16 *)cat, ldcat, col0);
  return launched("op2b_gnn_gather_pair") ? 0 : -1;
}

int op2b_gnn_aggregate(int N, int D, const int *off, const int *idx, const void *e, long lde,
                       void *out, long ldo, void *stream) {
  if (N < 0 || D <= 0 || D % 8 || lde % 8 || ldo % 8 || !aligned16(e) || !aligned16(out)) {
    set_error("op2b_gnn_aggregate: D and leading dims multiples of 8, 16-byte aligned arrays");
    return -1;
  }
  if (N == 0) return 0;
  k_aggregate<<<grid_for((long)N * (D / 8)), kBlock, 0, S_>>>(
      N, D, off, idx, (const __nv_bfloat16 *)e, lde, (__nv_bfloat16 *)out, ldo);
  return launched("op2b_gnn_aggregate") ? 0 : -1;
}

int op2b_gnn_to_bf16(int M, int D, const float *x, long ldx, void *y, long ldy, void *stream) {
  if (M < 0 || D <= 0 || D % 8 || ldx % 4 || ldy % 8 || !aligned16(x) || !aligned16(y)) {
    set_error("op2b_gnn_to_bf16: D a multiple of 8, aligned leading dims and arrays");
    return -1;
  }
  if (M == 0) return 0;
  k_to_bf16<<<grid_for((long)M * (D / 8)), kBlock, 0, S_>>>(M, D, x, ldx, (__nv_bfloat16 *)y,
                                                           ldy);
  return launched("op2b_gnn_to_bf16") ? 0 : -1;
}

int op2b_gnn_add_f32(int M, int D, float *acc, const float *x, long ldx, void *stream) {
  if (M < 0 || D <= 0 || D % 8 || ldx % 4 || !aligned16(acc) || !aligned16(x)) {
    set_error("op2b_gnn_add_f32: D a multiple of 8, aligned leading dims and arrays");
    return -1;
  }
  if (M == 0) return 0;
  k_add_f32<<<grid_for((long)M * (D / 8)), kBlock, 0, S_>>>(M, D, acc, x, ldx);
  return launched("op2b_gnn_add_f32") ? 0 : -1;
}

int op2b_gnn_edge_grad(int E, int D, const int *dst, float *dE, const float *dAgg, long ldagg,
                       void *dy, void *stream) {
  if (E < 0 || D <= 0 || D % 8 || ldagg % 4 || !aligned16(dE) || !aligned16(dAgg) ||
      !aligned16(dy)) {
    set_error("op2b_gnn_edge_grad: D a multiple of 8, aligned leading dims and arrays");
    return -1;
  }
  if (E == 0) return 0;
  k_edge_grad<<<grid_for((long)E * (D / 8)), kBlock, 0, S_>>>(E, D, dst, dE, dAgg, ldagg,
                                                             (__nv_bfloat16 *)dy);
  return launched("op2b_gnn_edge_grad") ? 0 : -1;
}

int op2b_gnn_cat_grad(int E, int N, int D, const float *dCat, long ldcat, float *dE,
                      const int *off, const int *idx, const int *rev, float *dH, void *stream) {
  if (E < 0 || N < 0 || D <= 0 || D % 8 || ldcat % 4 || ldcat < 3 * D || !aligned16(dCat) ||
      !aligned16(dE) || !aligned16(dH)) {
    set_error("op2b_gnn_cat_grad: D a multiple of 8, ldcat >= 3D, aligned arrays");
    return -1;
  }
  if (E > 0) {
    k_cat_grad_edges<<<grid_for((long)E * (D / 8)), kBlock, 0, S_>>>(E, D, dCat, ldcat, dE);
    if (!launched("op2b_gnn_cat_grad")) return -1;
  }
  if (N > 0) {
    k_cat_grad_nodes<<<grid_for((long)N * (D / 8)), kBlock, 0, S_>>>(N, D, dCat, ldcat, off, idx,
                                                                    rev, dH);
    if (!launched("op2b_gnn_cat_grad")) return -1;
  }
  return 0;
}

int op2b_gnn_colsum(int M, int N, const void *dz, long ld, float *db, void *stream) {
  if (M < 0 || N <= 0 || ld < N) {
    set_error("op2b_gnn_colsum: bad sizes");
    return -1;
  }
  if (M == 0) return 0;
  const int ncol = (N + 31) / 32;
  long rows = (long)M * ncol / (rt().nsm * 8) + 1;
  rows = ((rows + 63) / 64) * 64;
  const long nrb = (M + rows - 1) / rows;
  k_colsum<<<dim3((unsigned)nrb, ncol), kBlock, 0, S_>>>(M, N, (const __nv_bfloat16 *)dz, ld, db,
                                                         rows);
  return launched("op2b_gnn_colsum") ? 0 : -1;
}

int op2b_gnn_mse(int M, int D, const float *out, long ldo, const float *target, void *dy,
                 float *loss, float scale, void *stream) {
  if (M < 0 || D <= 0 || ldo < D) {
    set_error("op2b_gnn_mse: bad sizes");
    return -1;
  }
  if (M == 0) return 0;
  k_mse<<<grid_for((long)M * ldo), kBlock, 0, S_>>>(M, D, out, ldo, target,
                                                    (__nv_bfloat16 *)dy, loss, scale);
  return launched("op2b_gnn_mse") ? 0 : -1;
}

int op2b_gnn_adam(long n, float *p, float *g, float *m, float *v, void *pb, float lr_t,
                  float beta1, float beta2, float eps, float wd, void *stream) {
  if (n < 0) {
    set_error("op2b_gnn_adam: negative size");
    return -1;
  }
  if (n == 0) return 0;
  k_adam<<<grid_for(n), kBlock, 0, S_>>>(n, p, g, m, v, (__nv_bfloat16 *)pb, lr_t, beta1, beta2,
                                         eps, wd);
  return launched("op2b_gnn_adam") ? 0 : -1;
}

int op2b_gnn_memset(void *ptr, int value, long bytes, void *stream) {
  if (bytes < 0 || (bytes > 0 && !ptr)) {
    set_error("op2b_gnn_memset: bad pointer or size");
    return -1;
  }
  if (bytes == 0) return 0;
  return cuda_ok(cudaMemsetAsync(ptr, value, (size_t)bytes, S_), "op2b_gnn_memset") ? 0 : -1;
}

int op2b_gnn_decode_q(int ncell, const float *out, long ldo, const double *mean_std,
                      const double *qinf, double *q, void *stream) {
  if (ncell < 0 || ldo < 4) {
    set_error("op2b_gnn_decode_q: bad sizes");
    return -1;
  }
  if (ncell == 0) return 0;
  k_decode_q<<<grid_for((long)ncell * 4), kBlock, 0, S_>>>(ncell, out, ldo, mean_std, qinf, q);
  return launched("op2b_gnn_decode_q") ? 0 : -1;
}

}  // extern "C"
