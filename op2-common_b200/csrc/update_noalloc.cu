// op2b_update_noalloc: the update loop for callers that cannot allocate
// device memory.
//
// Who needs it: an application that hands all device memory to its own pool
// at start-up (so a later cudaMalloc inside a library call fails or breaks
// the pool's budget), and code on a latency-critical path that must not pay
// cudaMalloc/cudaFree, which synchronise the whole device.  Those callers
// pass their own device arrays and get the same arithmetic as
// op_par_loop("update", ...), without the library allocating anything.
//
// How: the reduction scratch (one partial per CTA plus the ticket counter)
// is a file-scope __device__ array of fixed size, loaded with the library and
// held by every GPU that loads it until the process exits:
//   kMaxBlocks + 1 slots of 32 bytes = 524,320 bytes per device.
// One thread per cell and 256 threads per CTA, so ncell is limited to
// kMaxBlocks * 256 = 4,194,304 cells; larger sizes are rejected.
//
// The array is shared by every call and keeps the previous call's contents:
// the ticket counter is cleared (cudaMemsetAsync on the caller's stream)
// before each launch, and the partials are written before they are read.
// Calls whose launches can overlap on the GPU (different streams, or
// different host threads) race on this one array and must be serialised by
// the caller.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>

#include "op2b.h"
#include "op2b_runtime.h"

namespace op2b {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 16384;
constexpr long long kMaxCells = (long long)kMaxBlocks * kThreads;
constexpr int kMaxDevices = 64;

struct Partial {
  double sum;
  double maxv;
  long long idx;
  long long pad;
};

// partials [0, kMaxBlocks), then one slot whose first word is the ticket
static __device__ __align__(256) Partial g_update_scratch[kMaxBlocks + 1];

// device address of g_update_scratch, looked up once per device
static Partial *g_scratch_addr[kMaxDevices] = {};

__device__ __forceinline__ void merge(double &s, double &m, long long &i, double s2, double m2,
                                      long long i2) {
  s += s2;
  if (m2 > m || (m2 == m && i2 < i)) {
    m = m2;
    i = i2;
  }
}

__device__ __forceinline__ void reduce_block(double &s, double &m, long long &i) {
  __shared__ double ss[kThreads / 32], sm[kThreads / 32];
  __shared__ long long si[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1)
    merge(s, m, i, __shfl_down_sync(0xffffffffu, s, o), __shfl_down_sync(0xffffffffu, m, o),
          __shfl_down_sync(0xffffffffu, i, o));
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    ss[w] = s;
    sm[w] = m;
    si[w] = i;
  }
  __syncthreads();
  if (w == 0) {
    s = 0.0;
    m = -INFINITY;
    i = LLONG_MAX;
    if (l < kThreads / 32) {
      s = ss[l];
      m = sm[l];
      i = si[l];
    }
    for (int o = 16; o > 0; o >>= 1)
      merge(s, m, i, __shfl_down_sync(0xffffffffu, s, o), __shfl_down_sync(0xffffffffu, m, o),
            __shfl_down_sync(0xffffffffu, i, o));
  }
  __syncthreads();
}

// update.h:1-19 for one cell per thread; the last CTA to finish folds the
// partials in CTA order and applies op_arg_gbl semantics to the caller's
// device outputs: rms += sum, and maxerr/errloc replaced when beaten.
__global__ void __launch_bounds__(kThreads)
k_update_noalloc(int ncell, const double *__restrict__ qold, double *__restrict__ q,
                 double *__restrict__ res, const double *__restrict__ adt, Partial *scratch,
                 double *rms, double *maxerr, int *errloc) {
  double s = 0.0, m = -INFINITY;
  long long i = LLONG_MAX;
  int n = blockIdx.x * kThreads + threadIdx.x;
  if (n < ncell) {
    const double2 *qo = reinterpret_cast<const double2 *>(qold + 4 * (size_t)n);
    double2 *r2 = reinterpret_cast<double2 *>(res + 4 * (size_t)n);
    double2 a = __ldg(qo), b = __ldg(qo + 1), ra = r2[0], rb = r2[1];
    double qv[4] = {a.x, a.y, b.x, b.y}, rv[4] = {ra.x, ra.y, rb.x, rb.y}, out[4];
    double adti = 1.0f / __ldg(adt + n);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      double del = adti * rv[k];
      out[k] = qv[k] - del;
      double sq = del * del;
      s += sq;
      if (sq > m) {
        m = sq;
        i = n;
      }
    }
    double2 *q2 = reinterpret_cast<double2 *>(q + 4 * (size_t)n);
    q2[0] = make_double2(out[0], out[1]);
    q2[1] = make_double2(out[2], out[3]);
    r2[0] = make_double2(0.0, 0.0);
    r2[1] = make_double2(0.0, 0.0);
  }
  reduce_block(s, m, i);
  __shared__ bool last;
  unsigned *ticket = reinterpret_cast<unsigned *>(scratch + kMaxBlocks);
  if (threadIdx.x == 0) {
    scratch[blockIdx.x] = Partial{s, m, i, 0};
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  s = 0.0;
  m = -INFINITY;
  i = LLONG_MAX;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kThreads) {
    const volatile Partial *p = scratch + b;
    merge(s, m, i, p->sum, p->maxv, p->idx);
  }
  reduce_block(s, m, i);
  if (threadIdx.x == 0) {
    *rms += s;
    if (m > *maxerr) {
      *maxerr = m;
      *errloc = (int)i;
    }
    *ticket = 0u;
  }
}

}  // namespace
}  // namespace op2b

using namespace op2b;

extern "C" int op2b_update_noalloc(int ncell, const double *qold, double *q, double *res,
                                   const double *adt, double *rms, double *maxerr, int *errloc,
                                   void *stream) {
  if (ncell < 0 || (long long)ncell > kMaxCells) {
    set_error("op2b_update_noalloc: ncell = %d is outside [0, %lld], the most cells the "
              "fixed %d-partial scratch holds (one cell per thread, %d threads per block)",
              ncell, kMaxCells, kMaxBlocks, kThreads);
    return -1;
  }
  if (ncell == 0) return 0;
  if (!qold || !q || !res || !adt || !rms || !maxerr || !errloc) {
    set_error("op2b_update_noalloc: every array and output must be a device pointer");
    return -1;
  }
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "op2b_update_noalloc: cudaGetDevice")) return -1;
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("op2b_update_noalloc: device ordinal %d above %d", dev, kMaxDevices - 1);
    return -1;
  }
  if (!g_scratch_addr[dev]) {
    // first call on this device, with the device current: resolve the
    // array's device address (host code may not use the symbol itself)
    Partial *ptr = nullptr;
    if (!cuda_ok(cudaGetSymbolAddress((void **)&ptr, g_update_scratch),
                 "op2b_update_noalloc: cudaGetSymbolAddress"))
      return -1;
    g_scratch_addr[dev] = ptr;
  }
  Partial *scratch = g_scratch_addr[dev];
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!cuda_ok(cudaMemsetAsync(scratch + kMaxBlocks, 0, sizeof(Partial), s),
               "op2b_update_noalloc: clearing the ticket"))
    return -1;
  int grid = (int)((ncell + kThreads - 1) / kThreads);
  k_update_noalloc<<<grid, kThreads, 0, s>>>(ncell, qold, q, res, adt, scratch, rms, maxerr,
                                             errloc);
  if (rt().initialised) rt().launches++;
  return cuda_ok(cudaGetLastError(), "op2b_update_noalloc: launch") ? 0 : -1;
}
