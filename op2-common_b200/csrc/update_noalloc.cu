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
//
// Host code cannot pass the array's name to a kernel (on the host it names a
// stand-in, not device memory), so the first call on a device, with that
// device current, asks cudaGetSymbolAddress for the device address and keeps
// it per device, tagged with the current context's unique ID: after the
// caller resets the device (a new context), the next call looks the address
// up again instead of using the old context's.  That look-up is not a stream
// operation, but it may load the module, so the first call on a device (and
// the first after a reset) must come before any stream capture.
//
// Arrays are read and written as 16-byte vectors, so qold, q and res must be
// 16-byte aligned (adt, rms and maxerr 8-byte, errloc 4-byte); a misaligned
// pointer is refused on the host, before anything is launched.
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <climits>
#include <cmath>
#include <cstdint>

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

// device address of g_update_scratch per device, and the ID of the context
// it was looked up in (0 = not looked up yet)
static std::atomic<Partial *> g_scratch_addr[kMaxDevices];
static std::atomic<unsigned long long> g_scratch_ctx[kMaxDevices];

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

// The unique ID of the calling thread's current context.  The two driver
// functions are found through the runtime (the library does not link the
// driver library itself, so it loads on machines without a GPU driver).
bool current_context_id(unsigned long long *id) {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static std::atomic<GetCurrent> get_current{nullptr};
  static std::atomic<GetId> get_id{nullptr};
  if (!get_current.load() || !get_id.load()) {
    void *a = nullptr, *b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b)
      return false;
    get_current.store(reinterpret_cast<GetCurrent>(a));
    get_id.store(reinterpret_cast<GetId>(b));
  }
  CUcontext ctx = nullptr;
  return get_current.load()(&ctx) == CUDA_SUCCESS && ctx &&
         get_id.load()(ctx, id) == CUDA_SUCCESS;
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
  const struct {
    const void *p;
    unsigned align;
    const char *name;
  } need[] = {{qold, 16, "qold"}, {q, 16, "q"},      {res, 16, "res"},      {adt, 8, "adt"},
              {rms, 8, "rms"},    {maxerr, 8, "maxerr"}, {errloc, 4, "errloc"}};
  for (const auto &a : need)
    if (reinterpret_cast<uintptr_t>(a.p) % a.align) {
      set_error("op2b_update_noalloc: %s = %p is not %u-byte aligned (the kernel accesses "
                "it in %u-byte units)",
                a.name, a.p, a.align, a.align);
      return -1;
    }
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "op2b_update_noalloc: cudaGetDevice")) return -1;
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("op2b_update_noalloc: device ordinal %d above %d", dev, kMaxDevices - 1);
    return -1;
  }
  // make the device's context current (created if this is the process's
  // first CUDA work on it) and read its unique ID
  if (!cuda_ok(cudaSetDevice(dev), "op2b_update_noalloc: cudaSetDevice")) return -1;
  unsigned long long ctx_id = 0;
  if (!current_context_id(&ctx_id)) {
    set_error("op2b_update_noalloc: no current CUDA context on device %d", dev);
    return -1;
  }
  Partial *scratch = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!scratch || g_scratch_ctx[dev].load(std::memory_order_acquire) != ctx_id) {
    // set-up, once per device and context, with the device current: resolve
    // the array's device address (host code may not use the symbol itself)
    Partial *ptr = nullptr;
    if (!cuda_ok(cudaGetSymbolAddress((void **)&ptr, g_update_scratch),
                 "op2b_update_noalloc: cudaGetSymbolAddress"))
      return -1;
    g_scratch_addr[dev].store(ptr, std::memory_order_release);
    g_scratch_ctx[dev].store(ctx_id, std::memory_order_release);
    scratch = ptr;
  }
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
