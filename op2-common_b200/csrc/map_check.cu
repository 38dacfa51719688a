// Device-side range check of a declared map (op_decl_map): the map is
// uploaded straight from the caller's array and checked where it lands, so a
// large map costs one transfer and one pass over HBM instead of a host loop
// before a staged copy.  Internal to libop2b.
#include <cuda_runtime.h>

#include "loops.h"

namespace op2b {

// *first_bad = the lowest index i with map[i] outside [0, nto) (unchanged if none)
__global__ void k_map_check(const int *__restrict__ map, long long n, int nto,
                            unsigned long long *first_bad) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int v = __ldcs(map + i);
    if (v < 0 || v >= nto) {
      atomicMin(first_bad, (unsigned long long)i);
      return;  // later entries of this thread cannot be lower
    }
  }
}

cudaError_t launch_map_check(const LaunchCtx &c, const int *map, long long n, int nto,
                             unsigned long long *first_bad) {
  if (n <= 0) return cudaSuccess;
  long long want = (n + 255) / 256, cap = (long long)c.nsm * 8;
  k_map_check<<<(unsigned)(want < cap ? want : cap), 256, 0, c.stream>>>(map, n, nto, first_bad);
  c.count();
  return cudaGetLastError();
}

}  // namespace op2b
