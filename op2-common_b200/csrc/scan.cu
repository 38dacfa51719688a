// Device scans for the setup code: a three-phase exclusive scan (per-block
// scans, a one-CTA scan of the block sums, the add-back) and the compaction of
// the nonzero positions of a count array built on it.  Internal to libop2b.
#include "scan.h"

namespace op2b {

__global__ void k_scan_blocks(const int *in, long long *out, long long n, long long *bsum) {
  __shared__ long long s[1024];
  long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  long long v = i < n ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    long long t = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == 1023) bsum[blockIdx.x] = s[1023];
}

// exclusive scan of the nb block sums by one CTA of 1024 threads: each thread
// sums a contiguous run, the runs' totals are scanned in shared memory, then
// each run is rewritten with its offsets; *total = the sum
__global__ void k_scan_bsum(long long *bsum, long long nb, long long *total) {
  __shared__ long long part[1024];
  const long long chunk = (nb + 1023) / 1024;
  const long long b0 = threadIdx.x * chunk, b1 = min(nb, b0 + chunk);
  long long acc = 0;
  for (long long b = b0; b < b1; b++) acc += bsum[b];
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    long long t = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += t;
    __syncthreads();
  }
  long long run = part[threadIdx.x] - acc;
  for (long long b = b0; b < b1; b++) {
    long long t = bsum[b];
    bsum[b] = run;
    run += t;
  }
  if (threadIdx.x == 1023) *total = part[1023];
}

__global__ void k_scan_add(long long *out, long long n, const long long *bsum) {
  long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += bsum[blockIdx.x];
}

long long scan_scratch_elems(long long n) { return (n + 1023) / 1024 + 1; }

bool scan_exclusive(const int *in, long long *out, long long n, cudaStream_t s,
                    long long *scratch) {
  long long nb = (n + 1023) / 1024;
  long long *bsum = scratch;
  if (!bsum && cudaMallocAsync(&bsum, sizeof(long long) * (nb + 1), s) != cudaSuccess)
    return false;
  if (nb > 0) {
    k_scan_blocks<<<(unsigned)nb, 1024, 0, s>>>(in, out, n, bsum);
    k_scan_bsum<<<1, 1024, 0, s>>>(bsum, nb, out + n);
    k_scan_add<<<(unsigned)nb, 1024, 0, s>>>(out, n, bsum);
  } else {
    cudaMemsetAsync(out, 0, sizeof(long long), s);
  }
  if (scratch) return cudaPeekAtLastError() == cudaSuccess;
  cudaFreeAsync(bsum, s);
  return cudaStreamSynchronize(s) == cudaSuccess;
}

__global__ void k_flag_nonzero(const int *cnt, int n, int *flag) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) flag[t] = cnt[t] > 0 ? 1 : 0;
}

__global__ void k_scatter_nonzero(const int *cnt, int n, const long long *pos, int *rows) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n && cnt[t] > 0) rows[pos[t]] = t;
}

bool compact_nonzero(const int *cnt, int n, int *rows, long long *pos, int *count,
                     cudaStream_t s) {
  int *flag = nullptr;
  if (cudaMallocAsync(&flag, sizeof(int) * ((size_t)n + 1), s) != cudaSuccess) return false;
  const unsigned g = (unsigned)((n + 255) / 256);
  if (n > 0) k_flag_nonzero<<<g, 256, 0, s>>>(cnt, n, flag);
  bool ok = scan_exclusive(flag, pos, n, s);
  if (ok && n > 0) k_scatter_nonzero<<<g, 256, 0, s>>>(cnt, n, pos, rows);
  long long total = 0;
  if (ok) cudaMemcpyAsync(&total, pos + n, sizeof(total), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(flag, s);
  ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
  *count = (int)total;
  return ok;
}

}  // namespace op2b
