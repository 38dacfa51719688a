// Halo packing for the partitioned single mesh: the device side of the
// reference's halo exchange (op2/src/mpi/op_mpi_rt_support.cpp:61-200,
// op_exchange_halo; its CUDA kernels export_halo_gather and
// import_halo_scatter, op2/src/mpi/op_mpi_cuda_kernels.cu:44-136).
//
// A partition's cells are its owned cells followed by its import halo,
// grouped by the rank that owns them, so what a neighbour sends lands in one
// contiguous slice of rows.  op2b_dat_pack gathers the rows of an export
// list into a contiguous buffer; op2b_dat_unpack writes a buffer into rows
// (a contiguous slice, or scattered by a list).  Listed rows outside the set
// are skipped, never accessed.  Rows are copied as 16-, 8-
// or 4-byte words, whichever the row size and the addresses allow.  Both run
// on the library's stream, after the runtime has settled any deferred or
// speculative work on the dat (they read and write it like a loop would).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "op2b.h"
#include "op2b_runtime.h"

namespace op2b {
namespace {

// a row outside [0, nrows) is skipped (its buffer row is left as it was)
template <typename W>
__global__ void k_pack_rows(const W *__restrict__ src, int nrows, const int *__restrict__ rows,
                            int n, int words, W *__restrict__ dst) {
  const long long total = (long long)n * words;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / words), w = (int)(i - (long long)r * words);
    const int row = rows[r];
    if (row >= 0 && row < nrows) dst[i] = src[(size_t)row * words + w];
  }
}

// a row outside [0, nrows) is skipped
template <typename W>
__global__ void k_unpack_rows(W *__restrict__ dst, int nrows, const int *__restrict__ rows,
                              int first, int n, int words, const W *__restrict__ src) {
  const long long total = (long long)n * words;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / words), w = (int)(i - (long long)r * words);
    const long long row = rows ? (long long)rows[r] : (long long)first + r;
    if (row >= 0 && row < nrows) dst[row * words + w] = src[i];
  }
}

int word_bytes(const void *a, const void *b, int row_bytes) {
  const uintptr_t m = reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b);
  if (row_bytes % 16 == 0 && m % 16 == 0) return 16;
  if (row_bytes % 8 == 0 && m % 8 == 0) return 8;
  return 4;
}

bool check(const char *what, op_dat dat, int n, const void *buf) {
  if (!dat || n < 0 || (n > 0 && !buf)) {
    set_error("%s: invalid dat, count or buffer", what);
    return false;
  }
  if (dat->size % 4) {
    set_error("%s: rows of %d bytes (a multiple of 4 is needed)", what, dat->size);
    return false;
  }
  return true;
}

}  // namespace
}  // namespace op2b

using namespace op2b;

extern "C" int op2b_dat_pack(op_dat dat, const int *rows, int n, void *buf) {
  Runtime &r = rt();
  if (!r.ready() || !check("op2b_dat_pack", dat, n, buf)) return -1;
  if (n == 0) return 0;
  if (!rows) {
    set_error("op2b_dat_pack: the row list is null");
    return -1;
  }
  const int wb = word_bytes(dat->data_d, buf, dat->size), words = dat->size / wb;
  const long long total = (long long)n * words;
  const unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, (long long)r.nsm * 8);
  if (wb == 16)
    k_pack_rows<uint4><<<grid, 256, 0, r.stream>>>((const uint4 *)dat->data_d, dat->set->size, rows, n, words,
                                                   (uint4 *)buf);
  else if (wb == 8)
    k_pack_rows<uint2><<<grid, 256, 0, r.stream>>>((const uint2 *)dat->data_d, dat->set->size, rows, n, words,
                                                   (uint2 *)buf);
  else
    k_pack_rows<unsigned><<<grid, 256, 0, r.stream>>>((const unsigned *)dat->data_d, dat->set->size,
                                                      rows, n, words, (unsigned *)buf);
  r.launches++;
  return cuda_ok(cudaGetLastError(), "op2b_dat_pack") ? 0 : -1;
}

extern "C" int op2b_dat_unpack(op_dat dat, const int *rows, int first, int n, const void *buf) {
  Runtime &r = rt();
  if (!r.ready() || !check("op2b_dat_unpack", dat, n, buf)) return -1;
  if (n == 0) return 0;
  if (!rows && (first < 0 || (long long)first + n > dat->set->size)) {
    set_error("op2b_dat_unpack: rows [%d, %lld) outside the set of %d", first,
              (long long)first + n, dat->set->size);
    return -1;
  }
  const int wb = word_bytes(dat->data_d, buf, dat->size), words = dat->size / wb;
  const long long total = (long long)n * words;
  const unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, (long long)r.nsm * 8);
  if (wb == 16)
    k_unpack_rows<uint4><<<grid, 256, 0, r.stream>>>((uint4 *)dat->data_d, dat->set->size, rows, first, n, words,
                                                     (const uint4 *)buf);
  else if (wb == 8)
    k_unpack_rows<uint2><<<grid, 256, 0, r.stream>>>((uint2 *)dat->data_d, dat->set->size, rows, first, n, words,
                                                     (const uint2 *)buf);
  else
    k_unpack_rows<unsigned><<<grid, 256, 0, r.stream>>>((unsigned *)dat->data_d, dat->set->size,
                                                        rows, first, n, words, (const unsigned *)buf);
  r.launches++;
  return cuda_ok(cudaGetLastError(), "op2b_dat_unpack") ? 0 : -1;
}
