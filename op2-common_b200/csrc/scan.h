// Device scans shared by the setup code (inverse maps, renumbering).
// Internal to libop2b.
#pragma once

#include <cuda_runtime.h>

namespace op2b {

// Exclusive scan of n ints into out[0..n] (out[n] = the total), on stream s.
// Asynchronous; uses a scratch of (n + 1023) / 1024 + 1 long longs that the
// caller provides (scan_scratch_elems), or allocates and frees one when
// scratch is null (then synchronous).
long long scan_scratch_elems(long long n);
bool scan_exclusive(const int *in, long long *out, long long n, cudaStream_t s,
                    long long *scratch = nullptr);

// rows[k] = the k-th index t (ascending) with cnt[t] > 0; *count (host) = how
// many.  pos is a scratch of n + 1 long longs.  Synchronous.
bool compact_nonzero(const int *cnt, int n, int *rows, long long *pos, int *count,
                     cudaStream_t s);

}  // namespace op2b
