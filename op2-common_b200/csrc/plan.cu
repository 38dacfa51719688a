// Execution plans built on the GPU: the op_plan_core of the reference
// (op2/src/core/op_rt_support.cpp:301-1126) re-designed as device kernels.
//
//   1. block partition: blocks of bsize elements (single rank: core = size)
//      -- :364-450 (bsize default MAX((24K/(64*maxbytes))*64, 256), :373-378)
//   2. per block and indirection: the referenced elements, sorted and made
//      unique (bitonic sort + scan in shared memory, one CTA per block) ->
//      ind_maps / ind_offs / ind_sizes; loc_maps by binary search -- :609-682
//   3. per block, greedy thread colouring in element order with 32-colour
//      passes over the targets of OP_INC/OP_RW arguments -- :684-754 (one
//      thread per block walks the block's elements; bitmasks in shared memory)
//   4. greedy block colouring in block order, 32-colour passes -- :798-884.
//      The sequence is inherently serial; one CTA walks the blocks, its
//      threads OR-reducing a block's mask in parallel -> bit-exact blk_col
//   5. ncolblk, blkmap (blocks grouped by colour, in block order) -- :886-922
//   6. shared-memory sizes per colour (:926-967); element permutation by
//      colour for OP_STAGE_PERMUTE / OP_COLOR2 (:756-796)
// Validation (op2b_plan_validate) re-checks the invariants of op_plan_check
// (:129-295) on the device and adds the colour checks the reference leaves
// empty: no two elements of a thread colour in a block, and no two blocks of
// a block colour, touch the same OP_INC/OP_RW target.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "op2b_plan.h"
#include "op2b_runtime.h"
#include "plan.h"

namespace op2b {

#define PLAN_MAX_ARGS 16
#define PLAN_MAX_INDS 8
#define PLAN_THREADS 256
#define PLAN_MAX_PART 4096

struct PlanParams {
  int nargs, ninds, nst;
  int exec_length, bsize, nblocks;
  const int *map[PLAN_MAX_ARGS];
  int mdim[PLAN_MAX_ARGS], idx[PLAN_MAX_ARGS], ind[PLAN_MAX_ARGS], incrw[PLAN_MAX_ARGS];
  int loc_slot[PLAN_MAX_ARGS];     // loc_map output slot of a staged arg, -1 otherwise
  int ind_nargs[PLAN_MAX_INDS];    // args using each indirection
  int ind_needed[PLAN_MAX_INDS];   // local numbering needed (staged or INC/RW)
  int ind_slot[PLAN_MAX_INDS];     // staged number of the indirection, -1 otherwise
  int ind_incrw[PLAN_MAX_INDS];    // some OP_INC/OP_RW arg uses it
  int ind_work_off[PLAN_MAX_INDS]; // offset of its colour bitmasks in shared memory
  int ind_to_size[PLAN_MAX_INDS];  // size of the target set
  int incrw_loc_off[PLAN_MAX_ARGS];// offset of an INC/RW arg's local indices in smem
  int buf_len;                     // power of two >= max gathered values of one indirection
  int work_len, loc_len;
  int jp;                          // Jones-Plassmann colouring instead of the serial greedy
};

// ------------------------------------------------------------------ helpers

__device__ void bitonic_sort(int *v, int n) {
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int ixj = i ^ j;
        if (ixj > i) {
          int a = v[i], b = v[ixj];
          bool up = (i & k) == 0;
          if ((a > b) == up) {
            v[i] = b;
            v[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Exclusive scan of flag[i] in [0, n) (n <= blockDim*chunks); returns total.
__device__ int block_exclusive_scan(const int *flag, int *pos, int n, int *s_tmp) {
  int T = blockDim.x;
  int chunk = (n + T - 1) / T;
  int beg = threadIdx.x * chunk, end = min(beg + chunk, n);
  int sum = 0;
  for (int i = beg; i < end; i++) sum += flag[i];
  // inclusive scan of per-thread sums
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int v = sum;
  for (int o = 1; o < 32; o <<= 1) {
    int u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) s_tmp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    int nw = (T + 31) >> 5;
    int w = lane < nw ? s_tmp[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int u = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += u;
    }
    if (lane < nw) s_tmp[lane] = w;
  }
  __syncthreads();
  int excl = v - sum + (warp > 0 ? s_tmp[warp - 1] : 0);
  int total = s_tmp[((T + 31) >> 5) - 1];
  for (int i = beg; i < end; i++) {
    pos[i] = excl;
    excl += flag[i];
  }
  __syncthreads();
  return total;
}

__device__ __forceinline__ void block_range(const PlanParams &p, int b, int &beg, int &n) {
  beg = b * p.bsize;
  n = min(p.bsize, p.exec_length - beg);
}

// Gather the targets of every arg using indirection m for the block's
// elements (arg order, then element order, as :615-621), pad, sort.
__device__ int gather_sorted(const PlanParams &p, int m, int beg, int n, int *buf) {
  int cnt = p.ind_nargs[m] * n;
  int pad = 1;
  while (pad < cnt) pad <<= 1;
  int k = 0;
  for (int a = 0; a < p.nargs; a++) {
    if (p.ind[a] != m) continue;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      buf[k * n + i] = p.map[a][p.idx[a] + (size_t)(beg + i) * p.mdim[a]];
    k++;
  }
  for (int i = cnt + threadIdx.x; i < pad; i += blockDim.x) buf[i] = INT_MAX;
  __syncthreads();
  bitonic_sort(buf, pad);
  return cnt;
}

// ------------------------------------------------------------------ kernel 1
// number of distinct targets per (block, needed indirection)
__global__ void k_plan_count(PlanParams p, int *counts) {
  extern __shared__ int sm[];
  int *buf = sm;
  int *flag = buf + p.buf_len;
  int *pos = flag + p.buf_len;
  __shared__ int s_tmp[32];
  int b = blockIdx.x, beg, n;
  block_range(p, b, beg, n);
  for (int m = 0; m < p.ninds; m++) {
    if (!p.ind_needed[m]) continue;
    int cnt = gather_sorted(p, m, beg, n, buf);
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) flag[i] = (i == 0 || buf[i] != buf[i - 1]);
    __syncthreads();
    int total = block_exclusive_scan(flag, pos, cnt, s_tmp);
    if (threadIdx.x == 0) counts[(size_t)b * p.ninds + m] = total;
    __syncthreads();
  }
}

// ------------------------------------------------------------------ Jones-Plassmann
// Parallel colouring, the alternative to the reference's serial greedy order
// (which the default plans keep, bit-exact).  Each round, every uncoloured
// element (or block) that holds the highest priority among the uncoloured
// ones sharing any of its OP_INC/OP_RW targets takes the lowest colour its
// already-coloured neighbours leave free; two winners of a round never share
// a target, so a round's choices cannot conflict.  Priorities are a hash of
// the index with the index as tie-break (unique, deterministic: the colouring
// is the same on every run).  Colours come 32 at a time, as in the greedy
// passes: a candidate whose neighbours hold all 32 colours of the pass waits
// for the next pass.  The result is checked like any plan by
// op2b_plan_validate (no two elements of a colour share a target).

__device__ __forceinline__ unsigned jp_hash(unsigned x) {
  // an integer mixing function (xorshift-multiply rounds)
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

__device__ __forceinline__ unsigned long long jp_prio(long long i) {
  return ((unsigned long long)jp_hash((unsigned)i ^ (unsigned)(i >> 32)) << 32) |
         (unsigned long long)(unsigned)(i + 1);
}

// thread colours of one block by CTA-parallel Jones-Plassmann in shared
// memory: work[] the colour masks of the block's local targets, tmax[] (as
// many ints) the round's highest priority per local target; up to 16
// elements per thread (blocks of at most 4096 elements)
__device__ void jp_thread_colours(const PlanParams &p, int b, int beg, int n, unsigned *work,
                                  const short *loc, int *tmax, int *thrcol, int *nthrcol) {
  __shared__ int s_ncolors;
  const int T = blockDim.x;
  for (int i = threadIdx.x; i < n; i += T) thrcol[beg + i] = -1;
  if (threadIdx.x == 0) s_ncolors = 0;
  // priorities below 2^31 (21 hash bits above the 12 index bits), unique in the block
  auto prio = [&](int i) { return (int)(((jp_hash((unsigned)(beg + i)) & 0x7ffffu) << 12) | i); };
  int base = 0;
  unsigned blocked = 0;  // per thread: bit k = its k-th element waits for the next pass
  for (;;) {
    for (int t = threadIdx.x; t < p.work_len; t += T) work[t] = 0u;
    blocked = 0;
    __syncthreads();
    for (;;) {
      for (int t = threadIdx.x; t < p.work_len; t += T) tmax[t] = -1;
      __syncthreads();
      for (int i = threadIdx.x, k = 0; i < n; i += T, k++) {
        if (thrcol[beg + i] != -1 || (blocked >> k & 1u)) continue;
        const int pr = prio(i);
        for (int a = 0; a < p.nargs; a++)
          if (p.incrw[a]) atomicMax(&tmax[p.ind_work_off[p.ind[a]] + loc[p.incrw_loc_off[a] + i]], pr);
      }
      __syncthreads();
      int active = 0;
      for (int i = threadIdx.x, k = 0; i < n; i += T, k++) {
        if (thrcol[beg + i] != -1 || (blocked >> k & 1u)) continue;
        const int pr = prio(i);
        bool win = true;
        unsigned mask = 0;
        for (int a = 0; a < p.nargs; a++)
          if (p.incrw[a]) {
            const int t = p.ind_work_off[p.ind[a]] + loc[p.incrw_loc_off[a] + i];
            win &= tmax[t] == pr;
            mask |= work[t];
          }
        if (!win) {
          active = 1;
          continue;
        }
        const int c = __ffs(~mask) - 1;
        if (c < 0) {
          blocked |= 1u << k;
          continue;
        }
        thrcol[beg + i] = base + c;
        atomicMax(&s_ncolors, base + c + 1);
        for (int a = 0; a < p.nargs; a++)
          if (p.incrw[a])
            atomicOr(&work[p.ind_work_off[p.ind[a]] + loc[p.incrw_loc_off[a] + i]], 1u << c);
      }
      if (!__syncthreads_or(active)) break;
    }
    if (!__syncthreads_or(blocked != 0)) break;
    base += 32;
  }
  if (threadIdx.x == 0) nthrcol[b] = s_ncolors;
}

// device-wide rounds over blocks (CTA b stands for plan block b) or over
// single elements (OP_COLOR2): the round's highest priority per target ...
__global__ void k_jp_block_max(PlanParams p, unsigned long long *const *tmax, const int *col,
                               const unsigned char *blocked) {
  const int b = blockIdx.x;
  if (col[b] != -1 || blocked[b]) return;
  int beg, n;
  block_range(p, b, beg, n);
  const unsigned long long pr = jp_prio(b);
  for (int a = 0; a < p.nargs; a++) {
    if (!p.incrw[a]) continue;
    unsigned long long *tm = tmax[p.ind[a]];
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      atomicMax(&tm[p.map[a][p.idx[a] + (size_t)(beg + i) * p.mdim[a]]], pr);
  }
}

// ... then each winner's colour; *active counts the candidates left waiting,
// *nblocked those that found the pass's 32 colours taken
__global__ void k_jp_block_win(PlanParams p, unsigned long long *const *tmax, unsigned *const *work,
                               int *col, unsigned char *blocked, int base, int *active,
                               int *nblocked, int *ncolors) {
  __shared__ unsigned s_or[32];
  const int b = blockIdx.x;
  if (col[b] != -1 || blocked[b]) return;
  int beg, n;
  block_range(p, b, beg, n);
  const unsigned long long pr = jp_prio(b);
  int lose = 0;
  unsigned mask = 0;
  for (int a = 0; a < p.nargs; a++) {
    if (!p.incrw[a]) continue;
    const unsigned long long *tm = tmax[p.ind[a]];
    const unsigned *w = work[p.ind[a]];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int t = p.map[a][p.idx[a] + (size_t)(beg + i) * p.mdim[a]];
      lose |= tm[t] != pr;
      mask |= w[t];
    }
  }
  if (__syncthreads_or(lose)) {
    if (threadIdx.x == 0) atomicAdd(active, 1);
    return;
  }
  mask = __reduce_or_sync(0xffffffffu, mask);
  if ((threadIdx.x & 31) == 0) s_or[threadIdx.x >> 5] = mask;
  __syncthreads();
  unsigned all = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) all |= s_or[w];
  const int c = __ffs(~all) - 1;
  if (c < 0) {
    if (threadIdx.x == 0) {
      blocked[b] = 1;
      atomicAdd(nblocked, 1);
    }
    return;
  }
  if (threadIdx.x == 0) {
    col[b] = base + c;
    atomicMax(ncolors, base + c + 1);
  }
  for (int a = 0; a < p.nargs; a++) {
    if (!p.incrw[a]) continue;
    unsigned *w = work[p.ind[a]];
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      atomicOr(&w[p.map[a][p.idx[a] + (size_t)(beg + i) * p.mdim[a]]], 1u << c);
  }
}

__global__ void k_jp_elem_max(PlanParams p, unsigned long long *const *tmax, const int *col,
                              const unsigned char *blocked) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < p.exec_length;
       e += gridDim.x * blockDim.x) {
    if (col[e] != -1 || blocked[e]) continue;
    const unsigned long long pr = jp_prio(e);
    for (int a = 0; a < p.nargs; a++)
      if (p.incrw[a]) atomicMax(&tmax[p.ind[a]][p.map[a][p.idx[a] + (size_t)e * p.mdim[a]]], pr);
  }
}

__global__ void k_jp_elem_win(PlanParams p, unsigned long long *const *tmax, unsigned *const *work,
                              int *col, unsigned char *blocked, int base, int *active,
                              int *nblocked, int *ncolors) {
  int act = 0, blk = 0, nc = 0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < p.exec_length;
       e += gridDim.x * blockDim.x) {
    if (col[e] != -1 || blocked[e]) continue;
    const unsigned long long pr = jp_prio(e);
    bool win = true;
    unsigned mask = 0;
    for (int a = 0; a < p.nargs; a++)
      if (p.incrw[a]) {
        const int t = p.map[a][p.idx[a] + (size_t)e * p.mdim[a]];
        win &= tmax[p.ind[a]][t] == pr;
        mask |= work[p.ind[a]][t];
      }
    if (!win) {
      act++;
      continue;
    }
    const int c = __ffs(~mask) - 1;
    if (c < 0) {
      blocked[e] = 1;
      blk++;
      continue;
    }
    col[e] = base + c;
    nc = max(nc, base + c + 1);
    for (int a = 0; a < p.nargs; a++)
      if (p.incrw[a]) atomicOr(&work[p.ind[a]][p.map[a][p.idx[a] + (size_t)e * p.mdim[a]]], 1u << c);
  }
  if (act) atomicAdd(active, act);
  if (blk) atomicAdd(nblocked, blk);
  if (nc) atomicMax(ncolors, nc);
}

// ------------------------------------------------------------------ kernel 2
// ind_maps + loc_maps (staged indirections) and the block's thread colours
__global__ void k_plan_fill(PlanParams p, const long long *ind_base, const int *ind_offs,
                            int *ind_map, short *loc_map, int *thrcol, int *nthrcol,
                            int *err) {
  extern __shared__ int sm[];
  int *buf = sm;
  int *flag = buf + p.buf_len;
  int *pos = flag + p.buf_len;
  unsigned *work = reinterpret_cast<unsigned *>(pos + p.buf_len);
  short *loc = reinterpret_cast<short *>(work + p.work_len);
  __shared__ int s_tmp[32];
  int b = blockIdx.x, beg, n;
  block_range(p, b, beg, n);
  for (int m = 0; m < p.ninds; m++) {
    if (!p.ind_needed[m]) continue;
    int cnt = gather_sorted(p, m, beg, n, buf);
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) flag[i] = (i == 0 || buf[i] != buf[i - 1]);
    __syncthreads();
    int total = block_exclusive_scan(flag, pos, cnt, s_tmp);
    // compact the distinct targets into flag[] (no longer needed as flags)
    for (int i = threadIdx.x; i < cnt; i += blockDim.x)
      if (i == 0 || buf[i] != buf[i - 1]) flag[pos[i]] = buf[i];
    __syncthreads();
    int *uniq = flag;
    int slot = p.ind_slot[m];
    if (slot >= 0) {
      long long o = ind_base[slot] + ind_offs[(size_t)b * p.nst + slot];
      for (int i = threadIdx.x; i < total; i += blockDim.x) ind_map[o + i] = uniq[i];
    }
    // local index of every (arg, element) of this indirection
    for (int a = 0; a < p.nargs; a++) {
      if (p.ind[a] != m) continue;
      bool need = p.loc_slot[a] >= 0 || p.incrw[a];
      if (!need) continue;
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int v = p.map[a][p.idx[a] + (size_t)(beg + i) * p.mdim[a]];
        int lo = 0, hi = total - 1;
        while (lo < hi) {
          int mid = (lo + hi) >> 1;
          if (uniq[mid] < v) lo = mid + 1;
          else hi = mid;
        }
        if (uniq[lo] != v || lo > 32767) atomicAdd(err, 1);
        if (p.loc_slot[a] >= 0) loc_map[(size_t)p.loc_slot[a] * p.exec_length + beg + i] = (short)lo;
        if (p.incrw[a]) loc[p.incrw_loc_off[a] + i] = (short)lo;
      }
    }
    __syncthreads();
  }
  if (p.jp) {
    jp_thread_colours(p, b, beg, n, work, loc, reinterpret_cast<int *>(loc) + (p.loc_len + 1) / 2,
                      thrcol, nthrcol);
    return;
  }
  // greedy thread colouring (:684-754): elements in order, 32 colours a pass
  if (threadIdx.x == 0) {
    for (int i = 0; i < n; i++) thrcol[beg + i] = -1;
    int ncolor = 0, ncolors = 0, repeat = 1;
    while (repeat) {
      repeat = 0;
      for (int i = 0; i < p.work_len; i++) work[i] = 0u;
      for (int i = 0; i < n; i++) {
        if (thrcol[beg + i] != -1) continue;
        unsigned mask = 0;
        for (int a = 0; a < p.nargs; a++)
          if (p.incrw[a]) mask |= work[p.ind_work_off[p.ind[a]] + loc[p.incrw_loc_off[a] + i]];
        int color = __ffs(~mask) - 1;
        if (color == -1) {
          repeat = 1;
        } else {
          thrcol[beg + i] = ncolor + color;
          ncolors = max(ncolors, ncolor + color + 1);
          unsigned bit = 1u << color;
          for (int a = 0; a < p.nargs; a++)
            if (p.incrw[a]) work[p.ind_work_off[p.ind[a]] + loc[p.incrw_loc_off[a] + i]] |= bit;
        }
      }
      ncolor += 32;
    }
    nthrcol[b] = ncolors;
  }
}

// ------------------------------------------------------------------ kernel 3
// greedy block colouring in block order (:798-884) by one CTA, then
// ncolblk and blkmap (:886-922).  work: one bitmask per target element of
// every OP_INC/OP_RW indirection.
__global__ void __launch_bounds__(1024)
k_block_colour_serial(PlanParams p, unsigned *const *work, int *blk_col, int *ncolblk,
                      int *blkmap, int *ncolors_out) {
  __shared__ unsigned s_or[32];
  __shared__ int s_color, s_repeat, s_ncolors, s_skip;
  int ncolor = 0;
  if (threadIdx.x == 0) {
    s_repeat = 1;
    s_ncolors = 0;
  }
  for (int b = threadIdx.x; b < p.nblocks; b += blockDim.x) blk_col[b] = -1;
  __syncthreads();
  while (s_repeat) {
    __syncthreads();
    if (threadIdx.x == 0) s_repeat = 0;
    for (int m = 0; m < p.ninds; m++)
      if (p.ind_incrw[m])
        for (int i = threadIdx.x; i < p.ind_to_size[m]; i += blockDim.x) work[m][i] = 0u;
    __syncthreads();
    for (int b = 0; b < p.nblocks; b++) {
      if (threadIdx.x == 0) s_skip = (blk_col[b] != -1);
      __syncthreads();
      if (s_skip) {
        __syncthreads();
        continue;
      }
      int beg, n;
      block_range(p, b, beg, n);
      unsigned mask = 0;
      for (int a = 0; a < p.nargs; a++) {
        if (!p.incrw[a]) continue;
        const unsigned *w = work[p.ind[a]];
        for (int i = threadIdx.x; i < n; i += blockDim.x)
          mask |= w[p.map[a][p.idx[a] + (size_t)(beg + i) * p.mdim[a]]];
      }
      mask = __reduce_or_sync(0xffffffffu, mask);
      if ((threadIdx.x & 31) == 0) s_or[threadIdx.x >> 5] = mask;
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned mm = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) mm |= s_or[w];
        int color = __ffs(~mm) - 1;
        if (color == -1) {
          s_repeat = 1;
        } else {
          blk_col[b] = ncolor + color;
          s_ncolors = max(s_ncolors, ncolor + color + 1);
        }
        s_color = color;
      }
      __syncthreads();
      if (s_color >= 0) {
        unsigned bit = 1u << s_color;
        for (int a = 0; a < p.nargs; a++) {
          if (!p.incrw[a]) continue;
          unsigned *w = work[p.ind[a]];
          for (int i = threadIdx.x; i < n; i += blockDim.x)
            atomicOr(&w[p.map[a][p.idx[a] + (size_t)(beg + i) * p.mdim[a]]], bit);
        }
      }
      __syncthreads();
    }
    ncolor += 32;
    __syncthreads();
  }
  // ncolblk and blkmap: blocks grouped by colour, each group in block order
  if (threadIdx.x == 0) {
    int nc = s_ncolors;
    *ncolors_out = nc;
    for (int c = 0; c < nc; c++) ncolblk[c] = 0;
    for (int b = 0; b < p.nblocks; b++) ncolblk[blk_col[b]]++;
    int acc = 0;
    for (int c = 0; c < nc; c++) {  // ncolblk temporarily holds exclusive starts
      int t = ncolblk[c];
      ncolblk[c] = acc;
      acc += t;
    }
    for (int b = 0; b < p.nblocks; b++) blkmap[ncolblk[blk_col[b]]++] = b;
    for (int c = nc - 1; c > 0; c--) ncolblk[c] -= ncolblk[c - 1];
  }
}

// shared memory per block (:926-967): sum of staged lists rounded up to 64 B
__global__ void k_plan_shared(PlanParams p, const int *ind_sizes, const int *dat_size,
                              const int *blk_col, int *nsharedCol, int *nshared) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= p.nblocks) return;
  int nbytes = 0;
  for (int s = 0; s < p.nst; s++)
    nbytes += ((ind_sizes[(size_t)b * p.nst + s] * dat_size[s]) + 63) & ~63;
  atomicMax(&nsharedCol[blk_col[b]], nbytes);
  atomicMax(nshared, nbytes);
}

// element permutation by thread colour within each block (:756-796);
// elements of equal colour keep their order
__global__ void k_plan_permute(PlanParams p, int *thrcol, const int *nthrcol,
                               const long long *coloff_base, int *col_reord, int *col_offsets) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= p.nblocks) return;
  int beg, n;
  block_range(p, b, beg, n);
  int nc = nthrcol[b];
  int *off = col_offsets + coloff_base[b];
  for (int c = 0; c <= nc; c++) off[c] = 0;
  for (int i = 0; i < n; i++) off[thrcol[beg + i] + 1]++;
  for (int c = 1; c <= nc; c++) off[c] += off[c - 1];
  // stable placement: position = start of colour + rank within colour
  for (int c = 0; c < nc; c++) {
    int k = off[c];
    for (int i = 0; i < n; i++)
      if (thrcol[beg + i] == c) col_reord[beg + k++] = i;
  }
  for (int i = 0; i < n; i++) thrcol[beg + i] = 0;
  for (int c = 0; c < nc; c++)
    for (int i = off[c]; i < off[c + 1]; i++) thrcol[beg + i] = c;
}

// flat element colouring of OP_COLOR2 (one block = the whole set, :684-754
// with bsize = exec_length): one device thread walks the set.
__global__ void k_color2_serial(PlanParams p, unsigned *const *work, int *thrcol, int *nthrcol) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int n = p.exec_length;
  for (int i = 0; i < n; i++) thrcol[i] = -1;
  int ncolor = 0, ncolors = 0, repeat = 1;
  while (repeat) {
    repeat = 0;
    for (int m = 0; m < p.ninds; m++)
      if (p.ind_incrw[m])
        for (int i = 0; i < p.ind_to_size[m]; i++) work[m][i] = 0u;
    for (int e = 0; e < n; e++) {
      if (thrcol[e] != -1) continue;
      unsigned mask = 0;
      for (int a = 0; a < p.nargs; a++)
        if (p.incrw[a]) mask |= work[p.ind[a]][p.map[a][p.idx[a] + (size_t)e * p.mdim[a]]];
      int color = __ffs(~mask) - 1;
      if (color == -1) {
        repeat = 1;
      } else {
        thrcol[e] = ncolor + color;
        ncolors = max(ncolors, ncolor + color + 1);
        for (int a = 0; a < p.nargs; a++)
          if (p.incrw[a]) work[p.ind[a]][p.map[a][p.idx[a] + (size_t)e * p.mdim[a]]] |= 1u << color;
      }
    }
    ncolor += 32;
  }
  nthrcol[0] = ncolors;
}

// ------------------------------------------------------------------ validation kernels

// op_plan_check ind_maps (:216-243): strictly increasing within a block, in range
__global__ void k_check_ind_maps(int nblocks, int nst, int slot, const int *ind_sizes,
                                 const int *ind_offs, const int *ind_map_s, int to_size,
                                 unsigned long long *err) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  int o = ind_offs[(size_t)b * nst + slot], s = ind_sizes[(size_t)b * nst + slot];
  int e = 0, last = -1;
  for (int i = 0; i < s; i++) {
    int v = ind_map_s[o + i];
    e += (v <= last) || v < 0;
    last = v;
  }
  e += (last >= to_size);
  if (e) atomicAdd(err, (unsigned long long)e);
}

// op_plan_check maps (:249-270): ind_map[loc_map[e] + ind_offs] == map value
__global__ void k_check_loc_maps(PlanParams p, int a, const short *loc, const int *ind_map_s,
                                 const int *ind_offs, unsigned long long *err) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= p.exec_length) return;
  int b = e / p.bsize;
  int slot = p.ind_slot[p.ind[a]];
  int g = ind_map_s[ind_offs[(size_t)b * p.nst + slot] + loc[e]];
  if (g != p.map[a][p.idx[a] + (size_t)e * p.mdim[a]]) atomicAdd(err, 1ull);
}

// thread colours: within a block no two elements of one colour share a
// target.  Sort (indirection, target, colour, element) keys; equal leading
// fields with different elements is a conflict.
__global__ void k_check_thread_colours(PlanParams p, const int *thrcol, unsigned long long *err) {
  extern __shared__ unsigned long long keys[];
  int b = blockIdx.x, beg, n;
  block_range(p, b, beg, n);
  int cnt = 0;
  for (int a = 0; a < p.nargs; a++)
    if (p.incrw[a]) cnt += n;
  int pad = 1;
  while (pad < cnt) pad <<= 1;
  int k = 0;
  for (int a = 0; a < p.nargs; a++) {
    if (!p.incrw[a]) continue;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      unsigned long long t = (unsigned)p.map[a][p.idx[a] + (size_t)(beg + i) * p.mdim[a]];
      unsigned long long c = (unsigned)thrcol[beg + i] & 0xfffu;
      keys[k * n + i] = ((unsigned long long)p.ind[a] << 60) | (t << 28) | (c << 16) |
                        (unsigned long long)i;
    }
    k++;
  }
  for (int i = cnt + threadIdx.x; i < pad; i += blockDim.x) keys[i] = ~0ull;
  __syncthreads();
  for (int kk = 2; kk <= pad; kk <<= 1)
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < pad; i += blockDim.x) {
        int ixj = i ^ j;
        if (ixj > i) {
          unsigned long long x = keys[i], y = keys[ixj];
          bool up = (i & kk) == 0;
          if ((x > y) == up) {
            keys[i] = y;
            keys[ixj] = x;
          }
        }
      }
      __syncthreads();
    }
  for (int i = 1 + threadIdx.x; i < cnt; i += blockDim.x) {
    unsigned long long x = keys[i - 1], y = keys[i];
    if ((x >> 16) == (y >> 16) && (x & 0xffffu) != (y & 0xffffu)) atomicAdd(err, 1ull);
  }
}

// block colours: blocks of colour c (one launch per colour) claim each
// target with atomicMax of (c+1, block); meeting another block of the same
// colour is a conflict.  Earlier colours hold smaller keys.
__global__ void k_check_block_colour(PlanParams p, int c, const int *blkmap, int first,
                                     int count, unsigned long long *const *owner,
                                     unsigned long long *err) {
  int j = blockIdx.x;
  if (j >= count) return;
  int b = blkmap[first + j];
  int beg, n;
  block_range(p, b, beg, n);
  unsigned long long key = ((unsigned long long)(c + 1) << 32) | (unsigned)b;
  for (int a = 0; a < p.nargs; a++) {
    if (!p.incrw[a]) continue;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int t = p.map[a][p.idx[a] + (size_t)(beg + i) * p.mdim[a]];
      unsigned long long old = atomicMax(&owner[p.ind[a]][t], key);
      if ((old >> 32) == (unsigned long long)(c + 1) && (unsigned)(old & 0xffffffffu) != (unsigned)b)
        atomicAdd(err, 1ull);
    }
  }
}

// ------------------------------------------------------------------ host side

static std::vector<std::unique_ptr<Plan>> &plan_cache() {
  static std::vector<std::unique_ptr<Plan>> v;
  return v;
}

template <typename T> static T *dalloc(size_t n, std::vector<void *> &owned) {
  void *p = nullptr;
  if (n == 0) n = 1;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
  owned.push_back(p);
  return static_cast<T *>(p);
}

Plan::~Plan() {
  for (void *p : owned) cudaFree(p);
}

static bool same_args(const Plan &pl, int nargs, const op_arg *args) {
  for (int m = 0; m < nargs; m++) {
    if (args[m].dat && pl.dats[m]) {
      if (args[m].dat->size != pl.dats[m]->size || args[m].dat->dim != pl.dats[m]->dim)
        return false;
    } else if (args[m].dat != pl.dats[m]) {
      return false;
    }
    if (args[m].map != pl.maps[m] || args[m].idx != pl.idxs[m] || args[m].acc != pl.accs[m])
      return false;
  }
  return true;
}

static void host_transfer(Plan &pl, const PlanParams &p, const op_arg *args, const int *inds) {
  // op_rt_support.cpp:969-1080 in its order of float additions
  op_plan &o = pl.pub;
  o.transfer = 0.f;
  o.transfer2 = 0.f;
  if (pl.staging == OP_COLOR2 || pl.staging == OP_STAGE_INC) return;
  int cl = rt().opt_cache_line > 0 ? rt().opt_cache_line : 128;
  for (int b = 0; b < o.nblocks; b++) {
    for (int m = 0; m < pl.nargs; m++) {
      if (!args[m].opt) continue;
      if (inds[m] < 0) {
        float fac = (pl.accs[m] == OP_READ || pl.accs[m] == OP_WRITE) ? 1.0f : 2.0f;
        if (pl.dats[m]) {
          o.transfer += fac * o.nelems[b] * pl.dats[m]->size;
          o.transfer2 += fac * o.nelems[b] * pl.dats[m]->size;
        }
      } else {
        o.transfer += o.nelems[b] * sizeof(short);
        o.transfer2 += o.nelems[b] * sizeof(short);
      }
    }
    for (int m = 0; m < pl.ninds; m++) {
      int m2 = 0;
      while (inds[m2] != m) m2++;
      if (!args[m2].opt) continue;
      float fac = (pl.accs[m2] == OP_READ || pl.accs[m2] == OP_WRITE) ? 1.0f : 2.0f;
      int sl = p.ind_slot[m];
      int sz = o.ind_sizes[m + b * pl.ninds];
      o.transfer += fac * sz * pl.dats[m2]->size;
      int e0 = o.ind_offs[m + b * pl.ninds], e1 = e0 + sz;
      int l_old = -1, l_new;
      for (int e = e0; e < e1; e++) {
        int i_map = o.ind_maps[sl][e];
        l_new = (i_map * pl.dats[m2]->size) / cl;
        if (l_new > l_old) o.transfer2 += fac * cl;
        l_old = l_new;
        l_new = ((i_map + 1) * pl.dats[m2]->size - 1) / cl;
        o.transfer2 += fac * (l_new - l_old) * cl;
        l_old = l_new;
      }
      fac = (pl.accs[m2] == OP_RW) ? 2.0f : 1.0f;
      o.transfer += fac * sz * sizeof(int);
      o.transfer2 += fac * sz * sizeof(int);
    }
  }
}

// Jones-Plassmann rounds over the plan's blocks (elem = false: one CTA a
// block) or its elements (elem = true, OP_COLOR2) until every candidate has
// a colour; col receives the colours, *ncolors_d their count.  Temporaries
// go to `temp` (freed by the caller after the stream has finished).
static bool jp_rounds(const PlanParams &p, bool elem, int *col, unsigned **work_ptrs,
                      unsigned **work_d, int *ncolors_d, std::vector<void *> &temp,
                      cudaStream_t s, int *rounds_out) {
  Runtime &r = rt();
  const int n = elem ? p.exec_length : p.nblocks;
  if (rounds_out) *rounds_out = 0;
  if (n <= 0) return cuda_ok(cudaMemsetAsync(ncolors_d, 0, sizeof(int), s), "op_plan_get: colouring");
  std::vector<unsigned long long *> tptrs(PLAN_MAX_INDS, nullptr);
  auto talloc = [&](size_t bytes) -> void * {
    void *q = nullptr;
    if (cudaMalloc(&q, bytes ? bytes : 1) != cudaSuccess) return nullptr;
    temp.push_back(q);
    return q;
  };
  for (int i = 0; i < p.ninds; i++)
    if (p.ind_incrw[i] &&
        !(tptrs[i] = (unsigned long long *)talloc(sizeof(unsigned long long) * p.ind_to_size[i])))
      return cuda_ok(cudaErrorMemoryAllocation, "op_plan_get: colouring");
  auto **tmax_d = (unsigned long long **)talloc(sizeof(void *) * PLAN_MAX_INDS);
  int *cnt_d = (int *)talloc(2 * sizeof(int));
  auto *blocked_d = (unsigned char *)talloc((size_t)n);
  if (!tmax_d || !cnt_d || !blocked_d)
    return cuda_ok(cudaErrorMemoryAllocation, "op_plan_get: colouring");
  cudaMemcpyAsync(tmax_d, tptrs.data(), sizeof(void *) * PLAN_MAX_INDS, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(col, 0xff, sizeof(int) * (size_t)n, s);  // -1: no colour yet
  cudaMemsetAsync(ncolors_d, 0, sizeof(int), s);
  const int grid = elem ? (int)std::min<long long>(((long long)n + 255) / 256, (long long)r.nsm * 8)
                        : n;
  int base = 0, rounds = 0;
  int cnt[2] = {0, 0};
  for (bool pass = true; pass;) {
    // a pass: its 32 colours free on every target, nobody waiting
    for (int i = 0; i < p.ninds; i++)
      if (work_ptrs[i]) cudaMemsetAsync(work_ptrs[i], 0, sizeof(unsigned) * p.ind_to_size[i], s);
    cudaMemsetAsync(blocked_d, 0, (size_t)n, s);
    cudaMemsetAsync(cnt_d + 1, 0, sizeof(int), s);
    // rounds go in batches between looks at the counters (a round after the
    // pass has finished finds no candidate and changes nothing); the batch
    // grows while candidates remain, so dense conflict graphs (hundreds of
    // rounds) pay few host round trips
    for (int batch = 1;; batch = std::min(2 * batch, 32)) {
      if ((rounds += batch) > 1000000) {
        set_error("op_plan_get: the parallel colouring did not finish");
        return false;
      }
      for (int k = 0; k < batch; k++) {
        for (int i = 0; i < p.ninds; i++)
          if (tptrs[i])
            cudaMemsetAsync(tptrs[i], 0, sizeof(unsigned long long) * p.ind_to_size[i], s);
        cudaMemsetAsync(cnt_d, 0, sizeof(int), s);
        if (elem) {
          k_jp_elem_max<<<grid, 256, 0, s>>>(p, tmax_d, col, blocked_d);
          k_jp_elem_win<<<grid, 256, 0, s>>>(p, tmax_d, work_d, col, blocked_d, base, cnt_d,
                                             cnt_d + 1, ncolors_d);
        } else {
          k_jp_block_max<<<grid, PLAN_THREADS, 0, s>>>(p, tmax_d, col, blocked_d);
          k_jp_block_win<<<grid, PLAN_THREADS, 0, s>>>(p, tmax_d, work_d, col, blocked_d, base,
                                                       cnt_d, cnt_d + 1, ncolors_d);
        }
        r.launches += 2;
      }
      if (!cuda_ok(cudaMemcpyAsync(cnt, cnt_d, 2 * sizeof(int), cudaMemcpyDeviceToHost, s),
                   "op_plan_get: colouring") ||
          !cuda_ok(cudaStreamSynchronize(s), "op_plan_get: colouring"))
        return false;
      if (cnt[0] == 0) break;  // nobody left waiting in this pass
    }
    pass = cnt[1] > 0;  // some found the pass's colours taken: the next 32
    base += 32;
  }
  if (rounds_out) *rounds_out = rounds;
  return true;
}

Plan *build_plan(const char *name, op_set set, int part_size, int nargs, op_arg *args, int ninds,
                 int *inds, int staging, int colouring) {
  Runtime &r = rt();
  if (!r.ready()) return nullptr;
  if (nargs > PLAN_MAX_ARGS || ninds > PLAN_MAX_INDS) {
    set_error("op_plan_get: at most %d arguments and %d indirections", PLAN_MAX_ARGS,
              PLAN_MAX_INDS);
    return nullptr;
  }
  if (staging < OP_STAGE_INC || staging > OP_COLOR2) {
    set_error("op_plan_get: unknown staging %d", staging);
    return nullptr;
  }
  for (auto &pl : plan_cache()) {
    if (pl->name == name && pl->set == set && pl->nargs == nargs && pl->ninds == ninds &&
        pl->part_size == part_size && pl->staging == staging && pl->colouring == colouring &&
        same_args(*pl, nargs, args)) {
      pl->pub.count++;
      return pl.get();
    }
  }
  auto pl = std::make_unique<Plan>();
  pl->name = name;
  pl->set = set;
  pl->nargs = nargs;
  pl->ninds = ninds;
  pl->part_size = part_size;
  pl->staging = staging;
  pl->colouring = colouring;
  for (int m = 0; m < nargs; m++) {
    pl->dats.push_back(args[m].dat);
    pl->maps.push_back(args[m].map);
    pl->idxs.push_back(args[m].idx);
    pl->accs.push_back(args[m].acc);
    pl->optflags.push_back(args[m].opt);
    pl->inds.push_back(inds[m]);
  }
  for (int m = 0; m < nargs; m++) {
    if (inds[m] >= ninds || (inds[m] >= 0 && (!args[m].map || !args[m].dat))) {
      set_error("op_plan_get(%s): inds[%d] = %d is not a valid indirection", name, m, inds[m]);
      return nullptr;
    }
    if (inds[m] >= 0 && !args[m].opt) {
      set_error("op_plan_get(%s): switched-off optional indirect arguments are not supported",
                name);
      return nullptr;
    }
  }
  int exec_length = set->size;
  // staged indirections, numbered by first use (:405-427)
  std::vector<int> inds_staged(nargs, -1), ind_to_staged(ninds, -1);
  int nst = 0, maxbytes = 0;
  auto staged_arg = [&](int m) {
    return inds[m] >= 0 && ((staging == OP_STAGE_INC && args[m].acc == OP_INC) ||
                            staging == OP_STAGE_ALL || staging == OP_STAGE_PERMUTE);
  };
  for (int m = 0; m < nargs; m++) {
    if (!staged_arg(m)) continue;
    maxbytes += args[m].dat->size;
    if (ind_to_staged[inds[m]] == -1) ind_to_staged[inds[m]] = nst++;
    inds_staged[m] = ind_to_staged[inds[m]];
  }
  int bsize = part_size;
  if (bsize == 0 && maxbytes > 0) bsize = std::max((24 * 1024 / (64 * maxbytes)) * 64, 256);
  else if (bsize == 0) bsize = 256;
  if (staging == OP_COLOR2) bsize = std::max(exec_length, 1);
  if (staging != OP_COLOR2 && bsize > PLAN_MAX_PART) {
    set_error("op_plan_get(%s): part size %d above the device builder's limit %d", name, bsize,
              PLAN_MAX_PART);
    return nullptr;
  }
  int nblocks = staging == OP_COLOR2 ? 1 : (exec_length + bsize - 1) / bsize;

  PlanParams p{};
  p.nargs = nargs;
  p.ninds = ninds;
  p.nst = nst;
  p.exec_length = exec_length;
  p.bsize = bsize;
  p.nblocks = nblocks;
  int nloc = 0;
  for (int m = 0; m < nargs; m++) {
    p.map[m] = args[m].map ? args[m].map->map_d : nullptr;
    p.mdim[m] = args[m].map ? args[m].map->dim : 1;
    p.idx[m] = args[m].idx;
    p.ind[m] = inds[m];
    p.incrw[m] = inds[m] >= 0 && (args[m].acc == OP_INC || args[m].acc == OP_RW);
    p.loc_slot[m] = (staging != OP_COLOR2 && inds_staged[m] >= 0) ? nloc++ : -1;
  }
  int work_len = 0, loc_len = 0, maxvals = 0;
  for (int i = 0; i < ninds; i++) {
    p.ind_slot[i] = ind_to_staged[i];
    int na = 0, incrw = 0, to = 0;
    for (int m = 0; m < nargs; m++)
      if (inds[m] == i) {
        na++;
        incrw |= p.incrw[m];
        to = args[m].map->to->size;
      }
    p.ind_nargs[i] = na;
    p.ind_incrw[i] = incrw;
    p.ind_to_size[i] = to;
    p.ind_needed[i] = staging != OP_COLOR2 && (ind_to_staged[i] >= 0 || incrw);
    if (p.ind_needed[i]) maxvals = std::max(maxvals, na * std::min(bsize, exec_length));
    if (incrw) {
      p.ind_work_off[i] = work_len;
      work_len += na * bsize;
    }
  }
  for (int m = 0; m < nargs; m++)
    if (p.incrw[m]) {
      p.incrw_loc_off[m] = loc_len;
      loc_len += bsize;
    }
  int buf_len = 1;
  while (buf_len < std::max(maxvals, 1)) buf_len <<= 1;
  p.buf_len = buf_len;
  p.work_len = work_len;
  p.loc_len = loc_len;
  p.jp = colouring == OP2B_COLOUR_JP;

  op_plan &o = pl->pub;
  memset(&o, 0, sizeof(o));
  o.set = set;
  o.nargs = nargs;
  o.ninds = ninds;
  o.ninds_staged = nst;
  o.part_size = part_size;
  o.nblocks = nblocks;
  o.count = 1;
  pl->bsize = bsize;
  pl->name_store = name;
  o.name = pl->name_store.c_str();

  cudaStream_t s = r.stream;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, s);
  auto &own = pl->owned;
  int *d_err = dalloc<int>(1, own);
  cudaMemsetAsync(d_err, 0, sizeof(int), s);
  size_t smem_count = sizeof(int) * 3 * (size_t)buf_len;
  size_t smem_fill = smem_count + sizeof(unsigned) * (size_t)work_len + sizeof(short) * (size_t)loc_len + 16;
  if (p.jp) smem_fill += sizeof(int) * (size_t)work_len + 4;  // the round's maxima per target
  // (OP_COLOR2 runs no per-block kernel: one block is the whole set)
  if (staging != OP_COLOR2 && smem_fill > 200 * 1024) {
    set_error("op_plan_get(%s): block of %d elements needs %zu bytes of shared memory", name,
              bsize, smem_fill);
    return nullptr;
  }
  if (staging != OP_COLOR2) {  // the per-block kernels (OP_COLOR2 runs neither)
    if (!cuda_ok(cudaFuncSetAttribute(k_plan_count, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem_count), "op_plan_get: shared memory") ||
        !cuda_ok(cudaFuncSetAttribute(k_plan_fill, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem_fill), "op_plan_get: shared memory"))
      return nullptr;
  }

  std::vector<int> h_counts;
  pl->thrcol_d = dalloc<int>(exec_length, own);
  pl->nthrcol_d = dalloc<int>(nblocks, own);
  pl->blk_col_d = dalloc<int>(nblocks, own);
  pl->blkmap_d = dalloc<int>(nblocks, own);
  int *ncolblk_d = dalloc<int>(std::max(nblocks, 1) + 1, own);
  std::vector<long long> ind_base(std::max(nst, 1), 0);
  std::vector<int> ind_offs((size_t)nblocks * std::max(nst, 1), 0),
      ind_sizes((size_t)nblocks * std::max(nst, 1), 0);
  std::vector<int> nindirect(std::max(ninds, 1), 0);
  long long total_ind = 0;
  bool ok = true;
  if (staging != OP_COLOR2 && nblocks > 0) {
    int *counts_d = dalloc<int>((size_t)nblocks * std::max(ninds, 1), own);
    cudaMemsetAsync(counts_d, 0, sizeof(int) * (size_t)nblocks * std::max(ninds, 1), s);
    k_plan_count<<<nblocks, PLAN_THREADS, smem_count, s>>>(p, counts_d);
    r.launches++;
    h_counts.resize((size_t)nblocks * std::max(ninds, 1));
    ok = cuda_ok(cudaMemcpyAsync(h_counts.data(), counts_d, sizeof(int) * h_counts.size(),
                                 cudaMemcpyDeviceToHost, s), "op_plan_get: counts") &&
         cuda_ok(cudaStreamSynchronize(s), "op_plan_get: counts");
    if (!ok) return nullptr;
    // ind_offs / ind_sizes / nindirect (:670-682)
    for (int i = 0; i < ninds; i++) {
      int sl = ind_to_staged[i];
      long long acc = 0;
      for (int b = 0; b < nblocks; b++) {
        int c = h_counts[(size_t)b * ninds + i];
        if (sl >= 0) {
          ind_offs[(size_t)b * nst + sl] = (int)acc;
          ind_sizes[(size_t)b * nst + sl] = c;
        }
        acc += c;
      }
      if (sl >= 0) nindirect[i] = (int)acc;
    }
    for (int sl = 0; sl < nst && sl < 8; sl++)
      for (int b = 0; b < nblocks; b++)
        pl->max_ind_size[sl] = std::max(pl->max_ind_size[sl], ind_sizes[(size_t)b * nst + sl]);
    for (int sl = 0; sl < nst; sl++) {
      int i = 0;
      while (ind_to_staged[i] != sl) i++;
      ind_base[sl] = total_ind;
      total_ind += nindirect[i];
    }
  }
  pl->ind_map_d = dalloc<int>((size_t)total_ind, own);
  pl->loc_map_d = dalloc<short>((size_t)std::max(nloc, 1) * exec_length, own);
  pl->ind_offs_d = dalloc<int>(ind_offs.size(), own);
  pl->ind_sizes_d = dalloc<int>(ind_sizes.size(), own);
  long long *ind_base_d = dalloc<long long>(ind_base.size(), own);
  cudaMemcpyAsync(pl->ind_offs_d, ind_offs.data(), sizeof(int) * ind_offs.size(), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(pl->ind_sizes_d, ind_sizes.data(), sizeof(int) * ind_sizes.size(), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(ind_base_d, ind_base.data(), sizeof(long long) * ind_base.size(), cudaMemcpyHostToDevice, s);

  // work bitmasks over every OP_INC/OP_RW target set
  std::vector<unsigned *> work_ptrs(PLAN_MAX_INDS, nullptr);
  for (int i = 0; i < ninds; i++)
    if (p.ind_incrw[i]) work_ptrs[i] = dalloc<unsigned>(p.ind_to_size[i], own);
  unsigned **work_d = dalloc<unsigned *>(PLAN_MAX_INDS, own);
  cudaMemcpyAsync(work_d, work_ptrs.data(), sizeof(unsigned *) * PLAN_MAX_INDS, cudaMemcpyHostToDevice, s);
  int *ncolors_d = dalloc<int>(1, own);

  std::vector<void *> temp;  // freed once the build has finished
  struct TempFree {
    std::vector<void *> &t;
    ~TempFree() {
      for (void *q : t) cudaFree(q);
    }
  } temp_free{temp};
  if (nblocks > 0) {
    if (staging != OP_COLOR2) {
      k_plan_fill<<<nblocks, PLAN_THREADS, smem_fill, s>>>(p, ind_base_d, pl->ind_offs_d,
                                                           pl->ind_map_d, pl->loc_map_d,
                                                           pl->thrcol_d, pl->nthrcol_d, d_err);
      r.launches++;
    } else if (p.jp) {
      if (!jp_rounds(p, true, pl->thrcol_d, work_ptrs.data(), work_d, pl->nthrcol_d, temp, s,
                     &pl->colour_rounds))
        return nullptr;
    } else {
      k_color2_serial<<<1, 32, 0, s>>>(p, work_d, pl->thrcol_d, pl->nthrcol_d);
      r.launches++;
    }
    if (p.jp && staging != OP_COLOR2) {
      // block colours by rounds, then ncolblk/blkmap (blocks grouped by
      // colour, in block order, :886-922) from them on the host
      if (!jp_rounds(p, false, pl->blk_col_d, work_ptrs.data(), work_d, ncolors_d, temp, s,
                     &pl->colour_rounds))
        return nullptr;
      std::vector<int> bc(nblocks);
      int nc = 0;
      if (!cuda_ok(cudaMemcpyAsync(bc.data(), pl->blk_col_d, sizeof(int) * nblocks,
                                   cudaMemcpyDeviceToHost, s), "op_plan_get: colouring") ||
          !cuda_ok(cudaMemcpyAsync(&nc, ncolors_d, sizeof(int), cudaMemcpyDeviceToHost, s),
                   "op_plan_get: colouring") ||
          !cuda_ok(cudaStreamSynchronize(s), "op_plan_get: colouring"))
        return nullptr;
      std::vector<int> ncb(std::max(nc, 1) + 1, 0), start(std::max(nc, 1) + 1, 0), bm(nblocks);
      for (int b = 0; b < nblocks; b++) ncb[bc[b]]++;
      for (int c = 1; c <= nc; c++) start[c] = start[c - 1] + ncb[c - 1];
      for (int b = 0; b < nblocks; b++) bm[start[bc[b]]++] = b;
      cudaMemcpyAsync(pl->blkmap_d, bm.data(), sizeof(int) * nblocks, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(ncolblk_d, ncb.data(), sizeof(int) * std::max(nc, 1), cudaMemcpyHostToDevice,
                      s);
      if (!cuda_ok(cudaStreamSynchronize(s), "op_plan_get: colouring")) return nullptr;
    } else {
      k_block_colour_serial<<<1, 1024, 0, s>>>(p, work_d, pl->blk_col_d, ncolblk_d, pl->blkmap_d,
                                               ncolors_d);
      r.launches++;
    }
  }
  int ncolors = 0, h_err = 0;
  cudaMemcpyAsync(&ncolors, ncolors_d, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (!cuda_ok(cudaStreamSynchronize(s), "op_plan_get: build")) return nullptr;
  if (nblocks == 0) ncolors = 0;
  if (h_err) {
    set_error("op_plan_get(%s): %d local indices out of range (block too large)", name, h_err);
    return nullptr;
  }
  if (staging == OP_COLOR2) ncolors = -1;  // set below from nthrcol[0]

  // shared memory sizes
  std::vector<int> dsz(std::max(nst, 1), 0);
  for (int m = 0; m < nargs; m++)
    if (inds_staged[m] >= 0) dsz[inds_staged[m]] = args[m].dat->size;
  int *dsz_d = dalloc<int>(dsz.size(), own);
  int nc_alloc = std::max(ncolors, 1);
  int *nsharedCol_d = dalloc<int>((size_t)nc_alloc + 1, own);
  cudaMemcpyAsync(dsz_d, dsz.data(), sizeof(int) * dsz.size(), cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(nsharedCol_d, 0, sizeof(int) * ((size_t)nc_alloc + 1), s);
  if (nblocks > 0 && staging != OP_COLOR2) {
    k_plan_shared<<<(nblocks + 255) / 256, 256, 0, s>>>(p, pl->ind_sizes_d, dsz_d, pl->blk_col_d,
                                                         nsharedCol_d, nsharedCol_d + nc_alloc);
    r.launches++;
  }
  // thread-colour permutation
  std::vector<long long> coloff_base;
  int *col_reord_d = nullptr, *col_offsets_d = nullptr;
  std::vector<int> h_nthrcol(nblocks);
  cudaMemcpyAsync(h_nthrcol.data(), pl->nthrcol_d, sizeof(int) * nblocks, cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  if ((staging == OP_STAGE_PERMUTE || staging == OP_COLOR2) && nblocks > 0) {
    long long acc = 0;
    for (int b = 0; b < nblocks; b++) {
      coloff_base.push_back(acc);
      acc += h_nthrcol[b] + 1;
    }
    long long *cb_d = dalloc<long long>(coloff_base.size(), own);
    cudaMemcpyAsync(cb_d, coloff_base.data(), sizeof(long long) * coloff_base.size(), cudaMemcpyHostToDevice, s);
    col_reord_d = dalloc<int>((size_t)exec_length + 16, own);
    pl->col_reord_d = col_reord_d;
    col_offsets_d = dalloc<int>((size_t)acc, own);
    cudaMemsetAsync(col_reord_d, 0, sizeof(int) * ((size_t)exec_length + 16), s);
    k_plan_permute<<<(nblocks + 127) / 128, 128, 0, s>>>(p, pl->thrcol_d, pl->nthrcol_d, cb_d,
                                                        col_reord_d, col_offsets_d);
    r.launches++;
    pl->col_offsets_len = acc;
  }
  cudaEventRecord(t1, s);
  if (!cuda_ok(cudaStreamSynchronize(s), "op_plan_get: build")) return nullptr;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  pl->build_ms = ms;
  r.stats[name].plan_ms += ms;

  // ---------------------------------------------------------------- host copies
  auto H = [&](std::vector<int> &v, const int *d, size_t n) {
    v.resize(std::max(n, (size_t)1));
    if (n) cudaMemcpy(v.data(), d, sizeof(int) * n, cudaMemcpyDeviceToHost);
  };
  if (staging == OP_COLOR2) ncolors = h_nthrcol.empty() ? 0 : h_nthrcol[0];
  pl->h_offset.resize(std::max(nblocks, 1));
  pl->h_nelems.resize(std::max(nblocks, 1));
  for (int b = 0; b < nblocks; b++) {
    pl->h_offset[b] = b * bsize;
    pl->h_nelems[b] = std::min(bsize, exec_length - b * bsize);
  }
  H(pl->h_thrcol, pl->thrcol_d, exec_length);
  pl->h_nthrcol = h_nthrcol;
  if (pl->h_nthrcol.empty()) pl->h_nthrcol.resize(1);
  H(pl->h_blkmap, pl->blkmap_d, nblocks);
  int nb_col = staging == OP_COLOR2 ? 1 : ncolors;
  H(pl->h_ncolblk, ncolblk_d, nb_col);
  std::vector<int> nsh;
  H(nsh, nsharedCol_d, (size_t)nc_alloc + 1);
  pl->h_nsharedCol.assign(nsh.begin(), nsh.begin() + std::max(nb_col, 1));
  // OP_COLOR2 reports the element colours as ncolors (:890-891) while there
  // is one block: pad the per-colour arrays with zeros to that length
  if ((int)pl->h_ncolblk.size() < std::max(ncolors, 1)) pl->h_ncolblk.resize(std::max(ncolors, 1), 0);
  if ((int)pl->h_nsharedCol.size() < std::max(ncolors, 1))
    pl->h_nsharedCol.resize(std::max(ncolors, 1), 0);
  H(pl->h_ind_map, pl->ind_map_d, (size_t)total_ind);
  pl->h_ind_offs = ind_offs;
  pl->h_ind_sizes = ind_sizes;
  pl->h_nindirect = nindirect;
  pl->h_loc_map.resize(std::max((size_t)nloc * exec_length, (size_t)1));
  if (nloc && exec_length)
    cudaMemcpy(pl->h_loc_map.data(), pl->loc_map_d, sizeof(short) * (size_t)nloc * exec_length,
               cudaMemcpyDeviceToHost);
  pl->h_ind_maps.assign(std::max(nst, 1), nullptr);
  for (int sl = 0; sl < nst; sl++) pl->h_ind_maps[sl] = pl->h_ind_map.data() + ind_base[sl];
  pl->h_loc_maps.assign(nargs, nullptr);
  for (int m = 0; m < nargs; m++)
    if (p.loc_slot[m] >= 0) pl->h_loc_maps[m] = pl->h_loc_map.data() + (size_t)p.loc_slot[m] * exec_length;
  if (col_reord_d) {
    H(pl->h_col_reord, col_reord_d, (size_t)exec_length + 16);
    H(pl->h_col_offsets_flat, col_offsets_d, (size_t)pl->col_offsets_len);
    pl->h_col_offsets.resize(nblocks);
    for (int b = 0; b < nblocks; b++) pl->h_col_offsets[b] = pl->h_col_offsets_flat.data() + coloff_base[b];
    // COLOR2 keeps colours on the permuted elements
    H(pl->h_thrcol, pl->thrcol_d, exec_length);
  }
  pl->h_inds_staged = inds_staged;
  pl->params_blob.resize(sizeof(PlanParams));
  memcpy(pl->params_blob.data(), &p, sizeof(PlanParams));

  o.maps = pl->maps.data();
  o.dats = pl->dats.data();
  o.idxs = pl->idxs.data();
  o.optflags = pl->optflags.data();
  o.accs = pl->accs.data();
  o.inds_staged = pl->h_inds_staged.data();
  o.nthrcol = pl->h_nthrcol.data();
  o.thrcol = pl->h_thrcol.data();
  o.col_reord = pl->h_col_reord.empty() ? nullptr : pl->h_col_reord.data();
  o.col_offsets = pl->h_col_offsets.empty() ? nullptr : pl->h_col_offsets.data();
  o.color2_offsets = (staging == OP_COLOR2 && !pl->h_col_offsets.empty()) ? pl->h_col_offsets[0] : nullptr;
  o.offset = pl->h_offset.data();
  o.ind_map = pl->h_ind_map.data();
  o.ind_maps = pl->h_ind_maps.data();
  o.ind_offs = pl->h_ind_offs.data();
  o.ind_sizes = pl->h_ind_sizes.data();
  o.nindirect = pl->h_nindirect.data();
  o.loc_map = pl->h_loc_map.data();
  o.loc_maps = pl->h_loc_maps.data();
  o.nelems = pl->h_nelems.data();
  o.ncolors = ncolors;
  o.ncolors_owned = (ncolors > 0 && staging != OP_COLOR2) ? ncolors : 0;
  o.ncolblk = pl->h_ncolblk.data();
  o.blkmap = pl->h_blkmap.data();
  o.nsharedCol = pl->h_nsharedCol.data();
  o.nshared = staging == OP_COLOR2 ? 0 : nsh[nc_alloc];
  host_transfer(*pl, p, args, inds);
  // indirect reductions keep ncolors_owned = ncolors in a single-rank run (:888-890)
  bool indirect_reduce = false;
  for (int m = 0; m < nargs; m++)
    indirect_reduce |= args[m].acc != OP_READ && args[m].acc != OP_WORK && args[m].argtype == OP_ARG_GBL;
  o.ncolors_owned = (indirect_reduce && ninds > 0) ? ncolors : 0;

  plan_cache().push_back(std::move(pl));
  return plan_cache().back().get();
}

int validate_plan(const Plan &pl, long detail[8]) {
  Runtime &r = rt();
  const op_plan &o = pl.pub;
  PlanParams p;
  memcpy(&p, pl.params_blob.data(), sizeof(PlanParams));
  long d[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // host-side structural checks (O(nblocks)): op_plan_check :149-201
  int nblock = 0;
  for (int c = 0; c < std::max(o.ncolors, 0) && pl.staging != OP_COLOR2; c++) nblock += o.ncolblk[c];
  if (pl.staging == OP_COLOR2) nblock = o.nblocks;
  long nelem = 0;
  for (int b = 0; b < nblock; b++) nelem += o.nelems[b];
  d[0] = nelem != pl.set->size;
  long ntot = 0;
  for (int b = 0; b < nblock; b++) {
    d[1] += o.offset[b] != ntot;
    ntot += o.nelems[b];
  }
  std::vector<int> bm(o.blkmap, o.blkmap + nblock);
  std::sort(bm.begin(), bm.end());
  for (int b = 0; b < nblock; b++) d[2] += bm[b] != b;
  for (int i = 0; i < o.ninds_staged; i++) {
    long t = 0;
    for (int b = 0; b < nblock; b++) {
      d[3] += o.ind_offs[i + b * o.ninds_staged] != t;
      t += o.ind_sizes[i + b * o.ninds_staged];
    }
  }
  cudaStream_t s = r.stream;
  std::vector<void *> own;
  unsigned long long *err_d = dalloc<unsigned long long>(4, own);
  cudaMemsetAsync(err_d, 0, 4 * sizeof(unsigned long long), s);
  if (pl.staging != OP_COLOR2 && o.nblocks > 0) {
    for (int i = 0; i < pl.ninds; i++) {
      int sl = p.ind_slot[i];
      if (sl < 0) continue;
      const int *base = pl.ind_map_d + (o.ind_maps[sl] - o.ind_map);
      k_check_ind_maps<<<(o.nblocks + 255) / 256, 256, 0, s>>>(o.nblocks, o.ninds_staged, sl,
                                                                pl.ind_sizes_d, pl.ind_offs_d,
                                                                base, p.ind_to_size[i], err_d);
    }
    for (int a = 0; a < pl.nargs; a++) {
      if (p.loc_slot[a] < 0) continue;
      int sl = p.ind_slot[p.ind[a]];
      const int *base = pl.ind_map_d + (o.ind_maps[sl] - o.ind_map);
      k_check_loc_maps<<<(p.exec_length + 255) / 256, 256, 0, s>>>(
          p, a, pl.loc_map_d + (size_t)p.loc_slot[a] * p.exec_length, base, pl.ind_offs_d,
          err_d + 1);
    }
    // thread colours (PERMUTE/COLOR2 keep sorted colours on permuted elements: skip)
    if (pl.staging != OP_STAGE_PERMUTE) {
      int cnt = 0;
      for (int a = 0; a < pl.nargs; a++) cnt += p.incrw[a] ? p.bsize : 0;
      int pad = 1;
      while (pad < cnt) pad <<= 1;
      size_t smem = sizeof(unsigned long long) * (size_t)pad;
      if (cnt > 0 && smem <= 200 * 1024) {
        cudaFuncSetAttribute(k_check_thread_colours, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        k_check_thread_colours<<<o.nblocks, 256, smem, s>>>(p, pl.thrcol_d, err_d + 2);
      }
    }
  }
  // block colours, one launch per colour
  if (pl.staging != OP_COLOR2 && o.ncolors > 0) {
    std::vector<unsigned long long *> owner(PLAN_MAX_INDS, nullptr);
    for (int i = 0; i < pl.ninds; i++)
      if (p.ind_incrw[i]) {
        owner[i] = dalloc<unsigned long long>(p.ind_to_size[i], own);
        cudaMemsetAsync(owner[i], 0, sizeof(unsigned long long) * p.ind_to_size[i], s);
      }
    unsigned long long **owner_d = dalloc<unsigned long long *>(PLAN_MAX_INDS, own);
    cudaMemcpyAsync(owner_d, owner.data(), sizeof(void *) * PLAN_MAX_INDS, cudaMemcpyHostToDevice, s);
    int first = 0;
    for (int c = 0; c < o.ncolors; c++) {
      if (o.ncolblk[c] > 0)
        k_check_block_colour<<<o.ncolblk[c], 256, 0, s>>>(p, c, pl.blkmap_d, first, o.ncolblk[c],
                                                           owner_d, err_d + 3);
      first += o.ncolblk[c];
    }
  }
  unsigned long long h[4] = {0, 0, 0, 0};
  cudaMemcpyAsync(h, err_d, sizeof(h), cudaMemcpyDeviceToHost, s);
  bool ok = cuda_ok(cudaStreamSynchronize(s), "op2b_plan_validate");
  for (void *q : own) cudaFree(q);
  if (!ok) return -1;
  d[4] = (long)h[0];
  d[5] = (long)h[1];
  d[6] = (long)h[2];
  d[7] = (long)h[3];
  long tot = 0;
  for (int i = 0; i < 8; i++) tot += d[i];
  if (detail)
    for (int i = 0; i < 8; i++) detail[i] = d[i];
  return (int)std::min(tot, (long)INT_MAX);
}

__global__ void k_count_blocks(int nst, int slot, const int *ind_sizes, const int *ind_offs,
                               const int *ind_map_s, int *cnt) {
  int b = blockIdx.x;
  int o = ind_offs[(size_t)b * nst + slot], s = ind_sizes[(size_t)b * nst + slot];
  for (int i = threadIdx.x; i < s; i += blockDim.x) atomicAdd(&cnt[ind_map_s[o + i]], 1);
}

__global__ void k_flag_shared(long long total, const int *ind_map_s, const int *cnt,
                              unsigned char *flag) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) flag[i] = cnt[ind_map_s[i]] > 1;
}

const int *plan_ind_map_slot(const Plan &pl, int slot) {
  return pl.ind_map_d + (pl.pub.ind_maps[slot] - pl.pub.ind_map);
}

int plan_max_ind_size(const Plan &pl, int slot) {
  int mx = 0;
  for (int b = 0; b < pl.pub.nblocks; b++)
    mx = std::max(mx, pl.pub.ind_sizes[(size_t)b * pl.pub.ninds_staged + slot]);
  return mx;
}

const unsigned char *plan_shared_flags(Plan &pl, int slot) {
  if ((int)pl.shared_d.size() <= slot) pl.shared_d.resize(slot + 1, nullptr);
  if (pl.shared_d[slot]) return pl.shared_d[slot];
  PlanParams p;
  memcpy(&p, pl.params_blob.data(), sizeof(PlanParams));
  int ind = -1;
  for (int i = 0; i < pl.ninds; i++)
    if (p.ind_slot[i] == slot) ind = i;
  if (ind < 0) return nullptr;
  long long total = 0;
  for (int b = 0; b < pl.pub.nblocks; b++)
    total += pl.pub.ind_sizes[(size_t)b * pl.pub.ninds_staged + slot];
  cudaStream_t s = rt().stream;
  int *cnt = dalloc<int>(p.ind_to_size[ind], pl.owned);
  unsigned char *flag = dalloc<unsigned char>((size_t)total, pl.owned);
  if (!cnt || !flag) return nullptr;
  cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)p.ind_to_size[ind], s);
  const int *im = plan_ind_map_slot(pl, slot);
  if (pl.pub.nblocks > 0) {
    k_count_blocks<<<pl.pub.nblocks, 256, 0, s>>>(pl.pub.ninds_staged, slot, pl.ind_sizes_d,
                                                  pl.ind_offs_d, im, cnt);
    k_flag_shared<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(total, im, cnt, flag);
  }
  if (!cuda_ok(cudaStreamSynchronize(s), "plan shared flags")) return nullptr;
  pl.shared_d[slot] = flag;
  return flag;
}

const Plan *find_plan(const op_plan *o) {
  for (auto &pl : plan_cache())
    if (&pl->pub == o) return pl.get();
  return nullptr;
}

void release_plans() { plan_cache().clear(); }

}  // namespace op2b

using namespace op2b;

extern "C" {

op_plan *op_plan_get_stage(char const *name, op_set set, int part_size, int nargs, op_arg *args,
                           int ninds, int *inds, int staging) {
  // the reference's greedy order (bit-exact plans) unless plan_mode 1 asks
  // for the parallel colouring
  Plan *pl = build_plan(name, set, part_size, nargs, args, ninds, inds, staging,
                        rt().opt_plan_mode == 1 ? OP2B_COLOUR_JP : OP2B_COLOUR_GREEDY);
  return pl ? &pl->pub : nullptr;
}

op_plan *op_plan_get_stage_upload(char const *name, op_set set, int part_size, int nargs,
                                  op_arg *args, int ninds, int *inds, int staging, int upload) {
  (void)upload;
  return op_plan_get_stage(name, set, part_size, nargs, args, ninds, inds, staging);
}

op_plan *op_plan_get(char const *name, op_set set, int part_size, int nargs, op_arg *args,
                     int ninds, int *inds) {
  return op_plan_get_stage(name, set, part_size, nargs, args, ninds, inds, OP_STAGE_ALL);
}

void op_plan_check(op_plan OP_plan, int ninds, int *inds) {
  (void)ninds;
  (void)inds;
  const Plan *pl = find_plan(&OP_plan);
  if (!pl) {
    for (auto &c : plan_cache())
      if (c->pub.thrcol == OP_plan.thrcol) pl = c.get();
  }
  if (!pl) {
    printf(" *** op_plan_check: unknown plan\n");
    return;
  }
  long d[8];
  int n = validate_plan(*pl, d);
  static const char *what[8] = {"nelems", "offset", "blkmap", "ind_offs", "ind_maps", "maps",
                                "thread colours", "block colours"};
  for (int i = 0; i < 8; i++)
    if (d[i]) printf(" *** op_plan_check: %ld %s error(s)\n", d[i], what[i]);
  if (n == 0 && rt().opt_diags > 6) printf(" *** op_plan_check: OK\n");
}

int op2b_plan_validate(const op_plan *plan, long detail[8]) {
  const Plan *pl = find_plan(plan);
  if (!pl) {
    set_error("op2b_plan_validate: unknown plan");
    return -1;
  }
  return validate_plan(*pl, detail);
}

double op2b_plan_build_ms(const op_plan *plan) {
  const Plan *pl = find_plan(plan);
  return pl ? pl->build_ms : -1.0;
}

const int *op2b_plan_device_blkmap(const op_plan *plan) {
  const Plan *pl = find_plan(plan);
  return pl ? pl->blkmap_d : nullptr;
}

const int *op2b_plan_device_thrcol(const op_plan *plan) {
  const Plan *pl = find_plan(plan);
  return pl ? pl->thrcol_d : nullptr;
}

void op2b_plan_release_all(void) {
  cudaStreamSynchronize(rt().stream);
  release_plans();
}

}  // extern "C"
