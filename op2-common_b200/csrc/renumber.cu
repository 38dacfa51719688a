// Mesh renumbering on the GPU: op_renumber of the reference
// (op2/src/externlib/op_renumber.cpp:224-505) with the base ordering from a
// GPU reverse Cuthill-McKee instead of PT-Scotch's Gibbs-Poole-Stockmeyer
// (SCOTCH_graphOrder with strategy "g", :452-461 -- a third-party library not
// in the reference tree).
//
//   1. graph of the base map's target set (:274-350): for a map from another
//      set (e.g. pecell, edges -> cells) two targets are adjacent when one
//      element maps to both; for a map onto its own set the rows are the
//      adjacency.  Built with a count / scan / fill / per-row sort+unique.
//   2. reverse Cuthill-McKee, by one CTA: George-Liu pseudo-peripheral start
//      (from a minimum-degree vertex, repeated BFS, min-degree vertex of the
//      last level, lowest id on ties), then BFS levels; a level's new vertices are ordered by
//      (position of their first parent in the previous level, degree, id) --
//      the order sequential Cuthill-McKee produces -- and the whole order is
//      reversed.  Each connected component starts from an unvisited vertex of
//      minimum degree (lowest id on ties).
//   3. propagation to the other sets, in the reference's recursive order over
//      the declared maps (propagate_reordering, :72-151):
//      * a map to -> from: elements sorted by the new index of their first
//        target, ties by original index (the reference leaves ties to qsort);
//      * else a map from -> to that covers `to`: first touch, walking `from`
//        in its new order.
//   4. reordering (reorder_set, :153-222): rows of maps from a set move,
//      entries of maps to a set are renumbered, dats on a set move; all on
//      the device, host copies of maps refreshed.
// The permutation of every set is kept so op_fetch_data_idx can return data
// in the application's original numbering.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>

#include "op2b_runtime.h"
#include "scan.h"

namespace op2b {

// ------------------------------------------------------------------ graph

__global__ void k_adj_count(int nfrom, int dim, const int *map, int nto, int *deg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nfrom) return;
  for (int a = 0; a < dim; a++) {
    int u = map[(size_t)i * dim + a];
    if (u < 0 || u >= nto) continue;
    for (int b = 0; b < dim; b++) {
      int v = map[(size_t)i * dim + b];
      if (b != a && v != u && v >= 0 && v < nto) atomicAdd(&deg[u], 1);
    }
  }
}

__global__ void k_adj_fill(int nfrom, int dim, const int *map, int nto, const long long *row,
                           int *fill, int *col) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nfrom) return;
  for (int a = 0; a < dim; a++) {
    int u = map[(size_t)i * dim + a];
    if (u < 0 || u >= nto) continue;
    for (int b = 0; b < dim; b++) {
      int v = map[(size_t)i * dim + b];
      if (b != a && v != u && v >= 0 && v < nto) col[row[u] + atomicAdd(&fill[u], 1)] = v;
    }
  }
}

// self map (to == from): the row of u lists its neighbours
__global__ void k_adj_self(int n, int dim, const int *map, int *deg, int *col) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  int k = 0;
  for (int a = 0; a < dim; a++) {
    int v = map[(size_t)u * dim + a];
    if (v >= 0 && v < n && v != u) col[(size_t)u * dim + k++] = v;
  }
  deg[u] = k;
}

// sort each row and drop duplicates; deg[u] becomes the unique count
__global__ void k_adj_unique(int n, const long long *row, int *col, int *deg) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  int *c = col + row[u];
  int m = deg[u];
  for (int i = 1; i < m; i++) {
    int v = c[i], j = i - 1;
    while (j >= 0 && c[j] > v) {
      c[j + 1] = c[j];
      j--;
    }
    c[j + 1] = v;
  }
  int k = 0;
  for (int i = 0; i < m; i++)
    if (i == 0 || c[i] != c[i - 1]) c[k++] = c[i];
  deg[u] = k;
}

// the first four neighbours of each vertex, -1 padded: one 16-byte load
__global__ void k_adj_ell(int n, const long long *row, const int *deg, const int *col,
                          int4 *ell) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const int d = deg[u];
  const int *c = col + row[u];
  ell[u] = make_int4(d > 0 ? c[0] : -1, d > 1 ? c[1] : -1, d > 2 ? c[2] : -1, d > 3 ? c[3] : -1);
}

// ------------------------------------------------------------------ RCM (one CTA)

struct RcmWork {
  int n;
  const long long *row;  // row start; row[u] + deg[u] = end
  const int *deg;
  const int *col;
  const int4 *ell;       // first four neighbours of each vertex, -1 padded
  int *newidx;           // CM position of each vertex, -1 = unvisited
  int *mark;             // BFS stamp of the pseudo-peripheral search
  int *lev_a, *lev_b;    // current and next level (positions from kLevShared on)
  int *pkey;             // first-parent position of a discovered vertex (INT_MAX = none)
  int *status;           // [0] = vertices ordered, [1] = error, [2] = walks, [3] = levels,
                         // [4] / [5] = microseconds in Cuthill-McKee / breadth-first walks
};

__device__ __forceinline__ unsigned long long rcm_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// thread 0 adds the time since prof[3] to prof[k] and restarts the lap
__device__ __forceinline__ void rcm_lap(unsigned long long *prof, int k) {
  if (threadIdx.x == 0) {
    const unsigned long long now = rcm_clock();
    prof[k] += now - prof[3];
    prof[3] = now;
  }
}

constexpr int kRcmThreads = 1024;
// Positions of a level below kLevShared live in shared memory, the rest in
// the global list: the levels of a 2-D mesh of a few million cells fit,
// and each level walk then reads its parents without a trip to L2.
constexpr int kLevShared = 16384;
constexpr size_t kRcmSmem = 2 * sizeof(int) * kLevShared;

struct Lev {
  int *s, *g;
  __device__ __forceinline__ int get(int j) const { return j < kLevShared ? s[j] : g[j]; }
  __device__ __forceinline__ void put(int j, int v) const {
    if (j < kLevShared) s[j] = v;
    else g[j] = v;
  }
};

// Exclusive block-wide scan of v (blockDim.x a multiple of 32, <= 1024);
// *total receives the sum over the block.
__device__ int rcm_block_scan(int v, int *total) {
  __shared__ int s_warp[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int t = lane < nw ? s_warp[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nw) s_warp[lane] = t;
  }
  __syncthreads();
  const int before = (wid > 0 ? s_warp[wid - 1] : 0) + x - v;
  *total = s_warp[nw - 1];
  __syncthreads();  // s_warp is reused by the next call
  return before;
}

constexpr int kB = 2;   // vertices a thread handles per round
constexpr int kNb = 4;  // neighbours per vertex loaded unrolled (the rest in a loop)

// A vertex is closed to a level walk once ordered before position `thr`
// (thr = INT_MAX: ordered at all).
__device__ __forceinline__ bool rcm_open(const RcmWork &w, int v, int thr) {
  const int p = w.newidx[v];
  return p < 0 || p >= thr;
}

// Degree, adjacency row and first kNb neighbours (-1 where there is none)
// of up to kB vertices u (-1 = none); the three loads of a vertex are
// independent of one another.
__device__ __forceinline__ void load_vertices(const RcmWork &w, const int (&u)[kB], int (&d)[kB],
                                              long long (&r)[kB], int (&v)[kB][kNb]) {
  static_assert(kNb == 4, "the neighbour table is four wide");
#pragma unroll
  for (int k = 0; k < kB; k++) {
    int4 nb = make_int4(-1, -1, -1, -1);
    d[k] = 0;
    r[k] = 0;
    if (u[k] >= 0) {
      nb = w.ell[u[k]];
      d[k] = w.deg[u[k]];
    }
    v[k][0] = nb.x;
    v[k][1] = nb.y;
    v[k][2] = nb.z;
    v[k][3] = nb.w;
  }
  // the adjacency row only where the neighbours do not fit the table
#pragma unroll
  for (int k = 0; k < kB; k++)
    if (d[k] > kNb) r[k] = w.row[u[k]];
}

// A vertex just placed in the next level: its neighbour-table entry and
// degree, read when that level is walked, start towards L2 now.
__device__ __forceinline__ void rcm_prefetch(const RcmWork &w, int v) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(w.ell + v));
  asm volatile("prefetch.global.L2 [%0];" ::"l"(w.deg + v));
}

// The first kNb unvisited neighbours of up to kB level vertices
// (cur[j0 + k * blockDim.x]); v = -1 where there is none.
struct LevelBatch {
  int d[kB];
  long long r[kB];
  int v[kB][kNb];
  // open: drop neighbours already ordered (Cuthill-McKee's walk); a
  // breadth-first search stays inside one component, none of whose
  // vertices is ordered before `thr`, and needs no such test
  __device__ void load(const RcmWork &w, const Lev &cur, int len, int j0, int thr = INT_MAX,
                       bool open = true) {
    int u[kB];
#pragma unroll
    for (int k = 0; k < kB; k++) {
      const int j = j0 + k * (int)blockDim.x;
      u[k] = j < len ? cur.get(j) : -1;
    }
    load_vertices(w, u, d, r, v);
    if (!open) return;
#pragma unroll
    for (int k = 0; k < kB; k++)
#pragma unroll
      for (int t = 0; t < kNb; t++)
        if (v[k][t] >= 0 && !rcm_open(w, v[k][t], thr)) v[k][t] = -1;
  }
};

// Up to kB consecutive parents j0 .. min(j0 + kB, je) - 1 of a level with
// their first kNb neighbours, each neighbour's claim (pkey) and degree.
struct ParentBatch {
  int d[kB];
  long long r[kB];
  int v[kB][kNb], pk[kB][kNb], vd[kB][kNb];
  __device__ void load(const RcmWork &w, const Lev &cur, int j0, int je) {
    int u[kB];
#pragma unroll
    for (int k = 0; k < kB; k++) u[k] = j0 + k < je ? cur.get(j0 + k) : -1;
    load_vertices(w, u, d, r, v);
#pragma unroll
    for (int k = 0; k < kB; k++)
#pragma unroll
      for (int t = 0; t < kNb; t++) {
        const int x = v[k][t];
        const bool open = x >= 0 && w.newidx[x] < 0;
        pk[k][t] = open ? w.pkey[x] : -1;
        vd[k][t] = open ? w.deg[x] : 0;
      }
  }
  // the same in two steps: the parents and their unordered neighbours
  // before the level's claims, the neighbours' claims and degrees after
  __device__ void load_open(const RcmWork &w, const Lev &cur, int j0, int je) {
    int u[kB];
#pragma unroll
    for (int k = 0; k < kB; k++) u[k] = j0 + k < je ? cur.get(j0 + k) : -1;
    load_vertices(w, u, d, r, v);
#pragma unroll
    for (int k = 0; k < kB; k++)
#pragma unroll
      for (int t = 0; t < kNb; t++)
        if (v[k][t] >= 0 && w.newidx[v[k][t]] >= 0) v[k][t] = -1;
  }
  __device__ void load_keys(const RcmWork &w) {
#pragma unroll
    for (int k = 0; k < kB; k++)
#pragma unroll
      for (int t = 0; t < kNb; t++) {
        const int x = v[k][t];
        pk[k][t] = x >= 0 ? w.pkey[x] : -1;
        vd[k][t] = x >= 0 ? w.deg[x] : 0;
      }
  }
  __device__ bool claimed(int k, int t, int j) const { return v[k][t] >= 0 && pk[k][t] == j; }
  // children of parent k (position j) that it claimed
  __device__ int count(const RcmWork &w, int k, int j) const {
    int c = 0;
#pragma unroll
    for (int t = 0; t < kNb; t++) c += claimed(k, t, j) ? 1 : 0;
    for (int t = kNb; t < d[k]; t++) {
      int x = w.col[r[k] + t];
      if (w.newidx[x] < 0 && w.pkey[x] == j) c++;
    }
    return c;
  }
};

// BFS from `start` over its component; marks with `stamp`.  (The vertices
// of other components are not reachable, and those of this one are either
// all unordered or, thr = the component's first position, ordered from thr
// on: no test of the order is needed.)  Returns the number of levels; the
// last level is left in *last (lev_a or lev_b).
__device__ int rcm_bfs(RcmWork &w, Lev cur, Lev nxt, int start, int stamp, Lev *last,
                       int *last_len, int thr = INT_MAX) {
  __shared__ int s_len, s_next;
  if (threadIdx.x == 0) {
    cur.put(0, start);
    w.mark[start] = stamp;
    s_len = 1;
  }
  __syncthreads();
  int nlev = 0;
  while (true) {
    int len = s_len;
    nlev++;
    if (threadIdx.x == 0) s_next = 0;
    __syncthreads();
    // kB vertices per thread per round, their first kNb neighbours unrolled:
    // every load of a round is independent of the others, so one round costs
    // a handful of memory latencies however many vertices it covers
    // (every thread runs the same rounds, so that the warp can combine its
    // appends: one shared-memory atomic per warp instead of one per vertex)
    for (int r0 = 0; r0 < len; r0 += kB * blockDim.x) {
      const int j0 = r0 + threadIdx.x;
      LevelBatch b;
      b.load(w, cur, len, j0, thr, false);
      // all exchanges first (none waits on another's result), then the appends
      int old[kB][kNb];
#pragma unroll
      for (int k = 0; k < kB; k++)
#pragma unroll
        for (int t = 0; t < kNb; t++)
          old[k][t] = b.v[k][t] >= 0 ? atomicExch(&w.mark[b.v[k][t]], stamp) : stamp;
      int cnt = 0;
#pragma unroll
      for (int k = 0; k < kB; k++)
#pragma unroll
        for (int t = 0; t < kNb; t++) cnt += old[k][t] != stamp ? 1 : 0;
      const int lane = threadIdx.x & 31;
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      int wbase = 0;
      if (lane == 31 && incl > 0) wbase = atomicAdd(&s_next, incl);
      int pos = __shfl_sync(0xffffffffu, wbase, 31) + incl - cnt;
#pragma unroll
      for (int k = 0; k < kB; k++)
#pragma unroll
        for (int t = 0; t < kNb; t++)
          if (old[k][t] != stamp) {
            rcm_prefetch(w, b.v[k][t]);
            nxt.put(pos++, b.v[k][t]);
          }
#pragma unroll
      for (int k = 0; k < kB; k++)
        for (int t = kNb; t < b.d[k]; t++) {  // vertices of higher degree
          int v = w.col[b.r[k] + t];
          if (atomicExch(&w.mark[v], stamp) != stamp) nxt.put(atomicAdd(&s_next, 1), v);
        }
    }
    __syncthreads();
    int nl = s_next;
    if (nl == 0) {
      *last = cur;
      *last_len = len;
      return nlev;
    }
    const Lev t = cur;
    cur = nxt;
    nxt = t;
    if (threadIdx.x == 0) s_len = nl;
    __syncthreads();
  }
}

// George-Liu candidate of a last level: minimum degree, lowest id on ties
__device__ int rcm_pick(const RcmWork &w, const Lev &last, int last_len) {
  __shared__ int s_best, s_bestdeg;
  if (threadIdx.x == 0) {
    s_best = INT_MAX;
    s_bestdeg = INT_MAX;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < last_len; j += blockDim.x)
    atomicMin(&s_bestdeg, w.deg[last.get(j)]);
  __syncthreads();
  for (int j = threadIdx.x; j < last_len; j += blockDim.x) {
    int v = last.get(j);
    if (w.deg[v] == s_bestdeg) atomicMin(&s_best, v);
  }
  __syncthreads();
  const int cand = s_best;
  __syncthreads();  // s_best is reused by the next call
  return cand;
}

// Parent k (level position j) of a batch appends its claimed children to
// the next level at pos, in sequential Cuthill-McKee's order, and places them.
__device__ __forceinline__ void rcm_place(RcmWork &w, const Lev &nxt, int &pos, int base, int v) {
  rcm_prefetch(w, v);
  nxt.put(pos, v);
  w.newidx[v] = base + pos;
  w.pkey[v] = INT_MAX;
  pos++;
}

__device__ __forceinline__ void rcm_emit(RcmWork &w, const ParentBatch &pb, int k, int j,
                                         const Lev &nxt, int &pos, int base) {
  if (pb.d[k] <= kNb) {
    // the claimed children's (degree capped at 63, id) keys, sorted in registers
    unsigned long long key[kNb];
#pragma unroll
    for (int t = 0; t < kNb; t++)
      key[t] = pb.claimed(k, t, j)
                   ? ((unsigned long long)(unsigned)min(pb.vd[k][t], 63) << 32) |
                         (unsigned)pb.v[k][t]
                   : ~0ull;
#pragma unroll
    for (int i = 1; i < kNb; i++)
#pragma unroll
      for (int m = i; m > 0; m--)
        if (key[m] < key[m - 1]) {
          unsigned long long x = key[m];
          key[m] = key[m - 1];
          key[m - 1] = x;
        }
#pragma unroll
    for (int t = 0; t < kNb; t++)
      if (key[t] != ~0ull) rcm_place(w, nxt, pos, base, (int)(key[t] & 0xffffffffull));
  } else {
    // higher degree: selection of the smallest claimed key above the last
    // (a child placed is no longer unordered: the test skips it as well)
    unsigned long long last = 0;
    bool any = false;
    while (true) {
      unsigned long long best = ~0ull;
      for (int t = 0; t < pb.d[k]; t++) {
        int v = w.col[pb.r[k] + t];
        if (w.newidx[v] < 0 && w.pkey[v] == j) {
          unsigned long long key =
              ((unsigned long long)(unsigned)min(w.deg[v], 63) << 32) | (unsigned)v;
          if ((!any || key > last) && key < best) best = key;
        }
      }
      if (best == ~0ull) break;
      rcm_place(w, nxt, pos, base, (int)(best & 0xffffffffull));
      last = best;
      any = true;
    }
  }
}

// Cuthill-McKee from `start`: appends its component to the order at
// s_pos (shared).  Its levels are the BFS levels from `start`: returns
// their number and leaves the last level in *last.
__device__ int rcm_cm(RcmWork &w, Lev cur, Lev nxt, int start, int &s_pos, int &s_len, Lev *last,
                      int *last_len, unsigned long long *prof) {
  if (threadIdx.x == 0) {
    cur.put(0, start);
    w.newidx[start] = s_pos++;
    s_len = 1;
  }
  __syncthreads();
  int nlev = 0;
  while (true) {
    const int len = s_len;
    const int base = s_pos;
    nlev++;
    const int chunk = (len + (int)blockDim.x - 1) / (int)blockDim.x;
    const int jb = min(len, (int)threadIdx.x * chunk), je = min(len, jb + chunk);
    if (chunk <= kB) {
      // a level of at most kB parents a thread: each thread loads its run of
      // parents once, claims their children, counts and places them -- the
      // steps below with the loads shared between them
      if (threadIdx.x == 0) prof[3] = rcm_clock();
      ParentBatch pb;
      pb.load_open(w, cur, jb, je);
#pragma unroll
      for (int k = 0; k < kB; k++) {
        const int j = jb + k;
        if (j >= je) break;
#pragma unroll
        for (int t = 0; t < kNb; t++)
          if (pb.v[k][t] >= 0) atomicMin(&w.pkey[pb.v[k][t]], j);
        for (int t = kNb; t < pb.d[k]; t++) {
          int v = w.col[pb.r[k] + t];
          if (w.newidx[v] < 0) atomicMin(&w.pkey[v], j);
        }
      }
      __syncthreads();
      rcm_lap(prof, 0);
      pb.load_keys(w);
      int mine = 0;
#pragma unroll
      for (int k = 0; k < kB; k++) mine += pb.count(w, k, jb + k);
      int nl = 0;
      int pos = rcm_block_scan(mine, &nl);
      rcm_lap(prof, 1);
      if (nl == 0) {
        *last = cur;
        *last_len = len;
        return nlev;
      }
#pragma unroll
      for (int k = 0; k < kB; k++) {
        const int j = jb + k;
        if (j >= je) break;
        rcm_emit(w, pb, k, j, nxt, pos, base);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        s_pos = base + nl;
        s_len = nl;
      }
      const Lev t = cur;
      cur = nxt;
      nxt = t;
      __syncthreads();
      rcm_lap(prof, 2);
      continue;
    }
    // first parent (lowest position in this level) of every new vertex
    for (int j0 = threadIdx.x; j0 < len; j0 += kB * blockDim.x) {
      LevelBatch b;
      b.load(w, cur, len, j0);
#pragma unroll
      for (int k = 0; k < kB; k++) {
        const int j = j0 + k * (int)blockDim.x;
#pragma unroll
        for (int t = 0; t < kNb; t++)
          if (b.v[k][t] >= 0) atomicMin(&w.pkey[b.v[k][t]], j);
        for (int t = kNb; t < b.d[k]; t++) {
          int v = w.col[b.r[k] + t];
          if (w.newidx[v] < 0) atomicMin(&w.pkey[v], j);
        }
      }
    }
    __syncthreads();
    // The next level is the parents' claimed vertices, parent by parent in
    // level order and, within a parent, by (degree capped at 63, id): the
    // order sequential Cuthill-McKee appends them in.  Each thread takes a
    // contiguous run of parents; a block scan of the runs' counts places
    // them, so no sort of the level is needed.
    int mine = 0;
    for (int j0 = jb; j0 < je; j0 += kB) {
      ParentBatch pb;
      pb.load(w, cur, j0, je);
#pragma unroll
      for (int k = 0; k < kB; k++) mine += pb.count(w, k, j0 + k);
    }
    int nl = 0;
    int pos = rcm_block_scan(mine, &nl);
    if (nl == 0) {
      *last = cur;
      *last_len = len;
      return nlev;
    }
    for (int j0 = jb; j0 < je; j0 += kB) {
      ParentBatch pb;
      pb.load(w, cur, j0, je);
#pragma unroll
      for (int k = 0; k < kB; k++) {
        const int j = j0 + k;
        if (j >= je) break;
        rcm_emit(w, pb, k, j, nxt, pos, base);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_pos = base + nl;
      s_len = nl;
    }
    const Lev t = cur;
    cur = nxt;
    nxt = t;
    __syncthreads();
  }
}

// An unvisited vertex of minimum degree, lowest id on ties (a corner of a
// structured mesh region: usually already pseudo-peripheral); -1 when every
// vertex is ordered.  Called by the whole CTA.
__device__ int rcm_min_degree(const RcmWork &w) {
  __shared__ unsigned long long s_key[kRcmThreads / 32];
  __shared__ int s_start;
  unsigned long long best = ~0ull;
  for (int v = threadIdx.x; v < w.n; v += blockDim.x)
    if (w.newidx[v] < 0) {
      const unsigned long long key = ((unsigned long long)(unsigned)w.deg[v] << 32) | (unsigned)v;
      best = key < best ? key : best;
    }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_down_sync(0xffffffffu, best, o);
    best = other < best ? other : best;
  }
  if ((threadIdx.x & 31) == 0) s_key[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); k++) best = s_key[k] < best ? s_key[k] : best;
    s_start = best == ~0ull ? -1 : (int)(best & 0xffffffffull);
  }
  __syncthreads();
  const int start = s_start;
  __syncthreads();  // s_key and s_start are reused by the next call
  return start;
}

// Reverse Cuthill-McKee of the first component is found by two CTAs at once
// (two kernels on two streams), which share nothing they write:
//   * k_rcm_search runs the plain George-Liu search: breadth-first walks
//     (w.mark, its own level lists) from the minimum-degree vertex, then from
//     the candidate of each last level (minimum degree, lowest id), while
//     the eccentricity grows, at most 8 candidates;
//   * k_rcm_first orders the component by Cuthill-McKee from the
//     minimum-degree vertex meanwhile (w.newidx, w.pkey, w.lev_a/b).
// When the search keeps the first vertex -- the usual case -- that order is
// the one the sequential algorithm builds; otherwise k_rcm_redo undoes it
// and orders from the vertex found.  k_rcm then takes the other components
// (if any) one after another in one CTA, each by Cuthill-McKee from its
// minimum-degree vertex followed by the breadth-first test of that order's
// last level (and the search, when the test finds a more eccentric vertex).
// rcm[0] = start found, [1] = first start, [2] = search walks, [3] = their
// levels, [4] = microseconds searching.
__global__ void __launch_bounds__(kRcmThreads) k_rcm_search(RcmWork w, int *lev_c, int *lev_d,
                                                            int *rcm) {
  extern __shared__ int s_lev[];  // 2 * kLevShared
  const Lev la{s_lev, lev_c}, lb{s_lev + kLevShared, lev_d};
  const unsigned long long t0 = rcm_clock();
  int start = rcm_min_degree(w);
  if (start < 0) return;
  const int start0 = start;
  Lev last;
  int last_len;
  int stamp = 1;
  int ecc = rcm_bfs(w, la, lb, start, stamp++, &last, &last_len);
  int walks = 1, levels = ecc;
  for (int round = 0; round < 8; round++) {
    const int cand = rcm_pick(w, last, last_len);
    const int e2 = rcm_bfs(w, la, lb, cand, stamp++, &last, &last_len);
    walks++;
    levels += e2;
    if (e2 <= ecc) break;
    ecc = e2;
    start = cand;
  }
  if (threadIdx.x == 0) {
    rcm[0] = start;
    rcm[1] = start0;
    rcm[2] = walks;
    rcm[3] = levels;
    rcm[4] = (int)((rcm_clock() - t0) / 1000);
  }
}

// Cuthill-McKee of the component of the minimum-degree vertex (start < 0) or
// of `start` after undoing the component ordered before (start >= 0).
// status[0] = vertices ordered, [2] = walks, [3] = levels, [4] = microseconds,
// [6..8] = the small levels' phases.
__global__ void __launch_bounds__(kRcmThreads) k_rcm_first(RcmWork w, int start) {
  extern __shared__ int s_lev[];
  __shared__ int s_len, s_pos;
  __shared__ unsigned long long s_prof[4];
  const Lev la{s_lev, w.lev_a}, lb{s_lev + kLevShared, w.lev_b};
  const unsigned long long t0 = rcm_clock();
  if (threadIdx.x == 0) {
    s_pos = 0;
    s_prof[0] = s_prof[1] = s_prof[2] = 0;
  }
  if (start >= 0) {  // undo: the search found a more eccentric start
    for (int v = threadIdx.x; v < w.n; v += blockDim.x)
      if (w.newidx[v] >= 0) w.newidx[v] = -1;
  }
  __syncthreads();
  if (start < 0) start = rcm_min_degree(w);
  if (start < 0) return;
  Lev last;
  int last_len;
  const int lv = rcm_cm(w, la, lb, start, s_pos, s_len, &last, &last_len, s_prof);
  __syncthreads();
  if (threadIdx.x == 0) {
    w.status[0] = s_pos;
    w.status[2] += 1;
    w.status[3] += lv;
    w.status[4] += (int)((rcm_clock() - t0) / 1000);
    w.status[6] += (int)(s_prof[0] / 1000);
    w.status[7] += (int)(s_prof[1] / 1000);
    w.status[8] += (int)(s_prof[2] / 1000);
  }
}

// The remaining components, from position status[0] on (see above).
__global__ void __launch_bounds__(kRcmThreads) k_rcm(RcmWork w) {
  extern __shared__ int s_lev[];  // 2 * kLevShared
  __shared__ int s_len;
  __shared__ int s_pos;
  const Lev la{s_lev, w.lev_a}, lb{s_lev + kLevShared, w.lev_b};
  int stamp = 1 << 20;  // above the search kernel's stamps
  int walks = 0;         // breadth-first and Cuthill-McKee walks (counted by every thread
  long long levels = 0;  // alike; thread 0 reports them)
  unsigned long long t_cm = 0, t_bfs = 0;
  __shared__ unsigned long long s_prof[4];
  if (threadIdx.x == 0) {
    s_prof[0] = s_prof[1] = s_prof[2] = 0;
    s_pos = w.status[0];
  }
  __syncthreads();
  while (s_pos < w.n) {
    int start = rcm_min_degree(w);
    if (start < 0) break;
    const int comp_base = s_pos;
    // George-Liu pseudo-peripheral vertex.  Its first BFS, from `start`, has
    // the levels of Cuthill-McKee from `start`: order the component from
    // `start` straight away and test that order's last level.  When the
    // candidate found there has no larger eccentricity -- the usual case --
    // the order stands; otherwise it is undone and the search goes on as
    // before.
    // Every walk starts in la; rcm_pick reads the last level (in la or lb)
    // before the next walk writes over either list.
    Lev last;
    int last_len;
    unsigned long long t0 = rcm_clock();
    int ecc = rcm_cm(w, la, lb, start, s_pos, s_len, &last, &last_len, s_prof);
    unsigned long long t1 = rcm_clock();
    t_cm += t1 - t0;
    int cand = rcm_pick(w, last, last_len);
    t0 = rcm_clock();
    int e2 = rcm_bfs(w, la, lb, cand, stamp++, &last, &last_len, comp_base);
    t_bfs += rcm_clock() - t0;
    walks += 2;
    levels += ecc + e2;
    if (e2 > ecc) {
      for (int v = threadIdx.x; v < w.n; v += blockDim.x)
        if (w.newidx[v] >= comp_base) w.newidx[v] = -1;
      __syncthreads();
      if (threadIdx.x == 0) s_pos = comp_base;
      __syncthreads();
      ecc = e2;
      start = cand;
      for (int round = 1; round < 8; round++) {
        cand = rcm_pick(w, last, last_len);
        t0 = rcm_clock();
        e2 = rcm_bfs(w, la, lb, cand, stamp++, &last, &last_len);
        t_bfs += rcm_clock() - t0;
        walks++;
        levels += e2;
        if (e2 <= ecc) break;  // no longer eccentricity: keep the current start
        ecc = e2;
        start = cand;
      }
      t0 = rcm_clock();
      levels += rcm_cm(w, la, lb, start, s_pos, s_len, &last, &last_len, s_prof);
      t_cm += rcm_clock() - t0;
      walks++;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    w.status[0] = s_pos;
    w.status[2] += walks;
    w.status[3] += (int)levels;
    w.status[4] += (int)(t_cm / 1000);
    w.status[5] += (int)(t_bfs / 1000);
    w.status[6] += (int)(s_prof[0] / 1000);
    w.status[7] += (int)(s_prof[1] / 1000);
    w.status[8] += (int)(s_prof[2] / 1000);
  }
}

// reverse: perm[v] = n - 1 - CM position
__global__ void k_reverse(int n, const int *cm, int *perm) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) perm[v] = n - 1 - cm[v];
}

// ------------------------------------------------------------------ propagation

// key of each `to` element: new index of its first target
__global__ void k_first_target_key(int n, int dim, const int *map, const int *perm_from,
                                   int *key, int *cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int k = perm_from[map[(size_t)i * dim]];
  key[i] = k;
  atomicAdd(&cnt[k], 1);
}

__global__ void k_bucket_fill(int n, const int *key, const long long *start, int *fill,
                              int *order) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int k = key[i];
  order[start[k] + atomicAdd(&fill[k], 1)] = i;
}

// sort each bucket by original index (stable order); perm[order[p]] = p
__global__ void k_bucket_sort(int nkeys, const long long *start, int *order, int *perm) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nkeys) return;
  long long b = start[k], e = start[k + 1];
  for (long long i = b + 1; i < e; i++) {
    int v = order[i];
    long long j = i - 1;
    while (j >= b && order[j] > v) {
      order[j + 1] = order[j];
      j--;
    }
    order[j + 1] = v;
  }
  for (long long i = b; i < e; i++) perm[order[i]] = (int)i;
}

// first touch: the `to` element reached first when walking `from` in its new
// order, slot by slot (:101-125) -- key = new position * dim + slot
__global__ void k_first_touch(int nfrom, int dim, const int *map, const int *perm_from, int nto,
                              int *key) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nfrom) return;
  for (int d = 0; d < dim; d++) {
    int t = map[(size_t)i * dim + d];
    if (t >= 0 && t < nto) atomicMin(&key[t], (int)((long long)perm_from[i] * dim + d));
  }
}

// elements of the target set no map entry reached (key still the memset
// pattern 0x7f7f7f7f), one atomic a warp
__global__ void k_count_unreached(int n, const int *key, int *missing) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool miss = i < n && key[i] == 0x7f7f7f7f;
  const unsigned b = __ballot_sync(0xffffffffu, miss);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(missing, __popc(b));
}

__global__ void k_flag_keys(int n, const int *key, int *flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[key[i]] = 1;
}

__global__ void k_rank_keys(int n, const int *key, const long long *pos, int *perm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) perm[i] = (int)pos[key[i]];
}

// ------------------------------------------------------------------ reordering

__global__ void k_move_rows(int n, int words, const int *src, int *dst, const int *perm) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * words) return;
  long long i = t / words, w = t % words;
  dst[(size_t)perm[i] * words + w] = src[t];
}

__global__ void k_renumber_entries(long long m, int *map, const int *perm) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < m) map[t] = perm[map[t]];
}

__global__ void k_gather_rows(int n, int words, const int *src, int *dst, const int *perm,
                              int low) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * words) return;
  long long j = t / words, w = t % words;
  dst[t] = src[(size_t)perm[low + j] * words + w];
}

// ------------------------------------------------------------------ host

struct Renumbering {
  std::map<int, int *> perm_d;  // set index -> device permutation (original -> current)
};

static Renumbering &ren() {
  static Renumbering r;
  return r;
}

static inline unsigned grid1(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// bandwidth statistics of a map (op_renumber's diagnostics): per element the
// largest difference between two of its targets; out[0] = max, out[1] = sum
__global__ void k_map_bandwidth(int n, int dim, const int *__restrict__ map,
                                unsigned long long *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  long long dist = 0;
  if (i < n) {
    const int *row = map + (size_t)i * dim;
    int lo = row[0], hi = row[0];
    for (int a = 1; a < dim; a++) {
      lo = min(lo, row[a]);
      hi = max(hi, row[a]);
    }
    dist = (long long)hi - lo;
  }
  unsigned long long mx = (unsigned long long)dist, sum = (unsigned long long)dist;
  for (int o = 16; o > 0; o >>= 1) {
    mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
    sum += __shfl_down_sync(0xffffffffu, sum, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, mx);
    atomicAdd(out + 1, sum);
  }
}

// RCM order of the base map's target set; perm[v] = new index of v
static bool base_rcm(op_map base, int *perm_d, cudaStream_t s) {
  op_set to = base->to;
  int n = to->size;
  std::vector<void *> tmp;
  auto A = [&](size_t bytes) {
    void *p = nullptr;
    if (cudaMallocAsync(&p, bytes ? bytes : 1, s) != cudaSuccess) return (void *)nullptr;
    tmp.push_back(p);
    return p;
  };
  auto cleanup = [&]() {
    cudaStreamSynchronize(s);
    for (void *p : tmp) cudaFreeAsync(p, s);
  };
  int *deg = (int *)A(sizeof(int) * (n + 1));
  long long *row = (long long *)A(sizeof(long long) * (n + 1));
  int *col = nullptr;
  if (!deg || !row) return cleanup(), false;
  cudaMemsetAsync(deg, 0, sizeof(int) * (n + 1), s);
  if (base->from == to) {
    col = (int *)A(sizeof(int) * (size_t)n * base->dim);
    k_adj_self<<<grid1(n), 256, 0, s>>>(n, base->dim, base->map_d, deg, col);
    // rows are dim apart
    std::vector<long long> h(n + 1);
    for (int u = 0; u <= n; u++) h[u] = (long long)u * base->dim;
    cudaMemcpyAsync(row, h.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
  } else {
    int nf = base->from->size;
    k_adj_count<<<grid1(nf), 256, 0, s>>>(nf, base->dim, base->map_d, n, deg);
    if (!scan_exclusive(deg, row, n, s)) return cleanup(), false;
    long long nnz = 0;
    cudaMemcpy(&nnz, row + n, sizeof(long long), cudaMemcpyDeviceToHost);
    col = (int *)A(sizeof(int) * (size_t)std::max(nnz, 1LL));
    int *fill = (int *)A(sizeof(int) * n);
    cudaMemsetAsync(fill, 0, sizeof(int) * n, s);
    k_adj_fill<<<grid1(nf), 256, 0, s>>>(nf, base->dim, base->map_d, n, row, fill, col);
  }
  k_adj_unique<<<grid1(n), 256, 0, s>>>(n, row, col, deg);
  RcmWork w{};
  w.n = n;
  w.row = row;
  w.deg = deg;
  w.col = col;
  int4 *ell = (int4 *)A(sizeof(int4) * n);
  w.ell = ell;
  w.newidx = (int *)A(sizeof(int) * n);
  w.mark = (int *)A(sizeof(int) * n);
  w.lev_a = (int *)A(sizeof(int) * n);
  w.lev_b = (int *)A(sizeof(int) * n);
  w.pkey = (int *)A(sizeof(int) * n);
  w.status = (int *)A(sizeof(int) * 9);
  int *lev_c = (int *)A(sizeof(int) * n), *lev_d = (int *)A(sizeof(int) * n);
  int *search = (int *)A(sizeof(int) * 5);
  if (!ell || !w.newidx || !w.mark || !w.lev_a || !w.lev_b || !w.pkey || !w.status || !lev_c ||
      !lev_d || !search)
    return cleanup(), false;
  k_adj_ell<<<grid1(n), 256, 0, s>>>(n, row, deg, col, ell);
  cudaMemsetAsync(w.newidx, 0xff, sizeof(int) * n, s);
  cudaMemsetAsync(w.mark, 0, sizeof(int) * n, s);
  cudaMemsetAsync(w.pkey, 0x7f, sizeof(int) * n, s);  // 0x7f7f7f7f > any position
  cudaMemsetAsync(w.status, 0, sizeof(int) * 9, s);
  cudaMemsetAsync(search, 0xff, sizeof(int) * 5, s);
  // pkey must read as "none": 0x7f7f7f7f is used as the no-parent value
  for (const void *kern : {(const void *)k_rcm, (const void *)k_rcm_first,
                           (const void *)k_rcm_search})
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRcmSmem) !=
        cudaSuccess) {
      cudaGetLastError();
      set_error("op_renumber: %zu bytes of shared memory refused", kRcmSmem);
      return cleanup(), false;
    }
  // the first component: the search on a second stream beside the ordering
  cudaStream_t aux = nullptr;
  cudaEvent_t ready = nullptr, found = nullptr;
  bool ok = cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&found, cudaEventDisableTiming) == cudaSuccess;
  int sr[5] = {-1, -1, 0, 0, 0};
  if (ok) {
    cudaEventRecord(ready, s);
    cudaStreamWaitEvent(aux, ready, 0);
    k_rcm_search<<<1, kRcmThreads, kRcmSmem, aux>>>(w, lev_c, lev_d, search);
    cudaEventRecord(found, aux);
    k_rcm_first<<<1, kRcmThreads, kRcmSmem, s>>>(w, -1);
    // the host copies of the reordered maps and dats come next: their pinned
    // staging buffers are pinned while the device orders
    if (rt().opt_host_mirror) stage_in_background();
    cudaStreamWaitEvent(s, found, 0);
    cudaMemcpyAsync(sr, search, sizeof(sr), cudaMemcpyDeviceToHost, s);
    ok = cudaStreamSynchronize(s) == cudaSuccess;
  }
  if (ok && sr[0] >= 0 && sr[0] != sr[1])  // a more eccentric start: order from it
    k_rcm_first<<<1, kRcmThreads, kRcmSmem, s>>>(w, sr[0]);
  if (ok) k_rcm<<<1, kRcmThreads, kRcmSmem, s>>>(w);  // the other components
  if (ok) k_reverse<<<grid1(n), 256, 0, s>>>(n, w.newidx, perm_d);
  int st[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (ok) cudaMemcpyAsync(st, w.status, sizeof(st), cudaMemcpyDeviceToHost, s);
  ok = ok && cudaStreamSynchronize(s) == cudaSuccess && st[0] == n;
  if (!ok) {
    cudaGetLastError();
    set_error("op_renumber: reverse Cuthill-McKee ordered %d of %d elements", st[0], n);
  }
  if (ok && rt().opt_diags > 2)
    fprintf(stderr, "op_renumber: Cuthill-McKee %d walks, %d levels, %d us ordering (small "
            "levels: %d us claims, %d us counts, %d us placing), %d us searching after; first "
            "component searched beside the ordering: %d walks, %d levels, %d us%s\n",
            st[2], st[3], st[4], st[6], st[7], st[8], st[5], sr[2], sr[3], sr[4],
            sr[0] != sr[1] ? " (start moved)" : "");
  if (aux) {
    cudaStreamSynchronize(aux);
    cudaStreamDestroy(aux);
  }
  if (ready) cudaEventDestroy(ready);
  if (found) cudaEventDestroy(found);
  cleanup();
  return ok;
}

// propagate_reordering (:72-151)
static void propagate(op_set from, op_set to, std::vector<int *> &perm, cudaStream_t s,
                      bool &ok) {
  Runtime &r = rt();
  if (!ok || to->size == 0) return;
  int n = to->size;
  if (!perm[to->index]) {
    for (auto &mp : r.maps) {  // a map to -> from: sort by first target's new index
      op_map m = mp.get();
      if (!m || m->to != from || m->from != to) continue;
      int *key, *cnt, *fill, *order, *pd;
      long long *start;
      int nk = from->size;
      cudaMallocAsync(&key, sizeof(int) * n, s);
      cudaMallocAsync(&cnt, sizeof(int) * (nk + 1), s);
      cudaMallocAsync(&fill, sizeof(int) * (nk + 1), s);
      cudaMallocAsync(&order, sizeof(int) * n, s);
      cudaMallocAsync(&start, sizeof(long long) * (nk + 1), s);
      cudaMallocAsync(&pd, sizeof(int) * n, s);
      cudaMemsetAsync(cnt, 0, sizeof(int) * (nk + 1), s);
      cudaMemsetAsync(fill, 0, sizeof(int) * (nk + 1), s);
      k_first_target_key<<<grid1(n), 256, 0, s>>>(n, m->dim, m->map_d, perm[from->index], key, cnt);
      ok = scan_exclusive(cnt, start, nk, s);
      k_bucket_fill<<<grid1(n), 256, 0, s>>>(n, key, start, fill, order);
      k_bucket_sort<<<grid1(nk), 256, 0, s>>>(nk, start, order, pd);
      ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
      cudaFreeAsync(key, s);
      cudaFreeAsync(cnt, s);
      cudaFreeAsync(fill, s);
      cudaFreeAsync(order, s);
      cudaFreeAsync(start, s);
      perm[to->index] = pd;
      break;
    }
  }
  if (!perm[to->index]) {
    for (auto &mp : r.maps) {  // a map from -> to covering `to`: first touch
      op_map m = mp.get();
      if (!m || m->to != to || m->from != from) continue;
      int *key, *flag, *missing, *pd;
      long long *pos;
      long long nslots = (long long)from->size * m->dim;
      cudaMallocAsync(&key, sizeof(int) * n, s);
      cudaMallocAsync(&flag, sizeof(int) * (nslots + 1), s);
      cudaMallocAsync(&missing, sizeof(int), s);
      cudaMallocAsync(&pos, sizeof(long long) * (nslots + 1), s);
      cudaMemsetAsync(key, 0x7f, sizeof(int) * n, s);
      cudaMemsetAsync(flag, 0, sizeof(int) * (nslots + 1), s);
      cudaMemsetAsync(missing, 0, sizeof(int), s);
      // 0x7f7f7f7f stands for "not reached"; map the sentinel to INT_MAX
      k_first_touch<<<grid1(from->size), 256, 0, s>>>(from->size, m->dim, m->map_d,
                                                       perm[from->index], n, key);
      int nmiss = 0;
      k_count_unreached<<<grid1(n), 256, 0, s>>>(n, key, missing);
      cudaMemcpyAsync(&nmiss, missing, sizeof(int), cudaMemcpyDeviceToHost, s);
      cudaStreamSynchronize(s);
      if (nmiss) {  // not onto: try the next map (:113-117)
        cudaFreeAsync(key, s);
        cudaFreeAsync(flag, s);
        cudaFreeAsync(missing, s);
        cudaFreeAsync(pos, s);
        continue;
      }
      k_flag_keys<<<grid1(n), 256, 0, s>>>(n, key, flag);
      ok = scan_exclusive(flag, pos, nslots, s);
      cudaMallocAsync(&pd, sizeof(int) * n, s);
      k_rank_keys<<<grid1(n), 256, 0, s>>>(n, key, pos, pd);
      ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
      cudaFreeAsync(key, s);
      cudaFreeAsync(flag, s);
      cudaFreeAsync(missing, s);
      cudaFreeAsync(pos, s);
      perm[to->index] = pd;
      break;
    }
  }
  if (!perm[to->index]) return;
  for (auto &mp : r.maps) {  // maps (*) -> to
    op_map m = mp.get();
    if (m && m->to == to && !perm[m->from->index]) propagate(to, m->from, perm, s, ok);
  }
  for (auto &mp : r.maps) {  // maps to -> (*)
    op_map m = mp.get();
    if (m && m->from == to && !perm[m->to->index]) propagate(to, m->to, perm, s, ok);
  }
}

// maximum and average over elements of the largest distance between two
// targets of one element (the figures op_renumber prints, :489-503), on the
// device from the map's device copy
static bool bandwidth(op_map base, long &mx, long &avg, cudaStream_t s) {
  mx = 0;
  avg = 0;
  const int n = base->from->size;
  if (n == 0) return true;
  Runtime &r = rt();
  unsigned long long *out = r.check_d + 1;  // two words of the runtime's check scratch
  unsigned long long h[2] = {0, 0};
  cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), s);
  k_map_bandwidth<<<grid1(n), 256, 0, s>>>(n, base->dim, base->map_d, out);
  cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return false;
  mx = (long)h[0];
  avg = (long)(h[1] / (unsigned long long)n);
  return true;
}

int renumber(op_map base, long stats[4]) {
  if (!rt().overlays.empty()) {
    set_error("op_renumber: overlay dats share storage across sets; renumber before "
              "declaring them");
    return -1;
  }
  Runtime &r = rt();
  if (!r.ready()) return -1;
  if (!base || !base->map_d) {
    set_error("op_renumber: invalid base map");
    return -1;
  }
  cudaStream_t s = r.stream;
  cudaStreamSynchronize(s);
  const auto t_begin = std::chrono::steady_clock::now();
  auto t_last = t_begin;
  auto lap = [&](const char *what) {  // phase times with diags > 2
    if (r.opt_diags <= 2) return;
    cudaStreamSynchronize(s);
    const auto now = std::chrono::steady_clock::now();
    fprintf(stderr, "op_renumber: %-22s %8.2f ms\n", what,
            std::chrono::duration<double, std::milli>(now - t_last).count());
    t_last = now;
  };
  // Reserve the temporaries' memory in the stream-ordered pool with one
  // allocation: the many allocations below are then carved from it instead of
  // each asking the driver (whose calls are slow and of uneven cost on a
  // device shared with other processes).  The estimate covers the graph and
  // Cuthill-McKee work arrays, the propagation keys and the largest moved row.
  {
    size_t nt = (size_t)base->to->size, nf = (size_t)base->from->size, d = (size_t)base->dim;
    size_t largest = 0;
    for (auto &dp : r.dats)
      if (dp) largest = std::max(largest, (size_t)dp->set->size * (size_t)dp->size);
    for (auto &mp : r.maps)
      if (mp) largest = std::max(largest, (size_t)mp->from->size * (size_t)mp->dim * sizeof(int));
    const size_t est = 64 * nt + 4 * nf * d * (d > 1 ? d - 1 : 1) + 32 * nf + largest;
    void *reserve = nullptr;
    if (cudaMallocAsync(&reserve, est, s) == cudaSuccess) cudaFreeAsync(reserve, s);
    else cudaGetLastError();  // no reservation: the allocations below ask one by one
  }
  // the base map's bandwidth before and after: for the caller's statistics
  // and the diagnostics only
  const bool want_bw = stats != nullptr || r.opt_diags > 1;
  long bmx = 0, bavg = 0;
  if (want_bw) bandwidth(base, bmx, bavg, s);
  lap("bandwidth before");
  std::vector<int *> perm(r.sets.size(), nullptr);
  op_set to = base->to;
  int *pb = nullptr;
  if (cudaMallocAsync(&pb, sizeof(int) * std::max(to->size, 1), s) != cudaSuccess) {
    set_error("op_renumber: out of device memory");
    return -1;
  }
  perm[to->index] = pb;
  if (!base_rcm(base, pb, s)) {
    cudaFree(pb);
    return -1;
  }
  lap("reverse Cuthill-McKee");
  bool ok = true;
  propagate(to, to, perm, s, ok);
  lap("propagation");
  if (!ok) {
    set_error("op_renumber: propagation failed");
    for (int *p : perm) cudaFree(p);
    return -1;
  }
  // reorder_set (:153-222) for every set that received a permutation
  for (auto &sp : r.sets) {
    op_set set = sp.get();
    if (!set || !perm[set->index] || set->size == 0) continue;
    const int *pd = perm[set->index];
    for (auto &mp : r.maps) {
      op_map m = mp.get();
      if (!m || !m->map_d) continue;
      if (m->from == set) {
        int *t;
        size_t bytes = sizeof(int) * (size_t)set->size * m->dim;
        cudaMallocAsync(&t, bytes, s);
        k_move_rows<<<grid1((long long)set->size * m->dim), 256, 0, s>>>(set->size, m->dim, m->map_d,
                                                                          t, pd);
        cudaMemcpyAsync(m->map_d, t, bytes, cudaMemcpyDeviceToDevice, s);
        cudaFreeAsync(t, s);
      }
    }
    for (auto &mp : r.maps) {
      op_map m = mp.get();
      if (!m || !m->map_d || m->to != set) continue;
      long long cnt = (long long)m->from->size * m->dim;
      k_renumber_entries<<<grid1(cnt), 256, 0, s>>>(cnt, m->map_d, pd);
    }
    for (auto &dp : r.dats) {
      op_dat d = dp.get();
      if (!d || d->set != set || !d->data_d) continue;
      if (d->size % 4) {
        set_error("op_renumber: dat %s has elements of %d bytes (not a multiple of 4)", d->name,
                  d->size);
        ok = false;
        continue;
      }
      int words = d->size / 4;
      size_t bytes = (size_t)set->size * d->size;
      int *t;
      cudaMallocAsync(&t, bytes, s);
      k_move_rows<<<grid1((long long)set->size * words), 256, 0, s>>>(
          set->size, words, reinterpret_cast<const int *>(d->data_d), t, pd);
      cudaMemcpyAsync(d->data_d, t, bytes, cudaMemcpyDeviceToDevice, s);
      cudaFreeAsync(t, s);
    }
  }
  lap("reordering");
  // host copies of the maps, and of the dats on reordered sets, follow the
  // device (the reference reorders dat->data and map->map on the host,
  // op_renumber.cpp:180-200)
  std::vector<HostDownload> mirrors;
  for (auto &mp : r.maps) {
    op_map m = mp.get();
    if (m && m->map_d && m->map)
      mirrors.push_back({m->map, m->map_d, sizeof(int) * (size_t)m->from->size * m->dim});
  }
  for (auto &dp : r.dats) {
    op_dat d = dp.get();
    // (a copy of zeros stays zeros in any order)
    if (d && d->data && d->data_d && perm[d->set->index] && !r.zero_mirror.count(d))
      mirrors.push_back({d->data, d->data_d, (size_t)d->set->size * d->size});
  }
  ok &= download_host_many(mirrors, "op_renumber: host copies of maps and dats");
  // compose with earlier renumberings: original -> current
  for (auto &sp : r.sets) {
    op_set set = sp.get();
    if (!set || !perm[set->index]) continue;
    auto it = ren().perm_d.find(set->index);
    if (it == ren().perm_d.end()) {
      ren().perm_d[set->index] = perm[set->index];
    } else {
      // current = perm[old current]
      long long n = set->size;
      int *t = it->second;
      k_renumber_entries<<<grid1(n), 256, 0, s>>>(n, t, perm[set->index]);
      cudaFreeAsync(perm[set->index], s);
    }
  }
  lap("host maps, composition");
  release_plans();  // plans and inverse maps refer to the old numbering
  release_inverse_maps();
  bool good = cuda_ok(cudaStreamSynchronize(s), "op_renumber") && ok;
  long amx = 0, aavg = 0;
  if (want_bw) bandwidth(base, amx, aavg, s);
  lap("release, bandwidth after");
  if (stats) {
    stats[0] = bmx;
    stats[1] = bavg;
    stats[2] = amx;
    stats[3] = aavg;
  }
  if (r.opt_diags > 1) {
    printf("Before renumbering: maximum bandwidth = %ld average bandwidth = %ld\n", bmx, bavg);
    printf("After renumbering: maximum bandwidth = %ld average bandwidth = %ld\n", amx, aavg);
  }
  return good ? 0 : -1;
}

void resolve_renumbering_for_fetch(op_dat) {}

void fetch_original_order(op_dat dat, char *dst, int low, int high) {
  Runtime &r = rt();
  if (!r.ready() || high < low) return;
  size_t cnt = (size_t)(high - low + 1);
  size_t bytes = cnt * dat->size;
  auto it = ren().perm_d.find(dat->set->index);
  if (it == ren().perm_d.end() || dat->size % 4) {
    download_host(dst, dat->data_d + (size_t)low * dat->size, bytes, "op_fetch_data_idx");
    return;
  }
  int *t = nullptr;
  if (!cuda_ok(cudaMallocAsync(&t, bytes, r.stream), "op_fetch_data_idx")) return;
  int words = dat->size / 4;
  k_gather_rows<<<grid1((long long)cnt * words), 256, 0, r.stream>>>(
      (int)cnt, words, reinterpret_cast<const int *>(dat->data_d), t, it->second, low);
  download_host(dst, t, bytes, "op_fetch_data_idx");
  cudaFreeAsync(t, r.stream);
}

void release_renumbering() {
  for (auto &kv : ren().perm_d) cudaFree(kv.second);
  ren().perm_d.clear();
}

int set_permutation(op_set set, int *host_perm) {
  auto it = ren().perm_d.find(set->index);
  if (it == ren().perm_d.end()) {
    for (int i = 0; i < set->size; i++) host_perm[i] = i;
    return 1;
  }
  return cuda_ok(cudaMemcpy(host_perm, it->second, sizeof(int) * (size_t)set->size,
                            cudaMemcpyDeviceToHost),
                 "op2b_set_permutation")
             ? 0
             : -1;
}

}  // namespace op2b

using namespace op2b;

extern "C" {

void op_renumber(op_map base) {
  if (renumber(base, nullptr) != 0 && !rt().opt_abort)
    fprintf(stderr, "op2b: %s\n", op2b_last_error());
}

void op_renumber_ptr(int *ptr) {
  auto it = rt().map_ptrs.find(ptr);
  if (it == rt().map_ptrs.end()) {
    set_error("op_renumber: op_map not found for %p pointer", (void *)ptr);
    fprintf(stderr, "op2b: %s\n", op2b_last_error());
    return;
  }
  op_renumber(it->second);
}

int op2b_renumber(op_map base, long stats[4]) { return renumber(base, stats); }

int op2b_set_permutation(op_set set, int *perm) {
  if (!set || !perm) {
    set_error("op2b_set_permutation: invalid arguments");
    return -1;
  }
  return set_permutation(set, perm);
}

}  // extern "C"
