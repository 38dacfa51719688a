// BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a) with FP32
// accumulation in tensor memory, for the learned warm start's MLPs.
//
//   C[M x N] = sum_k A(m, k) * B(n, k)          (A, B bf16; accumulate FP32)
//
// One CTA of 128 threads computes a 128 x NT tile (NT <= 128, multiple of 16):
//   * tensor memory: warp 0 allocates 128 columns; accumulator row m sits in
//     TMEM lane m, column n in TMEM column n (M = 128, cta_group::1);
//   * K is walked in tiles of 64; the CTA stages 16-byte chunks of A and B
//     from global memory into shared memory in the K-major layout with the
//     128-byte swizzle (one 128-byte row of 64 bf16 per tile row, 8-row
//     groups 1024 B apart, 16-byte chunks XOR-permuted by the row); a
//     transposed operand is transposed in registers on the way;
//   * two shared-memory stages: while the tensor core consumes one, the CTA
//     fills the other; one thread issues four tcgen05.mma (K = 16 each) per
//     tile and a tcgen05.commit to the stage's mbarrier, which the CTA waits
//     on before refilling that stage;
//   * epilogue: warp w reads rows 32w..32w+31 from TMEM (tcgen05.ld 32x32b,
//     16 columns at a time) and applies bias / SiLU / SiLU' / residual /
//     split-K atomics before storing.
// Every mbarrier wait is bounded in time (%globaltimer): on expiry the kernel
// records an error, stops issuing, waits (bounded) for its outstanding
// commits, frees its tensor memory and returns.
#include <algorithm>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "op2b_gnn.h"
#include "op2b_runtime.h"

namespace op2b {
namespace {

constexpr int kTileM = 128;
constexpr int kTileN = 128;
constexpr int kTileK = 64;
constexpr int kThreads = 128;
constexpr int kStageBytes = kTileM * kTileK * 2;  // one operand tile (16 KiB)
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s per mbarrier wait

// i over the first n of 16 columns, unrolled so per-column arrays stay in registers
#define FOR_LT_N(i) _Pragma("unroll") for (int i = 0; i < 16; i++) if (i < n)

struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16 *A;
  long a_m, a_k;
  const __nv_bfloat16 *B;
  long b_n, b_k;
  void *C;
  long ldc;
  const float *bias;
  __nv_bfloat16 *Z;
  const __nv_bfloat16 *R;
  long ldr;
  int epi;
  int k_per_split;
  int *err;
  int staged;  // k_gemm_ws<16>: C (and Z) 16-byte aligned rows: stores through shared memory
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// shared-memory matrix descriptor, version 1 (sm_100), K-major with the
// 128-byte swizzle (layout type 2 in bits 61-63): start address >> 4 in bits
// 0-13, leading byte offset >> 4 in 16-29 (unused by a swizzled K-major
// operand whose K step fits in the 128-byte row; 1 by convention), stride
// byte offset >> 4 in 32-45 (1024: the distance between 8-row groups)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// The same descriptor for an MN-major operand tile (128 MN x 64 K) as TMA
// writes it with the 128-byte swizzle: two boxes of 64 MN x 64 K, 8 KiB
// apart, each 64 rows of 128 bytes (64 MN values of one k) in 1024-byte
// groups of 8 rows.  In the canonical MN-major layout ((8,n),(8,k)) :
// ((1,LBO),(8,SBO)) in 16-byte units the leading byte offset is the 8 KiB
// between the two 64-wide MN blocks and the stride byte offset the 1024 bytes
// between groups of 8 k; a K step of 16 starts 2048 bytes further on.
__device__ __forceinline__ uint64_t umma_desc_mn(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)(8192 >> 4) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and B
// bf16 (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 in
// bits 17-22, M >> 4 in bits 24-28
__device__ __forceinline__ uint32_t umma_idesc(int nt) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nt >> 3) << 17) |
         ((uint32_t)(kTileM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while (!mbar_try(bar, parity))
    if (globaltimer() - t0 > kWaitNs) return false;
  return true;
}

// SiLU and its derivative with the fast exponential and division (a few
// ulp in FP32; the results are rounded to BF16).  Below z = -87 the
// denominator passes 2^126 and the fast division gives 0, as the values
// round to next to nothing anyway.
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = __fdividef(1.0f, 1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// bias[col .. col + n) into v (16-byte loads when aligned)
__device__ __forceinline__ void add_bias16(float *v, const float *bias, int col, int n) {
  const float *b = bias + col;
  if (n == 16 && (reinterpret_cast<uintptr_t>(b) & 15) == 0) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const float4 t = __ldg(reinterpret_cast<const float4 *>(b) + i);
      v[4 * i] += t.x;
      v[4 * i + 1] += t.y;
      v[4 * i + 2] += t.z;
      v[4 * i + 3] += t.w;
    }
  } else {
    FOR_LT_N(i) v[i] += b[i];
  }
}

// Shared-memory tile layout: K-major with the 128-byte swizzle.  Row r of the
// 128 x 64 tile is 128 bytes (64 bf16) at (r / 8) * 1024 + (r % 8) * 128; its
// 16-byte chunk j (k = 8j .. 8j+7) sits at chunk position j ^ (r % 8).  The
// XOR spreads both the k-contiguous and the transposed staging stores over
// all 32 banks; the tensor core undoes it from the descriptor's swizzle mode.
__device__ __forceinline__ uint32_t sw128(int row, int kc) {
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((kc ^ (row & 7)) << 4));
}

// Stage one operand tile (128 rows x 64 k); rows >= nrows and k >= kend read
// as zero.
__device__ __forceinline__ void stage_tile(uint8_t *dst, const __nv_bfloat16 *src, long s_row,
                                           long s_k, int row0, int nrows, int k0, int kend) {
  if (s_k == 1) {  // k contiguous: one 16-byte chunk = 8 k values of one row
    uint4 v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int c = threadIdx.x + i * kThreads;
      const int row = c >> 3, kc = c & 7;
      const int gr = row0 + row, gk = k0 + kc * 8;
      v[i] = make_uint4(0, 0, 0, 0);
      if (gr < nrows && gk < kend)
        v[i] = __ldg(reinterpret_cast<const uint4 *>(src + (long)gr * s_row + gk));
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int c = threadIdx.x + i * kThreads;
      *reinterpret_cast<uint4 *>(dst + sw128(c >> 3, c & 7)) = v[i];
    }
  } else {
    // rows contiguous: thread (rc, kc) loads the 8 x 8 block of rows
    // 8rc..8rc+7 and k 8kc..8kc+7 (eight 16-byte loads, one per k), transposes
    // it in registers and stores eight 16-byte row chunks
    const int kc = threadIdx.x & 7, rc = threadIdx.x >> 3;
    const int gr = row0 + rc * 8;
    uint32_t in[8][4];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int gk = k0 + kc * 8 + j;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (gk < kend && gr < nrows)
        v = __ldg(reinterpret_cast<const uint4 *>(src + (long)gk * s_k + gr));
      in[j][0] = v.x, in[j][1] = v.y, in[j][2] = v.z, in[j][3] = v.w;
    }
    // in[j] word w = (row 2w, row 2w+1) of k j; out[r] word w = (k 2w, k 2w+1) of row r
#pragma unroll
    for (int r2 = 0; r2 < 4; r2++) {
      uint32_t lo[4], hi[4];
#pragma unroll
      for (int w = 0; w < 4; w++) {
        lo[w] = __byte_perm(in[2 * w][r2], in[2 * w + 1][r2], 0x5410);
        hi[w] = __byte_perm(in[2 * w][r2], in[2 * w + 1][r2], 0x7632);
      }
      *reinterpret_cast<uint4 *>(dst + sw128(rc * 8 + 2 * r2, kc)) =
          make_uint4(lo[0], lo[1], lo[2], lo[3]);
      *reinterpret_cast<uint4 *>(dst + sw128(rc * 8 + 2 * r2 + 1, kc)) =
          make_uint4(hi[0], hi[1], hi[2], hi[3]);
    }
  }
}

__device__ __forceinline__ void store_bf16x16(__nv_bfloat16 *dst, const float *v, int n) {
  if (n == 16 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
    uint4 w[2];
    __nv_bfloat162 *p = reinterpret_cast<__nv_bfloat162 *>(w);
#pragma unroll
    for (int i = 0; i < 8; i++) p[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    reinterpret_cast<uint4 *>(dst)[0] = w[0];
    reinterpret_cast<uint4 *>(dst)[1] = w[1];
  } else {
    FOR_LT_N(i) dst[i] = __float2bfloat16(v[i]);
  }
}

__device__ __forceinline__ void load_bf16x16(const __nv_bfloat16 *src, float *v, int n) {
  if (n == 16 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
    uint4 w[2];
    w[0] = reinterpret_cast<const uint4 *>(src)[0];
    w[1] = reinterpret_cast<const uint4 *>(src)[1];
    const __nv_bfloat162 *p = reinterpret_cast<const __nv_bfloat162 *>(w);
#pragma unroll
    for (int i = 0; i < 8; i++) {
      float2 f = __bfloat1622float2(p[i]);
      v[2 * i] = f.x;
      v[2 * i + 1] = f.y;
    }
  } else {
    FOR_LT_N(i) v[i] = __bfloat162float(src[i]);
  }
}

__device__ void epilogue16(const GemmArgs &g, int row, int col, const uint32_t *r) {
  const int n = min(16, g.N - col);
  if (n <= 0) return;
  float v[16];
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
  const long o = (long)row * g.ldc + col;
  switch (g.epi) {
    case OP2B_EPI_STORE_F32: {
      float *c = reinterpret_cast<float *>(g.C) + o;
      if (g.bias) add_bias16(v, g.bias, col, n);
      if (n == 16 && (reinterpret_cast<uintptr_t>(c) & 15) == 0) {
#pragma unroll
        for (int i = 0; i < 4; i++)
          reinterpret_cast<float4 *>(c)[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2],
                                                         v[4 * i + 3]);
      } else {
        FOR_LT_N(i) c[i] = v[i];
      }
      return;
    }
    case OP2B_EPI_ATOMIC_F32: {
      float *c = reinterpret_cast<float *>(g.C) + o;
      FOR_LT_N(i) atomicAdd(c + i, v[i]);
      return;
    }
    case OP2B_EPI_BIAS_BF16: {
      if (g.bias) add_bias16(v, g.bias, col, n);
      if (g.R) {
        float rr[16];
        load_bf16x16(g.R + (long)row * g.ldr + col, rr, n);
        FOR_LT_N(i) v[i] += rr[i];
      }
      store_bf16x16(reinterpret_cast<__nv_bfloat16 *>(g.C) + o, v, n);
      return;
    }
    case OP2B_EPI_BIAS_SILU_BF16: {
      if (g.bias) add_bias16(v, g.bias, col, n);
      if (g.Z) store_bf16x16(g.Z + o, v, n);
      FOR_LT_N(i) v[i] = silu(v[i]);
      store_bf16x16(reinterpret_cast<__nv_bfloat16 *>(g.C) + o, v, n);
      return;
    }
    case OP2B_EPI_SILU_GRAD_BF16: {
      float z[16];
      load_bf16x16(g.R + (long)row * g.ldr + col, z, n);
      FOR_LT_N(i) v[i] *= silu_grad(z[i]);
      store_bf16x16(reinterpret_cast<__nv_bfloat16 *>(g.C) + o, v, n);
      return;
    }
    default:
      store_bf16x16(reinterpret_cast<__nv_bfloat16 *>(g.C) + o, v, n);
  }
}

__global__ void __launch_bounds__(kThreads, 1) k_gemm_tc(GemmArgs g) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ uint32_t s_taddr;
  __shared__ int s_fail;
  // the swizzle pattern repeats every 1024 bytes of shared address: align the
  // tiles to it (the launch reserves 1 KiB of slack)
  uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * kTileN;
  const int rem = g.N - n0;
  const int nt = rem >= kTileN ? kTileN : ((rem + 15) & ~15);
  const int kb = blockIdx.z * g.k_per_split;
  const int ke = min(g.K, kb + g.k_per_split);
  const int nk = ke > kb ? (ke - kb + kTileK - 1) / kTileK : 0;
  uint8_t *sA[2] = {smem, smem + 2 * kStageBytes};
  uint8_t *sB[2] = {smem + kStageBytes, smem + 3 * kStageBytes};
  const uint32_t bar[2] = {smem_u32(&bars[0]), smem_u32(&bars[1])};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    mbar_init(bar[0], 1);
    mbar_init(bar[1], 1);
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_taddr)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = s_taddr;
  const uint32_t idesc = umma_idesc(nt);
  uint32_t phase[2] = {0u, 0u};
  int pending[2] = {0, 0};  // commits on each stage not yet waited for
  int issued = 0;

  for (int kt = 0; kt < nk; kt++) {
    const int s = kt & 1;
    if (pending[s]) {  // the MMAs of tile kt-2 read this stage
      if (!mbar_wait(bar[s], phase[s])) s_fail = 1;
      phase[s] ^= 1u;
      pending[s] = 0;
    }
    __syncthreads();
    if (s_fail) break;
    const int k0 = kb + kt * kTileK;
    stage_tile(sA[s], g.A, g.a_m, g.a_k, m0, g.M, k0, ke);
    stage_tile(sB[s], g.B, g.b_n, g.b_k, n0, g.N, k0, ke);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(sA[s]), b0 = smem_u32(sB[s]);
#pragma unroll
      for (int j = 0; j < kTileK / 16; j++) {
        // K step j = 16 bf16 = 32 bytes along the (swizzled) 128-byte rows
        const uint64_t da = umma_desc(a0 + j * 32);
        const uint64_t db = umma_desc(b0 + j * 32);
        const uint32_t acc = (kt > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr),
            "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              bar[s])
          : "memory");
    }
    pending[s] = 1;
    issued = kt + 1;
  }
  // drain: wait for every commit not yet waited for (the later one covers all
  // earlier MMAs, but each arrival must land before the CTA exits)
  for (int i = 0; i < 2; i++) {
    const int s = (issued + i) & 1;  // older stage first
    if (pending[s]) {
      if (!mbar_wait(bar[s], phase[s])) s_fail = 1;
      pending[s] = 0;
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (!s_fail) {
    const int row = m0 + warp * 32 + lane;
    for (int cc = 0; cc < nt; cc += 16) {
      uint32_t r[16];
      if (issued > 0) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)cc));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int i = 0; i < 16; i++) r[i] = 0u;
      }
      if (row < g.M) epilogue16(g, row, n0 + cc, r);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(128u));
  if (threadIdx.x == 0 && s_fail) atomicExch(g.err, 1);
}

// ---------------------------------------------------------------------------
// The TMA-fed form, for K-major A and B (k contiguous in both: the forward
// products X W^T of the MLPs).  Operand tiles arrive by cp.async.bulk.tensor
// (a tensor map per operand, 128-byte swizzle -- the layout the tensor core
// reads through umma_desc -- and zero fill outside the matrix) into a ring of
// kTmaStages stages, so loads run up to three K tiles ahead of the MMAs:
//   * thread 0 (producer): waits until the MMAs of the tile that last used a
//     stage have completed (the stage's "empty" mbarrier, arrived by
//     tcgen05.commit), announces the stage's bytes on its "full" mbarrier and
//     issues the two tile loads, which complete the transaction;
//   * thread 32 (MMA issuer): waits for a stage's "full" mbarrier, issues the
//     four tcgen05.mma of the K tile and commits them to the stage's "empty"
//     mbarrier; after the last tile, one more commit to "done";
//   * then all four warps read the accumulator from TMEM and run the
//     epilogue as in k_gemm_tc.
// Three stages (96 KiB) let two CTAs share an SM, so one CTA's epilogue
// overlaps the other's loads.  No multicast: every CTA loads its own tiles.
// Every wait is bounded; on expiry the kernel records the error, stops
// issuing, waits (bounded) for the loads and MMAs already issued, frees its
// tensor memory and returns.
constexpr int kTmaStages = 3;

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__global__ void __launch_bounds__(kThreads, 2)
k_gemm_tma(GemmArgs g, const __grid_constant__ CUtensorMap ta,
           const __grid_constant__ CUtensorMap tb) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[2 * kTmaStages + 1];
  __shared__ uint32_t s_taddr;
  __shared__ int s_fail, s_loaded, s_mma;
  uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * kTileN;
  const int rem = g.N - n0;
  const int nt = rem >= kTileN ? kTileN : ((rem + 15) & ~15);
  const int kb = blockIdx.z * g.k_per_split;
  const int ke = min(g.K, kb + g.k_per_split);
  const int nk = ke > kb ? (ke - kb + kTileK - 1) / kTileK : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto full = [&](int st) { return smem_u32(&bars[st]); };
  auto empty = [&](int st) { return smem_u32(&bars[kTmaStages + st]); };
  const uint32_t done = smem_u32(&bars[2 * kTmaStages]);
  auto stage_a = [&](int st) { return smem_u32(smem + (size_t)st * 2 * kStageBytes); };
  auto stage_b = [&](int st) { return smem_u32(smem + (size_t)st * 2 * kStageBytes + kStageBytes); };

  if (threadIdx.x == 0) {
    for (int st = 0; st < kTmaStages; st++) {
      mbar_init(full(st), 1);
      mbar_init(empty(st), 1);
    }
    mbar_init(done, 1);
    s_fail = 0;
    s_loaded = 0;
    s_mma = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_taddr)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = s_taddr;

  if (threadIdx.x == 0) {  // producer
    int kt = 0;
    for (; kt < nk; kt++) {
      const int st = kt % kTmaStages;
      if (kt >= kTmaStages && !mbar_wait(empty(st), (uint32_t)((kt / kTmaStages - 1) & 1))) {
        atomicExch(&s_fail, 1);
        break;
      }
      if (*(volatile int *)&s_fail) break;
      mbar_expect_tx(full(st), 2 * kStageBytes);
      const int k0 = kb + kt * kTileK;
      tma_load_2d(stage_a(st), &ta, k0, m0, full(st));
      tma_load_2d(stage_b(st), &tb, k0, n0, full(st));
    }
    *(volatile int *)&s_loaded = kt;
  } else if (threadIdx.x == 32) {  // MMA issuer
    const uint32_t idesc = umma_idesc(nt);
    int kt = 0;
    for (; kt < nk; kt++) {
      const int st = kt % kTmaStages;
      if (!mbar_wait(full(st), (uint32_t)((kt / kTmaStages) & 1))) {
        atomicExch(&s_fail, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = stage_a(st), b0 = stage_b(st);
#pragma unroll
      for (int j = 0; j < kTileK / 16; j++) {
        const uint64_t da = umma_desc(a0 + j * 32);
        const uint64_t db = umma_desc(b0 + j * 32);
        const uint32_t acc = (kt > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr),
            "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              empty(st))
          : "memory");
    }
    *(volatile int *)&s_mma = kt;
    // one more commit: arrives when every MMA issued above has completed
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(done)
        : "memory");
  }
  __syncthreads();
  // every issued MMA has finished once "done" has arrived; the loads the MMA
  // issuer did not consume (after a failure) are waited for before exit
  if (threadIdx.x == 0) {
    if (!mbar_wait(done, 0u)) s_fail = 1;
    for (int kt = s_mma; kt < s_loaded; kt++)
      if (!mbar_wait(full(kt % kTmaStages), (uint32_t)((kt / kTmaStages) & 1))) {
        s_fail = 1;
        break;
      }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!s_fail) {
    const int row = m0 + warp * 32 + lane;
    for (int cc = 0; cc < nt; cc += 16) {
      uint32_t r[16];
      if (nk > 0) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)cc));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int i = 0; i < 16; i++) r[i] = 0u;
      }
      if (row < g.M) epilogue16(g, row, n0 + cc, r);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(128u));
  if (threadIdx.x == 0 && s_fail) atomicExch(g.err, 1);
}

// ---------------------------------------------------------------------------
// The persistent, warp-specialised form of the TMA-fed kernel (engine 2 by
// default).  One CTA per SM walks the output tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... (M tiles fastest, so CTAs running together
// share their B tile in L2), and its roles run side by side:
//   * warp 0, lane 0: TMA producer over a kWsStages-deep operand ring that
//     continues from one tile into the next;
//   * warp 1, lane 0: MMA issuer.  The accumulator alternates between two
//     128-column halves of tensor memory, so the MMAs of tile i+1 run while
//     the epilogue drains tile i; a half is reused once the epilogue warps
//     have read it (the "acc empty" mbarrier, one arrival per warp);
//   * EW epilogue warps (2 .. EW + 1; EW = 8 or 16).  Warp w reads TMEM
//     lanes 32 (w % 4) .. 32 (w % 4) + 31 (the lane quarter the hardware
//     lets it access), columns [c0, c0 + 128 / (EW / 4)) with c0 set by
//     (w - 2) / 4, and stores those parts of the rows as k_gemm_tma does;
//     two or four warps per scheduler keep the epilogue's arithmetic and
//     stores from being the bound.
// The K order of every tile's MMAs is the same as in k_gemm_tma and
// k_gemm_tc, so the three give identical results.  Every wait is bounded and
// also ends when another role has recorded a failure; on failure the CTA
// waits (bounded) for its issued loads and MMAs, frees tensor memory and
// returns.
constexpr int kWsStages = 4;

__device__ __forceinline__ bool mbar_wait_or_fail(uint32_t bar, uint32_t parity,
                                                  const volatile int *fail) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while (!mbar_try(bar, parity)) {
    if (*fail) return false;
    if (globaltimer() - t0 > kWaitNs) return false;
  }
  return true;
}

struct WsTile {
  int m0, n0, nt, kb, nk;
};

__device__ __forceinline__ WsTile ws_tile(const GemmArgs &g, int t, int mtiles, int ntiles) {
  WsTile w;
  const int mb = t % mtiles, rest = t / mtiles;
  w.m0 = mb * kTileM;
  w.n0 = (rest % ntiles) * kTileN;
  const int kz = rest / ntiles;
  const int rem = g.N - w.n0;
  w.nt = rem >= kTileN ? kTileN : ((rem + 15) & ~15);
  w.kb = kz * g.k_per_split;
  const int ke = min(g.K, w.kb + g.k_per_split);
  w.nk = ke > w.kb ? (ke - w.kb + kTileK - 1) / kTileK : 0;
  return w;
}

// The persistent kernel's epilogue through shared memory (16 epilogue warps,
// 32 rows x 32 columns a warp a tile, taken in two halves of 16 columns).
// Each lane computes its row's values with the arithmetic of epilogue16 and
// writes them into the warp's staging rows (padded: 16-byte accesses free of
// bank conflicts); the warp then stores whole row segments -- four lanes a
// 64-byte BF16 row, eight a 128-byte FP32 row -- instead of each lane its own
// row 16 bytes at a time.  Two staging areas: C, and Z for bias + SiLU.
// Z's BF16 rows follow C's BF16 rows; FP32 rows of C (no Z) take the space of both.
constexpr int kEpiRowF32 = 32 * 4 + 16, kEpiRowBf16 = 32 * 2 + 16;
constexpr int kEpiAreaBytes = 32 * kEpiRowBf16;  // offset of Z's area
constexpr int kEpiStageBytes =
    32 * kEpiRowF32 > 2 * kEpiAreaBytes ? 32 * kEpiRowF32 : 2 * kEpiAreaBytes;  // per warp

__device__ __forceinline__ void stage_bf16x16(uint8_t *area, int lane, int h, const float *v) {
#pragma unroll
  for (int j = 0; j < 2; j++) {
    uint4 w;
    __nv_bfloat162 *p = reinterpret_cast<__nv_bfloat162 *>(&w);
#pragma unroll
    for (int i = 0; i < 4; i++) p[i] = __floats2bfloat162_rn(v[8 * j + 2 * i], v[8 * j + 2 * i + 1]);
    *reinterpret_cast<uint4 *>(area + lane * kEpiRowBf16 + h * 32 + j * 16) = w;
  }
}

__device__ __forceinline__ void stage_f32x16(uint8_t *area, int lane, int h, const float *v) {
#pragma unroll
  for (int j = 0; j < 4; j++)
    *reinterpret_cast<float4 *>(area + lane * kEpiRowF32 + h * 64 + j * 16) =
        make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
}

__device__ __forceinline__ void store_rows_bf16(const uint8_t *area, int lane, int ncols,
                                                __nv_bfloat16 *dst, long ld, int row0, int col0,
                                                int M) {
  const int seg = lane & 3;
#pragma unroll
  for (int pass = 0; pass < 4; pass++) {
    const int r = pass * 8 + (lane >> 2);
    if (row0 + r < M && seg * 8 < ncols)
      *reinterpret_cast<uint4 *>(dst + (long)(row0 + r) * ld + col0 + seg * 8) =
          *reinterpret_cast<const uint4 *>(area + r * kEpiRowBf16 + seg * 16);
  }
}

__device__ __forceinline__ void store_rows_f32(const uint8_t *area, int lane, int ncols,
                                               float *dst, long ld, int row0, int col0, int M) {
  const int seg = lane & 7;
#pragma unroll
  for (int pass = 0; pass < 8; pass++) {
    const int r = pass * 4 + (lane >> 3);
    if (row0 + r < M && seg * 4 < ncols)
      *reinterpret_cast<float4 *>(dst + (long)(row0 + r) * ld + col0 + seg * 4) =
          *reinterpret_cast<const float4 *>(area + r * kEpiRowF32 + seg * 16);
  }
}

// half h (columns col0 + 16h ..) of the lane's row into the staging areas
__device__ __forceinline__ void epilogue_half(const GemmArgs &g, uint8_t *stage, int lane,
                                              int row, int col, int n, int h, float *v) {
  uint8_t *areaC = stage, *areaZ = stage + kEpiAreaBytes;
  const bool live = row < g.M;
  switch (g.epi) {
    case OP2B_EPI_STORE_F32:
      if (g.bias && n > 0) add_bias16(v, g.bias, col, n);
      stage_f32x16(areaC, lane, h, v);
      return;
    case OP2B_EPI_BIAS_BF16:
      if (g.bias && n > 0) add_bias16(v, g.bias, col, n);
      if (g.R && live && n > 0) {
        float rr[16];
        load_bf16x16(g.R + (long)row * g.ldr + col, rr, n);
        FOR_LT_N(i) v[i] += rr[i];
      }
      stage_bf16x16(areaC, lane, h, v);
      return;
    case OP2B_EPI_BIAS_SILU_BF16:
      if (g.bias && n > 0) add_bias16(v, g.bias, col, n);
      stage_bf16x16(areaZ, lane, h, v);
#pragma unroll
      for (int i = 0; i < 16; i++) v[i] = silu(v[i]);
      stage_bf16x16(areaC, lane, h, v);
      return;
    case OP2B_EPI_SILU_GRAD_BF16:
      if (live && n > 0) {
        float z[16];
        load_bf16x16(g.R + (long)row * g.ldr + col, z, n);
        FOR_LT_N(i) v[i] *= silu_grad(z[i]);
      }
      stage_bf16x16(areaC, lane, h, v);
      return;
    default:
      stage_bf16x16(areaC, lane, h, v);
  }
}

// the staged rows of the warp out to C (and Z)
__device__ __forceinline__ void epilogue_store(const GemmArgs &g, const uint8_t *stage, int lane,
                                               int row0, int col0, int ncols) {
  if (g.epi == OP2B_EPI_STORE_F32) {
    store_rows_f32(stage, lane, ncols, reinterpret_cast<float *>(g.C), g.ldc, row0, col0, g.M);
    return;
  }
  if (g.epi == OP2B_EPI_BIAS_SILU_BF16 && g.Z)
    store_rows_bf16(stage + kEpiAreaBytes, lane, ncols, g.Z, g.ldc, row0, col0, g.M);
  store_rows_bf16(stage, lane, ncols, reinterpret_cast<__nv_bfloat16 *>(g.C), g.ldc, row0, col0,
                  g.M);
}

template <int EW, bool AMN, bool BMN>
__global__ void __launch_bounds__(64 + 32 * EW, 1)
k_gemm_ws(GemmArgs g, const __grid_constant__ CUtensorMap ta,
          const __grid_constant__ CUtensorMap tb, int mtiles, int ntiles, int ntotal) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // full[kWsStages], empty[kWsStages], acc_full[2], acc_empty[2], done
  __shared__ __align__(8) uint64_t bars[2 * kWsStages + 5];
  __shared__ uint32_t s_taddr;
  __shared__ int s_fail, s_loaded, s_mma;
  uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto full = [&](int st) { return smem_u32(&bars[st]); };
  auto empty = [&](int st) { return smem_u32(&bars[kWsStages + st]); };
  auto acc_full = [&](int b) { return smem_u32(&bars[2 * kWsStages + b]); };
  auto acc_empty = [&](int b) { return smem_u32(&bars[2 * kWsStages + 2 + b]); };
  const uint32_t done = smem_u32(&bars[2 * kWsStages + 4]);
  auto stage_a = [&](int st) { return smem_u32(smem + (size_t)st * 2 * kStageBytes); };
  auto stage_b = [&](int st) { return smem_u32(smem + (size_t)st * 2 * kStageBytes + kStageBytes); };
  volatile int *fail = &s_fail;

  if (threadIdx.x == 0) {
    for (int st = 0; st < kWsStages; st++) {
      mbar_init(full(st), 1);
      mbar_init(empty(st), 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(acc_full(b), 1);
      mbar_init(acc_empty(b), EW);
    }
    mbar_init(done, 1);
    s_fail = 0;
    s_loaded = 0;
    s_mma = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_taddr)),
                 "r"(256u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = s_taddr;

  if (threadIdx.x == 0) {  // producer
    int it = 0;
    for (int t = blockIdx.x; t < ntotal && !*fail; t += gridDim.x) {
      const WsTile w = ws_tile(g, t, mtiles, ntiles);
      for (int kt = 0; kt < w.nk; kt++, it++) {
        const int st = it % kWsStages;
        if (it >= kWsStages &&
            !mbar_wait_or_fail(empty(st), (uint32_t)((it / kWsStages - 1) & 1), fail)) {
          atomicExch(&s_fail, 1);
          break;
        }
        mbar_expect_tx(full(st), 2 * kStageBytes);
        const int k0 = w.kb + kt * kTileK;
        if (AMN) {  // two 64 (MN) x 64 (K) boxes
          tma_load_2d(stage_a(st), &ta, w.m0, k0, full(st));
          tma_load_2d(stage_a(st) + kStageBytes / 2, &ta, w.m0 + 64, k0, full(st));
        } else {
          tma_load_2d(stage_a(st), &ta, k0, w.m0, full(st));
        }
        if (BMN) {
          tma_load_2d(stage_b(st), &tb, w.n0, k0, full(st));
          tma_load_2d(stage_b(st) + kStageBytes / 2, &tb, w.n0 + 64, k0, full(st));
        } else {
          tma_load_2d(stage_b(st), &tb, k0, w.n0, full(st));
        }
      }
    }
    *(volatile int *)&s_loaded = it;
  } else if (threadIdx.x == 32) {  // MMA issuer
    int it = 0, i = 0;
    for (int t = blockIdx.x; t < ntotal && !*fail; t += gridDim.x, i++) {
      const WsTile w = ws_tile(g, t, mtiles, ntiles);
      const int b = i & 1;
      if (i >= 2 && !mbar_wait_or_fail(acc_empty(b), (uint32_t)(((i >> 1) - 1) & 1), fail)) {
        atomicExch(&s_fail, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t idesc =
          umma_idesc(w.nt) | (AMN ? 1u << 15 : 0u) | (BMN ? 1u << 16 : 0u);  // MN-major
      const uint32_t d = taddr + (uint32_t)(b * kTileN);
      bool ok = true;
      for (int kt = 0; kt < w.nk; kt++, it++) {
        const int st = it % kWsStages;
        if (!mbar_wait_or_fail(full(st), (uint32_t)((it / kWsStages) & 1), fail)) {
          atomicExch(&s_fail, 1);
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = stage_a(st), b0 = stage_b(st);
#pragma unroll
        for (int j = 0; j < kTileK / 16; j++) {
          const uint64_t da = AMN ? umma_desc_mn(a0 + j * 2048) : umma_desc(a0 + j * 32);
          const uint64_t db = BMN ? umma_desc_mn(b0 + j * 2048) : umma_desc(b0 + j * 32);
          const uint32_t acc = (kt > 0 || j > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
              "l"(da), "l"(db), "r"(idesc), "r"(acc));
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                empty(st))
            : "memory");
      }
      if (!ok) break;
      // the tile's accumulator is complete once these MMAs have finished
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              acc_full(b))
          : "memory");
    }
    *(volatile int *)&s_mma = it;
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(done)
        : "memory");
  } else if (warp >= 2) {  // epilogue
    const int quarter = warp & 3;
    constexpr int kCols = kTileN / (EW / 4);
    const int c0 = ((warp - 2) >> 2) * kCols;
    // the warp's staging rows, after the operand ring (EW == 16 only)
    uint8_t *epi_stage = smem + (size_t)kWsStages * 2 * kStageBytes + (warp - 2) * kEpiStageBytes;
    int i = 0;
    for (int t = blockIdx.x; t < ntotal; t += gridDim.x, i++) {
      const WsTile w = ws_tile(g, t, mtiles, ntiles);
      const int b = i & 1;
      bool ok = mbar_wait_or_fail(acc_full(b), (uint32_t)((i >> 1) & 1), fail);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) {
        if (lane == 0) atomicExch(&s_fail, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int row = w.m0 + quarter * 32 + lane;
      const uint32_t src = taddr + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * kTileN);
      const int ce = min(w.nt, c0 + kCols);
      if (c0 >= ce) {  // nothing of this tile in the warp's columns
        __syncwarp();
        if (lane == 0)
          asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(acc_empty(b)) : "memory");
        continue;
      }
      if (EW == 16 && g.staged) {  // 32 columns: the row-coalesced epilogue
        // the warp's columns of the matrix (nt is rounded up to 16; N is not)
        const int nv = min(ce, g.N - w.n0) - c0;
#pragma unroll 1
        for (int h = 0; h < 2; h++) {
          uint32_t r[16];
#pragma unroll
          for (int k = 0; k < 16; k++) r[k] = 0u;
          if (w.nk > 0 && c0 + 16 * h < ce) {
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                  "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                  "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(src + (uint32_t)(c0 + 16 * h)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          }
          if (h == 1) {  // the warp's part has been read: the MMAs may reuse it
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
              asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(acc_empty(b))
                           : "memory");
          }
          float v[16];
#pragma unroll
          for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
          epilogue_half(g, epi_stage, lane, row, w.n0 + c0 + 16 * h,
                        min(16, nv - 16 * h), h, v);
        }
        __syncwarp();
        epilogue_store(g, epi_stage, lane, w.m0 + quarter * 32, w.n0 + c0, nv);
        __syncwarp();
        continue;
      }
      for (int cc = c0; cc < ce; cc += 16) {
        uint32_t r[16];
        if (w.nk > 0) {
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
              "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
              : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
              : "r"(src + (uint32_t)cc));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        } else {
#pragma unroll
          for (int k = 0; k < 16; k++) r[k] = 0u;
        }
        if (cc + 16 >= ce) {  // the warp's part has been read: the MMAs may reuse it
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0)
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(acc_empty(b))
                         : "memory");
        }
        if (row < g.M) epilogue16(g, row, w.n0 + cc, r);
      }
    }
  }
  __syncthreads();
  // every issued MMA has finished once "done" has arrived; loads the MMA
  // issuer did not consume (after a failure) are waited for before exit
  if (threadIdx.x == 0) {
    if (!mbar_wait(done, 0u)) s_fail = 1;
    for (int it = s_mma; it < s_loaded; it++)
      if (!mbar_wait(full(it % kWsStages), (uint32_t)((it / kWsStages) & 1))) {
        s_fail = 1;
        break;
      }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(256u));
  }
  if (threadIdx.x == 0 && s_fail) atomicExch(g.err, 1);
}

// the same product on the CUDA cores (FP32 accumulation), as a cross-check
__global__ void k_gemm_simt(GemmArgs g) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x, row = blockIdx.y;
  if (col >= g.N || row >= g.M) return;
  float acc = 0.f;
  for (int k = 0; k < g.K; k++)
    acc += __bfloat162float(g.A[row * g.a_m + k * g.a_k]) *
           __bfloat162float(g.B[col * g.b_n + k * g.b_k]);
  reinterpret_cast<float *>(g.C)[(long)row * g.ldc + col] = acc;
}

int *g_err_dev[16] = {};

// cuTensorMapEncodeTiled, found through the runtime (the library does not
// link the driver library itself)
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                 const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                 const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled() {
  static EncodeTiled fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
    cudaGetLastError();
  }
  return fn;
}

// a K-major bf16 operand (rows x K, row stride `ld` elements) as a tensor map
// of 64 x 128 boxes with the 128-byte swizzle; false if it cannot be encoded
bool operand_map(CUtensorMap *m, const void *base, int rows, int K, long ld) {
  EncodeTiled enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kTileK, (cuuint32_t)kTileM};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// an MN-major bf16 operand (K rows of `mn` contiguous values, row stride `ld`
// elements) as a tensor map of 64 (MN) x 64 (K) boxes with the 128-byte
// swizzle; false if it cannot be encoded
bool operand_map_mn(CUtensorMap *m, const void *base, int mn, int K, long ld) {
  EncodeTiled enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)mn, (cuuint64_t)K};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {64, (cuuint32_t)kTileK};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

template <int EW, bool AMN, bool BMN>
cudaError_t launch_ws(const GemmArgs &g, const CUtensorMap &ta, const CUtensorMap &tb,
                      dim3 grid, int nsm, cudaStream_t s) {
  const size_t smem_w =
      (size_t)kWsStages * 2 * kStageBytes + (EW == 16 ? 16 * kEpiStageBytes : 0) + 1024;
  static bool attr[16] = {};  // per device, once
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 16) return cudaErrorInvalidDevice;
  if (!attr[dev]) {
    cudaError_t e = cudaFuncSetAttribute(k_gemm_ws<EW, AMN, BMN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_w);
    if (e != cudaSuccess) return e;
    attr[dev] = true;
  }
  const long long total = (long long)grid.x * grid.y * grid.z;
  const int ctas = (int)std::min<long long>(total, nsm > 0 ? nsm : 148);
  k_gemm_ws<EW, AMN, BMN><<<ctas, 64 + 32 * EW, smem_w, s>>>(g, ta, tb, (int)grid.x,
                                                             (int)grid.y, (int)total);
  return cudaGetLastError();
}

}  // namespace
}  // namespace op2b

using namespace op2b;

extern "C" int op2b_gemm_bf16(int M, int N, int K, const void *A, long a_m, long a_k,
                              const void *B, long b_n, long b_k, void *C, long ldc, int epi,
                              const float *bias, void *Z, const void *R, long ldr, int split_k,
                              int engine, void *stream) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) {
    set_error("op2b_gemm_bf16: empty or null operands (M=%d N=%d K=%d)", M, N, K);
    return -1;
  }
  if ((a_m != 1 && a_k != 1) || (b_n != 1 && b_k != 1) || N % 8 ||
      ((a_k == 1 || b_k == 1) && K % 8)) {
    set_error("op2b_gemm_bf16: each operand needs a unit stride; N, and K of a k-contiguous "
              "operand, multiples of 8");
    return -1;
  }
  if ((a_k != 1 && (M % 8 || a_k % 8)) || (b_k != 1 && (N % 8 || b_k % 8)) ||
      (a_k == 1 && a_m % 8) || (b_k == 1 && b_n % 8)) {
    set_error("op2b_gemm_bf16: rows of 16-byte chunks need strides and transposed row counts "
              "that are multiples of 8");
    return -1;
  }
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) {
    set_error("op2b_gemm_bf16: A and B must be 16-byte aligned");
    return -1;
  }
  if (epi < OP2B_EPI_STORE_F32 || epi > OP2B_EPI_SILU_GRAD_BF16 ||
      (epi == OP2B_EPI_SILU_GRAD_BF16 && !R)) {
    set_error("op2b_gemm_bf16: bad epilogue %d (SILU_GRAD needs R)", epi);
    return -1;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 16) {
    set_error("op2b_gemm_bf16: device %d out of range", dev);
    return -1;
  }
  if (!g_err_dev[dev]) {
    if (!cuda_ok(cudaMalloc(&g_err_dev[dev], sizeof(int)), "op2b_gemm_bf16: error flag"))
      return -1;
    cudaMemset(g_err_dev[dev], 0, sizeof(int));
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  GemmArgs g{M,   N,   K,   (const __nv_bfloat16 *)A, a_m, a_k, (const __nv_bfloat16 *)B,
             b_n, b_k, C,   ldc, bias, (__nv_bfloat16 *)Z,     (const __nv_bfloat16 *)R,
             ldr, epi, 0,   g_err_dev[dev]};
  {  // rows of C (and Z) that 16-byte stores can cover
    const long esize = epi == OP2B_EPI_STORE_F32 ? 4 : 2;
    g.staged = rt().opt_gemm_rows && epi != OP2B_EPI_ATOMIC_F32 &&
               (reinterpret_cast<uintptr_t>(C) & 15) == 0 && (ldc * esize) % 16 == 0 &&
               (reinterpret_cast<uintptr_t>(Z) & 15) == 0;
  }
  if (engine == 1) {
    if (epi != OP2B_EPI_STORE_F32) {
      set_error("op2b_gemm_bf16: the CUDA-core path stores FP32 only");
      return -1;
    }
    k_gemm_simt<<<dim3((N + 127) / 128, M), 128, 0, s>>>(g);
    if (rt().initialised) rt().launches++;
    return cuda_ok(cudaGetLastError(), "op2b_gemm_bf16") ? 0 : -1;
  }
  if (split_k < 1) split_k = 1;
  const int kps = ((K + split_k - 1) / split_k + kTileK - 1) / kTileK * kTileK;
  split_k = (K + kps - 1) / kps;
  if (split_k > 1 && epi != OP2B_EPI_ATOMIC_F32) {
    set_error("op2b_gemm_bf16: split-K needs the atomic FP32 epilogue");
    return -1;
  }
  if (split_k > 65535) {
    set_error("op2b_gemm_bf16: split_k above 65535");
    return -1;
  }
  g.k_per_split = kps;
  dim3 grid((M + kTileM - 1) / kTileM, (N + kTileN - 1) / kTileN, split_k);
  // the TMA-fed kernels (engine 2 asks for them; engine 0 takes them when the
  // option gemm_tma is on): the persistent kernel for any layout of A and B
  // (k-contiguous operands as K-major tiles, the others as MN-major tiles),
  // the one-tile-per-CTA kernel for k-contiguous operands
  const bool a_mn = a_k != 1, b_mn = b_k != 1;
  const bool ws = rt().opt_gemm_ws != 0;
  if (engine == 2 || (engine == 0 && rt().opt_gemm_tma)) {
    CUtensorMap ta, tb;
    const bool mapped = (a_mn ? operand_map_mn(&ta, A, M, K, a_k) : operand_map(&ta, A, M, K, a_m)) &&
                        (b_mn ? operand_map_mn(&tb, B, N, K, b_k) : operand_map(&tb, B, N, K, b_n));
    if ((a_mn || b_mn) && !ws) {
      if (engine == 2) {
        set_error("op2b_gemm_bf16: engine 2 with gemm_persistent 0 needs k-contiguous A and B");
        return -1;
      }
    } else if (mapped) {
      const long long total = (long long)grid.x * grid.y * grid.z;
      if (total > 0x7fffffffLL) {
        set_error("op2b_gemm_bf16: too many output tiles");
        return -1;
      }
      cudaError_t e;
      if (ws) {
        int nsm = 0;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (a_mn && b_mn) e = launch_ws<16, true, true>(g, ta, tb, grid, nsm, s);
        else if (a_mn) e = launch_ws<16, true, false>(g, ta, tb, grid, nsm, s);
        else if (b_mn) e = launch_ws<16, false, true>(g, ta, tb, grid, nsm, s);
        else if (rt().opt_gemm_ws == 2) e = launch_ws<16, false, false>(g, ta, tb, grid, nsm, s);
        else e = launch_ws<8, false, false>(g, ta, tb, grid, nsm, s);
      } else {
        const size_t smem_t = (size_t)kTmaStages * 2 * kStageBytes + 1024;
        static bool attr_t[16] = {};
        e = cudaSuccess;
        if (!attr_t[dev]) {
          e = cudaFuncSetAttribute(k_gemm_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem_t);
          attr_t[dev] = e == cudaSuccess;
        }
        if (e == cudaSuccess) {
          k_gemm_tma<<<grid, kThreads, smem_t, s>>>(g, ta, tb);
          e = cudaGetLastError();
        }
      }
      if (rt().initialised) rt().launches++;
      return cuda_ok(e, "op2b_gemm_bf16") ? 0 : -1;
    } else if (engine == 2) {
      set_error("op2b_gemm_bf16: the operands cannot be described as tensor maps");
      return -1;
    }
  }
  const size_t smem = 4 * (size_t)kStageBytes + 1024;
  static bool attr[16] = {};
  if (!attr[dev]) {
    if (!cuda_ok(cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem),
                 "op2b_gemm_bf16: shared memory attribute"))
      return -1;
    attr[dev] = true;
  }
  k_gemm_tc<<<grid, kThreads, smem, s>>>(g);
  if (rt().initialised) rt().launches++;
  return cuda_ok(cudaGetLastError(), "op2b_gemm_bf16") ? 0 : -1;
}

extern "C" int op2b_gemm_error(int reset) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 16 || !g_err_dev[dev]) return 0;
  int h = 0;
  cudaMemcpy(&h, g_err_dev[dev], sizeof(int), cudaMemcpyDeviceToHost);
  if (reset) cudaMemset(g_err_dev[dev], 0, sizeof(int));
  return h;
}
