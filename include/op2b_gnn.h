/* Learned warm start for Airfoil: kernels of a message-passing graph network
 * (encode - process - decode) trained and evaluated on the GPU.
 *
 * The reference has no counterpart: OP2's Airfoil starts every solve from the
 * freestream state (apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:204-210).
 * This header adds the kernels that let a caller predict the initial q on the
 * solver's own mesh graph (cells are graph nodes, interior edges pecell are
 * graph edges in both directions) and then run the unchanged op_par_loop
 * iteration from it.  All pointers are device pointers; every entry point is
 * asynchronous on `stream` (a cudaStream_t, null = legacy default stream) and
 * returns 0, or -1 with op2b_last_error() set.  Matrices are row-major with an
 * explicit leading dimension (elements).  bf16 = IEEE bfloat16 (2 bytes).
 */
#ifndef OP2B_GNN_H
#define OP2B_GNN_H

#ifdef __cplusplus
extern "C" {
#endif

/* epilogues of op2b_gemm_bf16 (acc = the FP32 accumulator of C(m, n)) */
#define OP2B_EPI_STORE_F32 0      /* C (float) = acc (+ bias[n] when bias given) */
#define OP2B_EPI_ATOMIC_F32 1     /* C (float) += acc, atomically (split-K) */
#define OP2B_EPI_STORE_BF16 2     /* C (bf16) = acc */
#define OP2B_EPI_BIAS_BF16 3      /* C (bf16) = acc + bias[n] (+ R(m, n) when R given) */
#define OP2B_EPI_BIAS_SILU_BF16 4 /* Z (bf16) = acc + bias[n]; C (bf16) = silu(Z) */
#define OP2B_EPI_SILU_GRAD_BF16 5 /* C (bf16) = acc * silu'(R(m, n)) */

/* C(m, n) = sum_k A(m, k) B(n, k) on the tensor cores (tcgen05.mma kind::f16,
 * bf16 operands, FP32 accumulation in tensor memory), then the epilogue `epi`.
 * A(m, k) = A[m*a_m + k*a_k], B(n, k) = B[n*b_n + k*b_k]: each operand has one
 * unit stride (k-contiguous rows, or transposed).  N a multiple of 8, and K
 * when an operand is k-contiguous; a transposed operand needs its row count
 * (M or N) a multiple of 8; strides multiples of 8; A, B 16-byte aligned.
 * `bias`: N floats or null.  `Z`: pre-activation output of
 * OP2B_EPI_BIAS_SILU_BF16 (bf16, leading dim ldc) or null.  `R`, `ldr`: the
 * residual (OP2B_EPI_BIAS_BF16) or the pre-activation whose silu' multiplies
 * the product (OP2B_EPI_SILU_GRAD_BF16), bf16.  split_k > 1 splits K over
 * CTAs and requires OP2B_EPI_ATOMIC_F32.  engine 0 = tensor cores, 1 = CUDA
 * cores (FP32 store only; a cross-check of the tensor-core path), 2 = tensor
 * cores fed by TMA (k-contiguous A and B only; engine 0 takes this path too
 * when the option gemm_tma is set).
 * Replaces: nothing in the reference (no learned component). */
int op2b_gemm_bf16(int M, int N, int K, const void *A, long a_m, long a_k, const void *B,
                   long b_n, long b_k, void *C, long ldc, int epi, const float *bias, void *Z,
                   const void *R, long ldr, int split_k, int engine, void *stream);

/* Nonzero if a tensor-core GEMM gave up waiting on its tensor-core commit (a
 * bounded wait ran out); reset clears the flag.  Synchronises the device. */
int op2b_gemm_error(int reset);

/* cat[k, col0 : col0+D] = h[src[k], :D]; cat[k, col0+D : col0+2D] = h[dst[k], :D]
 * (bf16; D a multiple of 8).  The edge-model input [e_k, h_src, h_dst]. */
int op2b_gnn_gather_pair(int E, int D, const int *src, const int *dst, const void *h, long ldh,
                         void *cat, long ldcat, int col0, void *stream);

/* out[n, :D] = sum over j in [off[n], off[n+1]) of e[idx[j], :D], FP32 sums in
 * a fixed order, stored as bf16: the aggregation of incoming edge messages. */
int op2b_gnn_aggregate(int N, int D, const int *off, const int *idx, const void *e, long lde,
                       void *out, long ldo, void *stream);

/* y (bf16) = x (float), M x D; x may be strided. */
int op2b_gnn_to_bf16(int M, int D, const float *x, long ldx, void *y, long ldy, void *stream);

/* acc (float, M x D, ld D) += x (float, leading dim ldx) */
int op2b_gnn_add_f32(int M, int D, float *acc, const float *x, long ldx, void *stream);

/* Backward of the aggregation plus the residual: for every edge k
 * dE[k, :] += dAgg[dst[k], :] (float); dy[k, :] = bf16(dE[k, :]). */
int op2b_gnn_edge_grad(int E, int D, const int *dst, float *dE, const float *dAgg, long ldagg,
                       void *dy, void *stream);

/* Backward of the edge-model input [e_k, h_src, h_dst] (dCat: E x 3D float,
 * leading dim ldcat): dE[k] += dCat[k, :D] for every edge k, and for every node n
 * dH[n] += sum over incoming edges k (off/idx) of dCat[k, 2D:3D] + dCat[rev[k], D:2D]
 * (rev[k] = the edge in the opposite direction, whose source is n). */
int op2b_gnn_cat_grad(int E, int N, int D, const float *dCat, long ldcat, float *dE,
                      const int *off, const int *idx, const int *rev, float *dH, void *stream);

/* db[n] += sum_m dz[m, n], dz bf16 (M x N, leading dim ld). */
int op2b_gnn_colsum(int M, int N, const void *dz, long ld, float *db, void *stream);

/* Mean-squared error of out[:, :D] (float, leading dim ldo) against target
 * (float, M x D): dy[m, c] = bf16(2 * scale * (out - target)) for c < D and 0
 * for D <= c < ldo; loss[0] += scale * sum (out - target)^2. */
int op2b_gnn_mse(int M, int D, const float *out, long ldo, const float *target, void *dy,
                 float *loss, float scale, void *stream);

/* One Adam(W) step over n parameters: FP32 master p, moments m, v, gradient g;
 * also writes the bf16 copy pb (null to skip) and zeroes g.  lr_t is the
 * bias-corrected step size; wd the decoupled decay of this step (p *= 1 - wd,
 * AdamW's lr * weight_decay). */
int op2b_gnn_adam(long n, float *p, float *g, float *m, float *v, void *pb, float lr_t,
                  float beta1, float beta2, float eps, float wd, void *stream);

/* bytes of ptr set to value (cudaMemsetAsync on stream). */
int op2b_gnn_memset(void *ptr, int value, long bytes, void *stream);

/* q (double, ncell x 4) = qinf + mean + std * out[:, :4] (out float, leading
 * dim ldo; mean_std = 4 means then 4 standard deviations; qinf 4 doubles). */
int op2b_gnn_decode_q(int ncell, const float *out, long ldo, const double *mean_std,
                      const double *qinf, double *q, void *stream);

#ifdef __cplusplus
}
#endif
#endif
