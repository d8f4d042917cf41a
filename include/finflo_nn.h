/* finflo_nn.h -- C-ABI of the learned warm start's tensor-core kernels
 * (libfinflo_nn.so, sm_100a).
 *
 * The reference has no counterpart: FINFLO starts every run from a free
 * stream or a restart file (RSTART).  These entry points train and evaluate
 * the small network that predicts a starting flow field for a new case from
 * its parameters; the prediction is handed to the solver as its initial
 * state, and the solver still iterates to the same tolerance.
 *
 * Conventions: every pointer is a device address; BF16 arrays are 16-bit
 * values (bfloat16) passed as void*; FP32 arrays are float*.  Row-major
 * matrices with a leading dimension in elements.  All work is enqueued on
 * `stream` (a cudaStream_t, or NULL for the default stream); nothing is
 * allocated.  Return 0 or one of the FFNN_ERR_* codes.
 */
#ifndef FINFLO_NN_H
#define FINFLO_NN_H

#ifdef __cplusplus
extern "C" {
#endif

#define FFNN_ERR_ARG 1      /* bad shape, stride or alignment */
#define FFNN_ERR_CUDA 2     /* a CUDA call failed */
#define FFNN_ERR_TIMEOUT 3  /* a bounded device wait gave up */

/* Z[M,N] = A[M,K] * B[N,K]^T (+ bias[N]) in FP32 accumulation on the 5th
 * generation tensor cores; BF16 operands, both K-contiguous (lda, ldb >= K,
 * multiples of 8; A, B 16-byte aligned; K a multiple of 16).
 * zf (FP32, ldz): the pre-activation result, stored, or added atomically when
 * atomic = 1 (required when ksplit < K: the K range is split over CTAs).
 * yb (BF16, ldy): act(Z) with act 0 = identity, 1 = SiLU.  Either output may
 * be NULL, not both. */
int ffnn_gemm(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias, int act,
              float *zf, int ldz, int atomic, void *yb, int ldy, int ksplit, void *stream);

/* dz = dy * SiLU'(z) element-wise over n values; dzb (BF16) and/or dzf (FP32). */
int ffnn_silu_bwd(const float *dy, const float *z, long n, void *dzb, float *dzf, void *stream);

/* out[c] += sum_r x[r*ld + c] for c < cols (bias gradients). */
int ffnn_colsum(const float *x, int rows, int cols, int ld, float *out, void *stream);

/* BF16 transpose: out[c*ldo + r] = in[r*ldi + c]; rows rows..rows_pad-1 of
 * the result are written as zeros. */
int ffnn_transpose(const void *in, int rows, int cols, int ldi, void *out, int ldo, int rows_pad, void *stream);

/* FP32 -> BF16 (round to nearest even). */
int ffnn_to_bf16(const float *in, long n, void *out, void *stream);

/* Mean-squared error of pred[rows, ld] (first cols columns) against
 * tgt[rows, cols]: *loss += mean((pred - tgt)^2), grad (BF16 [rows, ld]) =
 * d loss / d pred, zero in the padding columns; gradf (FP32, may be NULL)
 * the same gradient in FP32. */
int ffnn_mse(const float *pred, int ld, const float *tgt, int rows, int cols, void *grad, float *gradf,
             float *loss, void *stream);

/* One Adam step (bias-corrected; wd * w added to the gradient) on FP32 master
 * weights w[n] with moments m, v; writes the BF16 copy w16 and, when
 * rows > 0, the BF16 transpose w16t of w viewed as [rows, n/rows]. */
int ffnn_adam(float *w, const float *g, float *m, float *v, long n, float lr, float b1, float b2, float eps,
              int step, float wd, void *w16, void *w16t, int rows, void *stream);

/* FFNN_ERR_TIMEOUT if any kernel of the library gave up a bounded wait since
 * the last reset (reset = 1 clears the word). */
int ffnn_error(int reset);

#ifdef __cplusplus
}
#endif

#endif
