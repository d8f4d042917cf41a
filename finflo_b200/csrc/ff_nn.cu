// BF16 tensor-core kernels of the learned warm start (sm_100a): the network
// that predicts an initial flow field from the case parameters is trained
// and evaluated with these kernels only.
//
//   ffnn_gemm     C[M,N] = A[M,K] * B[N,K]^T (+ bias, SiLU), BF16 operands,
//                 FP32 accumulation in tensor memory (tcgen05.mma, one
//                 elected thread per CTA, operands staged in shared memory
//                 in the canonical K-major core-matrix layout, completion
//                 through an mbarrier, accumulator read back with
//                 tcgen05.ld); split-K with FP32 atomics for the weight
//                 gradients, whose reduction runs over all voxels.
//   element-wise  SiLU backward, column sums (bias gradients), transposes,
//                 casts, mean-squared-error gradient, Adam.
//
// Every device wait is bounded: on time-out the kernel sets the error word,
// waits (bounded) for its own tensor-core work, frees its tensor memory and
// returns; the host reads the word with ffnn_error().
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/finflo_nn.h"

namespace {

constexpr int GM = 128;        // rows of a CTA tile (tcgen05 M)
constexpr int GKT = 64;        // K elements staged per iteration (4 MMAs of K = 16)
constexpr int GTHREADS = 128;  // 4 warps: one per 32 TMEM lanes
constexpr long kSpin = 1L << 26;

__device__ int g_err;          // first error of any kernel of this file

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for one phase of an mbarrier; false on time-out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long it = 0; it < kSpin; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Shared-memory matrix descriptor, K-major without swizzle: core matrices
// of 8 rows x 16 bytes; lbo = byte distance of the two core matrices along
// K that one MMA (K = 16) reads, sbo = byte distance of 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version of sm_100
  return d;                 // base offset 0, legacy LBO mode, no swizzle
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D.
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float v[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }

}  // namespace

namespace {

struct GemmArgs {
  const __nv_bfloat16* A;   // [M, K] row-major (K contiguous), lda elements per row
  const __nv_bfloat16* B;   // [N, K] row-major, ldb
  int lda, ldb, M, N, K;
  int nt;                   // columns of a CTA tile: multiple of 16, <= 256
  int ksplit;               // K elements per split (a multiple of GKT)
  const float* bias;        // [N] or null
  int act;                  // 0: none, 1: SiLU on the bf16 output
  float* zf;                // FP32 output (pre-activation) or null
  int ldz;
  int atomic;               // 1: zf += (split-K partial sums)
  __nv_bfloat16* yb;        // BF16 output (after the activation) or null
  int ldy;
};

// Shared memory of one stage: A tile [128 x 64] then B tile [nt x 64], each in
// core-matrix order: element (r, k) at (r/8)*1024 + (k/8)*128 + (r%8)*16 + (k%8)*2.
constexpr uint32_t kLBO = 128, kSBO = (GKT / 8) * 128;

__device__ __forceinline__ uint32_t core_off(int r, int c8) { return (r >> 3) * kSBO + c8 * kLBO + (r & 7) * 16; }

__global__ void __launch_bounds__(GTHREADS) k_gemm_bf16(GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * GM, n0 = blockIdx.y * g.nt;
  const int kb = blockIdx.z * g.ksplit, ke = min(g.K, kb + g.ksplit);
  const uint32_t abytes = GM * GKT * 2, bbytes = g.nt * GKT * 2, sbytes = abytes + bbytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * sbytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
  const uint32_t sbase = smem_u32(smem), bar0 = smem_u32(bars), bar1 = bar0 + 8;
  uint32_t ncol = 32;
  while ((int)ncol < g.nt) ncol <<= 1;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(ncol)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = instr_desc(GM, g.nt);
  const int nk = ke > kb ? (ke - kb + GKT - 1) / GKT : 0;
  bool ok = true;
  for (int it = 0; it < nk && ok; it++) {
    const int b = it & 1;
    if (it >= 2) {   // the MMAs that read this stage two iterations ago are done
      bool w = mbar_wait(b ? bar1 : bar0, ((it >> 1) - 1) & 1);
      if (__syncthreads_or(!w)) { ok = false; break; }
    }
    const int k0 = kb + it * GKT, klen = min(GKT, ke - k0);
    const int nc8 = klen >> 3;
    unsigned char* sa = smem + b * sbytes;
    unsigned char* sb = sa + abytes;
    // A tile: 128 rows x nc8 chunks of 8 elements (16 bytes), zero past M
    for (int q = tid; q < GM * nc8; q += GTHREADS) {
      const int r = q / nc8, c8 = q % nc8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (m0 + r < g.M) v = *reinterpret_cast<const uint4*>(g.A + (size_t)(m0 + r) * g.lda + k0 + c8 * 8);
      *reinterpret_cast<uint4*>(sa + core_off(r, c8)) = v;
    }
    for (int q = tid; q < g.nt * nc8; q += GTHREADS) {
      const int r = q / nc8, c8 = q % nc8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (n0 + r < g.N) v = *reinterpret_cast<const uint4*>(g.B + (size_t)(n0 + r) * g.ldb + k0 + c8 * 8);
      *reinterpret_cast<uint4*>(sb + core_off(r, c8)) = v;
    }
    proxy_fence();   // generic-proxy stores -> visible to the tensor core's reads
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a_addr = sbase + b * sbytes, b_addr = a_addr + abytes;
      for (int s = 0; s < (klen >> 4); s++) {
        const uint64_t ad = smem_desc(a_addr + s * 2 * kLBO, kLBO, kSBO);
        const uint64_t bd = smem_desc(b_addr + s * 2 * kLBO, kLBO, kSBO);
        mma_bf16(tmem, ad, bd, idesc, (it > 0 || s > 0) ? 1u : 0u);
      }
      mma_commit(b ? bar1 : bar0);
    }
  }
  // the last commit tracks every MMA issued before it
  bool done = nk == 0;
  if (nk > 0) {
    const int last = nk - 1;
    done = mbar_wait((last & 1) ? bar1 : bar0, (last >> 1) & 1);
  }
  if (__syncthreads_or(!done || !ok)) {
    if (tid == 0) atomicCAS(&g_err, 0, 1);
    ok = false;
  }
  tc_fence_after();
  if (ok && nk > 0) {
    const int row = m0 + warp * 32 + lane;
    for (int c = 0; c < g.nt / 8; c++) {
      float v[8];
      tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 8), v);
      if (row >= g.M) continue;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int col = n0 + c * 8 + j;
        if (col >= g.N) break;
        float z = v[j] + (g.bias ? g.bias[col] : 0.f);
        if (g.zf) {
          if (g.atomic) atomicAdd(g.zf + (size_t)row * g.ldz + col, z);
          else g.zf[(size_t)row * g.ldz + col] = z;
        }
        if (g.yb) g.yb[(size_t)row * g.ldy + col] = __float2bfloat16_rn(g.act == 1 ? silu(z) : z);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncol) : "memory");
}

}  // namespace

namespace {

// dz = dy * silu'(z), written as BF16 (the next GEMM's operand) and FP32.
__global__ void k_silu_bwd(const float* __restrict__ dy, const float* __restrict__ z, long n, __nv_bfloat16* dzb,
                           float* dzf) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float zi = z[i], s = 1.f / (1.f + __expf(-zi));
    const float d = dy[i] * s * (1.f + zi * (1.f - s));
    if (dzb) dzb[i] = __float2bfloat16_rn(d);
    if (dzf) dzf[i] = d;
  }
}

// out[c] += sum over rows of x[r * ld + c] (bias gradients).
__global__ void k_colsum(const float* __restrict__ x, int rows, int cols, int ld, float* out) {
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) s += x[(size_t)r * ld + c];
  atomicAdd(out + c, s);
}

// out[c * ldo + r] = in[r * ldi + c] for r < rows, c < cols; rows padded
// with zeros up to rows_pad (so that the transposed operand's K is a
// multiple of the GEMM's K step).
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, int rows, int cols, int ldi,
                                 __nv_bfloat16* out, int ldo, int rows_pad) {
  __shared__ __nv_bfloat16 t[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    t[y][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * ldi + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (c < cols && r < rows_pad) out[(size_t)c * ldo + r] = t[threadIdx.x][y];
  }
}

__global__ void k_f32_to_bf16(const float* __restrict__ in, long n, __nv_bfloat16* out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

// Mean-squared error of pred [rows, ld] (first cols columns) against
// target [rows, cols]: loss += sum((p - t)^2) / count, grad = 2 (p - t) / count
// as BF16 [rows, ld] with zero padding columns (and as FP32 when gradf is set).
__global__ void k_mse(const float* __restrict__ pred, int ld, const float* __restrict__ tgt, int rows, int cols,
                      float inv_count, __nv_bfloat16* grad, float* gradf, float* loss) {
  float s = 0.f;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (long)rows * ld; i += (long)gridDim.x * blockDim.x) {
    const long r = i / ld;
    const int c = (int)(i % ld);
    float g = 0.f;
    if (c < cols) {
      const float d = pred[i] - tgt[r * cols + c];
      s += d * d;
      g = 2.f * d * inv_count;
    }
    grad[i] = __float2bfloat16_rn(g);
    if (gradf) gradf[i] = g;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_count);
}

// Adam on FP32 master weights w [n]; w16 gets the BF16 copy and, when
// rows > 0, w16t the BF16 transpose of w viewed as [rows, n / rows].
__global__ void k_adam(float* w, const float* __restrict__ g, float* m, float* v, long n, float lr, float b1,
                       float b2, float eps, float c1, float c2, float wd, __nv_bfloat16* w16, __nv_bfloat16* w16t,
                       int rows) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16_rn(wi);
    if (w16t && rows > 0) {
      const long cols = n / rows, r = i / cols, c = i % cols;
      w16t[c * rows + r] = __float2bfloat16_rn(wi);
    }
  }
}

int g_smem_set[64];   // dynamic shared memory granted to k_gemm_bf16, per device

inline int blocks_for(long n, int t) { return (int)min((n + t - 1) / t, (long)148 * 16); }

}  // namespace

extern "C" {

int ffnn_gemm(const void* A, int lda, const void* B, int ldb, int M, int N, int K, const float* bias, int act,
              float* zf, int ldz, int atomic, void* yb, int ldy, int ksplit, void* stream) {
  if (!A || !B || M < 1 || N < 1 || K < 16 || (K % 16) || (lda % 8) || (ldb % 8) || lda < K || ldb < K)
    return FFNN_ERR_ARG;
  if (((uintptr_t)A & 15) || ((uintptr_t)B & 15) || (!zf && !yb) || (atomic && !zf)) return FFNN_ERR_ARG;
  if (ksplit <= 0 || ksplit >= K) ksplit = K;
  else ksplit = (ksplit + GKT - 1) / GKT * GKT;
  if (ksplit < K && !atomic) return FFNN_ERR_ARG;   // partial sums need the atomic epilogue
  GemmArgs g;
  g.A = (const __nv_bfloat16*)A; g.B = (const __nv_bfloat16*)B;
  g.lda = lda; g.ldb = ldb; g.M = M; g.N = N; g.K = K;
  g.nt = N <= 256 ? (N + 15) / 16 * 16 : 256;
  g.ksplit = ksplit;
  g.bias = bias; g.act = act; g.zf = zf; g.ldz = ldz; g.atomic = atomic;
  g.yb = (__nv_bfloat16*)yb; g.ldy = ldy;
  // tensor-memory columns of a CTA; shared memory sized so that the CTAs
  // resident on one SM never ask for more than its 512 columns
  int ncol = 32;
  while (ncol < g.nt) ncol <<= 1;
  size_t smem = 2 * (size_t)(GM + g.nt) * GKT * 2 + 64;
  const size_t floor_ = ncol >= 256 ? 80 * 1024 : (ncol >= 128 ? 48 * 1024 : (ncol >= 64 ? 28 * 1024 : 0));
  if (smem < floor_) smem = floor_;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return FFNN_ERR_CUDA;
  if (g_smem_set[dev] < (int)smem) {
    if (cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024) != cudaSuccess)
      return FFNN_ERR_CUDA;
    g_smem_set[dev] = 100 * 1024;
  }
  dim3 grid((M + GM - 1) / GM, (N + g.nt - 1) / g.nt, (K + ksplit - 1) / ksplit);
  k_gemm_bf16<<<grid, GTHREADS, smem, (cudaStream_t)stream>>>(g);
  return cudaGetLastError() == cudaSuccess ? 0 : FFNN_ERR_CUDA;
}

int ffnn_silu_bwd(const float* dy, const float* z, long n, void* dzb, float* dzf, void* stream) {
  if (n <= 0) return 0;
  k_silu_bwd<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(dy, z, n, (__nv_bfloat16*)dzb, dzf);
  return cudaGetLastError() == cudaSuccess ? 0 : FFNN_ERR_CUDA;
}

int ffnn_colsum(const float* x, int rows, int cols, int ld, float* out, void* stream) {
  if (rows <= 0 || cols <= 0) return 0;
  dim3 grid(min(rows, 1024), (cols + 127) / 128);
  k_colsum<<<grid, 128, 0, (cudaStream_t)stream>>>(x, rows, cols, ld, out);
  return cudaGetLastError() == cudaSuccess ? 0 : FFNN_ERR_CUDA;
}

int ffnn_transpose(const void* in, int rows, int cols, int ldi, void* out, int ldo, int rows_pad, void* stream) {
  if (rows_pad < rows || ldo < rows_pad) return FFNN_ERR_ARG;
  dim3 grid((rows_pad + 31) / 32, (cols + 31) / 32);
  k_transpose_bf16<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in, rows, cols, ldi,
                                                                  (__nv_bfloat16*)out, ldo, rows_pad);
  return cudaGetLastError() == cudaSuccess ? 0 : FFNN_ERR_CUDA;
}

int ffnn_to_bf16(const float* in, long n, void* out, void* stream) {
  if (n <= 0) return 0;
  k_f32_to_bf16<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(in, n, (__nv_bfloat16*)out);
  return cudaGetLastError() == cudaSuccess ? 0 : FFNN_ERR_CUDA;
}

int ffnn_mse(const float* pred, int ld, const float* tgt, int rows, int cols, void* grad, float* gradf, float* loss,
             void* stream) {
  if (rows <= 0 || cols <= 0 || ld < cols) return FFNN_ERR_ARG;
  long n = (long)rows * ld;
  k_mse<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(pred, ld, tgt, rows, cols, 1.f / ((float)rows * cols),
                                                              (__nv_bfloat16*)grad, gradf, loss);
  return cudaGetLastError() == cudaSuccess ? 0 : FFNN_ERR_CUDA;
}

int ffnn_adam(float* w, const float* g, float* m, float* v, long n, float lr, float b1, float b2, float eps,
              int step, float wd, void* w16, void* w16t, int rows, void* stream) {
  if (n <= 0 || step < 1) return FFNN_ERR_ARG;
  const float c1 = 1.f / (1.f - powf(b1, (float)step)), c2 = 1.f / (1.f - powf(b2, (float)step));
  k_adam<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2, wd,
                                                               (__nv_bfloat16*)w16, (__nv_bfloat16*)w16t, rows);
  return cudaGetLastError() == cudaSuccess ? 0 : FFNN_ERR_CUDA;
}

int ffnn_error(int reset) {
  int e = 0;
  if (cudaMemcpyFromSymbol(&e, g_err, sizeof(int)) != cudaSuccess) return FFNN_ERR_CUDA;
  if (reset) {
    int z = 0;
    if (cudaMemcpyToSymbol(g_err, &z, sizeof(int)) != cudaSuccess) return FFNN_ERR_CUDA;
  }
  return e ? FFNN_ERR_TIMEOUT : 0;
}

}  // extern "C"
