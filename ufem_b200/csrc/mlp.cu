// The warm-start network: a 3-layer GELU MLP (n_in -> H -> H -> n_out) that
// maps a Monte Carlo sample's random parameters to coefficients on a POD
// basis of earlier solutions.  No counterpart in the reference (the closest
// hook is the disabled warm start of monte_linear_solver, fem/fem_mont.c:493-504).
//
// Every matrix product, forward and backward, runs on the 5th-generation
// tensor cores through one hand-written kernel, k_gemm_tc:
//   C[M x N] = A[M x K] . B[N x K]^T   (BF16 operands, FP32 accumulation)
// * A and B are staged from global memory (any element strides, so the
//   backward products read transposed operands without copies) into shared
//   memory in the canonical no-swizzle K-major layout of the UMMA
//   descriptors: 8-row x 16-byte core matrices, K-adjacent core matrices
//   128 B apart (LBO), 8-row groups KC/8 * 128 B apart (SBO).  A thread
//   stages a whole core matrix with eight 16-byte loads (K-contiguous
//   operands directly, M-contiguous ones through an 8 x 8 register
//   transpose); two operand stages let the next K chunk be staged while the
//   tensor cores work on the current one;
// * one elected thread issues tcgen05.mma.cta_group::1.kind::f16 (M = 128,
//   N <= 256, K = 16 per instruction) into an FP32 accumulator in tensor
//   memory (TMEM) and tcgen05.commit arrives on an mbarrier; all waits are
//   bounded (an iteration limit sets an error flag and the kernel still
//   frees its TMEM);
// * the epilogue reads the accumulator with tcgen05.ld.32x32b (warp w owns
//   TMEM lanes 32w..32w+31 = rows of the tile) and applies bias, GELU or the
//   GELU derivative.
// Master weights and Adam moments are FP32; BF16 copies feed the GEMMs.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "tcgen05.cuh"
#include "ufem_internal.h"

namespace ufem {
namespace {

constexpr int kTileM = 128;   // UMMA M (TMEM lanes)
constexpr int kMaxN = 256;    // UMMA N per CTA (TMEM columns)
constexpr int kKC = 64;       // K chunk staged per round
constexpr int kGemmThreads = 128;
constexpr long kSpinLimit = 1L << 26;

// the stream every launch of this file goes to: 0 for the public calls, the
// capture stream while a training step is being recorded as a CUDA graph
static cudaStream_t g_stream = 0;

struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16 *A;
  long a_sm, a_sk;  // A(m, k) = A[m * a_sm + k * a_sk]
  const __nv_bfloat16 *B;
  long b_sn, b_sk;  // B(n, k) = B[n * b_sn + k * b_sk]
  int epi;          // 0: C = acc; 1: Z = acc + bias, H = gelu(Z); 2: C = acc + bias;
                    // 3: D = acc * gelu'(Zin) -> C (FP32) and H (BF16)
  float *C;
  long ldc;
  const float *bias;
  float *Z;         // epi 1: pre-activation out; epi 3: pre-activation in
  __nv_bfloat16 *H; // epi 1/3: BF16 copy of the output
  long ldh;
  int *err;
};

using tc::smem_u32;

// byte offset of element (r, k) of an R x KC tile in the core-matrix layout
__device__ __forceinline__ uint32_t cm_offset(int r, int k) { return tc::cm_offset(r, k, kKC); }

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// 8 x 8 transpose of BF16 values held as 8 rows of 16 bytes: in[k] holds
// rows m = 0..7 of column k, out[m] holds columns k = 0..7 of row m.  Pairs
// of 16-bit halves are exchanged with byte permutes; the rest is renaming.
__device__ __forceinline__ void transpose8x8_bf16(const uint4 (&in)[8], uint4 (&out)[8]) {
  uint32_t w[8][4];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    w[k][0] = in[k].x; w[k][1] = in[k].y; w[k][2] = in[k].z; w[k][3] = in[k].w;
  }
  uint32_t o[8][4];
#pragma unroll
  for (int kp = 0; kp < 4; kp++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint32_t a = w[2 * kp][j], b = w[2 * kp + 1][j];  // rows 2j, 2j+1 of columns 2kp, 2kp+1
      o[2 * j][kp] = __byte_perm(a, b, 0x5410);               // row 2j: columns 2kp, 2kp+1
      o[2 * j + 1][kp] = __byte_perm(a, b, 0x7632);           // row 2j+1
    }
#pragma unroll
  for (int m = 0; m < 8; m++) out[m] = make_uint4(o[m][0], o[m][1], o[m][2], o[m][3]);
}

// Stages rows [r_base, r_base + nrows) x columns [k0, k0 + KC) of an operand
// X(r, k) = src[r * s_r + k * s_k] (rows >= r_lim and columns >= K read 0)
// into the core-matrix layout.  One 8 x 8 core matrix per thread step: a
// K-contiguous operand is read as 8 rows of 16 bytes, an R-contiguous one
// (the backward products' transposed operands) as 8 columns of 16 bytes and
// transposed in registers; edge and unaligned tiles element by element.
__device__ __forceinline__ void stage_operand(const __nv_bfloat16 *__restrict__ src, long s_r, long s_k, int r_base,
                                              int r_lim, int K, int k0, int nrows, uint8_t *dst) {
  const bool kvec = s_k == 1 && (s_r & 7) == 0 && ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
  const bool rvec = s_r == 1 && (s_k & 7) == 0 && ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
  const int ntiles = (nrows / 8) * (kKC / 8);
  for (int t = threadIdx.x; t < ntiles; t += kGemmThreads) {
    const int r0 = (t / (kKC / 8)) * 8, kk = (t % (kKC / 8)) * 8;
    const int gr = r_base + r0, gk = k0 + kk;
    const bool full = gr + 8 <= r_lim && gk + 8 <= K;
    uint8_t *d = dst + cm_offset(r0, kk);  // the tile's 8 rows of 16 bytes
    if (full && kvec) {
#pragma unroll
      for (int i = 0; i < 8; i++)
        *reinterpret_cast<uint4 *>(d + 16 * i) =
            __ldg(reinterpret_cast<const uint4 *>(src + (long)(gr + i) * s_r + gk));
    } else if (full && rvec) {
      uint4 in[8], out[8];
#pragma unroll
      for (int i = 0; i < 8; i++) in[i] = __ldg(reinterpret_cast<const uint4 *>(src + gr + (long)(gk + i) * s_k));
      transpose8x8_bf16(in, out);
#pragma unroll
      for (int i = 0; i < 8; i++) *reinterpret_cast<uint4 *>(d + 16 * i) = out[i];
    } else {
      for (int i = 0; i < 8; i++)
        for (int e = 0; e < 8; e++) {
          __nv_bfloat16 v = __float2bfloat16(0.0f);
          if (gr + i < r_lim && gk + e < K) v = src[(long)(gr + i) * s_r + (long)(gk + e) * s_k];
          *reinterpret_cast<__nv_bfloat16 *>(d + 16 * i + 2 * e) = v;
        }
    }
  }
}

// Two operand stages: the next K chunk is staged while the tensor cores work
// on the current one; the MMAs of a stage arrive on that stage's mbarrier.
constexpr int kStageA = kTileM * kKC * 2;        // 16 KB
constexpr int kStageBytes = kStageA + kMaxN * kKC * 2;  // + 32 KB

__global__ void __launch_bounds__(kGemmThreads) k_gemm_tc(GemmArgs g) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int s_bad;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kTileM;
  const int N = g.N;
  const int ncols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  if (threadIdx.x == 0) {
    s_bad = 0;
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base, ncols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::idesc_bf16(kTileM, N);
  const uint32_t sbo = (kKC / 8) * 128;
  uint32_t phase[2] = {0u, 0u};
  const int nchunks = (g.K + kKC - 1) / kKC;
  auto stage = [&](int c) {
    uint8_t *sA = smem + (c & 1) * kStageBytes;
    stage_operand(g.A, g.a_sm, g.a_sk, m0, g.M, g.K, c * kKC, kTileM, sA);
    stage_operand(g.B, g.b_sn, g.b_sk, 0, N, g.K, c * kKC, N, sA + kStageA);
  };
  stage(0);
  for (int c = 0; c < nchunks; c++) {
    const int buf = c & 1;
    // make the generic-proxy shared stores visible to the tensor core
    tc::fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc::fence_after_sync();
      const uint8_t *sA = smem + buf * kStageBytes, *sB = sA + kStageA;
      for (int ks = 0; ks < kKC / 16; ks++) {
        const uint64_t da = tc::desc_kmajor(tc::smem_u32(sA) + ks * 256, 128, sbo);
        const uint64_t db = tc::desc_kmajor(tc::smem_u32(sB) + ks * 256, 128, sbo);
        tc::mma_bf16(tmem, da, db, idesc, c > 0 || ks > 0);
      }
      tc::commit(&mbar[buf]);
    }
    if (c + 1 < nchunks) {
      const int nb = buf ^ 1;
      // the other stage is free once the MMAs of chunk c - 1 have read it
      if (c >= 1) {
        if (!tc::mbar_wait(&mbar[nb], phase[nb], kSpinLimit)) s_bad = 1;
        phase[nb] ^= 1u;
      }
      __syncthreads();
      if (s_bad) break;
      stage(c + 1);
    }
  }
  // the last commit arrives once every MMA of the block has completed
  if (!s_bad) {
    const int lb = (nchunks - 1) & 1;
    if (!tc::mbar_wait(&mbar[lb], phase[lb], kSpinLimit)) s_bad = 1;
  }
  __syncthreads();
  tc::fence_after_sync();
  if (!s_bad) {
    // epilogue: warp w owns TMEM lanes 32w..32w+31 = rows m0+32w+lane
    const int m = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < N; c0 += 32) {
      uint32_t v[32];
      tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (m < g.M) {
#pragma unroll
        for (int j = 0; j < 32; j++) {
          const int n = c0 + j;
          if (n >= N) break;
          float a = __uint_as_float(v[j]);
          switch (g.epi) {
            case 0:
              g.C[(long)m * g.ldc + n] = a;
              break;
            case 1: {
              const float z = a + g.bias[n];
              g.Z[(long)m * g.ldc + n] = z;
              g.H[(long)m * g.ldh + n] = __float2bfloat16(gelu(z));
              break;
            }
            case 2:
              g.C[(long)m * g.ldc + n] = a + g.bias[n];
              break;
            default: {
              const float d = a * gelu_grad(g.Z[(long)m * g.ldc + n]);
              g.C[(long)m * g.ldc + n] = d;
              g.H[(long)m * g.ldh + n] = __float2bfloat16(d);
              break;
            }
          }
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
  if (threadIdx.x == 0 && s_bad) atomicExch(g.err, 1);
}

// The two operand stages take 96 KB; the request is padded to 100 KB so that
// at most two CTAs share an SM, which keeps their TMEM allocations (<= 256
// columns each) within the SM's 512 columns without any CTA waiting.
constexpr size_t kGemmSmem = 100 * 1024;
static_assert(2 * (size_t)kStageBytes <= kGemmSmem, "operand stages exceed the shared-memory request");

// ---- small elementwise kernels ---------------------------------------------
__global__ void k_to_bf16_pad(long rows, int cols, int ld_out, const float *__restrict__ x,
                              __nv_bfloat16 *__restrict__ y) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= rows * ld_out) return;
  long r = t / ld_out;
  int c = (int)(t % ld_out);
  y[t] = __float2bfloat16(c < cols ? x[r * cols + c] : 0.0f);
}

__global__ void k_f32_to_bf16(long n, const float *__restrict__ x, __nv_bfloat16 *__restrict__ y) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t < n) y[t] = __float2bfloat16(x[t]);
}

// dY = 2 (Y - T) / (B * n_out) and the per-row squared error
__global__ void k_loss_grad(long B, int n_out, const float *__restrict__ Y, const float *__restrict__ T,
                            float *__restrict__ dY, __nv_bfloat16 *__restrict__ dYb, float *__restrict__ rowloss) {
  long b = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (b >= B) return;
  const float scale = 2.0f / (float)(B * n_out);
  float s = 0.0f;
  for (int o = 0; o < n_out; o++) {
    const float d = Y[b * n_out + o] - T[b * n_out + o];
    s += d * d;
    dY[b * n_out + o] = scale * d;
    dYb[b * n_out + o] = __float2bfloat16(scale * d);
  }
  rowloss[b] = s;
}

// column sums of a row-major [B][n] matrix (bias gradients), fixed order
__global__ void k_colsum(long B, int n, const float *__restrict__ x, float *__restrict__ out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  float s = 0.0f;
  for (long b = 0; b < B; b++) s += x[b * n + c];
  out[c] = s;
}

__global__ void k_sum(long n, const float *__restrict__ x, float *__restrict__ out) {
  __shared__ float sh[256];
  float s = 0.0f;
  for (long i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// Adam with the learning rate taken from a per-step schedule and the bias
// corrections from the device step counter, so that one captured training
// step can be replayed (CUDA graph) without host arguments.
__global__ void k_adam_sched(long n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m1,
                             float *__restrict__ m2, const float *__restrict__ sched, const long *__restrict__ step,
                             float b1, float b2, float eps, const unsigned char *__restrict__ frozen) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n || (frozen && frozen[i])) return;
  const long s = *step;
  const float lr = sched[s];
  const float c1 = 1.0f - powf(b1, (float)(s + 1)), c2 = 1.0f - powf(b2, (float)(s + 1));
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// end of a replayed step: add its loss to the running sum, advance the step
__global__ void k_step_tail(const float *__restrict__ loss, float *__restrict__ acc, long *__restrict__ step) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    *acc += *loss;
    *step += 1;
  }
}

// minibatch rows of a replayed step: rows perm[b * B + r], b = step mod (steps per epoch)
__global__ void k_gather_step(long B, int ncol, const long *__restrict__ perm, const long *__restrict__ step,
                              long steps_per_epoch, const float *__restrict__ src, float *__restrict__ dst) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= B * ncol) return;
  const long r = t / ncol, b = (*step) % steps_per_epoch;
  dst[t] = src[perm[b * B + r] * ncol + (t % ncol)];
}

__global__ void k_adam(long n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m1,
                       float *__restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2,
                       const unsigned char *__restrict__ frozen) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n || (frozen && frozen[i])) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

}  // namespace
}  // namespace ufem

using namespace ufem;

// ---------------------------------------------------------------------------
struct ufem_mlp {
  int n_in = 0, n_inp = 0, H = 0, n_out = 0;  // n_inp: n_in padded to 32
  long nparam = 0;
  // FP32 master parameters (flat: W1 [H][n_inp], b1, W2 [H][H], b2, W3 [n_out][H], b3)
  DBuf<float> w, grad, m1, m2;
  DBuf<unsigned char> frozen;  // padded input columns of W1 stay zero
  DBuf<__nv_bfloat16> wb;      // BF16 copies of W1, W2, W3
  long oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0;
  long step = 0;
  // activations for a batch
  long cap = 0;
  DBuf<__nv_bfloat16> X, H1, H2, dYb, dZ2b, dZ1b;
  DBuf<float> Z1, Z2, Y, dY, dZ2, dZ1, dH, rowloss, scal;
  DBuf<int> err;
};

namespace {

int gemm_configure() {
  static bool configured = false;
  if (!configured) {
    UFEM_CUDA_TRY(cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem));
    configured = true;
  }
  return UFEM_AF_OK;
}

int launch_gemm(const GemmArgs &a) {
  if (a.N > kMaxN || a.N % 16 != 0) {
    set_error("tensor-core GEMM: N must be a multiple of 16 up to 256");
    return UFEM_AF_ERR_SIZ;
  }
  int rv = gemm_configure();
  if (rv != UFEM_AF_OK) return rv;
  dim3 grid((unsigned)((a.M + kTileM - 1) / kTileM));
  k_gemm_tc<<<grid, kGemmThreads, kGemmSmem, g_stream>>>(a);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

int ensure_batch(ufem_mlp *p, long B) {
  if (B <= p->cap) return UFEM_AF_OK;
  int rv;
  const long H = p->H;
  if ((rv = p->X.alloc(B * p->n_inp)) || (rv = p->H1.alloc(B * H)) || (rv = p->H2.alloc(B * H)) ||
      (rv = p->dYb.alloc(B * p->n_out)) || (rv = p->dZ2b.alloc(B * H)) || (rv = p->dZ1b.alloc(B * H)) ||
      (rv = p->Z1.alloc(B * H)) || (rv = p->Z2.alloc(B * H)) || (rv = p->Y.alloc(B * p->n_out)) ||
      (rv = p->dY.alloc(B * p->n_out)) || (rv = p->dZ2.alloc(B * H)) || (rv = p->dZ1.alloc(B * H)) ||
      (rv = p->dH.alloc(B * H)) || (rv = p->rowloss.alloc(B)) || (rv = p->scal.alloc(4)))
    return rv;
  p->cap = B;
  return UFEM_AF_OK;
}

int refresh_bf16(ufem_mlp *p) {
  const long n1 = (long)p->H * p->n_inp, n2 = (long)p->H * p->H, n3 = (long)p->n_out * p->H;
  k_f32_to_bf16<<<(unsigned)((n1 + 255) / 256), 256, 0, g_stream>>>(n1, p->w.p + p->oW1, p->wb.p);
  k_f32_to_bf16<<<(unsigned)((n2 + 255) / 256), 256, 0, g_stream>>>(n2, p->w.p + p->oW2, p->wb.p + n1);
  k_f32_to_bf16<<<(unsigned)((n3 + 255) / 256), 256, 0, g_stream>>>(n3, p->w.p + p->oW3, p->wb.p + n1 + n2);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

GemmArgs gemm(int M, int N, int K, const __nv_bfloat16 *A, long a_sm, long a_sk, const __nv_bfloat16 *B, long b_sn,
              long b_sk, int epi, float *C, long ldc, const float *bias, float *Z, __nv_bfloat16 *H, long ldh,
              int *err) {
  GemmArgs a;
  a.M = M; a.N = N; a.K = K; a.A = A; a.a_sm = a_sm; a.a_sk = a_sk; a.B = B; a.b_sn = b_sn; a.b_sk = b_sk;
  a.epi = epi; a.C = C; a.ldc = ldc; a.bias = bias; a.Z = Z; a.H = H; a.ldh = ldh; a.err = err;
  return a;
}

int forward(ufem_mlp *p, long B, const float *d_x) {
  int rv;
  const int H = p->H;
  const __nv_bfloat16 *W1 = p->wb.p, *W2 = W1 + (long)H * p->n_inp, *W3 = W2 + (long)H * H;
  k_to_bf16_pad<<<(unsigned)((B * p->n_inp + 255) / 256), 256, 0, g_stream>>>(B, p->n_in, p->n_inp, d_x, p->X.p);
  // Z1 = X W1^T + b1, H1 = gelu(Z1)
  if ((rv = launch_gemm(gemm((int)B, H, p->n_inp, p->X.p, p->n_inp, 1, W1, p->n_inp, 1, 1, nullptr, H,
                             p->w.p + p->ob1, p->Z1.p, p->H1.p, H, p->err.p))))
    return rv;
  // Z2 = H1 W2^T + b2, H2 = gelu(Z2)
  if ((rv = launch_gemm(gemm((int)B, H, H, p->H1.p, H, 1, W2, H, 1, 1, nullptr, H, p->w.p + p->ob2, p->Z2.p,
                             p->H2.p, H, p->err.p))))
    return rv;
  // Y = H2 W3^T + b3
  return launch_gemm(gemm((int)B, p->n_out, H, p->H2.p, H, 1, W3, H, 1, 2, p->Y.p, p->n_out, p->w.p + p->ob3,
                          nullptr, nullptr, 0, p->err.p));
}

// gradients of the mean squared error into p->grad; the loss into p->scal[0]
int backward(ufem_mlp *p, long B, const float *d_t) {
  int rv;
  const int H = p->H, O = p->n_out;
  const __nv_bfloat16 *W2 = p->wb.p + (long)H * p->n_inp, *W3 = W2 + (long)H * H;
  k_loss_grad<<<(unsigned)((B + 127) / 128), 128, 0, g_stream>>>(B, O, p->Y.p, d_t, p->dY.p, p->dYb.p, p->rowloss.p);
  k_sum<<<1, 256, 0, g_stream>>>(B, p->rowloss.p, p->scal.p);
  float *gW1 = p->grad.p + p->oW1, *gb1 = p->grad.p + p->ob1, *gW2 = p->grad.p + p->oW2;
  float *gb2 = p->grad.p + p->ob2, *gW3 = p->grad.p + p->oW3, *gb3 = p->grad.p + p->ob3;
  // dW3 = dY^T H2 (O x H, K = B); db3 = colsum(dY)
  if ((rv = launch_gemm(gemm(O, H, (int)B, p->dYb.p, 1, O, p->H2.p, 1, H, 0, gW3, H, nullptr, nullptr, nullptr, 0,
                             p->err.p))))
    return rv;
  k_colsum<<<(O + 127) / 128, 128, 0, g_stream>>>(B, O, p->dY.p, gb3);
  // dZ2 = (dY W3) * gelu'(Z2)   (B x H, K = O)
  if ((rv = launch_gemm(gemm((int)B, H, O, p->dYb.p, O, 1, W3, 1, H, 3, p->dZ2.p, H, nullptr, p->Z2.p, p->dZ2b.p,
                             H, p->err.p))))
    return rv;
  // dW2 = dZ2^T H1 (H x H, K = B); db2
  if ((rv = launch_gemm(gemm(H, H, (int)B, p->dZ2b.p, 1, H, p->H1.p, 1, H, 0, gW2, H, nullptr, nullptr, nullptr, 0,
                             p->err.p))))
    return rv;
  k_colsum<<<(H + 127) / 128, 128, 0, g_stream>>>(B, H, p->dZ2.p, gb2);
  // dZ1 = (dZ2 W2) * gelu'(Z1)   (B x H, K = H)
  if ((rv = launch_gemm(gemm((int)B, H, H, p->dZ2b.p, H, 1, W2, 1, H, 3, p->dZ1.p, H, nullptr, p->Z1.p, p->dZ1b.p,
                             H, p->err.p))))
    return rv;
  // dW1 = dZ1^T X (H x n_inp, K = B); db1
  if ((rv = launch_gemm(gemm(H, p->n_inp, (int)B, p->dZ1b.p, 1, H, p->X.p, 1, p->n_inp, 0, gW1, p->n_inp, nullptr,
                             nullptr, nullptr, 0, p->err.p))))
    return rv;
  k_colsum<<<(H + 127) / 128, 128, 0, g_stream>>>(B, H, p->dZ1.p, gb1);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

int check_mlp_err(ufem_mlp *p) {
  int h = 0;
  UFEM_CUDA_TRY(cudaMemcpy(&h, p->err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    set_error("tensor-core GEMM: MMA completion wait timed out");
    return UFEM_AF_ERR;
  }
  return UFEM_AF_OK;
}

}  // namespace

namespace ufem {

// Trains the network for `epochs` passes over (X [ntrain][n_in], T
// [ntrain][n_out]) in minibatches of bs rows, reshuffled every epoch (seeded),
// with the per-step learning rates `sched` (epochs * ntrain / bs values).  One
// training step -- minibatch gather, forward, backward, Adam, BF16 refresh --
// is recorded once as a CUDA graph on its own stream and replayed for every
// step; the host only uploads each epoch's permutation and reads each
// epoch's summed loss.  loss_first / loss_last: mean squared error of the
// first and last epoch (per output, as ufem_mlp_train_step reports it).
int mlp_train_graph(ufem_mlp *p, long ntrain, int bs, const float *d_X, const float *d_T,
                    const std::vector<float> &sched, int epochs, unsigned long long seed, float *loss_first,
                    float *loss_last, long *steps) {
  int rv;
  const long nb = ntrain / bs;
  const long total = (long)epochs * nb;
  if (nb < 1 || (long)sched.size() < total) {
    set_error("mlp_train_graph: need at least one minibatch and a learning rate per step");
    return UFEM_AF_ERR_SIZ;
  }
  DBuf<long> perm, step;
  DBuf<float> d_sched, acc, Xb, Tb;
  if ((rv = ensure_batch(p, bs)) || (rv = perm.alloc(ntrain)) || (rv = step.alloc(1)) ||
      (rv = d_sched.upload(sched.data(), total)) || (rv = acc.alloc(1)) ||
      (rv = Xb.alloc((size_t)bs * p->n_in)) || (rv = Tb.alloc((size_t)bs * p->n_out)) || (rv = gemm_configure()))
    return rv;
  UFEM_CUDA_TRY(cudaMemset(step.p, 0, sizeof(long)));
  cudaStream_t st;
  UFEM_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int fail = UFEM_AF_OK;
  // ---- record one step ------------------------------------------------------
  g_stream = st;
  cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) {
    const long nx = (long)bs * p->n_in, nt = (long)bs * p->n_out;
    k_gather_step<<<(unsigned)((nx + 255) / 256), 256, 0, st>>>(bs, p->n_in, perm.p, step.p, nb, d_X, Xb.p);
    k_gather_step<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(bs, p->n_out, perm.p, step.p, nb, d_T, Tb.p);
    if ((fail = forward(p, bs, Xb.p)) == UFEM_AF_OK && (fail = backward(p, bs, Tb.p)) == UFEM_AF_OK) {
      k_adam_sched<<<(unsigned)((p->nparam + 255) / 256), 256, 0, st>>>(p->nparam, p->w.p, p->grad.p, p->m1.p,
                                                                         p->m2.p, d_sched.p, step.p, 0.9f, 0.999f,
                                                                         1e-8f, p->frozen.p);
      if ((fail = refresh_bf16(p)) == UFEM_AF_OK) k_step_tail<<<1, 32, 0, st>>>(p->scal.p, acc.p, step.p);
    }
    ce = cudaStreamEndCapture(st, &graph);
  }
  g_stream = 0;
  if (fail == UFEM_AF_OK && ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
  if (fail != UFEM_AF_OK || ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(st);
    if (fail == UFEM_AF_OK) set_error(std::string("MLP training graph: ") + cudaGetErrorString(ce));
    return fail != UFEM_AF_OK ? fail : UFEM_AF_ERR;
  }
  // ---- replay ----------------------------------------------------------------
  std::mt19937_64 rng(seed);
  std::vector<long> idx(ntrain);
  for (long i = 0; i < ntrain; i++) idx[i] = i;
  const float norm = 1.0f / ((float)nb * (float)bs * (float)p->n_out);
  for (int ep = 0; ep < epochs && ce == cudaSuccess; ep++) {
    std::shuffle(idx.begin(), idx.end(), rng);
    ce = cudaMemcpyAsync(perm.p, idx.data(), ntrain * sizeof(long), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(acc.p, 0, sizeof(float), st);
    for (long b = 0; b < nb && ce == cudaSuccess; b++) ce = cudaGraphLaunch(exec, st);
    float h = 0.0f;
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&h, acc.p, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ep == 0 && loss_first) *loss_first = h * norm;
    if (loss_last) *loss_last = h * norm;
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  cudaStreamDestroy(st);
  if (ce != cudaSuccess) {
    set_error(std::string("MLP training replay: ") + cudaGetErrorString(ce));
    return UFEM_AF_ERR;
  }
  p->step += total;
  if (steps) *steps = total;
  return check_mlp_err(p);
}

}  // namespace ufem

extern "C" {

int ufem_mlp_create(int n_in, int n_hidden, int n_out, unsigned long long seed, ufem_mlp **out) {
  if (n_in < 1 || n_in > 32 || n_hidden < 16 || n_hidden > 256 || n_hidden % 16 || n_out < 16 || n_out > 256 ||
      n_out % 16) {
    set_error("ufem_mlp_create: n_in <= 32; n_hidden and n_out multiples of 16 up to 256");
    return UFEM_AF_ERR_SIZ;
  }
  ufem_mlp *p = new ufem_mlp();
  p->n_in = n_in;
  p->n_inp = 32;
  p->H = n_hidden;
  p->n_out = n_out;
  const long H = n_hidden;
  p->oW1 = 0;
  p->ob1 = p->oW1 + H * p->n_inp;
  p->oW2 = p->ob1 + H;
  p->ob2 = p->oW2 + H * H;
  p->oW3 = p->ob2 + H;
  p->ob3 = p->oW3 + (long)n_out * H;
  p->nparam = p->ob3 + n_out;
  // He-style uniform initialisation, seeded; padded input columns zero and frozen
  std::mt19937_64 rng(seed);
  std::vector<float> w(p->nparam, 0.0f);
  std::vector<unsigned char> fr(p->nparam, 0);
  auto fill = [&](long off, long rows, long cols, long fan_in, long valid_cols) {
    const float lim = std::sqrt(6.0f / (float)fan_in);
    std::uniform_real_distribution<float> u(-lim, lim);
    for (long r = 0; r < rows; r++)
      for (long c = 0; c < cols; c++) {
        if (c < valid_cols) w[off + r * cols + c] = u(rng);
        else fr[off + r * cols + c] = 1;
      }
  };
  fill(p->oW1, H, p->n_inp, n_in, n_in);
  fill(p->oW2, H, H, H, H);
  fill(p->oW3, n_out, H, H, H);
  int rv;
  if ((rv = p->w.upload(w.data(), w.size())) || (rv = p->grad.alloc(p->nparam)) || (rv = p->m1.alloc(p->nparam)) ||
      (rv = p->m2.alloc(p->nparam)) || (rv = p->frozen.upload(fr.data(), fr.size())) ||
      (rv = p->wb.alloc(H * p->n_inp + H * H + (long)n_out * H)) || (rv = p->err.alloc(1))) {
    delete p;
    return rv;
  }
  cudaMemset(p->m1.p, 0, p->nparam * sizeof(float));
  cudaMemset(p->m2.p, 0, p->nparam * sizeof(float));
  cudaMemset(p->err.p, 0, sizeof(int));
  if ((rv = refresh_bf16(p)) != UFEM_AF_OK) {
    delete p;
    return rv;
  }
  *out = p;
  return UFEM_AF_OK;
}

void ufem_mlp_free(ufem_mlp *p) { delete p; }

long ufem_mlp_num_params(const ufem_mlp *p) { return p->nparam; }

int ufem_mlp_get_params(const ufem_mlp *p, float *h) {
  UFEM_CUDA_TRY(cudaMemcpy(h, p->w.p, p->nparam * sizeof(float), cudaMemcpyDeviceToHost));
  return UFEM_AF_OK;
}

int ufem_mlp_set_params(ufem_mlp *p, const float *h) {
  UFEM_CUDA_TRY(cudaMemcpy(p->w.p, h, p->nparam * sizeof(float), cudaMemcpyHostToDevice));
  return refresh_bf16(p);
}

int ufem_mlp_forward(ufem_mlp *p, long nbatch, const float *d_x, float *d_y) {
  int rv;
  if ((rv = ensure_batch(p, nbatch)) || (rv = forward(p, nbatch, d_x))) return rv;
  UFEM_CUDA_TRY(cudaMemcpy(d_y, p->Y.p, nbatch * p->n_out * sizeof(float), cudaMemcpyDeviceToDevice));
  return check_mlp_err(p);
}

int ufem_mlp_gradients(ufem_mlp *p, long nbatch, const float *d_x, const float *d_t, float *h_grad, float *loss) {
  int rv;
  if ((rv = ensure_batch(p, nbatch)) || (rv = forward(p, nbatch, d_x)) || (rv = backward(p, nbatch, d_t))) return rv;
  if ((rv = check_mlp_err(p)) != UFEM_AF_OK) return rv;
  if (h_grad) UFEM_CUDA_TRY(cudaMemcpy(h_grad, p->grad.p, p->nparam * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss) {
    float s = 0;
    UFEM_CUDA_TRY(cudaMemcpy(&s, p->scal.p, sizeof(float), cudaMemcpyDeviceToHost));
    *loss = s / (float)(nbatch * p->n_out);
  }
  return UFEM_AF_OK;
}

int ufem_mlp_train_step(ufem_mlp *p, long nbatch, const float *d_x, const float *d_t, float lr, float *loss) {
  int rv;
  if ((rv = ensure_batch(p, nbatch)) || (rv = forward(p, nbatch, d_x)) || (rv = backward(p, nbatch, d_t))) return rv;
  p->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)p->step), c2 = 1.0f - std::pow(b2, (float)p->step);
  k_adam<<<(unsigned)((p->nparam + 255) / 256), 256, 0, g_stream>>>(p->nparam, p->w.p, p->grad.p, p->m1.p, p->m2.p, lr, b1, b2,
                                                       1e-8f, c1, c2, p->frozen.p);
  if ((rv = refresh_bf16(p)) != UFEM_AF_OK) return rv;
  if (loss) {
    float s = 0;
    UFEM_CUDA_TRY(cudaMemcpy(&s, p->scal.p, sizeof(float), cudaMemcpyDeviceToHost));
    *loss = s / (float)(nbatch * p->n_out);
  }
  return check_mlp_err(p);
}

// C = A . B^T on the tensor cores, for tests of the GEMM itself: A [M x K]
// and B [N x K] row-major BF16, C [M x N] row-major FP32 (device pointers).
int ufem_tc_gemm_bf16(int M, int N, int K, const void *d_A, const void *d_B, float *d_C) {
  DBuf<int> err;
  int rv;
  if ((rv = err.alloc(1)) != UFEM_AF_OK) return rv;
  UFEM_CUDA_TRY(cudaMemset(err.p, 0, sizeof(int)));
  GemmArgs a = gemm(M, N, K, (const __nv_bfloat16 *)d_A, K, 1, (const __nv_bfloat16 *)d_B, K, 1, 0, d_C, N, nullptr,
                    nullptr, nullptr, 0, err.p);
  if ((rv = launch_gemm(a)) != UFEM_AF_OK) return rv;
  int h = 0;
  UFEM_CUDA_TRY(cudaMemcpy(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    set_error("tensor-core GEMM: MMA completion wait timed out");
    return UFEM_AF_ERR;
  }
  return UFEM_AF_OK;
}

}  // extern "C"
