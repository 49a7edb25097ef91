// Learned warm start for the batched Monte Carlo solve.  No counterpart in
// the reference: its only hook is the disabled warm start of
// monte_linear_solver (fem/fem_mont.c:493-504, the femVecClone of the
// previous solution into u before femEqsCGwSSOR).
//
// Pipeline, every step on the GPU:
//   1. the batched solver (batch.cu) solves ntrain samples from zero; their
//      solutions U [ndof][ntrain] stay on the device;
//   2. POD basis Phi [ndof][r] of the first nsnap solutions: randomised
//      subspace iteration (Halko, Martinsson & Tropp, SIAM Review 53, 2011,
//      algorithm 4.4) with l = r + 16 columns, every product orthonormalised
//      through the eigen-decomposition of its Gram matrix (twice), then a
//      Rayleigh-Ritz step that orders the modes by energy; when the
//      snapshots span fewer than r directions above 1e-12 of the largest
//      singular value, the missing modes are zero columns;
//   3. targets: the coefficients Phi^T u of every training solution divided
//      by the sample's load scale (the solution is linear in the load),
//      standardised per mode; inputs: the chosen ifld columns, log|.| where
//      asked, standardised;
//   4. the MLP (mlp.cu: tcgen05 BF16 GEMMs, FP32 accumulation, Adam) is
//      trained on them for a number of epochs with a cosine learning rate;
//   5. a warm-started solve runs the MLP on the new samples' inputs, forms
//      u0 = scale * Phi c in FP64 and hands it to the batched PCG as the
//      initial guess, with the iteration cap set to the largest count the
//      cold training solves needed.  A sample that does not converge within
//      it (the guess made the iterations regress) is solved again from zero
//      by the same batched solver and reported UFEM_ST_FALLBACK.
//
// Dense FP64 products run in one generic tiled kernel (k_gemm_f64) with a
// split K dimension whose partial sums are added in a fixed order, so every
// result is identical run to run.  The l x l symmetric eigenproblems run in
// one thread block (k_jacobi_eig): cyclic Jacobi with the round-robin
// ordering, l/2 disjoint rotations per round.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "ufem_internal.h"

namespace ufem {

namespace {

// ---------------------------------------------------------------------------
// C(m, n) = alpha * sum_k A(m, k) B(k, n), any element strides
// ---------------------------------------------------------------------------
constexpr int kGT = 64;   // output tile (kGT x kGT), 4 x 4 per thread
constexpr int kGK = 16;   // K chunk staged in shared memory
constexpr int kMaxSplits = 64;

struct G64 {
  int M, N;
  long K;
  const double *A;
  long sam, sak;
  const double *B;
  long sbk, sbn;
  double *C;
  long scm, scn;
  double alpha;
  int splits;
  double *part;  // [splits][M][N] when splits > 1
};

__global__ void __launch_bounds__(256) k_gemm_f64(G64 g) {
  __shared__ double As[kGK][kGT + 1];
  __shared__ double Bs[kGK][kGT + 1];
  const int m0 = blockIdx.x * kGT, n0 = blockIdx.y * kGT;
  const long per = (g.K + g.splits - 1) / g.splits;
  const long kbeg = (long)blockIdx.z * per, kend = min(g.K, kbeg + per);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const bool a_kfast = (g.sak == 1), b_kfast = (g.sbk == 1);
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
  for (long kb = kbeg; kb < kend; kb += kGK) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = threadIdx.x + 256 * q;
      int mm, kk;
      if (a_kfast) { kk = e % kGK; mm = e / kGK; }
      else { mm = e % kGT; kk = e / kGT; }
      const long gk = kb + kk;
      const int gm = m0 + mm;
      As[kk][mm] = (gm < g.M && gk < kend) ? g.A[(size_t)gm * g.sam + (size_t)gk * g.sak] : 0.0;
      int nn;
      if (b_kfast) { kk = e % kGK; nn = e / kGK; }
      else { nn = e % kGT; kk = e / kGT; }
      const long gk2 = kb + kk;
      const int gn = n0 + nn;
      Bs[kk][nn] = (gn < g.N && gk2 < kend) ? g.B[(size_t)gk2 * g.sbk + (size_t)gn * g.sbn] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; kk++) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int gm = m0 + ty + 16 * i, gn = n0 + tx + 16 * j;
      if (gm >= g.M || gn >= g.N) continue;
      if (g.splits == 1) g.C[(size_t)gm * g.scm + (size_t)gn * g.scn] = g.alpha * acc[i][j];
      else g.part[((size_t)blockIdx.z * g.M + gm) * g.N + gn] = acc[i][j];
    }
}

__global__ void k_split_sum(int M, int N, int splits, const double *__restrict__ part, double alpha,
                            double *__restrict__ C, long scm, long scn) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long)M * N) return;
  const int m = (int)(e / N), n = (int)(e % N);
  double t = 0.0;
  for (int s = 0; s < splits; s++) t += part[(size_t)s * M * N + e];
  C[(size_t)m * scm + (size_t)n * scn] = alpha * t;
}

// Launches k_gemm_f64; splits the K range when the output has few tiles.
int gemm_f64(int M, int N, long K, const double *A, long sam, long sak, const double *B, long sbk, long sbn,
             double *C, long scm, long scn, DBuf<double> &part, double alpha = 1.0) {
  if (M <= 0 || N <= 0) return UFEM_AF_OK;
  G64 g;
  g.M = M; g.N = N; g.K = K; g.A = A; g.sam = sam; g.sak = sak; g.B = B; g.sbk = sbk; g.sbn = sbn;
  g.C = C; g.scm = scm; g.scn = scn; g.alpha = alpha; g.splits = 1; g.part = nullptr;
  const long tiles = (long)((M + kGT - 1) / kGT) * ((N + kGT - 1) / kGT);
  if (tiles < 296 && K > 512) {
    long s = (296 + tiles - 1) / tiles;
    s = std::min<long>(s, K / 256);
    s = std::min<long>(s, kMaxSplits);
    g.splits = (int)std::max<long>(1, s);
  }
  if (g.splits > 1) {
    int rv = part.ensure((size_t)g.splits * M * N);
    if (rv != UFEM_AF_OK) return rv;
    g.part = part.p;
  }
  dim3 grid((unsigned)((M + kGT - 1) / kGT), (unsigned)((N + kGT - 1) / kGT), (unsigned)g.splits);
  k_gemm_f64<<<grid, 256>>>(g);
  if (g.splits > 1) {
    const long tot = (long)M * N;
    k_split_sum<<<(unsigned)((tot + 255) / 256), 256>>>(M, N, g.splits, part.p, alpha, C, scm, scn);
  }
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

// ---------------------------------------------------------------------------
// symmetric eigen-decomposition of an l x l matrix (l even, <= kMaxL) in one
// block: cyclic Jacobi, round-robin ordering (l - 1 rounds of l/2 disjoint
// rotations per sweep), rotation of Numerical Recipes (Press et al., 11.1):
// theta = (a_qq - a_pp) / (2 a_pq), t = sgn(theta) / (|theta| + sqrt(theta^2 + 1)),
// c = 1 / sqrt(t^2 + 1), s = t c; A <- P^T A P, V <- V P.  A is kept in
// shared memory; V too up to kSmemL, beyond that transposed in the global
// workspace Vg (row p = column p of V, so a rotation reads two contiguous
// rows; the l x l doubles stay in L2).
// ---------------------------------------------------------------------------
constexpr int kMaxL = 144;
constexpr int kSmemL = 96;
constexpr int kJacThreads = 512;

template <bool VG>
__global__ void __launch_bounds__(kJacThreads) k_jacobi_eig(int l, const double *__restrict__ Ain,
                                                            double *__restrict__ Vout, double *__restrict__ lam,
                                                            int max_sweeps, int *__restrict__ sweeps_out,
                                                            double *__restrict__ Vg) {
  extern __shared__ double sm[];
  const int ld = l + 1;
  double *A = sm;                        // [l][ld]
  double *V = sm + l * ld;               // [l][ld] (shared-memory V only)
  double *cs = VG ? V : V + l * ld;      // [l/2][2]
  int *pq = (int *)(cs + l);             // [l/2][2]
  __shared__ double red[kJacThreads];
  __shared__ int s_done;
  const int half = l / 2;
  for (int e = threadIdx.x; e < l * l; e += blockDim.x) {
    const int i = e / l, j = e % l;
    A[i * ld + j] = 0.5 * (Ain[i * l + j] + Ain[j * l + i]);
    if (VG) Vg[i * l + j] = (i == j) ? 1.0 : 0.0;
    else V[i * ld + j] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  int sweep = 0;
  for (; sweep < max_sweeps; sweep++) {
    // convergence test: off-diagonal mass against the diagonal
    double off = 0.0, dia = 0.0;
    for (int e = threadIdx.x; e < l * l; e += blockDim.x) {
      const int i = e / l, j = e % l;
      const double v = A[i * ld + j];
      if (i == j) dia += v * v;
      else off += v * v;
    }
    red[threadIdx.x] = off;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    const double off_t = red[0];
    __syncthreads();
    red[threadIdx.x] = dia;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    const double dia_t = red[0];
    if (threadIdx.x == 0) s_done = (off_t <= 1e-30 * dia_t) || !(off_t > 0.0);
    __syncthreads();
    if (s_done) break;
    for (int round = 0; round < l - 1; round++) {
      if (threadIdx.x < half) {
        const int k = threadIdx.x;
        int p, q;
        if (k == 0) { p = round; q = l - 1; }
        else { p = (round + k) % (l - 1); q = (round - k + (l - 1)) % (l - 1); }
        if (p > q) { const int t = p; p = q; q = t; }
        const double apq = A[p * ld + q], app = A[p * ld + p], aqq = A[q * ld + q];
        double c = 1.0, s = 0.0;
        if (fabs(apq) > 1e-300 && fabs(apq) > 1e-18 * sqrt(fabs(app * aqq))) {
          const double theta = (aqq - app) / (2.0 * apq);
          double t;
          if (fabs(theta) > 1e150) t = 0.5 / theta;
          else t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          c = 1.0 / sqrt(t * t + 1.0);
          s = t * c;
        }
        pq[2 * k] = p; pq[2 * k + 1] = q;
        cs[2 * k] = c; cs[2 * k + 1] = s;
      }
      __syncthreads();
      // rows p, q of A
      for (int e = threadIdx.x; e < half * l; e += blockDim.x) {
        const int k = e / l, j = e % l;
        const int p = pq[2 * k], q = pq[2 * k + 1];
        const double c = cs[2 * k], s = cs[2 * k + 1];
        const double a = A[p * ld + j], b = A[q * ld + j];
        A[p * ld + j] = c * a - s * b;
        A[q * ld + j] = s * a + c * b;
      }
      __syncthreads();
      // columns p, q of A and of V
      for (int e = threadIdx.x; e < half * l; e += blockDim.x) {
        const int k = e / l, i = e % l;
        const int p = pq[2 * k], q = pq[2 * k + 1];
        const double c = cs[2 * k], s = cs[2 * k + 1];
        double a = A[i * ld + p], b = A[i * ld + q];
        A[i * ld + p] = c * a - s * b;
        A[i * ld + q] = s * a + c * b;
        if (VG) {
          a = Vg[p * l + i];
          b = Vg[q * l + i];
          Vg[p * l + i] = c * a - s * b;
          Vg[q * l + i] = s * a + c * b;
        } else {
          a = V[i * ld + p];
          b = V[i * ld + q];
          V[i * ld + p] = c * a - s * b;
          V[i * ld + q] = s * a + c * b;
        }
      }
      __syncthreads();
    }
  }
  for (int e = threadIdx.x; e < l * l; e += blockDim.x) {
    const int i = e / l, j = e % l;
    Vout[i * l + j] = VG ? Vg[j * l + i] : V[i * ld + j];
  }
  for (int j = threadIdx.x; j < l; j += blockDim.x) lam[j] = A[j * ld + j];
  if (threadIdx.x == 0 && sweeps_out) *sweeps_out = sweep;
}

size_t jacobi_smem(int l) {
  const int nmat = l <= kSmemL ? 2 : 1;
  return (size_t)(nmat * l * (l + 1) + l) * sizeof(double) + (size_t)l * sizeof(int);
}

// eigen-decomposition of dA [l x l] -> dV (columns), dlam; dVg: l x l scratch (l > kSmemL)
int jacobi_eig(int l, const double *dA, double *dV, double *dlam, int *dsweeps, double *dVg) {
  const size_t smem = jacobi_smem(l);
  if (l <= kSmemL) {
    UFEM_CUDA_TRY(cudaFuncSetAttribute(k_jacobi_eig<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_jacobi_eig<false><<<1, kJacThreads, smem>>>(l, dA, dV, dlam, 60, dsweeps, nullptr);
  } else {
    UFEM_CUDA_TRY(cudaFuncSetAttribute(k_jacobi_eig<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_jacobi_eig<true><<<1, kJacThreads, smem>>>(l, dA, dV, dlam, 60, dsweeps, dVg);
  }
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

// T[i][c] = V[i][perm[c]] * scale[c]   (l rows, rc columns)
__global__ void k_cols_perm_scale(int l, int rc, const double *__restrict__ V, const int *__restrict__ perm,
                                  const double *__restrict__ scale, double *__restrict__ T) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= l * rc) return;
  const int i = e / rc, c = e % rc;
  T[e] = V[i * l + perm[c]] * scale[c];
}

// ---------------------------------------------------------------------------
// features, targets, statistics
// ---------------------------------------------------------------------------
// raw[s][f] = ifld[s][col[f]] (log|.| where asked)
__global__ void k_feat_raw(long nsamp, int nf, long ilen, const double *__restrict__ ifld, const long *__restrict__ col,
                           const int *__restrict__ lg, double *__restrict__ raw) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nsamp * nf) return;
  const long s = e / nf;
  const int f = (int)(e % nf);
  double v = ifld[s * ilen + col[f]];
  if (lg[f] == 2) v = v != 0.0 ? 1.0 / v : 0.0;  // compliance-like inputs (1/E)
  else if (lg[f]) v = log(fabs(v));
  raw[e] = v;
}

// per-column mean and standard deviation (each column summed in row order)
__global__ void k_col_stats(long nrow, int ncol, const double *__restrict__ X, double *__restrict__ mean,
                            double *__restrict__ sd) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  double s = 0.0;
  for (long r = 0; r < nrow; r++) s += X[r * ncol + c];
  const double mu = s / (double)nrow;
  double v = 0.0;
  for (long r = 0; r < nrow; r++) {
    const double d = X[r * ncol + c] - mu;
    v += d * d;
  }
  v /= (double)nrow;
  mean[c] = mu;
  sd[c] = v > 0.0 ? sqrt(v) : 1.0;
}

// network input rows: standardised features, zero-padded to ldx columns (FP32)
__global__ void k_standardise(long nsamp, int nf, int ldx, const double *__restrict__ raw,
                              const double *__restrict__ mean, const double *__restrict__ sd, float *__restrict__ X) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nsamp * ldx) return;
  const long s = e / ldx;
  const int f = (int)(e % ldx);
  X[e] = f < nf ? (float)((raw[s * nf + f] - mean[f]) / sd[f]) : 0.0f;
}

// per-sample load scale (1 when no scale column)
__global__ void k_scale(long nsamp, long ilen, long col, const double *__restrict__ ifld, double *__restrict__ sc) {
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsamp) return;
  sc[s] = col >= 0 ? ifld[s * ilen + col] : 1.0;
}

// c[s][k] /= sc[s]
__global__ void k_div_scale(long nsamp, int r, const double *__restrict__ sc, double *__restrict__ c) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nsamp * r) return;
  const double d = sc[e / r];
  c[e] = d != 0.0 ? c[e] / d : 0.0;
}

__global__ void k_mul(long n, double f, double *__restrict__ c) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) c[e] *= f;
}

// FP32 targets t = (c - mean) / sd
__global__ void k_targets(long nsamp, int r, const double *__restrict__ c, const double *__restrict__ mean,
                          const double *__restrict__ sd, float *__restrict__ t) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nsamp * r) return;
  const int k = (int)(e % r);
  t[e] = (float)((c[e] - mean[k]) / sd[k]);
}

// Least-squares part of the coefficient model: a full quadratic polynomial
// in the standardised features xs (1, xs_f, xs_i xs_j for i <= j),
// lin(x)[k] = sum_j W[j][k] phi_j(xs).  The MLP learns only what this misses,
// so its BF16 arithmetic and its fitting error act on a small residual
// instead of the whole coefficient.  nterms(nf) = 1 + nf + nf (nf + 1) / 2.
// With fewer than 4 training samples per quadratic term the model keeps the
// linear terms only (quad = 0).
__host__ __device__ __forceinline__ int poly_terms(int nf, int quad) { return 1 + nf + (quad ? nf * (nf + 1) / 2 : 0); }

__device__ __forceinline__ void poly_features(int nf, int quad, const double *__restrict__ raw,
                                              const double *__restrict__ fmean, const double *__restrict__ fsd,
                                              double *phi) {
  double xs[32];
  for (int f = 0; f < nf; f++) xs[f] = (raw[f] - fmean[f]) / fsd[f];
  int j = 0;
  phi[j++] = 1.0;
  for (int f = 0; f < nf; f++) phi[j++] = xs[f];
  if (quad)
    for (int a = 0; a < nf; a++)
      for (int b = a; b < nf; b++) phi[j++] = xs[a] * xs[b];
}

__device__ __forceinline__ double lin_model(int nf, int quad, int r, int k, const double *__restrict__ raw,
                                            const double *__restrict__ fmean, const double *__restrict__ fsd,
                                            const double *__restrict__ W) {
  double xs[32];
  for (int f = 0; f < nf; f++) xs[f] = (raw[f] - fmean[f]) / fsd[f];
  double t = W[k];
  int j = 1;
  for (int f = 0; f < nf; f++) t = fma(xs[f], W[(size_t)(j++) * r + k], t);
  if (quad)
    for (int a = 0; a < nf; a++)
      for (int b = a; b < nf; b++) t = fma(xs[a] * xs[b], W[(size_t)(j++) * r + k], t);
  return t;
}

// network outputs -> coefficients: c[s][k] = (lin(x_s)[k] + y * sd + mean) * sc[s]
// (W == nullptr: no least-squares part)
__global__ void k_coeffs(long nsamp, int r, int nf, int quad, const float *__restrict__ y, const double *__restrict__ mean,
                         const double *__restrict__ sd, const double *__restrict__ raw,
                         const double *__restrict__ fmean, const double *__restrict__ fsd,
                         const double *__restrict__ W, const double *__restrict__ sc, double gscale,
                         double *__restrict__ c) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nsamp * r) return;
  const int k = (int)(e % r);
  const long s = e / r;
  const double lin = W ? lin_model(nf, quad, r, k, raw + s * nf, fmean, fsd, W) : 0.0;
  c[e] = (lin + (double)y[e] * sd[k] + mean[k]) * sc[s] * gscale;
}

// design matrix of the least-squares model: D[s] = phi(xs_s), one thread per sample
__global__ void k_design(long nsamp, int nf, int quad, const double *__restrict__ raw, const double *__restrict__ fmean,
                         const double *__restrict__ fsd, double *__restrict__ D) {
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsamp) return;
  poly_features(nf, quad, raw + s * nf, fmean, fsd, D + s * poly_terms(nf, quad));
}

// c[s][k] -= lin(x_s)[k]: the residual the MLP is trained on
__global__ void k_lin_resid(long nsamp, int r, int nf, int quad, const double *__restrict__ raw,
                            const double *__restrict__ fmean, const double *__restrict__ fsd,
                            const double *__restrict__ W, double *__restrict__ c) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nsamp * r) return;
  c[e] -= lin_model(nf, quad, r, (int)(e % r), raw + (e / r) * nf, fmean, fsd, W);
}

// rows of a row-major matrix picked by idx (minibatches)
template <typename T>
__global__ void k_gather_rows(long nrow, int ncol, const long *__restrict__ idx, const T *__restrict__ src,
                              T *__restrict__ dst) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nrow * ncol) return;
  const long r = e / ncol;
  dst[e] = src[idx[r] * ncol + (e % ncol)];
}

// rows of src scattered back to the rows idx of a row-major matrix
template <typename T>
__global__ void k_scatter_rows(long nrow, int ncol, const long *__restrict__ idx, const T *__restrict__ src,
                               T *__restrict__ dst) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nrow * ncol) return;
  const long r = e / ncol;
  dst[idx[r] * ncol + (e % ncol)] = src[e];
}

// Ordering score of a sample: the spread (standard deviation) over its E
// variables of log(a_v / mean a_v).  Samples far from the mean operator --
// the coarse space's -- need more PCG iterations (correlation 0.77 on the
// zone beam), and a group of 128 samples iterates until its slowest one.
__global__ void k_order_score(long nsamp, long ilen, int nmult, const double *__restrict__ ifld,
                              const int *__restrict__ mcol, const double *__restrict__ log_abar,
                              double *__restrict__ score) {
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsamp) return;
  double m1 = 0.0, m2 = 0.0;
  for (int v = 1; v < nmult; v++) {
    const double t = log(fabs(ifld[s * ilen + mcol[v]])) - log_abar[v];
    m1 += t;
    m2 += t * t;
  }
  const double k = (double)max(1, nmult - 1);
  score[s] = m2 / k - (m1 / k) * (m1 / k);
}

// |u0_s - u_s| / |u_s| per sample, both [n][S], in two passes with a fixed
// order: k_rel_err_part sums a chunk of rows for 32 samples per block (8
// warps stride the chunk, combined in warp order), k_rel_err adds the chunks.
constexpr int kErrChunks = 64;
__global__ void __launch_bounds__(256) k_rel_err_part(long n, int S, const double *__restrict__ u0,
                                                      const double *__restrict__ u, double *__restrict__ part) {
  __shared__ double sa[8][32], sb[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int s = blockIdx.x * 32 + lane;  // S is a multiple of 128
  const long per = (n + gridDim.y - 1) / gridDim.y;
  const long i0 = (long)blockIdx.y * per, i1 = min(n, i0 + per);
  double a = 0.0, b = 0.0;
  for (long i = i0 + w; i < i1; i += 8) {
    const double x = u[i * S + s], d = u0[i * S + s] - x;
    a += d * d;
    b += x * x;
  }
  sa[w][lane] = a;
  sb[w][lane] = b;
  __syncthreads();
  if (w == 0) {
    double ta = 0.0, tb = 0.0;
    for (int k = 0; k < 8; k++) {
      ta += sa[k][lane];
      tb += sb[k][lane];
    }
    part[((size_t)blockIdx.y * S + s) * 2] = ta;
    part[((size_t)blockIdx.y * S + s) * 2 + 1] = tb;
  }
}
__global__ void k_rel_err(int nch, int S, int nsamp, const double *__restrict__ part, double *__restrict__ err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsamp) return;
  double a = 0.0, b = 0.0;
  for (int c = 0; c < nch; c++) {
    a += part[((size_t)c * S + s) * 2];
    b += part[((size_t)c * S + s) * 2 + 1];
  }
  err[s] = b > 0.0 ? sqrt(a / b) : sqrt(a);
}

// [n][S] (first nsamp columns) -> [nsamp][n]
__global__ void k_to_sample_major(long n, int S, long nsamp, const double *__restrict__ src, double *__restrict__ dst) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * nsamp) return;
  const long i = e / nsamp, s = e % nsamp;
  dst[s * n + i] = src[i * S + s];
}

// Y [n][r] = K_v Phi: the part of the implicit stiffness that multiplier v
// scales (supported rows and columns are zero in the unit blocks; Phi is zero
// on supported DOFs, so the identity rows add nothing to Phi^T K Phi).
// thread per (block row I, column k)
template <int B>
__global__ void k_zone_apply(int nbr, int r, const int *__restrict__ crow, const double *__restrict__ cval,
                             int cstride, int v, const double *__restrict__ Phi, double *__restrict__ Y) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)nbr * r) return;
  const int I = (int)(t / r), k = (int)(t % r);
  double y[B];
#pragma unroll
  for (int a = 0; a < B; a++) y[a] = 0.0;
  for (int c = crow[I]; c < crow[I + 1]; c++) {
    const double *w = cval + (size_t)c * cstride;
    const long long key = (long long)w[B * B];
    if ((int)(key >> 32) != v) continue;
    const int J = (int)(key & 0xffffffffLL);
#pragma unroll
    for (int a = 0; a < B; a++)
#pragma unroll
      for (int b = 0; b < B; b++) y[a] += w[a * B + b] * Phi[(size_t)(J * B + b) * r + k];
  }
#pragma unroll
  for (int a = 0; a < B; a++) Y[(size_t)(I * B + a) * r + k] = y[a];
}

// Prow[j][k] = Phi[row_j][k]: the basis rows of the randomised loads
__global__ void k_phi_rows(int nrow, int r, const int *__restrict__ rows, const double *__restrict__ Phi,
                           double *__restrict__ Prow) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrow * r) return;
  Prow[t] = Phi[(size_t)rows[t / r] * r + (t % r)];
}

// The POD-Galerkin coefficients of one sample per block: A = sum_v a_v G_v
// (a_0 = 1, a_v = the sample's E of variable v), b = Phi^T F0 + sum_j
// f_j Phi[row_j], A c = b by Cholesky in shared memory.  Directions with a
// pivot below 1e-13 of the largest diagonal (zero basis columns) get c = 0.
constexpr int kMaxR = 128;
constexpr int kRedThreads = 256;
// A is kept as a packed lower triangle, row i at i (i + 1) / 2 (66 KB at
// r = 128, so three samples share an SM); warps own rows (assembly and the
// Cholesky updates read and write along a row), one warp does both
// triangular solves.
__device__ __forceinline__ int tri(int i) { return i * (i + 1) / 2; }

__global__ void __launch_bounds__(kRedThreads) k_reduced_solve(long nsamp, int r, int nmult, long ilen,
                                                               const double *__restrict__ ifld,
                                                               const int *__restrict__ mcol,
                                                               const double *__restrict__ G,
                                                               const double *__restrict__ PF0, int novr,
                                                               const int *__restrict__ ovar,
                                                               const double *__restrict__ Prow, int ldg,
                                                               double *__restrict__ c_out) {
  extern __shared__ double s_A[];  // packed lower triangle of the r x r system
  __shared__ double bb[kMaxR];
  __shared__ double av[64];
  __shared__ int skip[kMaxR];
  __shared__ double s_dmax;
  constexpr int kW = kRedThreads / 32;
  const long s = blockIdx.x;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const double *row = ifld + s * ilen;
  for (int v = tid; v < nmult; v += blockDim.x) av[v] = (v == 0) ? 1.0 : row[mcol[v]];
  __syncthreads();
  // A[i][k] = sum_v a_v G_v[i][k], k <= i: warp w takes rows w, w + kW, ...
  for (int i = warp; i < r; i += kW)
    for (int k = lane; k <= i; k += 32) {
      const double *g = G + (size_t)i * ldg + k;  // leading r x r block of each ldg x ldg operator
      double t = 0.0;
#pragma unroll 4
      for (int v = 0; v < nmult; v++) t = fma(av[v], __ldg(g + (size_t)v * ldg * ldg), t);
      s_A[tri(i) + k] = t;
    }
  for (int i = tid; i < r; i += blockDim.x) {
    double t = PF0[i];
    for (int j = 0; j < novr; j++) t += row[ovar[j]] * Prow[(size_t)j * ldg + i];
    bb[i] = t;
  }
  __syncthreads();
  if (warp == 0) {
    double m = 0.0;
    for (int i = lane; i < r; i += 32) m = fmax(m, fabs(s_A[tri(i) + i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) s_dmax = m;
  }
  __syncthreads();
  const double dmax = s_dmax;
  // right-looking Cholesky, L in the packed lower triangle
  for (int j = 0; j < r; j++) {
    // column j below the diagonal scaled by 1 / L_jj (every thread reads the
    // pivot; it is rewritten only in the next phase)
    const double d = s_A[tri(j) + j];
    const bool sk = !(d > 1e-13 * dmax);
    const double inv = sk ? 0.0 : 1.0 / sqrt(d);
    for (int i = j + 1 + tid; i < r; i += blockDim.x) s_A[tri(i) + j] *= inv;
    __syncthreads();
    if (tid == 0) {
      s_A[tri(j) + j] = sk ? 1.0 : sqrt(d);
      skip[j] = sk;
    }
    // trailing update A[i][k] -= L[i][j] L[k][j], j < k <= i, along rows
    for (int i = j + 1 + warp; i < r; i += kW) {
      const double lij = s_A[tri(i) + j];
      for (int k = j + 1 + lane; k <= i; k += 32) s_A[tri(i) + k] = fma(-lij, s_A[tri(k) + j], s_A[tri(i) + k]);
    }
    __syncthreads();
  }
  // L y = b, then L^T c = y, by warp 0 (bb holds y, then c)
  if (warp == 0) {
    for (int j = 0; j < r; j++) {
      const double y = skip[j] ? 0.0 : bb[j] / s_A[tri(j) + j];
      __syncwarp();
      if (lane == 0) bb[j] = y;
      for (int i = j + 1 + lane; i < r; i += 32) bb[i] = fma(-s_A[tri(i) + j], y, bb[i]);
      __syncwarp();
    }
    for (int i = r - 1; i >= 0; i--) {
      const double c = skip[i] ? 0.0 : bb[i] / s_A[tri(i) + i];
      __syncwarp();
      if (lane == 0) bb[i] = c;
      for (int k = lane; k < i; k += 32) bb[k] = fma(-s_A[tri(i) + k], c, bb[k]);
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = tid; i < r; i += blockDim.x) c_out[s * r + i] = bb[i];
}

int grid1(long n, int b = 256) { return (int)((n + b - 1) / b); }

}  // namespace

}  // namespace ufem

using namespace ufem;

struct ufem_warm {
  ufem_model *m = nullptr;
  ufem_warm_options o;
  int r = 0, l = 0;   // guess / MLP modes; subspace width of the POD fit
  int rb = 0;         // basis columns computed: max(n_modes, n_coarse) (phi row stride)
  long n = 0;
  ufem_mlp *mlp = nullptr;
  bool trained = false;
  long cold_cap = 0;
  int train_precision = -1;  // the cap holds for solves at this precision
  // POD-Galerkin operators (when the model has at most 64 E variables)
  bool galerkin = false;
  int nmult = 0;
  DBuf<double> Gv, PF0, Prow;
  DBuf<int> d_mcol, d_ovar;
  int novr = 0;
  double guess_scale = 1.0;
  int coarse_modes = 0;                   // modes of the preconditioner's coarse space
  DBuf<double> log_abar;                  // log of the training samples' mean multipliers (sample ordering)
  DBuf<double> score, ifperm, ofperm;
  DBuf<int> stperm;
  DBuf<long> itperm, sperm;
  // basis and normalisation
  DBuf<double> phi;                       // [n][r]
  DBuf<double> fmean, fsd, cmean, csd;    // feature / coefficient statistics
  DBuf<double> linW;                      // [terms][r] least-squares (quadratic) model of the coefficients
  DBuf<double> design, gram;              // [ntrain][terms] design matrix; normal equations
  int lin_quad = 0;                       // the least-squares model has the quadratic terms
  DBuf<long> fcol;
  DBuf<int> flog;
  std::vector<double> sigma2;             // Rayleigh-Ritz energies of the modes
  // scratch
  DBuf<double> U, Y, Q, Z, G, V, lam, T, scale, part, raw, sc, c;
  DBuf<int> perm, sweeps;
  DBuf<float> X, Tt, Yo;
  DBuf<double> ifsub, u0, uf, err, errpart;
  DBuf<double> Vg;                        // eigenvector scratch of the larger bases
  DBuf<double> ofsub;
  DBuf<int> stsub;
  DBuf<long> itsub;
  DBuf<int> st;
  DBuf<long> it;
};

namespace ufem {

int mc_solve_device(int nmesh, ufem_model *const *models, const long *nsamp, const double *const *d_ifld,
                    double *const *d_ofld, int *const *d_status, long *const *d_iters,
                    const double *const *d_u_guess, double *const *d_u_out, const ufem_mc_options *opt_in);

namespace {

// eigen-decomposition of the l x l matrix w->G; columns of w->V sorted by
// descending eigenvalue through w->perm, eigenvalues (sorted) into lam_sorted
int sym_eig_sorted(ufem_warm *w, int l, std::vector<double> &lam_sorted, std::vector<int> &order) {
  int rv;
  if (l > kSmemL && (rv = w->Vg.ensure((size_t)l * l))) return rv;
  if ((rv = jacobi_eig(l, w->G.p, w->V.p, w->lam.p, w->sweeps.p, w->Vg.p))) return rv;
  std::vector<double> lam(l);
  UFEM_CUDA_TRY(cudaMemcpy(lam.data(), w->lam.p, l * sizeof(double), cudaMemcpyDeviceToHost));
  order.resize(l);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return lam[a] > lam[b]; });
  lam_sorted.resize(l);
  for (int j = 0; j < l; j++) lam_sorted[j] = lam[order[j]];
  return UFEM_AF_OK;
}

// Yin [rows][l] -> out [rows][l] with orthonormal columns spanning Yin:
// T = V Lambda^-1/2 from the eigen-decomposition of the Gram matrix Yin^T Yin
// (directions whose eigenvalue is below 1e-24 of the largest, i.e. singular
// values below 1e-12 of the largest, become zero columns), out = Yin T; done
// twice so the columns are orthonormal to working precision.  tmp: rows*l.
int orthonormalise(ufem_warm *w, long rows, int l, const double *Yin, double *out, double *tmp) {
  int rv;
  const double *src = Yin;
  for (int pass = 0; pass < 2; pass++) {
    if ((rv = gemm_f64(l, l, rows, src, 1, l, src, l, 1, w->G.p, l, 1, w->part))) return rv;
    std::vector<double> lam;
    std::vector<int> order;
    if ((rv = sym_eig_sorted(w, l, lam, order))) return rv;
    std::vector<double> scale(l, 0.0);
    const double lmax = std::max(lam[0], 0.0);
    for (int j = 0; j < l; j++) scale[j] = (lmax > 0.0 && lam[j] > 1e-24 * lmax) ? 1.0 / std::sqrt(lam[j]) : 0.0;
    if ((rv = w->perm.upload(order.data(), l)) || (rv = w->scale.upload(scale.data(), l))) return rv;
    k_cols_perm_scale<<<grid1((long)l * l), 256>>>(l, l, w->V.p, w->perm.p, w->scale.p, w->T.p);
    double *dst = (pass == 0) ? tmp : out;
    if ((rv = gemm_f64((int)rows, l, l, src, l, 1, w->T.p, l, 1, dst, l, 1, w->part))) return rv;
    src = dst;
  }
  return UFEM_AF_OK;
}

// POD basis of the first nsnap columns of U [n][S]: randomised range finder
// with power iterations, every product followed by an orthonormalisation
// (Halko, Martinsson & Tropp 2011, algorithm 4.4), then Rayleigh-Ritz.
int fit_basis(ufem_warm *w, int S, long nsnap) {
  int rv;
  const long n = w->n;
  const int l = w->l, r = w->rb;  // every basis column (guess and coarse space)
  const long big = std::max<long>(nsnap, n);
  if ((rv = w->Y.ensure((size_t)big * l)) || (rv = w->Q.ensure((size_t)n * l)) ||
      (rv = w->Z.ensure((size_t)big * l)) || (rv = w->G.ensure((size_t)l * l)) ||
      (rv = w->V.ensure((size_t)l * l)) || (rv = w->lam.ensure(l)) || (rv = w->T.ensure((size_t)l * l)) ||
      (rv = w->scale.ensure(l)) || (rv = w->perm.ensure(l)) || (rv = w->sweeps.ensure(1)) ||
      (rv = w->phi.ensure((size_t)n * r)))
    return rv;
  // Omega [nsnap][l], seeded standard normal
  std::mt19937_64 rng(w->o.seed ^ 0x5eed0f0dULL);
  std::normal_distribution<double> nd(0.0, 1.0);
  std::vector<double> om((size_t)nsnap * l);
  for (auto &v : om) v = nd(rng);
  DBuf<double> d_om, zq;
  if ((rv = d_om.upload(om.data(), om.size())) || (rv = zq.ensure((size_t)nsnap * l))) return rv;
  // Q = orth(U Omega)
  if ((rv = gemm_f64((int)n, l, nsnap, w->U.p, S, 1, d_om.p, l, 1, w->Y.p, l, 1, w->part))) return rv;
  if ((rv = orthonormalise(w, n, l, w->Y.p, w->Q.p, w->Z.p))) return rv;
  for (int it = 0; it < w->o.power_iters; it++) {
    // Zq = orth(U^T Q) [nsnap][l]; Q = orth(U Zq)
    if ((rv = gemm_f64((int)nsnap, l, n, w->U.p, 1, S, w->Q.p, l, 1, w->Y.p, l, 1, w->part))) return rv;
    if ((rv = orthonormalise(w, nsnap, l, w->Y.p, zq.p, w->Z.p))) return rv;
    if ((rv = gemm_f64((int)n, l, nsnap, w->U.p, S, 1, zq.p, l, 1, w->Y.p, l, 1, w->part))) return rv;
    if ((rv = orthonormalise(w, n, l, w->Y.p, w->Q.p, w->Z.p))) return rv;
  }
  // Rayleigh-Ritz: Z = U^T Q, H = Z^T Z, H = W mu W^T, Phi = Q W[:, :r]
  if ((rv = gemm_f64((int)nsnap, l, n, w->U.p, 1, S, w->Q.p, l, 1, w->Z.p, l, 1, w->part))) return rv;
  if ((rv = gemm_f64(l, l, nsnap, w->Z.p, 1, l, w->Z.p, l, 1, w->G.p, l, 1, w->part))) return rv;
  std::vector<double> mu;
  std::vector<int> order;
  if ((rv = sym_eig_sorted(w, l, mu, order))) return rv;
  std::vector<double> one(r, 1.0);
  if ((rv = w->perm.upload(order.data(), l)) || (rv = w->scale.upload(one.data(), r))) return rv;
  k_cols_perm_scale<<<grid1((long)l * r), 256>>>(l, r, w->V.p, w->perm.p, w->scale.p, w->T.p);
  if ((rv = gemm_f64((int)n, r, l, w->Q.p, l, 1, w->T.p, r, 1, w->phi.p, r, 1, w->part))) return rv;
  w->sigma2.assign(mu.begin(), mu.begin() + r);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

// The POD-Galerkin operators of the model's affine stiffness K = sum_v a_v K_v:
// G_v = Phi^T K_v Phi for every multiplier v, Phi^T F0 and the basis rows of
// the randomised loads.  Only for models with at most 64 E variables (the
// per-sample reduced system then costs nmult r^2 to assemble).
int build_galerkin(ufem_warm *w) {
  int rv;
  McImplicitView v;
  if ((rv = mc_implicit_view(w->m, &v))) return rv;
  w->galerkin = false;
  if (v.nmult > 64) return UFEM_AF_OK;
  const int r = w->rb;  // operators of every basis column; the guess uses the leading n_modes
  const long n = w->n;
  DBuf<double> Y;
  if ((rv = Y.ensure((size_t)n * r)) || (rv = w->Gv.ensure((size_t)v.nmult * r * r)) || (rv = w->PF0.ensure(r)))
    return rv;
  for (int m = 0; m < v.nmult; m++) {
    if (v.B == 3)
      k_zone_apply<3><<<grid1((long)v.nbr * r), 256>>>(v.nbr, r, v.crow, v.cval, v.cstride, m, w->phi.p, Y.p);
    else
      k_zone_apply<2><<<grid1((long)v.nbr * r), 256>>>(v.nbr, r, v.crow, v.cval, v.cstride, m, w->phi.p, Y.p);
    if ((rv = gemm_f64(r, r, n, w->phi.p, 1, r, Y.p, r, 1, w->Gv.p + (size_t)m * r * r, r, 1, w->part))) return rv;
  }
  if ((rv = gemm_f64(r, 1, n, w->phi.p, 1, r, v.F0, 1, 1, w->PF0.p, 1, 1, w->part))) return rv;
  w->novr = (int)v.ovr_row.size();
  if (w->novr > 0) {
    DBuf<int> rows;
    if ((rv = rows.upload(v.ovr_row.data(), w->novr)) || (rv = w->d_ovar.upload(v.ovr_var.data(), w->novr)) ||
        (rv = w->Prow.ensure((size_t)w->novr * r)))
      return rv;
    k_phi_rows<<<grid1((long)w->novr * r), 256>>>(w->novr, r, rows.p, w->phi.p, w->Prow.p);
    UFEM_CUDA_TRY(cudaDeviceSynchronize());
  }
  if ((rv = w->d_mcol.upload(v.mult_col.data(), v.mult_col.size()))) return rv;
  w->nmult = v.nmult;
  w->galerkin = true;
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

// Coarse space of the batched PCG's preconditioner from the leading rc POD
// modes: Wc = Phi_c L^-T with L L^T = Phi_c^T Kbar Phi_c, Kbar the stiffness
// at the training samples' mean multipliers (sum_v mean(a_v) G_v, the
// Galerkin operators above), so Wc Wc^T = Phi_c (Phi_c^T Kbar Phi_c)^-1
// Phi_c^T.  One operator serves every sample: the preconditioner only has to
// be a fixed symmetric positive definite map.  Pivots below 1e-13 of the
// largest drop their mode.
int build_coarse(ufem_warm *w, long ntrain, const double *d_ifld) {
  // only modes that carry solution content: energy above 1e-20 of the first
  // (singular values 1e-10 of the first, far above the error of snapshots
  // solved to 1e-11) -- beyond the family's numerical rank a mode is solver
  // noise, and the additive correction would lift it to the top of the
  // preconditioned spectrum; a multiple of 16 (the MMA's N granularity)
  int rc = std::min(w->o.n_coarse, w->rb);
  {
    int keep = 0;
    while (keep < rc && keep < (int)w->sigma2.size() && w->sigma2[keep] > 1e-20 * w->sigma2[0]) keep++;
    rc = keep / 16 * 16;
  }
  w->coarse_modes = 0;
  if (!w->galerkin || rc < 16) return ufem_mc_set_coarse(w->m, 0, nullptr);
  int rv;
  const int r = w->rb, nmult = w->nmult;
  const long ilen = w->m->mc_ilen;
  std::vector<int> mcol(nmult);
  std::vector<double> ifl((size_t)ntrain * ilen), G((size_t)nmult * r * r);
  UFEM_CUDA_TRY(cudaMemcpy(mcol.data(), w->d_mcol.p, nmult * sizeof(int), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(ifl.data(), d_ifld, ifl.size() * sizeof(double), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(G.data(), w->Gv.p, G.size() * sizeof(double), cudaMemcpyDeviceToHost));
  std::vector<double> abar(nmult, 1.0);
  for (int v = 1; v < nmult; v++) {
    double t = 0.0;
    for (long s = 0; s < ntrain; s++) t += ifl[(size_t)s * ilen + mcol[v]];
    abar[v] = t / (double)ntrain;
  }
  {
    std::vector<double> la(nmult);
    for (int v = 0; v < nmult; v++) la[v] = std::log(std::fabs(abar[v]));
    if ((rv = w->log_abar.upload(la.data(), nmult))) return rv;
  }
  // Ebar (rc x rc), then its Cholesky factor in place (lower triangle)
  std::vector<double> L((size_t)rc * rc, 0.0);
  for (int i = 0; i < rc; i++)
    for (int j = 0; j < rc; j++) {
      double t = 0.0;
      for (int v = 0; v < nmult; v++) t += abar[v] * G[(size_t)v * r * r + (size_t)i * r + j];
      L[(size_t)i * rc + j] = t;
    }
  double dmax = 0.0;
  for (int i = 0; i < rc; i++) dmax = std::max(dmax, std::fabs(L[(size_t)i * rc + i]));
  std::vector<char> skip(rc, 0);
  for (int j = 0; j < rc; j++) {
    double d = L[(size_t)j * rc + j];
    for (int k = 0; k < j; k++) d -= L[(size_t)j * rc + k] * L[(size_t)j * rc + k];
    skip[j] = !(d > 1e-13 * dmax);
    const double ljj = skip[j] ? 1.0 : std::sqrt(d);
    L[(size_t)j * rc + j] = ljj;
    for (int i = j + 1; i < rc; i++) {
      double t = L[(size_t)i * rc + j];
      for (int k = 0; k < j; k++) t -= L[(size_t)i * rc + k] * L[(size_t)j * rc + k];
      L[(size_t)i * rc + j] = skip[j] ? 0.0 : t / ljj;
    }
    for (int k = 0; k < j; k++) L[(size_t)k * rc + j] = 0.0;
  }
  // T = L^-T (column j of T = row j of L^-1); a dropped mode is a zero column
  std::vector<double> T((size_t)rc * rc, 0.0);
  for (int j = 0; j < rc; j++) {
    // solve L y = e_j; y = column j of L^-1 = row j of T
    std::vector<double> y(rc, 0.0);
    for (int i = j; i < rc; i++) {
      double t = (i == j) ? 1.0 : 0.0;
      for (int k = j; k < i; k++) t -= L[(size_t)i * rc + k] * y[k];
      y[i] = t / L[(size_t)i * rc + i];
    }
    for (int i = 0; i < rc; i++) T[(size_t)j * rc + i] = y[i];
  }
  for (int j = 0; j < rc; j++)
    if (skip[j])
      for (int i = 0; i < rc; i++) T[(size_t)i * rc + j] = 0.0;
  DBuf<double> dT, Wc;
  if ((rv = dT.upload(T.data(), T.size())) || (rv = Wc.ensure((size_t)w->n * rc))) return rv;
  // Wc [n][rc] = Phi[:, :rc] T
  if ((rv = gemm_f64((int)w->n, rc, rc, w->phi.p, r, 1, dT.p, rc, 1, Wc.p, rc, 1, w->part))) return rv;
  if ((rv = ufem_mc_set_coarse(w->m, rc, Wc.p))) return rv;
  w->coarse_modes = rc;
  return UFEM_AF_OK;
}

// standardised network inputs of nsamp samples into w->X (FP32 [nsamp][n_feat]);
// with fit = true the feature statistics are (re)computed from these samples
int make_inputs(ufem_warm *w, long nsamp, const double *d_ifld, bool fit) {
  int rv;
  const int nf = w->o.n_feat;
  if ((rv = w->raw.ensure((size_t)nsamp * nf)) || (rv = w->X.ensure((size_t)nsamp * nf)) ||
      (rv = w->sc.ensure(nsamp)))
    return rv;
  k_feat_raw<<<grid1(nsamp * nf), 256>>>(nsamp, nf, w->m->mc_ilen, d_ifld, w->fcol.p, w->flog.p, w->raw.p);
  if (fit) k_col_stats<<<1, 32>>>(nsamp, nf, w->raw.p, w->fmean.p, w->fsd.p);
  k_standardise<<<grid1(nsamp * nf), 256>>>(nsamp, nf, nf, w->raw.p, w->fmean.p, w->fsd.p, w->X.p);
  k_scale<<<grid1(nsamp), 256>>>(nsamp, w->m->mc_ilen, w->o.scale_col, d_ifld, w->sc.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

int padded_S(long nsamp) { return (int)std::max<long>(128, (nsamp + 127) / 128 * 128); }

// u0 [n][S] = Phi c^T for nsamp samples: c from the MLP (inputs in w->X /
// w->sc), or from the POD-Galerkin system of each sample (guess mode 1)
// The coefficient model's least-squares part, fitted over the training
// samples (normal equations (D^T D + lambda I) W = D^T C, D the quadratic
// design matrix of the standardised features, formed on the GPU and solved
// by Cholesky on the host: 1 + nf + nf (nf + 1) / 2 unknowns, 171 for 17
// inputs, shared by every mode); c becomes the
// residual, and the MLP's targets are that residual over one common scale
// (its RMS over samples and modes), so the network's squared error is the
// squared error of the coefficients themselves -- the error of the guess
// in the 2-norm, Phi being orthonormal.
int fit_linear(ufem_warm *w, long ntrain) {
  int rv;
  const int r = w->r, nf = w->o.n_feat;
  w->lin_quad = ntrain >= 4L * poly_terms(nf, 1) ? 1 : 0;
  const int nd = poly_terms(nf, w->lin_quad);
  if ((rv = w->design.ensure((size_t)ntrain * nd)) || (rv = w->gram.ensure((size_t)nd * (nd + r))) ||
      (rv = w->linW.ensure((size_t)nd * r)))
    return rv;
  k_design<<<grid1(ntrain, 128), 128>>>(ntrain, nf, w->lin_quad, w->raw.p, w->fmean.p, w->fsd.p, w->design.p);
  // G = D^T D [nd][nd], H = D^T C [nd][r]
  if ((rv = gemm_f64(nd, nd, ntrain, w->design.p, 1, nd, w->design.p, nd, 1, w->gram.p, nd, 1, w->part)) ||
      (rv = gemm_f64(nd, r, ntrain, w->design.p, 1, nd, w->c.p, r, 1, w->gram.p + (size_t)nd * nd, r, 1, w->part)))
    return rv;
  std::vector<double> G((size_t)nd * nd), H((size_t)nd * r);
  UFEM_CUDA_TRY(cudaMemcpy(G.data(), w->gram.p, G.size() * sizeof(double), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(H.data(), w->gram.p + (size_t)nd * nd, H.size() * sizeof(double), cudaMemcpyDeviceToHost));
  double tr = 0.0;
  for (int i = 0; i < nd; i++) tr += G[(size_t)i * nd + i];
  for (int i = 0; i < nd; i++) G[(size_t)i * nd + i] += 1e-12 * tr / nd;  // keeps a constant feature solvable
  // Cholesky G = L L^T (lower, in place)
  for (int j = 0; j < nd; j++) {
    double d = G[(size_t)j * nd + j];
    for (int k = 0; k < j; k++) d -= G[(size_t)j * nd + k] * G[(size_t)j * nd + k];
    if (!(d > 0.0)) {
      set_error("warm start: the linear coefficient model's normal equations are not positive definite");
      return UFEM_AF_ERR;
    }
    const double ljj = std::sqrt(d);
    G[(size_t)j * nd + j] = ljj;
    for (int i = j + 1; i < nd; i++) {
      double t = G[(size_t)i * nd + j];
      for (int k = 0; k < j; k++) t -= G[(size_t)i * nd + k] * G[(size_t)j * nd + k];
      G[(size_t)i * nd + j] = t / ljj;
    }
  }
  for (int k = 0; k < r; k++) {  // L y = h, L^T w = y, column by column
    std::vector<double> y(nd);
    for (int i = 0; i < nd; i++) {
      double t = H[(size_t)i * r + k];
      for (int j = 0; j < i; j++) t -= G[(size_t)i * nd + j] * y[j];
      y[i] = t / G[(size_t)i * nd + i];
    }
    for (int i = nd - 1; i >= 0; i--) {
      double t = y[i];
      for (int j = i + 1; j < nd; j++) t -= G[(size_t)j * nd + i] * H[(size_t)j * r + k];
      H[(size_t)i * r + k] = t / G[(size_t)i * nd + i];
    }
  }
  UFEM_CUDA_TRY(cudaMemcpy(w->linW.p, H.data(), H.size() * sizeof(double), cudaMemcpyHostToDevice));
  k_lin_resid<<<grid1(ntrain * r), 256>>>(ntrain, r, nf, w->lin_quad, w->raw.p, w->fmean.p, w->fsd.p, w->linW.p,
                                          w->c.p);
  // one common scale for every mode: the RMS of the residual
  k_col_stats<<<1, 128>>>(ntrain, r, w->c.p, w->cmean.p, w->csd.p);
  std::vector<double> mu(r), sd(r);
  UFEM_CUDA_TRY(cudaMemcpy(mu.data(), w->cmean.p, r * sizeof(double), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(sd.data(), w->csd.p, r * sizeof(double), cudaMemcpyDeviceToHost));
  double ms = 0.0;
  for (int k = 0; k < r; k++) ms += sd[k] * sd[k] + mu[k] * mu[k];
  const double scale = ms > 0.0 ? std::sqrt(ms / r) : 1.0;
  for (int k = 0; k < r; k++) sd[k] = scale;
  UFEM_CUDA_TRY(cudaMemcpy(w->csd.p, sd.data(), r * sizeof(double), cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

int make_guess(ufem_warm *w, long nsamp, int S, const double *d_ifld) {
  int rv;
  const int r = w->r;
  if ((rv = w->Yo.ensure((size_t)nsamp * r)) || (rv = w->c.ensure((size_t)nsamp * r)) ||
      (rv = w->u0.ensure((size_t)w->n * S)))
    return rv;
  if (w->o.guess_mode == 1 && w->galerkin) {
    const size_t smem = (size_t)r * (r + 1) / 2 * sizeof(double);
    static size_t configured = 0;
    if (configured < smem) {
      UFEM_CUDA_TRY(cudaFuncSetAttribute(k_reduced_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      configured = smem;
    }
    k_reduced_solve<<<(unsigned)nsamp, kRedThreads, smem>>>(nsamp, r, w->nmult, w->m->mc_ilen, d_ifld, w->d_mcol.p, w->Gv.p,
                                                     w->PF0.p, w->novr, w->d_ovar.p, w->Prow.p, w->rb, w->c.p);
    if (w->guess_scale != 1.0) k_mul<<<grid1(nsamp * r), 256>>>(nsamp * r, w->guess_scale, w->c.p);
  } else {
    if (w->o.guess_mode == 2) {  // the least-squares part alone: a zero network output
      UFEM_CUDA_TRY(cudaMemsetAsync(w->Yo.p, 0, (size_t)nsamp * r * sizeof(float)));
    } else if ((rv = ufem_mlp_forward(w->mlp, nsamp, w->X.p, w->Yo.p))) {
      return rv;
    }
    k_coeffs<<<grid1(nsamp * r), 256>>>(nsamp, r, w->o.n_feat, w->lin_quad, w->Yo.p, w->cmean.p, w->csd.p, w->raw.p, w->fmean.p,
                                        w->fsd.p, w->linW.p, w->sc.p, w->guess_scale, w->c.p);
  }
  if (S > nsamp) UFEM_CUDA_TRY(cudaMemsetAsync(w->u0.p, 0, (size_t)w->n * S * sizeof(double)));
  // u0(i, s) = sum_k Phi[i][k] c[s][k]
  return gemm_f64((int)w->n, (int)nsamp, r, w->phi.p, w->rb, 1, w->c.p, 1, r, w->u0.p, S, 1, w->part);
}

}  // namespace
}  // namespace ufem

extern "C" {

void ufem_warm_default_options(ufem_warm_options *o) {
  std::memset(o, 0, sizeof(*o));
  o->n_modes = 64;
  o->n_hidden = 256;
  o->n_feat = 0;
  o->scale_col = -1;
  o->n_snapshots = 512;
  o->power_iters = 2;
  o->epochs = 400;
  o->batch = 256;
  o->lr = 2e-3f;
  o->seed = 20261203ULL;
  o->guess_mode = 0;
  o->n_coarse = 64;
  o->snap_tol = 1e-11;
  o->order_samples = 1;
}

int ufem_warm_create(ufem_model *m, const ufem_warm_options *o, ufem_warm **out) {
  if (!m || !o || !out) return UFEM_AF_ERR_EMP;
  if (m->mc_ilen <= 0) {
    set_error("ufem_warm_create: the model has no Monte Carlo variable table");
    return UFEM_AF_ERR_EMP;
  }
  if (o->n_modes < 16 || o->n_modes % 16 || std::max(o->n_modes, o->n_coarse) + 16 > kMaxL || o->n_feat < 1 ||
      o->n_feat > 32 ||
      o->n_hidden < 16 || o->n_hidden > 256 || o->n_hidden % 16 || o->batch < 1 ||
      o->n_snapshots < std::max(o->n_modes, o->n_coarse) + 16 ||
      o->n_coarse < 0 || o->n_coarse % 16) {
    set_error("ufem_warm_create: n_modes a multiple of 16 up to 128, 1..32 inputs, n_hidden a multiple of 16 up to "
              "256, n_coarse a multiple of 16 up to 128, n_snapshots >= max(n_modes, n_coarse) + 16");
    return UFEM_AF_ERR_SIZ;
  }
  for (int f = 0; f < o->n_feat; f++)
    if (o->feat_cols[f] < 0 || o->feat_cols[f] >= m->mc_ilen) {
      set_error("ufem_warm_create: input column out of range");
      return UFEM_AF_ERR_SIZ;
    }
  if (o->scale_col >= m->mc_ilen) {
    set_error("ufem_warm_create: scale column out of range");
    return UFEM_AF_ERR_SIZ;
  }
  ufem_warm *w = new ufem_warm();
  w->m = m;
  w->o = *o;
  w->r = o->n_modes;
  w->rb = std::max(o->n_modes, o->n_coarse);
  w->l = w->rb + 16;
  w->n = m->nDOFAct;
  int rv;
  std::vector<int> lg(o->n_feat);
  for (int f = 0; f < o->n_feat; f++) lg[f] = o->feat_log[f] == 2 ? 2 : (o->feat_log[f] ? 1 : 0);
  if ((rv = w->fcol.upload(o->feat_cols, o->n_feat)) || (rv = w->flog.upload(lg.data(), o->n_feat)) ||
      (rv = w->fmean.ensure(32)) || (rv = w->fsd.ensure(32)) || (rv = w->cmean.ensure(w->r)) ||
      (rv = w->csd.ensure(w->r)) ||
      (rv = ufem_mlp_create(o->n_feat, o->n_hidden, w->r, o->seed, &w->mlp))) {
    delete w;
    return rv;
  }
  *out = w;
  return UFEM_AF_OK;
}

void ufem_warm_free(ufem_warm *w) {
  if (!w) return;
  if (w->mlp) ufem_mlp_free(w->mlp);
  delete w;
}

int ufem_warm_train(ufem_warm *w, long ntrain, const double *d_ifld, const ufem_mc_options *opt,
                    ufem_warm_train_stats *ts) {
  if (!w || !d_ifld) return UFEM_AF_ERR_EMP;
  if (ntrain < w->o.n_snapshots || ntrain < w->o.batch) {
    set_error("ufem_warm_train: need at least n_snapshots and batch training samples");
    return UFEM_AF_ERR_SIZ;
  }
  int rv;
  ufem_warm_train_stats st;
  std::memset(&st, 0, sizeof(st));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto ms_since = [&](cudaEvent_t a) {
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, e1);
    return (double)ms;
  };
  const long n = w->n;
  const int r = w->r;
  ufem_model *m = w->m;
  // 1. cold batched solves of every training sample -> U [n][ntrain], Jacobi
  // PCG alone (the cap of the warm runs is the cold iteration count)
  ufem_mc_options cold;
  if (opt) cold = *opt;
  else ufem_mc_default_options(&cold);
  cold.coarse = 0;
  cudaEventRecord(e0);
  if ((rv = w->U.ensure((size_t)n * ntrain)) || (rv = w->st.ensure(ntrain)) || (rv = w->it.ensure(ntrain))) return rv;
  // the first n_snapshots samples (the POD snapshots) at snap_tol: the tail
  // modes of the basis then hold solution content rather than solver error
  ufem_mc_options snap = cold;
  if (w->o.snap_tol > 0.0) snap.tol = std::min(cold.tol, w->o.snap_tol);
  const long nsnap = std::min<long>(w->o.n_snapshots, ntrain);
  {
    DBuf<double> uchunk;
    const long chunk = 4096;
    for (long c0 = 0; c0 < ntrain;) {
      const bool is_snap = c0 < nsnap;
      const long cn = std::min(chunk, (is_snap ? nsnap : ntrain) - c0);
      const int S = padded_S(cn);
      if ((rv = uchunk.ensure((size_t)n * S))) return rv;
      const double *pin = d_ifld + c0 * m->mc_ilen;
      double *pu = uchunk.p;
      int *ps = w->st.p + c0;
      long *pi = w->it.p + c0;
      if ((rv = mc_solve_device(1, &m, &cn, &pin, nullptr, &ps, &pi, nullptr, &pu, is_snap ? &snap : &cold)))
        return rv;
      UFEM_CUDA_TRY(cudaMemcpy2DAsync(w->U.p + c0, ntrain * sizeof(double), uchunk.p, S * sizeof(double),
                                      cn * sizeof(double), n, cudaMemcpyDeviceToDevice));
      c0 += cn;
    }
  }
  {
    std::vector<int> hs(ntrain);
    std::vector<long> hi(ntrain);
    UFEM_CUDA_TRY(cudaMemcpy(hs.data(), w->st.p, ntrain * sizeof(int), cudaMemcpyDeviceToHost));
    UFEM_CUDA_TRY(cudaMemcpy(hi.data(), w->it.p, ntrain * sizeof(long), cudaMemcpyDeviceToHost));
    long mx = 0, cnt = 0;
    double sum = 0;
    // the cap of the warm runs: the cold iteration counts at the caller's
    // tolerance (the snapshots' counts when every sample is a snapshot)
    const bool all_snap = nsnap >= ntrain || snap.tol == cold.tol;
    for (long s = 0; s < ntrain; s++) {
      if (hs[s] != UFEM_ST_CONVERGED) {
        set_error("ufem_warm_train: a training sample did not converge");
        return UFEM_AF_ERR;
      }
      if (s < nsnap && !all_snap) continue;
      mx = std::max(mx, hi[s]);
      sum += (double)hi[s];
      cnt++;
    }
    w->cold_cap = mx;
    w->train_precision = cold.precision;
    st.cold_iters_max = mx;
    st.cold_iters_mean = sum / (double)std::max<long>(1, cnt);
  }
  st.ms_solve = ms_since(e0);
  // 2. POD basis from the first n_snapshots solutions
  cudaEventRecord(e0);
  if ((rv = fit_basis(w, (int)ntrain, w->o.n_snapshots)) || (rv = build_galerkin(w)) ||
      (rv = build_coarse(w, ntrain, d_ifld)))
    return rv;
  st.ms_basis = ms_since(e0);
  st.coarse_modes = w->coarse_modes;
  for (int k = 0; k < r && k < 80; k++) st.sigma2[k] = w->sigma2[k];
  // 3. inputs and targets
  cudaEventRecord(e0);
  if ((rv = make_inputs(w, ntrain, d_ifld, true))) return rv;
  if ((rv = w->c.ensure((size_t)ntrain * r)) || (rv = w->Tt.ensure((size_t)ntrain * r))) return rv;
  // c[s][k] = sum_i U[i][s] Phi[i][k]
  if ((rv = gemm_f64((int)ntrain, r, n, w->U.p, 1, ntrain, w->phi.p, w->rb, 1, w->c.p, r, 1, w->part))) return rv;
  k_div_scale<<<grid1(ntrain * r), 256>>>(ntrain, r, w->sc.p, w->c.p);
  if ((rv = fit_linear(w, ntrain))) return rv;
  k_targets<<<grid1(ntrain * r), 256>>>(ntrain, r, w->c.p, w->cmean.p, w->csd.p, w->Tt.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  // 4. training: shuffled minibatches, cosine learning rate; every step is
  // the replay of one recorded CUDA graph
  const int bs = w->o.batch;
  const long nb = ntrain / bs;
  const long total = (long)w->o.epochs * nb;
  std::vector<float> sched(std::max<long>(1, total));
  for (long step = 0; step < total; step++) {
    const double frac = (double)step / (double)std::max<long>(1, total);
    sched[step] = (float)(w->o.lr * (0.02 + 0.98 * 0.5 * (1.0 + std::cos(3.14159265358979323846 * frac))));
  }
  if ((rv = mlp_train_graph(w->mlp, ntrain, bs, w->X.p, w->Tt.p, sched, w->o.epochs, w->o.seed ^ 0x7a11ULL,
                            &st.loss_first, &st.loss_last, &st.steps)))
    return rv;
  st.ms_train = ms_since(e0);
  st.epochs = w->o.epochs;
  w->trained = true;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ts) *ts = st;
  return UFEM_AF_OK;
}

int ufem_warm_guess(ufem_warm *w, long nsamp, const double *d_ifld, double *d_u0) {
  if (!w || !d_ifld || !d_u0) return UFEM_AF_ERR_EMP;
  if (!w->trained) {
    set_error("ufem_warm_guess: the warm start is not trained");
    return UFEM_AF_ERR;
  }
  int rv;
  const int S = padded_S(nsamp);
  if ((rv = make_inputs(w, nsamp, d_ifld, false)) || (rv = make_guess(w, nsamp, S, d_ifld))) return rv;
  k_to_sample_major<<<grid1(w->n * nsamp), 256>>>(w->n, S, nsamp, w->u0.p, d_u0);
  UFEM_CUDA_TRY(cudaGetLastError());
  UFEM_CUDA_TRY(cudaDeviceSynchronize());
  return UFEM_AF_OK;
}

}  // extern "C"

namespace {
// the warm-started solve of the samples in the given order
int warm_solve_ordered(ufem_warm *w, long nsamp, const double *d_ifld, double *d_ofld, int *d_status, long *d_iters,
                       const ufem_mc_options *opt_in, ufem_warm_stats *ws) {
  int rv;
  ufem_mc_options opt;
  if (opt_in) opt = *opt_in;
  else ufem_mc_default_options(&opt);
  ufem_warm_stats st;
  std::memset(&st, 0, sizeof(st));
  st.nsamp = nsamp;
  cudaEvent_t e0, e1, e2, e3;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
  ufem_model *m = w->m;
  const long n = w->n;
  const int S = padded_S(nsamp);
  if ((rv = w->uf.ensure((size_t)n * S)) || (rv = w->st.ensure(nsamp)) || (rv = w->it.ensure(nsamp)) ||
      (rv = w->err.ensure(nsamp)))
    return rv;
  int *pst = d_status ? d_status : w->st.p;
  long *pit = d_iters ? d_iters : w->it.p;
  cudaEventRecord(e0);
  // guess
  if ((rv = make_inputs(w, nsamp, d_ifld, false)) || (rv = make_guess(w, nsamp, S, d_ifld))) return rv;
  cudaEventRecord(e1);
  // warm-started batched solve, capped at the cold iteration count seen in
  // training at the same precision (other precisions: the caller's cap)
  ufem_mc_options wopt = opt;
  const bool capped = w->cold_cap > 0 && opt.precision == w->train_precision;
  if (capped) wopt.max_iters = std::min(opt.max_iters, w->cold_cap);
  {
    const double *pg = w->u0.p;
    double *pu = w->uf.p;
    if ((rv = mc_solve_device(1, &m, &nsamp, &d_ifld, &d_ofld, &pst, &pit, &pg, &pu, &wopt))) return rv;
    ufem_mc_stats ms;
    ufem_mc_get_stats(&ms);
    st.kernel_launches += ms.kernel_launches;
    st.pcg_ms = ms.ms_pcg;
    st.pcg_bytes = ms.pcg_bytes;
    st.pcg_launches = ms.pcg_launches;
  }
  st.kernel_launches += 4 + 3 + 1 + 1;  // inputs (3), MLP forward (4), coefficients, u0 = Phi c
  cudaEventRecord(e2);
  // fallback: samples that did not converge from the guess, again from zero
  std::vector<int> hs(nsamp);
  UFEM_CUDA_TRY(cudaMemcpy(hs.data(), pst, nsamp * sizeof(int), cudaMemcpyDeviceToHost));
  std::vector<long> fb;
  for (long s = 0; s < nsamp; s++)
    if (hs[s] != UFEM_ST_CONVERGED) fb.push_back(s);
  st.fallbacks = (long)fb.size();
  if (!fb.empty()) {
    const long nf = (long)fb.size();
    const long ilen = m->mc_ilen, olen = std::max<long>(1, m->mc_olen);
    DBuf<long> d_idx;
    if ((rv = d_idx.upload(fb.data(), nf)) || (rv = w->ifsub.ensure((size_t)nf * ilen)) ||
        (rv = w->ofsub.ensure((size_t)nf * olen)) || (rv = w->stsub.ensure(nf)) || (rv = w->itsub.ensure(nf)))
      return rv;
    k_gather_rows<double><<<grid1(nf * ilen), 256>>>(nf, (int)ilen, d_idx.p, d_ifld, w->ifsub.p);
    const double *pin = w->ifsub.p;
    double *pof = w->ofsub.p;
    int *ps = w->stsub.p;
    long *pi = w->itsub.p;
    DBuf<double> ufb;
    const int Sf = padded_S(nf);
    if ((rv = ufb.ensure((size_t)n * Sf))) return rv;
    double *pu = ufb.p;
    // from zero, FP32 SpMV products (precision 4) converge poorly: the
    // fallback forms the products in FP64 (precision 3)
    ufem_mc_options fopt = opt;
    if (fopt.precision == 4) fopt.precision = 3;
    if ((rv = mc_solve_device(1, &m, &nf, &pin, d_ofld ? &pof : nullptr, &ps, &pi, nullptr, &pu, &fopt))) return rv;
    ufem_mc_stats ms;
    ufem_mc_get_stats(&ms);
    st.kernel_launches += ms.kernel_launches + 1;  // + the input gather
    std::vector<int> fst(nf);
    std::vector<long> fit(nf), wit(nsamp);
    std::vector<double> fof((size_t)nf * olen);
    UFEM_CUDA_TRY(cudaMemcpy(fst.data(), ps, nf * sizeof(int), cudaMemcpyDeviceToHost));
    UFEM_CUDA_TRY(cudaMemcpy(fit.data(), pi, nf * sizeof(long), cudaMemcpyDeviceToHost));
    UFEM_CUDA_TRY(cudaMemcpy(wit.data(), pit, nsamp * sizeof(long), cudaMemcpyDeviceToHost));
    if (d_ofld && m->mc_olen > 0)
      UFEM_CUDA_TRY(cudaMemcpy(fof.data(), pof, (size_t)nf * olen * sizeof(double), cudaMemcpyDeviceToHost));
    for (long j = 0; j < nf; j++) {
      const long s = fb[j];
      hs[s] = fst[j] == UFEM_ST_CONVERGED ? UFEM_ST_FALLBACK : fst[j];
      wit[s] += fit[j];  // iterations spent on this sample: the capped warm run + the cold one
      if (d_ofld && m->mc_olen > 0)
        UFEM_CUDA_TRY(cudaMemcpy(d_ofld + s * m->mc_olen, fof.data() + j * olen, m->mc_olen * sizeof(double),
                                 cudaMemcpyHostToDevice));
      UFEM_CUDA_TRY(cudaMemcpy2DAsync(w->uf.p + s, S * sizeof(double), ufb.p + j, Sf * sizeof(double),
                                      sizeof(double), n, cudaMemcpyDeviceToDevice));
    }
    UFEM_CUDA_TRY(cudaMemcpy(pst, hs.data(), nsamp * sizeof(int), cudaMemcpyHostToDevice));
    UFEM_CUDA_TRY(cudaMemcpy(pit, wit.data(), nsamp * sizeof(long), cudaMemcpyHostToDevice));
  }
  cudaEventRecord(e3);
  // guess error against the converged solution
  if ((rv = w->errpart.ensure((size_t)kErrChunks * S * 2))) return rv;
  k_rel_err_part<<<dim3((unsigned)(S / 32), kErrChunks), 256>>>(n, S, w->u0.p, w->uf.p, w->errpart.p);
  k_rel_err<<<grid1(nsamp, 128), 128>>>(kErrChunks, S, (int)nsamp, w->errpart.p, w->err.p);
  st.kernel_launches += 2;
  UFEM_CUDA_TRY(cudaGetLastError());
  std::vector<double> he(nsamp);
  std::vector<long> hi(nsamp);
  UFEM_CUDA_TRY(cudaMemcpy(he.data(), w->err.p, nsamp * sizeof(double), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(hi.data(), pit, nsamp * sizeof(long), cudaMemcpyDeviceToHost));
  double se = 0, si = 0;
  for (long s = 0; s < nsamp; s++) {
    se += he[s];
    st.guess_err_max = std::max(st.guess_err_max, he[s]);
    si += (double)hi[s];
    st.iters_max = std::max(st.iters_max, hi[s]);
  }
  st.guess_err_mean = nsamp ? se / (double)nsamp : 0.0;
  st.iters_mean = nsamp ? si / (double)nsamp : 0.0;
  st.cold_cap = capped ? w->cold_cap : opt.max_iters;
  float a = 0, b = 0, c = 0;
  cudaEventElapsedTime(&a, e0, e1);
  cudaEventElapsedTime(&b, e1, e2);
  cudaEventElapsedTime(&c, e2, e3);
  st.ms_guess = a;
  st.ms_solve = b;
  st.ms_fallback = c;
  st.ms_total = (double)a + b + c;
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2); cudaEventDestroy(e3);
  if (ws) *ws = st;
  return UFEM_AF_OK;
}
}  // namespace

extern "C" {

// Samples are solved in the order of their ordering score (stable, so the
// same batch gives the same grouping every run) and the outputs returned in
// the caller's order: similar samples share a 128-sample group.
int ufem_warm_solve(ufem_warm *w, long nsamp, const double *d_ifld, double *d_ofld, int *d_status, long *d_iters,
                    const ufem_mc_options *opt_in, ufem_warm_stats *ws) {
  if (!w || !d_ifld) return UFEM_AF_ERR_EMP;
  if (!w->trained) {
    set_error("ufem_warm_solve: the warm start is not trained");
    return UFEM_AF_ERR;
  }
  if (!w->o.order_samples || !w->galerkin || w->nmult < 2 || !w->log_abar.p || nsamp <= 128)
    return warm_solve_ordered(w, nsamp, d_ifld, d_ofld, d_status, d_iters, opt_in, ws);
  int rv;
  const long ilen = w->m->mc_ilen, olen = w->m->mc_olen;
  if ((rv = w->score.ensure(nsamp)) || (rv = w->sperm.ensure(nsamp)) || (rv = w->ifperm.ensure((size_t)nsamp * ilen)) ||
      (rv = w->stperm.ensure(nsamp)) || (rv = w->itperm.ensure(nsamp)) ||
      (rv = w->ofperm.ensure((size_t)nsamp * std::max<long>(1, olen))))
    return rv;
  k_order_score<<<grid1(nsamp), 256>>>(nsamp, ilen, w->nmult, d_ifld, w->d_mcol.p, w->log_abar.p, w->score.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  std::vector<double> sc(nsamp);
  UFEM_CUDA_TRY(cudaMemcpy(sc.data(), w->score.p, nsamp * sizeof(double), cudaMemcpyDeviceToHost));
  for (auto &x : sc)
    if (!std::isfinite(x)) x = HUGE_VAL;  // non-finite inputs last
  std::vector<long> perm(nsamp);
  std::iota(perm.begin(), perm.end(), 0L);
  std::stable_sort(perm.begin(), perm.end(), [&](long a, long b) { return sc[a] < sc[b]; });
  if ((rv = w->sperm.upload(perm.data(), nsamp))) return rv;
  k_gather_rows<double><<<grid1(nsamp * ilen), 256>>>(nsamp, (int)ilen, w->sperm.p, d_ifld, w->ifperm.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  if ((rv = warm_solve_ordered(w, nsamp, w->ifperm.p, d_ofld ? w->ofperm.p : nullptr, w->stperm.p, w->itperm.p,
                               opt_in, ws)))
    return rv;
  if (d_ofld && olen > 0)
    k_scatter_rows<double><<<grid1(nsamp * olen), 256>>>(nsamp, (int)olen, w->sperm.p, w->ofperm.p, d_ofld);
  if (d_status) k_scatter_rows<int><<<grid1(nsamp), 256>>>(nsamp, 1, w->sperm.p, w->stperm.p, d_status);
  if (d_iters) k_scatter_rows<long><<<grid1(nsamp), 256>>>(nsamp, 1, w->sperm.p, w->itperm.p, d_iters);
  UFEM_CUDA_TRY(cudaGetLastError());
  if (ws) ws->kernel_launches += 5;
  return UFEM_AF_OK;
}

int ufem_warm_set_guess_mode(ufem_warm *w, int mode) {
  if (!w) return UFEM_AF_ERR_EMP;
  if (mode < 0 || mode > 2) {
    set_error("ufem_warm_set_guess_mode: 0 (MLP), 1 (POD-Galerkin) or 2 (least-squares part alone)");
    return UFEM_AF_ERR_VAL;
  }
  w->o.guess_mode = mode;
  return UFEM_AF_OK;
}

int ufem_warm_set_guess_scale(ufem_warm *w, double factor) {
  if (!w) return UFEM_AF_ERR_EMP;
  w->guess_scale = factor;
  return UFEM_AF_OK;
}

int ufem_warm_get_basis(const ufem_warm *w, double *h_phi, double *h_sigma2) {
  if (!w) return UFEM_AF_ERR_EMP;
  if (!w->trained) {
    set_error("ufem_warm_get_basis: the warm start is not trained");
    return UFEM_AF_ERR;
  }
  if (h_phi)
    UFEM_CUDA_TRY(cudaMemcpy2D(h_phi, w->r * sizeof(double), w->phi.p, w->rb * sizeof(double), w->r * sizeof(double),
                               w->n, cudaMemcpyDeviceToHost));
  if (h_sigma2) std::memcpy(h_sigma2, w->sigma2.data(), w->r * sizeof(double));
  return UFEM_AF_OK;
}

// FP64 dense product through the warm start's GEMM kernel, for its tests:
// C [M x N] = A [M x K] . B [K x N], all row-major device arrays.
int ufem_dgemm_f64(int M, int N, long K, const double *d_A, const double *d_B, double *d_C) {
  DBuf<double> part;
  int rv = gemm_f64(M, N, K, d_A, K, 1, d_B, N, 1, d_C, N, 1, part);
  if (rv) return rv;
  UFEM_CUDA_TRY(cudaDeviceSynchronize());
  return UFEM_AF_OK;
}

// Symmetric eigen-decomposition through the warm start's one-block Jacobi
// kernel, for its tests: A [l x l] (l even, <= 144) -> V [l x l] (columns =
// eigenvectors, unsorted), lam [l].  Host arrays.
int ufem_sym_eig(int l, const double *h_A, double *h_V, double *h_lam, int *sweeps) {
  if (l < 2 || l % 2 || l > kMaxL) {
    set_error("ufem_sym_eig: l even, 2..144");
    return UFEM_AF_ERR_SIZ;
  }
  DBuf<double> A, V, lam, Vg;
  DBuf<int> sw;
  int rv;
  if ((rv = A.upload(h_A, (size_t)l * l)) || (rv = V.ensure((size_t)l * l)) || (rv = lam.ensure(l)) ||
      (rv = sw.ensure(1)) || (rv = Vg.ensure((size_t)l * l)))
    return rv;
  if ((rv = jacobi_eig(l, A.p, V.p, lam.p, sw.p, Vg.p))) return rv;
  UFEM_CUDA_TRY(cudaMemcpy(h_V, V.p, (size_t)l * l * sizeof(double), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(h_lam, lam.p, l * sizeof(double), cudaMemcpyDeviceToHost));
  if (sweeps) UFEM_CUDA_TRY(cudaMemcpy(sweeps, sw.p, sizeof(int), cudaMemcpyDeviceToHost));
  return UFEM_AF_OK;
}

}  // extern "C"
