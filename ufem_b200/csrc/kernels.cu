// Element integration, colour-ordered assembly, supports and the result pass
// for libufem_gpu.so (sm_100a, FP64).
//
// Reference behaviour restated:
//   quad K_e   stiffp fem/fem_e002.c:346-760: 2x2 Gauss at +-0.577350569189626
//              (the reference's literal, fem/fem_e002.c:164), plane stress
//              when the thickness is > 0 else plane strain (fem/fem_stf2.c:43-89),
//              dvolu = detJ * t.
//   brick K_e  e009_stiff fem/fem_e009.c:261-635: 3x3x3 Gauss with the
//              15-digit constants of e008_init_gauss (fem/fem_e008.c:481-488),
//              J from the natural-coordinate derivatives (fem/fem_e009.c:106-205),
//              isotropic D (fem/fem_pl3d.c:32-57).
//   assembly   femLocKM_e fem/fem_mloc.c:163-221 into the block-sparse K.
//   supports   femApplyDisp fem/fem_loads.c:116-262.
//   results    fem_fill_K(AF_YES) fem/fem_sol.c:748-880: sigma = D B u_e at
//              every integration point, F_e = sum B^T sigma dV, reactions.
//
// Design: one element per warp.  The Gauss weights and shape-function
// derivatives are staged in shared memory once per block.  Lane l owns the
// node pairs (l/8, l%8) and (l/8+4, l%8) of a brick (16 pairs of a quad) and
// accumulates their 3x3 (2x2) blocks of
//     K_ab = sum_ip w detJ (lambda g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I),
// the closed form of H^T D H for isotropic D (plane: B^T D B written out).
// The product order makes K_ba exactly K_ab^T bit for bit.  Elements are
// launched colour by colour (no two elements of a colour share a node), so
// each block receives at most one update per launch: plain read-modify-write,
// no atomics, and a fixed summation order -> deterministic FP64 assembly.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "ufem_internal.h"

namespace ufem {

namespace {

__constant__ double c_brick_gp[3] = {-0.774596669241483, 0.000000000000000, 0.774596669241483};
__constant__ double c_brick_gw[3] = {0.555555555555556, 0.888888888888889, 0.555555555555556};
__constant__ double c_brick_nc[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                        {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
constexpr double QUAD_GP = 0.577350569189626;

constexpr int EPB = 4;  // elements (warps) per block

// Natural-coordinate derivatives dN_n/dxi_d at the 27 points, ordered x
// outer, y, z inner (fem/fem_e009.c:369-385), and the point weights.
__device__ void brick_tables(double (*s_dN)[8][3], double *s_w) {
  for (int t = threadIdx.x; t < 27 * 8; t += blockDim.x) {
    int ip = t >> 3, n = t & 7;
    int i = ip / 9, j = (ip / 3) % 3, k = ip % 3;
    double x = c_brick_gp[i], y = c_brick_gp[j], z = c_brick_gp[k];
    double xv = c_brick_nc[n][0], yv = c_brick_nc[n][1], zv = c_brick_nc[n][2];
    s_dN[ip][n][0] = 0.125 * xv * (1.0 + yv * y) * (1.0 + zv * z);
    s_dN[ip][n][1] = 0.125 * yv * (1.0 + xv * x) * (1.0 + zv * z);
    s_dN[ip][n][2] = 0.125 * zv * (1.0 + xv * x) * (1.0 + yv * y);
    if (n == 0) s_w[ip] = c_brick_gw[i] * c_brick_gw[j] * c_brick_gw[k];
  }
}

// Jacobian, its determinant and inverse at point ip for element coords X.
__device__ __forceinline__ double brick_jinv(const double (*s_dN)[8][3], int ip, const double (*X)[3],
                                             double inv[3][3]) {
  double J[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double s = 0.0;
#pragma unroll
      for (int n = 0; n < 8; n++) s += s_dN[ip][n][a] * X[n][c];
      J[a][c] = s;
    }
  double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  double id = 1.0 / det;
  inv[0][0] = c00 * id;
  inv[1][0] = c01 * id;
  inv[2][0] = c02 * id;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  return det;
}

__device__ __forceinline__ void brick_grad(const double (*s_dN)[8][3], int ip, int n, const double inv[3][3],
                                           double g[3]) {
#pragma unroll
  for (int d = 0; d < 3; d++)
    g[d] = inv[d][0] * s_dN[ip][n][0] + inv[d][1] * s_dN[ip][n][1] + inv[d][2] * s_dN[ip][n][2];
}

// Adds w*(lam g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I) to K (row-major 3x3).
__device__ __forceinline__ void brick_pair(double K[9], const double ga[3], const double gb[3], double w,
                                           double lam, double mu) {
  double dot = __dadd_rn(__dadd_rn(__dmul_rn(ga[0], gb[0]), __dmul_rn(ga[1], gb[1])), __dmul_rn(ga[2], gb[2]));
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      // explicitly rounded so that the mirrored lane forms the same value
      double tij = __dmul_rn(ga[i], gb[j]);
      double tji = __dmul_rn(ga[j], gb[i]);
      double v = __dadd_rn(__dmul_rn(lam, tij), __dmul_rn(mu, tji));
      if (i == j) v = __dadd_rn(v, __dmul_rn(mu, dot));
      K[i * 3 + j] += w * v;
    }
}

// MODE 0: scatter into the block-sparse K (one colour per launch).
// MODE 1: store the element matrix densely (eLen x 24 x 24) instead.
template <int MODE>
__global__ void __launch_bounds__(EPB * 32) k_brick_stiff(const int *__restrict__ elems, int nelem,
                                                          const double *__restrict__ xyz,
                                                          const int *__restrict__ enodes,
                                                          const double *__restrict__ eE,
                                                          const double *__restrict__ eNu,
                                                          const int *__restrict__ emap, double *__restrict__ val,
                                                          double *__restrict__ Ke, int *__restrict__ err) {
  __shared__ double s_dN[27][8][3];
  __shared__ double s_w[27];
  __shared__ double s_x[EPB][8][3];
  brick_tables(s_dN, s_w);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * EPB + warp;
  if (idx >= nelem) return;
  const int e = elems ? elems[idx] : idx;
  if (lane < 24) s_x[warp][lane / 3][lane % 3] = xyz[3 * (size_t)enodes[(size_t)e * 8 + lane / 3] + lane % 3];
  __syncwarp();
  const double E = eE[e], nu = eNu[e];
  const double lam = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));  // d2, fem/fem_pl3d.c:37
  const double mu = E / (2.0 * (1 + nu));                           // d3, fem/fem_pl3d.c:38
  const int a0 = lane >> 3, c = lane & 7, a1 = a0 + 4;
  double K0[9], K1[9];
#pragma unroll
  for (int t = 0; t < 9; t++) K0[t] = K1[t] = 0.0;
  bool bad = false;
  for (int ip = 0; ip < 27; ip++) {
    double inv[3][3];
    double det = brick_jinv(s_dN, ip, s_x[warp], inv);
    if (!(det > 0.0)) bad = true;  // fem/fem_e009.c:87-94
    double w = det * s_w[ip];
    double ga0[3], ga1[3], gc[3];
    brick_grad(s_dN, ip, a0, inv, ga0);
    brick_grad(s_dN, ip, a1, inv, ga1);
    brick_grad(s_dN, ip, c, inv, gc);
    brick_pair(K0, ga0, gc, w, lam, mu);
    brick_pair(K1, ga1, gc, w, lam, mu);
  }
  if (bad && lane == 0) atomicExch(err, UFEM_AF_ERR_VAL);
  if (MODE == 0) {
    double *b0 = val + (size_t)emap[(size_t)e * 64 + a0 * 8 + c] * 9;
    double *b1 = val + (size_t)emap[(size_t)e * 64 + a1 * 8 + c] * 9;
#pragma unroll
    for (int t = 0; t < 9; t++) {
      b0[t] += K0[t];
      b1[t] += K1[t];
    }
  } else {
    double *k = Ke + (size_t)e * 576;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        k[(3 * a0 + i) * 24 + 3 * c + j] = K0[i * 3 + j];
        k[(3 * a1 + i) * 24 + 3 * c + j] = K1[i * 3 + j];
      }
  }
}

// Plane D of D_HookIso_planeRaw (fem/fem_stf2.c:43-89): d00, d01, d11, d22.
__device__ __forceinline__ void plane_D(double E, double nu, double thick, double D[4]) {
  if (thick > 0.0) {
    double Mul = E / (1 - (nu * nu));
    D[0] = Mul;
    D[1] = Mul * nu;
    D[2] = Mul;
    D[3] = Mul * 0.5 * (1 - nu);
  } else {
    double Mul = E / ((1 + nu) * (1 - (2 * nu)));
    D[0] = Mul * (1 - nu);
    D[1] = Mul * nu;
    D[2] = Mul * (1 - nu);
    D[3] = Mul * 0.5 * (1 - nu);
  }
}

// Cartesian derivatives of the 4 shape functions at (s,t) (sfr + jacob,
// fem/fem_e002.c:53-66, :195-255); returns detJ.
__device__ __forceinline__ double quad_cartd(const double (*X)[2], double s, double t, double g[4][2]) {
  double dS[4] = {(-1.0 + t) * 0.25, (+1.0 - t) * 0.25, (+1.0 + t) * 0.25, (-1.0 - t) * 0.25};
  double dT[4] = {(-1.0 + s) * 0.25, (-1.0 - s) * 0.25, (+1.0 + s) * 0.25, (+1.0 - s) * 0.25};
  double j00 = 0, j01 = 0, j10 = 0, j11 = 0;
#pragma unroll
  for (int n = 0; n < 4; n++) {
    j00 += dS[n] * X[n][0];
    j01 += dS[n] * X[n][1];
    j10 += dT[n] * X[n][0];
    j11 += dT[n] * X[n][1];
  }
  double det = j00 * j11 - j01 * j10;
  double i00 = j11 / det, i11 = j00 / det, i01 = -j01 / det, i10 = -j10 / det;
#pragma unroll
  for (int n = 0; n < 4; n++) {
    g[n][0] = i00 * dS[n] + i01 * dT[n];
    g[n][1] = i10 * dS[n] + i11 * dT[n];
  }
  return det;
}

template <int MODE>
__global__ void __launch_bounds__(EPB * 32) k_quad_stiff(const int *__restrict__ elems, int nelem,
                                                         const double *__restrict__ xyz,
                                                         const int *__restrict__ enodes,
                                                         const double *__restrict__ eE,
                                                         const double *__restrict__ eNu,
                                                         const double *__restrict__ eThick,
                                                         const int *__restrict__ emap, double *__restrict__ val,
                                                         double *__restrict__ Ke, int *__restrict__ err) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * EPB + warp;
  if (idx >= nelem || lane >= 16) return;
  const int e = elems ? elems[idx] : idx;
  double X[4][2];
#pragma unroll
  for (int n = 0; n < 4; n++) {
    size_t q = (size_t)enodes[(size_t)e * 4 + n];
    X[n][0] = xyz[3 * q];
    X[n][1] = xyz[3 * q + 1];
  }
  const double thick = eThick[e];
  double D[4];
  plane_D(eE[e], eNu[e], thick, D);
  const int a = lane >> 2, c = lane & 3;
  double K[4] = {0, 0, 0, 0};
  bool bad = false;
  const double gp[2] = {-QUAD_GP, QUAD_GP};
#pragma unroll
  for (int ig = 0; ig < 2; ig++)
#pragma unroll
    for (int jg = 0; jg < 2; jg++) {
      double g[4][2];
      double det = quad_cartd(X, gp[ig], gp[jg], g);
      if (!(det > 0.0)) bad = true;  // fem/fem_e002.c:223-229
      double dv = det;
      if (thick > 0.0) dv = dv * thick;
      double ax = g[a][0], ay = g[a][1], cx = g[c][0], cy = g[c][1];
      // explicitly rounded: block (c,a) forms exactly the transpose of (a,c)
      double pxx = __dmul_rn(ax, cx), pyy = __dmul_rn(ay, cy);
      double pxy = __dmul_rn(ax, cy), pyx = __dmul_rn(ay, cx);
      K[0] += dv * __dadd_rn(__dmul_rn(D[0], pxx), __dmul_rn(D[3], pyy));
      K[1] += dv * __dadd_rn(__dmul_rn(D[1], pxy), __dmul_rn(D[3], pyx));
      K[2] += dv * __dadd_rn(__dmul_rn(D[1], pyx), __dmul_rn(D[3], pxy));
      K[3] += dv * __dadd_rn(__dmul_rn(D[2], pyy), __dmul_rn(D[3], pxx));
    }
  if (bad && lane == 0) atomicExch(err, UFEM_AF_ERR_VAL);
  if (MODE == 0) {
    double *bk = val + (size_t)emap[(size_t)e * 16 + lane] * 4;
#pragma unroll
    for (int t = 0; t < 4; t++) bk[t] += K[t];
  } else {
    double *k = Ke + (size_t)e * 64;
    k[(2 * a) * 8 + 2 * c] = K[0];
    k[(2 * a) * 8 + 2 * c + 1] = K[1];
    k[(2 * a + 1) * 8 + 2 * c] = K[2];
    k[(2 * a + 1) * 8 + 2 * c + 1] = K[3];
  }
}

// Zero-valued supports: rows and columns of fixed DOFs become identity
// (femMatSetZeroRow/Col + K[P][P] = 1, fem/fem_loads.c:158-166).
template <int B>
__global__ void k_bc_mask(long nnzb, const int *__restrict__ blkrow, const int *__restrict__ colind,
                          const unsigned char *__restrict__ fixed, double *__restrict__ val) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= nnzb * B * B) return;
  long k = t / (B * B);
  int e = (int)(t % (B * B));
  long row = (long)blkrow[k] * B + e / B, col = (long)colind[k] * B + e % B;
  if (fixed[row] | fixed[col]) val[t] = (row == col) ? 1.0 : 0.0;
}

__global__ void k_zero_fixed(long n, const unsigned char *__restrict__ fixed, double *__restrict__ F,
                             double *__restrict__ u) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n && fixed[i]) {
    F[i] = 0.0;
    u[i] = 0.0;
  }
}

// Supports in input order when some prescribed value is nonzero: one block
// walks the list exactly as fem_add_disps/femApplyDisp do (fem/fem_loads.c:116-262).
template <int B>
__global__ void k_bc_sequential(int nbc, const int *__restrict__ bc_row, const double *__restrict__ bc_val,
                                const int *__restrict__ rowptr, const int *__restrict__ colind,
                                const int *__restrict__ diagblk, double *__restrict__ val, double *__restrict__ F,
                                double *__restrict__ u, double *__restrict__ fval) {
  for (int q = 0; q < nbc; q++) {
    const int P = bc_row[q];
    const double v = bc_val[q];
    const int I = P / B, a = P % B;
    const int k0 = rowptr[I], k1 = rowptr[I + 1];
    __syncthreads();
    if (threadIdx.x == 0) fval[q] = F[P];
    __syncthreads();
    if (v != 0.0) {
      // F[i] += -1.0 * K[i][P] * u_val for every row i (fem/fem_loads.c:211-221)
      for (int t = threadIdx.x; t < (k1 - k0) * B; t += blockDim.x) {
        int k = k0 + t / B, r = t % B, J = colind[k];
        int lo = rowptr[J], hi = rowptr[J + 1] - 1;
        while (lo < hi) {
          int mid = (lo + hi) >> 1;
          if (colind[mid] < I) lo = mid + 1; else hi = mid;
        }
        double kij = val[(size_t)lo * B * B + r * B + a];
        F[(size_t)J * B + r] += (-1.0 * kij * v);
      }
      __syncthreads();
    }
    // zero row P and column P
    for (int t = threadIdx.x; t < (k1 - k0) * B; t += blockDim.x) {
      int k = k0 + t / B, c = t % B, J = colind[k];
      val[(size_t)k * B * B + a * B + c] = 0.0;
      int lo = rowptr[J], hi = rowptr[J + 1] - 1;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (colind[mid] < I) lo = mid + 1; else hi = mid;
      }
      val[(size_t)lo * B * B + c * B + a] = 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double *d = val + (size_t)diagblk[I] * B * B + a * B + a;
      if (v == 0.0) {
        *d = 1.0;
        u[P] = v;
        F[P] = v;
      } else {
        u[P] = v;
        if (fabs(F[P] / v) > FEM_ZERO) {
          *d = F[P] / v;
        } else {
          *d = 1.0;
          F[P] = v;
        }
      }
    }
  }
}

// Result pass for bricks: warp per element, lane = integration point.
__global__ void __launch_bounds__(EPB * 32) k_brick_results(const int *__restrict__ elems, int nelem,
                                                            const double *__restrict__ xyz,
                                                            const int *__restrict__ enodes,
                                                            const int *__restrict__ node_rank,
                                                            const double *__restrict__ eE,
                                                            const double *__restrict__ eNu,
                                                            const double *__restrict__ u, double *__restrict__ sig,
                                                            double *__restrict__ vm, double *__restrict__ fint) {
  __shared__ double s_dN[27][8][3];
  __shared__ double s_w[27];
  __shared__ double s_x[EPB][8][3];
  __shared__ double s_u[EPB][24];
  __shared__ int s_dof[EPB][8];
  brick_tables(s_dN, s_w);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * EPB + warp;
  if (idx >= nelem) return;
  const int e = elems ? elems[idx] : idx;
  if (lane < 8) s_dof[warp][lane] = 3 * node_rank[enodes[(size_t)e * 8 + lane]];
  if (lane < 24) s_x[warp][lane / 3][lane % 3] = xyz[3 * (size_t)enodes[(size_t)e * 8 + lane / 3] + lane % 3];
  __syncwarp();
  if (lane < 24) s_u[warp][lane] = u[s_dof[warp][lane / 3] + lane % 3];
  __syncwarp();
  const double E = eE[e], nu = eNu[e];
  const double d1 = (E * (1.0 - nu)) / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const double d2 = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const double d3 = E / (2.0 * (1 + nu));
  double f[24];
#pragma unroll
  for (int t = 0; t < 24; t++) f[t] = 0.0;
  if (lane < 27) {
    const int ip = lane;
    double inv[3][3];
    double det = brick_jinv(s_dN, ip, s_x[warp], inv);
    double w = det * s_w[ip];
    double g[8][3];
#pragma unroll
    for (int n = 0; n < 8; n++) brick_grad(s_dN, ip, n, inv, g[n]);
    double ex = 0, ey = 0, ez = 0, gyz = 0, gzx = 0, gxy = 0;
#pragma unroll
    for (int n = 0; n < 8; n++) {
      double ux = s_u[warp][3 * n], uy = s_u[warp][3 * n + 1], uz = s_u[warp][3 * n + 2];
      ex += g[n][0] * ux;
      ey += g[n][1] * uy;
      ez += g[n][2] * uz;
      gyz += g[n][2] * uy + g[n][1] * uz;
      gzx += g[n][2] * ux + g[n][0] * uz;
      gxy += g[n][1] * ux + g[n][0] * uy;
    }
    double sx = d1 * ex + d2 * ey + d2 * ez;
    double sy = d2 * ex + d1 * ey + d2 * ez;
    double sz = d2 * ex + d2 * ey + d1 * ez;
    double tyz = d3 * gyz, tzx = d3 * gzx, txy = d3 * gxy;
    double *o = sig + ((size_t)e * 27 + ip) * 6;
    o[0] = sx; o[1] = sy; o[2] = sz; o[3] = tyz; o[4] = tzx; o[5] = txy;
    // von Mises (fdbResComp_vonMisesStress, fdb/fdb_cres.c:404-435, in invariant form)
    vm[(size_t)e * 27 + ip] = sqrt(0.5 * ((sx - sy) * (sx - sy) + (sy - sz) * (sy - sz) + (sz - sx) * (sz - sx)) +
                                   3.0 * (tyz * tyz + tzx * tzx + txy * txy));
#pragma unroll
    for (int n = 0; n < 8; n++) {
      f[3 * n] = w * (g[n][0] * sx + g[n][1] * txy + g[n][2] * tzx);
      f[3 * n + 1] = w * (g[n][1] * sy + g[n][0] * txy + g[n][2] * tyz);
      f[3 * n + 2] = w * (g[n][2] * sz + g[n][1] * tyz + g[n][0] * tzx);
    }
  }
#pragma unroll
  for (int t = 0; t < 24; t++) {
    double v = f[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    f[t] = v;
  }
  if (fint && lane < 24) {
    double mine = 0.0;
#pragma unroll
    for (int t = 0; t < 24; t++)
      if (t == lane) mine = f[t];
    fint[s_dof[warp][lane / 3] + lane % 3] += mine;
  }
}

__global__ void __launch_bounds__(EPB * 32) k_quad_results(const int *__restrict__ elems, int nelem,
                                                           const double *__restrict__ xyz,
                                                           const int *__restrict__ enodes,
                                                           const int *__restrict__ node_rank,
                                                           const double *__restrict__ eE,
                                                           const double *__restrict__ eNu,
                                                           const double *__restrict__ eThick,
                                                           const double *__restrict__ u, double *__restrict__ sig,
                                                           double *__restrict__ vm, double *__restrict__ fint) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * EPB + warp;
  if (idx >= nelem) return;
  const int e = elems ? elems[idx] : idx;
  double X[4][2], ue[8];
  int dof[4];
#pragma unroll
  for (int n = 0; n < 4; n++) {
    size_t q = (size_t)enodes[(size_t)e * 4 + n];
    X[n][0] = xyz[3 * q];
    X[n][1] = xyz[3 * q + 1];
    dof[n] = 2 * node_rank[q];
    ue[2 * n] = u[dof[n]];
    ue[2 * n + 1] = u[dof[n] + 1];
  }
  const double thick = eThick[e];
  double D[4];
  plane_D(eE[e], eNu[e], thick, D);
  double f[8];
#pragma unroll
  for (int t = 0; t < 8; t++) f[t] = 0.0;
  if (lane < 4) {
    const double gp[2] = {-QUAD_GP, QUAD_GP};
    double g[4][2];
    double det = quad_cartd(X, gp[lane >> 1], gp[lane & 1], g);
    double dv = det;
    if (thick > 0.0) dv = dv * thick;
    double ex = 0, ey = 0, gxy = 0;
#pragma unroll
    for (int n = 0; n < 4; n++) {
      ex += g[n][0] * ue[2 * n];
      ey += g[n][1] * ue[2 * n + 1];
      gxy += g[n][1] * ue[2 * n] + g[n][0] * ue[2 * n + 1];
    }
    double sx = D[0] * ex + D[1] * ey, sy = D[1] * ex + D[2] * ey, txy = D[3] * gxy;
    double *o = sig + ((size_t)e * 4 + lane) * 3;
    o[0] = sx; o[1] = sy; o[2] = txy;
    vm[(size_t)e * 4 + lane] = sqrt(sx * sx - sx * sy + sy * sy + 3.0 * txy * txy);
#pragma unroll
    for (int n = 0; n < 4; n++) {
      f[2 * n] = dv * (g[n][0] * sx + g[n][1] * txy);
      f[2 * n + 1] = dv * (g[n][1] * sy + g[n][0] * txy);
    }
  }
#pragma unroll
  for (int t = 0; t < 8; t++) {
    double v = f[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    f[t] = v;
  }
  if (fint && lane < 8) {
    double mine = 0.0;
#pragma unroll
    for (int t = 0; t < 8; t++)
      if (t == lane) mine = f[t];
    fint[dof[lane / 2] + lane % 2] += mine;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
int upload_model(ufem_model *m) {
  // the element nodes, pattern, scatter map, colour groups and block rows
  // are already on the device (gpu_build_pattern)
  int rv;
  if ((rv = m->d_xyz.upload(m->xyz.data(), m->xyz.size())) != UFEM_AF_OK) return rv;
  if ((rv = m->d_eE.upload(m->eE.data(), m->eE.size())) != UFEM_AF_OK) return rv;
  if ((rv = m->d_eNu.upload(m->eNu.data(), m->eNu.size())) != UFEM_AF_OK) return rv;
  if ((rv = m->d_eThick.upload(m->eThick.data(), m->eThick.size())) != UFEM_AF_OK) return rv;
  if ((rv = m->d_fixed.upload(m->fixedMask.data(), m->fixedMask.size())) != UFEM_AF_OK) return rv;
  if ((rv = m->d_val.alloc((size_t)m->nnzb * m->b * m->b)) != UFEM_AF_OK) return rv;
  if ((rv = m->d_F.alloc(m->nDOFAct)) != UFEM_AF_OK) return rv;
  if ((rv = m->d_u.alloc(m->nDOFAct)) != UFEM_AF_OK) return rv;
  UFEM_CUDA_TRY(cudaMemset(m->d_u.p, 0, m->nDOFAct * sizeof(double)));
  UFEM_CUDA_TRY(cudaMemset(m->d_F.p, 0, m->nDOFAct * sizeof(double)));
  m->assembled = m->bcs_applied = false;
  return UFEM_AF_OK;
}

static int check_err_flag(int *d_err) {
  int h = 0;
  UFEM_CUDA_TRY(cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) {
    set_error("non-positive Jacobian determinant in an element");
    return h;
  }
  return UFEM_AF_OK;
}

int gpu_fill_K(ufem_model *m) {
  DBuf<int> d_err;
  int rv;
  if ((rv = d_err.alloc(1)) != UFEM_AF_OK) return rv;
  UFEM_CUDA_TRY(cudaMemset(d_err.p, 0, sizeof(int)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  UFEM_CUDA_TRY(cudaMemsetAsync(m->d_val.p, 0, m->d_val.n * sizeof(double)));
  for (int c = 0; c < m->ncolours; c++) {
    int n = m->colour_ptr[c + 1] - m->colour_ptr[c];
    if (n == 0) continue;
    const int *el = m->d_colour_elems.p + m->colour_ptr[c];
    int grid = (n + EPB - 1) / EPB;
    if (m->etype == 2)
      k_quad_stiff<0><<<grid, EPB * 32>>>(el, n, m->d_xyz.p, m->d_enodes.p, m->d_eE.p, m->d_eNu.p, m->d_eThick.p,
                                          m->d_emap.p, m->d_val.p, nullptr, d_err.p);
    else
      k_brick_stiff<0><<<grid, EPB * 32>>>(el, n, m->d_xyz.p, m->d_enodes.p, m->d_eE.p, m->d_eNu.p, m->d_emap.p,
                                           m->d_val.p, nullptr, d_err.p);
  }
  UFEM_CUDA_TRY(cudaGetLastError());
  cudaEventRecord(e1);
  UFEM_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  m->ms_fill = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if ((rv = check_err_flag(d_err.p)) != UFEM_AF_OK) return rv;
  m->assembled = true;
  m->bcs_applied = false;
  return UFEM_AF_OK;
}

int gpu_element_matrices(ufem_model *m, double *hKe) {
  int s = m->nn * m->b, rv;
  DBuf<double> d_ke;
  DBuf<int> d_err;
  if ((rv = d_ke.alloc((size_t)m->eLen * s * s)) != UFEM_AF_OK) return rv;
  if ((rv = d_err.alloc(1)) != UFEM_AF_OK) return rv;
  UFEM_CUDA_TRY(cudaMemset(d_err.p, 0, sizeof(int)));
  int grid = (int)((m->eLen + EPB - 1) / EPB);
  if (m->etype == 2)
    k_quad_stiff<1><<<grid, EPB * 32>>>(nullptr, (int)m->eLen, m->d_xyz.p, m->d_enodes.p, m->d_eE.p, m->d_eNu.p,
                                        m->d_eThick.p, nullptr, nullptr, d_ke.p, d_err.p);
  else
    k_brick_stiff<1><<<grid, EPB * 32>>>(nullptr, (int)m->eLen, m->d_xyz.p, m->d_enodes.p, m->d_eE.p, m->d_eNu.p,
                                         nullptr, nullptr, d_ke.p, d_err.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  UFEM_CUDA_TRY(cudaMemcpy(hKe, d_ke.p, (size_t)m->eLen * s * s * sizeof(double), cudaMemcpyDeviceToHost));
  return check_err_flag(d_err.p);
}

// Element matrices with E = 1 for every element (K_e is linear in E for the
// isotropic D), written densely to d_out (eLen*s*s, FP64).
int element_matrices_unitE(ufem_model *m, double *d_out) {
  int rv;
  DBuf<double> ones;
  DBuf<int> d_err;
  std::vector<double> h(m->eLen, 1.0);
  if ((rv = ones.upload(h.data(), h.size())) != UFEM_AF_OK) return rv;
  if ((rv = d_err.alloc(1)) != UFEM_AF_OK) return rv;
  UFEM_CUDA_TRY(cudaMemset(d_err.p, 0, sizeof(int)));
  int grid = (int)((m->eLen + EPB - 1) / EPB);
  if (m->etype == 2)
    k_quad_stiff<1><<<grid, EPB * 32>>>(nullptr, (int)m->eLen, m->d_xyz.p, m->d_enodes.p, ones.p, m->d_eNu.p,
                                        m->d_eThick.p, nullptr, nullptr, d_out, d_err.p);
  else
    k_brick_stiff<1><<<grid, EPB * 32>>>(nullptr, (int)m->eLen, m->d_xyz.p, m->d_enodes.p, ones.p, m->d_eNu.p,
                                         nullptr, nullptr, d_out, d_err.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  UFEM_CUDA_TRY(cudaDeviceSynchronize());
  return check_err_flag(d_err.p);
}

int gpu_add_loads(ufem_model *m) {
  UFEM_CUDA_TRY(cudaMemcpy(m->d_F.p, m->F_loads.data(), m->nDOFAct * sizeof(double), cudaMemcpyHostToDevice));
  return UFEM_AF_OK;
}

template <int B>
static int bc_launch(ufem_model *m) {
  if (!m->has_nonzero_bc) {
    long tot = m->nnzb * B * B;
    k_bc_mask<B><<<(unsigned)((tot + 255) / 256), 256>>>(m->nnzb, m->d_blkrow.p, m->d_colind.p, m->d_fixed.p,
                                                         m->d_val.p);
    k_zero_fixed<<<(unsigned)((m->nDOFAct + 255) / 256), 256>>>(m->nDOFAct, m->d_fixed.p, m->d_F.p, m->d_u.p);
    UFEM_CUDA_TRY(cudaGetLastError());
    // F at the time of each support: F after loads, 0 once a DOF was fixed
    std::vector<unsigned char> seen(m->nDOFAct, 0);
    m->reacFval.assign(m->reacRow.size(), 0.0);
    for (size_t r = 0; r < m->reacRow.size(); r++) {
      int p = m->reacRow[r];
      m->reacFval[r] = seen[p] ? 0.0 : m->F_loads[p];
      seen[p] = 1;
    }
    return UFEM_AF_OK;
  }
  std::vector<int> rows;
  std::vector<double> vals;
  std::vector<int> reac_slot;
  for (const auto &l : m->loads) {
    if (l.type != 1) continue;
    long p = m->dof(l.node * KNOWN_DOFS + l.dir - 1);
    rows.push_back((int)(p - 1));
    vals.push_back(l.val);
  }
  DBuf<int> d_rows;
  DBuf<double> d_vals, d_fval;
  int rv;
  if ((rv = d_rows.upload(rows.data(), rows.size())) != UFEM_AF_OK) return rv;
  if ((rv = d_vals.upload(vals.data(), vals.size())) != UFEM_AF_OK) return rv;
  if ((rv = d_fval.alloc(rows.size())) != UFEM_AF_OK) return rv;
  k_bc_sequential<B><<<1, 256>>>((int)rows.size(), d_rows.p, d_vals.p, m->d_rowptr.p, m->d_colind.p, m->d_diagblk.p,
                                 m->d_val.p, m->d_F.p, m->d_u.p, d_fval.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  std::vector<double> fval(rows.size());
  UFEM_CUDA_TRY(cudaMemcpy(fval.data(), d_fval.p, rows.size() * sizeof(double), cudaMemcpyDeviceToHost));
  m->reacFval.clear();
  for (size_t q = 0; q < rows.size(); q++)
    if (vals[q] == 0.0) m->reacFval.push_back(fval[q]);
  return UFEM_AF_OK;
}

int gpu_add_disps(ufem_model *m) {
  if (!m->assembled) {
    set_error("add_disps before fill_K");
    return UFEM_AF_ERR;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  int rv = (m->b == 2) ? bc_launch<2>(m) : bc_launch<3>(m);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  m->ms_bc = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rv == UFEM_AF_OK) m->bcs_applied = true;
  return rv;
}

int gpu_results(ufem_model *m) {
  int rv;
  int nip = (m->etype == 2) ? 4 : 27, ns = (m->etype == 2) ? 3 : 6;
  if (m->d_sig.n != (size_t)m->eLen * nip * ns && (rv = m->d_sig.alloc((size_t)m->eLen * nip * ns)) != UFEM_AF_OK)
    return rv;
  if (m->d_vm.n != (size_t)m->eLen * nip && (rv = m->d_vm.alloc((size_t)m->eLen * nip)) != UFEM_AF_OK) return rv;
  if (m->d_fint.n != (size_t)m->nDOFAct && (rv = m->d_fint.alloc(m->nDOFAct)) != UFEM_AF_OK) return rv;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  UFEM_CUDA_TRY(cudaMemsetAsync(m->d_fint.p, 0, m->nDOFAct * sizeof(double)));
  for (int c = 0; c < m->ncolours; c++) {
    int n = m->colour_ptr[c + 1] - m->colour_ptr[c];
    if (n == 0) continue;
    const int *el = m->d_colour_elems.p + m->colour_ptr[c];
    int grid = (n + EPB - 1) / EPB;
    if (m->etype == 2)
      k_quad_results<<<grid, EPB * 32>>>(el, n, m->d_xyz.p, m->d_enodes.p, m->d_noderank.p, m->d_eE.p, m->d_eNu.p,
                                         m->d_eThick.p, m->d_u.p, m->d_sig.p, m->d_vm.p, m->d_fint.p);
    else
      k_brick_results<<<grid, EPB * 32>>>(el, n, m->d_xyz.p, m->d_enodes.p, m->d_noderank.p, m->d_eE.p, m->d_eNu.p,
                                          m->d_u.p, m->d_sig.p, m->d_vm.p, m->d_fint.p);
  }
  UFEM_CUDA_TRY(cudaGetLastError());
  cudaEventRecord(e1);
  UFEM_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  m->ms_results = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // reactions: (0 - F at support time) + internal force (fem/fem_loads.c:205, fem/fem_sol.c:826-852)
  m->reacVal.assign(m->reacRow.size(), 0.0);
  if (!m->reacRow.empty()) {
    std::vector<double> fint(m->nDOFAct);
    UFEM_CUDA_TRY(cudaMemcpy(fint.data(), m->d_fint.p, m->nDOFAct * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t r = 0; r < m->reacRow.size(); r++) {
      double fv = r < m->reacFval.size() ? m->reacFval[r] : 0.0;
      m->reacVal[r] = (0.0 - fv) + fint[m->reacRow[r]];
    }
  }
  return UFEM_AF_OK;
}

}  // namespace ufem
