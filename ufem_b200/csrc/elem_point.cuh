// Strains and stresses at one result point of one element, for the Monte
// Carlo output passes (batch.cu k_outputs, mcout.cu).  The result points and
// their order are the element integration loops': quad 2x2 Gauss points
// (fem/fem_e002.c:489-499, point = 2 igaus + jgaus, 0-based), brick 3x3x3
// Gauss points (fem/fem_e009.c:366-378, point = 9 i + 3 j + k, 0-based).
//
// point_grad_*: the Cartesian shape-function gradients at the point, the
// geometry part that is the same for every sample; point_values_*: strains
// eps = B u_e and stresses sig = D eps from them, in the reference's stored
// component order (quad: SX, SY, SXY | EX, EY, EXY; brick: SX, SY, SZ, SYZ,
// SZX, SXY | EX, EY, EZ, EYZ, EZX, EXY).
#pragma once

namespace ufem {
namespace ep {

// result points the reference stores per element (femGetRepVal reads index
// idx + res_rp * (k - 1) < rvals, fem/fem_accs.c:263-273, with res_rp/rvals
// 22/76 quad fem/fem_e002.c:942,1024; 20/378 brick fem/fem_e009.c:825,880;
// 32/702 brick with foundation fem/fem_e010.c:41,82): the same count for
// every stress and strain code
constexpr int kStoredQuad = 4, kStoredBrick = 19, kStoredBrickW = 22;
constexpr int kMaxStored = 22;

__device__ __forceinline__ void point_grad_brick(const double *__restrict__ xyz, const int *__restrict__ en, int ip,
                                                 double *__restrict__ G) {
  const double gp[3] = {-0.774596669241483, 0.0, 0.774596669241483};
  const double nc[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                           {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  const double x = gp[ip / 9], y = gp[(ip / 3) % 3], z = gp[ip % 3];
  double dN[8][3], X[8][3], J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int n = 0; n < 8; n++) {
    dN[n][0] = 0.125 * nc[n][0] * (1.0 + nc[n][1] * y) * (1.0 + nc[n][2] * z);
    dN[n][1] = 0.125 * nc[n][1] * (1.0 + nc[n][0] * x) * (1.0 + nc[n][2] * z);
    dN[n][2] = 0.125 * nc[n][2] * (1.0 + nc[n][0] * x) * (1.0 + nc[n][1] * y);
    for (int d = 0; d < 3; d++) X[n][d] = xyz[3 * (size_t)en[n] + d];
  }
  for (int a = 0; a < 3; a++)
    for (int c = 0; c < 3; c++)
      for (int n = 0; n < 8; n++) J[a][c] += dN[n][a] * X[n][c];
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1], c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2],
               c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double id = 1.0 / (J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02);
  const double inv[3][3] = {{c00 * id, (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id,
                             (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id},
                            {c01 * id, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id,
                             (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id},
                            {c02 * id, (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id,
                             (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id}};
  for (int n = 0; n < 8; n++)
    for (int d = 0; d < 3; d++) G[3 * n + d] = inv[d][0] * dN[n][0] + inv[d][1] * dN[n][1] + inv[d][2] * dN[n][2];
}

__device__ __forceinline__ void point_grad_quad(const double *__restrict__ xyz, const int *__restrict__ en, int ip,
                                                double *__restrict__ G) {
  const double qg = 0.577350569189626;  // the reference's Gauss abscissa, fem/fem_e002.c:164
  const double sx_ = (ip >> 1) ? qg : -qg, tx_ = (ip & 1) ? qg : -qg;
  const double dS[4] = {(-1.0 + tx_) * 0.25, (1.0 - tx_) * 0.25, (1.0 + tx_) * 0.25, (-1.0 - tx_) * 0.25};
  const double dT[4] = {(-1.0 + sx_) * 0.25, (-1.0 - sx_) * 0.25, (1.0 + sx_) * 0.25, (1.0 - sx_) * 0.25};
  double j00 = 0, j01 = 0, j10 = 0, j11 = 0;
  for (int n = 0; n < 4; n++) {
    const double X0 = xyz[3 * (size_t)en[n]], X1 = xyz[3 * (size_t)en[n] + 1];
    j00 += dS[n] * X0; j01 += dS[n] * X1; j10 += dT[n] * X0; j11 += dT[n] * X1;
  }
  const double det = j00 * j11 - j01 * j10;
  for (int n = 0; n < 4; n++) {
    G[2 * n] = (j11 / det) * dS[n] + (-j01 / det) * dT[n];
    G[2 * n + 1] = (-j10 / det) * dS[n] + (j00 / det) * dT[n];
  }
}

// D of the isotropic solid (fem/fem_pl3d.c:32-60): d[0] diagonal normal,
// d[1] off-diagonal normal, d[2] shear; per element and sample
__device__ __forceinline__ void elem_D_brick(double Ee, double nu, double *__restrict__ d) {
  d[0] = (Ee * (1.0 - nu)) / ((1.0 + nu) * (1.0 - 2.0 * nu));
  d[1] = (Ee * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
  d[2] = Ee / (2.0 * (1 + nu));
}

// plane D: thick > 0 plane stress, else plane strain (fem/fem_e002.c:400-407,
// fem/fem_stf2.c:43-89); d = D11, D12, D22, D33
__device__ __forceinline__ void elem_D_quad(double Ee, double nu, double thick, double *__restrict__ d) {
  if (thick > 0.0) {
    const double Mul = Ee / (1 - nu * nu);
    d[0] = Mul; d[1] = Mul * nu; d[2] = Mul; d[3] = Mul * 0.5 * (1 - nu);
  } else {
    const double Mul = Ee / ((1 + nu) * (1 - 2 * nu));
    d[0] = Mul * (1 - nu); d[1] = Mul * nu; d[2] = Mul * (1 - nu); d[3] = Mul * 0.5 * (1 - nu);
  }
}

// v[0..5]: SX, SY, SZ, SYZ, SZX, SXY; v[6..11]: EX, EY, EZ, EYZ, EZX, EXY
__device__ __forceinline__ void point_values_brick(const double *__restrict__ G, const double *__restrict__ ue,
                                                   const double *__restrict__ d, double *__restrict__ v) {
  double ep[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int n = 0; n < 8; n++) {
    const double g0 = G[3 * n], g1 = G[3 * n + 1], g2 = G[3 * n + 2];
    const double ux = ue[3 * n], uy = ue[3 * n + 1], uz = ue[3 * n + 2];
    ep[0] += g0 * ux; ep[1] += g1 * uy; ep[2] += g2 * uz;
    ep[3] += g2 * uy + g1 * uz; ep[4] += g2 * ux + g0 * uz; ep[5] += g1 * ux + g0 * uy;
  }
  v[0] = d[0] * ep[0] + d[1] * ep[1] + d[1] * ep[2];
  v[1] = d[1] * ep[0] + d[0] * ep[1] + d[1] * ep[2];
  v[2] = d[1] * ep[0] + d[1] * ep[1] + d[0] * ep[2];
  v[3] = d[2] * ep[3]; v[4] = d[2] * ep[4]; v[5] = d[2] * ep[5];
#pragma unroll
  for (int c = 0; c < 6; c++) v[6 + c] = ep[c];
}

// v[0..2]: SX, SY, SXY; v[3..5]: EX, EY, EXY
__device__ __forceinline__ void point_values_quad(const double *__restrict__ G, const double *__restrict__ ue,
                                                  const double *__restrict__ d, double *__restrict__ v) {
  double ex = 0, ey = 0, gxy = 0;
#pragma unroll
  for (int n = 0; n < 4; n++) {
    const double gx = G[2 * n], gy = G[2 * n + 1], ux = ue[2 * n], uy = ue[2 * n + 1];
    ex += gx * ux; ey += gy * uy; gxy += gy * ux + gx * uy;
  }
  v[0] = d[0] * ex + d[1] * ey; v[1] = d[1] * ex + d[2] * ey; v[2] = d[3] * gxy;
  v[3] = ex; v[4] = ey; v[5] = gxy;
}

// 3 J2 of the stored stress vector, the square of the von Mises stress that
// fem_asse_mat_vmis compares with |F_YC| (sqrt(3 J2) < |F_YC|, J2 of
// stress2D_J2 fem/fem_ch2d.c:46-57 or stress3D_J2 fem/fem_chen.c:54-74):
// 3 J2 = ((sx-sy)^2 + sx^2 + sy^2) / 2 + 3 txy^2 (plane),
//        ((sx-sy)^2 + (sy-sz)^2 + (sz-sx)^2) / 2 + 3 (tyz^2 + tzx^2 + txy^2) (solid).
// Callers test 3 J2 < F_YC^2, the same order for non-negative values, and a
// NaN stress fails both forms.
__device__ __forceinline__ double vmis2_quad(const double *v) {
  const double a = v[0] - v[1];
  return 0.5 * (a * a + v[0] * v[0] + v[1] * v[1]) + 3.0 * (v[2] * v[2]);
}
__device__ __forceinline__ double vmis2_brick(const double *v) {
  const double a = v[0] - v[1], b = v[1] - v[2], c = v[2] - v[0];
  return 0.5 * (a * a + b * b + c * c) + 3.0 * (v[5] * v[5] + v[4] * v[4] + v[3] * v[3]);
}

}  // namespace ep
}  // namespace ufem
