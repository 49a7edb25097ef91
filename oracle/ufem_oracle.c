/*
 * ufem_oracle.c -- CPU restatement of the reference uFEM linear static path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker for the CUDA path: tests,
 * the smoke check and the CPU-baseline leg of the benchmark may call it; the
 * product (ufem_b200/csrc, libufem_gpu.so) never links, loads or calls it.
 *
 * It restates, in the reference's own floating-point operation order (plain
 * C, no FMA contraction), so that its results are bit-identical to the
 * reference built from source (pinned by tests/test_oracle.py against dumps
 * of oracle/_ref/serial/ref_harness, committed as tests/golden/):
 *
 *   quad element matrix      stiffp / sfr / jacob / bmatp / dbe / mirrorK
 *                            fem/fem_e002.c:39-346, 346-760
 *   plane D                  D_HookIso_planeRaw, fem/fem_stf2.c:43-89
 *   brick element matrix     e009_stiff, fem/fem_e009.c:261-635, with
 *                            e008_init_gauss fem/fem_e008.c:470-489,
 *                            femLUinverse fem/fem_math.c:2285-2466
 *   3-D D                    femD_3D_iso, fem/fem_pl3d.c:32-57
 *   DOF numbering            fem_dofs, fem/fem_sol.c:1263-1395
 *   row-slot sizes           femKhit, fem/fem_mloc.c:83-116
 *   scatter                  femLocKM_e fem/fem_mloc.c:163-221 ->
 *                            femMatPutAdd fem/fem_math.c:185-236
 *   nodal forces / supports  femApplyNLoad fem/fem_loads.c:343,
 *                            femApplyDisp fem/fem_loads.c:116-262
 *   Jacobi PCG               femEqsCGwJ fem/fem_eqs.c:88-247
 *   SSOR PCG                 femEqsCGwSSOR fem/fem_eqs.c:1001-1217
 *   Jacobi BiCGStab          femEqsBiCCSwJ fem/fem_eqs.c:262-468
 *   norms                    femMatNormBig fem/fem_math.c:1856,
 *                            femVecNormBig :2022, femVecVecMultBig :1017
 *   result pass              fem_fill_K(AF_YES) fem/fem_sol.c:748-990
 *                            (stresses sigma = D B u_e at every integration
 *                            point, internal forces, reactions)
 *
 * Return codes are the reference's AF_* values (fem/fem.h:41-52).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define AF_OK 0
#define AF_ERR (-1)
#define AF_ERR_VAL (-3)
#define AF_ERR_MEM (-4)
#define AF_ERR_TYP (-5)
#define AF_ERR_SIZ (-9)
#define AF_ERR_BIG (-11)
#define AF_ERR_ZER (-13)
#define FEM_ZERO 1e-17
#define FEM_TINY_VAL 1.0e-20
#define KNOWN_DOFS 7

/* ------------------------------------------------------------------------ */
/* element matrices                                                         */
/* ------------------------------------------------------------------------ */

/* plane D, fem/fem_stf2.c:43-89 (problem 0 = plane stress, 1 = plane strain) */
static int plane_D(double E, double nu, int problem, double D[3][3])
{
  double Mul;
  memset(D, 0, 9 * sizeof(double));
  if ((nu <= 0.0) || (nu >= 1)) return AF_ERR_VAL;
  if (problem == 0) {
    Mul = E / (1 - (nu * nu));
    D[0][0] = Mul; D[0][1] = Mul * nu; D[1][0] = Mul * nu; D[1][1] = Mul;
    D[2][2] = Mul * 0.5 * (1 - nu);
  } else {
    Mul = E / ((1 + nu) * (1 - (2 * nu)));
    D[0][0] = Mul * (1 - nu); D[0][1] = Mul * nu; D[1][0] = Mul * nu;
    D[1][1] = Mul * (1 - nu); D[2][2] = Mul * 0.5 * (1 - nu);
  }
  return AF_OK;
}

/* 2x2 Gauss abscissa of fem/fem_e002.c:164 (the literal, typo included) */
static const double QUAD_GP = 0.577350569189626;

/* shape derivatives, Jacobian and cartesian derivatives at (s,t):
 * sfr fem/fem_e002.c:53-66, jacob fem/fem_e002.c:195-255 */
static int quad_cartd(const double *xy, double s, double t, double cartd[2][4], double *djacb)
{
  double deriv[2][4], xjacm[2][2], xjaci[2][2];
  int i, j, n;
  deriv[0][0] = (-1.0 + t) * 0.25; deriv[0][1] = (+1.0 - t) * 0.25;
  deriv[0][2] = (+1.0 + t) * 0.25; deriv[0][3] = (-1.0 - t) * 0.25;
  deriv[1][0] = (-1.0 + s) * 0.25; deriv[1][1] = (-1.0 - s) * 0.25;
  deriv[1][2] = (+1.0 + s) * 0.25; deriv[1][3] = (+1.0 - s) * 0.25;
  for (i = 0; i < 2; i++)
    for (j = 0; j < 2; j++) {
      xjacm[i][j] = 0;
      for (n = 0; n < 4; n++) xjacm[i][j] += deriv[i][n] * xy[2 * n + j];
    }
  *djacb = (xjacm[0][0] * xjacm[1][1]) - (xjacm[0][1] * xjacm[1][0]);
  if (*djacb <= 0) return AF_ERR_VAL;
  xjaci[0][0] = xjacm[1][1] / (*djacb);
  xjaci[1][1] = xjacm[0][0] / (*djacb);
  xjaci[0][1] = -xjacm[0][1] / (*djacb);
  xjaci[1][0] = -xjacm[1][0] / (*djacb);
  for (i = 0; i < 2; i++)
    for (n = 0; n < 4; n++) {
      cartd[i][n] = 0;
      for (j = 0; j < 2; j++) cartd[i][n] += (xjaci[i][j] * deriv[j][n]);
    }
  return AF_OK;
}

/* B matrix, bmatp fem/fem_e002.c:260-285 */
static void quad_B(double cartd[2][4], double B[3][8])
{
  int n;
  for (n = 0; n < 4; n++) {
    B[0][2 * n] = cartd[0][n]; B[0][2 * n + 1] = 0.0;
    B[1][2 * n] = 0.0;         B[1][2 * n + 1] = cartd[1][n];
    B[2][2 * n] = cartd[1][n]; B[2][2 * n + 1] = cartd[0][n];
  }
}

/* quad element stiffness, stiffp Mode=AF_NO, fem/fem_e002.c:346-760 */
int orc_quad_ke(const double *xy, double E, double nu, double thick, double *Ke)
{
  double posgp[2], cartd[2][4], B[3][8], DB[3][8], D[3][3], djacb, dvolu;
  int ig, jg, i, j, k, rv, problem = (thick <= 0.0) ? 1 : 0;
  posgp[0] = -QUAD_GP;
  posgp[1] = -1 * posgp[0];   /* gaussq mirror, fem/fem_e002.c:176-181 */
  memset(Ke, 0, 64 * sizeof(double));
  for (ig = 0; ig < 2; ig++)
    for (jg = 0; jg < 2; jg++) {
      /* sfr(nnode, etasp=posgp[jgaus], exitsp=posgp[igaus]): s = posgp[ig], t = posgp[jg] */
      if ((rv = quad_cartd(xy, posgp[ig], posgp[jg], cartd, &djacb)) != AF_OK) return rv;
      dvolu = djacb * 1.0 * 1.0;
      if (thick > 0.0) dvolu = dvolu * thick;
      quad_B(cartd, B);
      if ((rv = plane_D(E, nu, problem, D)) != AF_OK) return rv;
      for (i = 0; i < 3; i++)
        for (j = 0; j < 8; j++) {
          DB[i][j] = 0.0;
          for (k = 0; k < 3; k++) DB[i][j] += D[i][k] * B[k][j];
        }
      for (i = 0; i < 8; i++)
        for (j = i; j < 8; j++)
          for (k = 0; k < 3; k++) Ke[i * 8 + j] += B[k][i] * DB[k][j] * dvolu;
    }
  for (i = 0; i < 8; i++)
    for (j = 0; j < i; j++) Ke[i * 8 + j] = Ke[j * 8 + i];
  return AF_OK;
}

/* brick natural coordinates, e009_fill_coords fem/fem_e009.c:36-70 */
static const double BRICK_NC[8][3] = {
  {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
  {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
/* 3-point Gauss rule, e008_init_gauss fem/fem_e008.c:481-488 */
static const double BRICK_GP[3] = {-0.774596669241483, 0.000000000000000, 0.774596669241483};
static const double BRICK_GW[3] = {0.555555555555556, 0.888888888888889, 0.555555555555556};

/* shape-function derivative d N_n / d xi_d, e009_p_a fem/fem_e009.c:106-145 */
static double brick_dN(int d, int n, double x, double y, double z)
{
  double xv = BRICK_NC[n][0], yv = BRICK_NC[n][1], zv = BRICK_NC[n][2];
  switch (d) {
    case 0: return (0.125 * xv * (1.0 + yv * y) * (1.0 + zv * z));
    case 1: return (0.125 * yv * (1.0 + xv * x) * (1.0 + zv * z));
    default: return (0.125 * zv * (1.0 + xv * x) * (1.0 + yv * y));
  }
}

/* Crout LU with implicit pivoting and the inverse by column back-substitution:
 * femLUdecomp fem/fem_math.c:2285-2378, femLUback :2388-2430, femLUinverse
 * :2440-2466 (the classic ludcmp/lubksb pair), 3x3 only. */
static int lu_inverse3(double a[3][3])
{
  double vv[3], big, dum, sum, temp, col[3], b[3][3];
  int i, j, k, imax = 0, idx[3], ii, ip;
  const int n = 3;
  for (i = 0; i < n; i++) {
    big = 0.0;
    for (j = 0; j < n; j++) if ((temp = fabs(a[i][j])) > big) big = temp;
    if (big == 0.0) return AF_ERR_VAL;
    vv[i] = 1.0 / big;
  }
  for (j = 0; j < n; j++) {
    for (i = 0; i < j; i++) {
      sum = a[i][j];
      for (k = 0; k < i; k++) sum -= (a[i][k] * a[k][j]);
      a[i][j] = sum;
    }
    big = 0.0;
    for (i = j; i < n; i++) {
      sum = a[i][j];
      for (k = 0; k < j; k++) sum -= (a[i][k] * a[k][j]);
      a[i][j] = sum;
      if ((dum = vv[i] * fabs(sum)) >= big) { big = dum; imax = i; }
    }
    if (j != imax) {
      for (k = 0; k < n; k++) { dum = a[imax][k]; a[imax][k] = a[j][k]; a[j][k] = dum; }
      vv[imax] = vv[j];
    }
    idx[j] = imax;
    if (a[j][j] == 0.0) a[j][j] = FEM_TINY_VAL;
    if (j != n - 1) {
      dum = 1.0 / a[j][j];
      for (i = j + 1; i < n; i++) a[i][j] = (dum * a[i][j]);
    }
  }
  for (j = 0; j < n; j++) {
    for (i = 0; i < n; i++) col[i] = 0.0;
    col[j] = 1.0;
    ii = -1;
    for (i = 0; i < n; i++) {
      ip = idx[i];
      sum = col[ip];
      col[ip] = col[i];
      if (ii >= 0) {
        for (k = ii; k <= i - 1; k++) sum -= a[i][k] * col[k];
      } else if (sum) {
        ii = i;
      }
      col[i] = sum;
    }
    for (i = n - 1; i >= 0; i--) {
      sum = col[i];
      for (k = i + 1; k < n; k++) sum -= a[i][k] * col[k];
      col[i] = (sum / a[i][i]);
    }
    for (i = 0; i < n; i++) b[i][j] = col[i];
  }
  for (i = 0; i < n; i++)
    for (j = 0; j < n; j++) a[i][j] = b[i][j];
  return AF_OK;
}

static void iso_D3(double Ex, double nu, double D[6][6])
{
  double d1, d2, d3;
  d1 = (Ex * (1.0 - nu)) / ((1.0 + nu) * (1.0 - 2.0 * nu));
  d2 = (Ex * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
  d3 = Ex / (2.0 * (1 + nu));
  memset(D, 0, 36 * sizeof(double));
  D[0][0] = D[1][1] = D[2][2] = d1;
  D[0][1] = D[0][2] = D[1][0] = D[2][0] = D[1][2] = D[2][1] = d2;
  D[3][3] = D[4][4] = D[5][5] = d3;
}

/* H (strain-displacement) matrix and integration multiplier at one point:
 * e009_fill_J fem/fem_e009.c:189-205, e009_jac_det :76-100,
 * e009_fill_H :207-258 (active #else branch: rows 4/5/6 = yz/zx/xy) */
static int brick_H(const double *xyz, int i, int j, int k, double H[6][24], double *mult)
{
  double jac[3][3], x = BRICK_GP[i], y = BRICK_GP[j], z = BRICK_GP[k], val, vi, detj;
  double h11, h22, h33;
  int a, b, n, rv;
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++) {
      val = 0.0;
      for (n = 0; n < 8; n++) {
        vi = brick_dN(a, n, x, y, z);
        vi *= xyz[3 * n + b];
        val += vi;
      }
      jac[a][b] = 0.0 + val;
    }
  detj = jac[0][0] * jac[1][1] * jac[2][2] + jac[1][0] * jac[2][1] * jac[0][2] +
         jac[0][1] * jac[1][2] * jac[2][0] + -jac[2][0] * jac[1][1] * jac[0][2] -
         jac[0][0] * jac[1][2] * jac[2][1] - jac[2][2] * jac[1][0] * jac[0][1];
  if (detj <= 0.0) return AF_ERR_VAL;
  *mult = detj * BRICK_GW[i] * BRICK_GW[j] * BRICK_GW[k];
  if ((rv = lu_inverse3(jac)) != AF_OK) return rv;
  memset(H, 0, 6 * 24 * sizeof(double));
  for (n = 0; n < 8; n++) {
    h11 = h22 = h33 = 0.0;
    for (a = 0; a < 3; a++) {
      h11 += jac[0][a] * brick_dN(a, n, x, y, z);
      h22 += jac[1][a] * brick_dN(a, n, x, y, z);
      h33 += jac[2][a] * brick_dN(a, n, x, y, z);
    }
    H[0][3 * n] = h11; H[1][3 * n + 1] = h22; H[2][3 * n + 2] = h33;
    H[5][3 * n] = h22; H[5][3 * n + 1] = h11;
    H[3][3 * n + 1] = h33; H[3][3 * n + 2] = h22;
    H[4][3 * n] = h33; H[4][3 * n + 2] = h11;
  }
  return AF_OK;
}

/* brick element stiffness, e009_stiff Mode=AF_NO, fem/fem_e009.c:261-635:
 * K_e += mult * ((H^T D) H) at 27 points, x outer, then y, z inner */
int orc_brick_ke(const double *xyz, double E, double nu, double *Ke)
{
  double H[6][24], D[6][6], HTD[24][6], Ki, mult, val;
  int i, j, k, a, b, c, rv;
  iso_D3(E, nu, D);
  memset(Ke, 0, 576 * sizeof(double));
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++)
      for (k = 0; k < 3; k++) {
        if ((rv = brick_H(xyz, i, j, k, H, &mult)) != AF_OK) return rv;
        for (a = 0; a < 24; a++)
          for (b = 0; b < 6; b++) {
            val = 0;
            for (c = 0; c < 6; c++) val += H[c][a] * D[c][b];
            HTD[a][b] = val;
          }
        for (a = 0; a < 24; a++)
          for (b = 0; b < 24; b++) {
            val = 0;
            for (c = 0; c < 6; c++) val += HTD[a][c] * H[c][b];
            Ki = val;
            Ke[a * 24 + b] += mult * Ki;
          }
      }
  return AF_OK;
}

/* ------------------------------------------------------------------------ */
/* model tables                                                             */
/* ------------------------------------------------------------------------ */

typedef struct {
  long nLen, eLen, rsLen, mpLen, nlLen;
  double *xyz;                      /* nLen x 3 */
  long *eType, *eRS, *eMP, *eNodes; /* eNodes: eLen x nn */
  long nn;                          /* nodes per element (uniform) */
  long *rsFrom, *rsCnt; double *rsVal;
  long *mpType, *mpFrom, *mpCnt; double *mpVal;
  long *nlNode, *nlType, *nlDir; double *nlVal;
  /* solution state */
  long nDOFAct, *nDOFfld;
  long rows, Klen, *frompos, *defpos, *pos; double *Kdata;
  double *F, *u;
  long resRLen, *resRnode, *resRdof; double *resRval;
} orc_model;

static long *ldup(const long *p, long n) { long *q = (long *)malloc((n > 0 ? n : 1) * sizeof(long)); if (n > 0) memcpy(q, p, n * sizeof(long)); return q; }
static double *ddup(const double *p, long n) { double *q = (double *)malloc((n > 0 ? n : 1) * sizeof(double)); if (n > 0) memcpy(q, p, n * sizeof(double)); return q; }

void *orc_model_new(long nLen, const double *xyz, long eLen, long nn, const long *eType,
                    const long *eRS, const long *eMP, const long *eNodes, long rsLen,
                    const long *rsFrom, const long *rsCnt, const double *rsVal, long rsLenL,
                    long mpLen, const long *mpType, const long *mpFrom, const long *mpCnt,
                    const double *mpVal, long mpLenL, long nlLen, const long *nlNode,
                    const long *nlType, const long *nlDir, const double *nlVal)
{
  orc_model *m = (orc_model *)calloc(1, sizeof(orc_model));
  m->nLen = nLen; m->eLen = eLen; m->nn = nn; m->rsLen = rsLen; m->mpLen = mpLen; m->nlLen = nlLen;
  m->xyz = ddup(xyz, 3 * nLen);
  m->eType = ldup(eType, eLen); m->eRS = ldup(eRS, eLen); m->eMP = ldup(eMP, eLen);
  m->eNodes = ldup(eNodes, eLen * nn);
  m->rsFrom = ldup(rsFrom, rsLen); m->rsCnt = ldup(rsCnt, rsLen); m->rsVal = ddup(rsVal, rsLenL);
  m->mpType = ldup(mpType, mpLen); m->mpFrom = ldup(mpFrom, mpLen); m->mpCnt = ldup(mpCnt, mpLen);
  m->mpVal = ddup(mpVal, mpLenL);
  m->nlNode = ldup(nlNode, nlLen); m->nlType = ldup(nlType, nlLen); m->nlDir = ldup(nlDir, nlLen);
  m->nlVal = ddup(nlVal, nlLen);
  return m;
}

void orc_model_free(void *mv)
{
  orc_model *m = (orc_model *)mv;
  if (!m) return;
  free(m->xyz); free(m->eType); free(m->eRS); free(m->eMP); free(m->eNodes);
  free(m->rsFrom); free(m->rsCnt); free(m->rsVal); free(m->mpType); free(m->mpFrom);
  free(m->mpCnt); free(m->mpVal); free(m->nlNode); free(m->nlType); free(m->nlDir);
  free(m->nlVal); free(m->nDOFfld); free(m->frompos); free(m->defpos); free(m->pos);
  free(m->Kdata); free(m->F); free(m->u); free(m->resRnode); free(m->resRdof); free(m->resRval);
  free(m);
}

/* element data lookups (femGetRepVal fem/fem_accs.c:196-288):
 * material type 1 value order DENS, EX, NU (fem/fem_m001.c:38),
 * quad real set order HEIGHT, ... (fem/fem_e002.c:1019) */
static double mat_val(orc_model *m, long e, int idx)
{
  long p = m->eMP[e];
  return (idx < m->mpCnt[p]) ? m->mpVal[m->mpFrom[p] + idx] : 0.0;
}
static double rs_val(orc_model *m, long e, int idx)
{
  long p = m->eRS[e];
  if (m->rsLen <= 0 || p < 0 || p >= m->rsLen) return 0.0;
  return (idx < m->rsCnt[p]) ? m->rsVal[m->rsFrom[p] + idx] : 0.0;
}
static int elem_dofs(long t) { return t == 2 ? 2 : 3; }
static int elem_nodes(long t) { return t == 2 ? 4 : 8; }

static int elem_ke(orc_model *m, long e, double *Ke)
{
  double c[24];
  long t = m->eType[e];
  int n, nn = elem_nodes(t);
  for (n = 0; n < nn; n++) {
    long q = m->eNodes[e * m->nn + n];
    c[3 * n] = m->xyz[3 * q]; c[3 * n + 1] = m->xyz[3 * q + 1]; c[3 * n + 2] = m->xyz[3 * q + 2];
  }
  if (t == 2) {
    double xy[8];
    for (n = 0; n < 4; n++) { xy[2 * n] = c[3 * n]; xy[2 * n + 1] = c[3 * n + 1]; }
    return orc_quad_ke(xy, mat_val(m, e, 1), mat_val(m, e, 2), rs_val(m, e, 0), Ke);
  }
  if (t == 9 || t == 10) {
    if (t == 10 && rs_val(m, e, 0) > 0.0) return AF_ERR_TYP;  /* Winkler springs not restated */
    return orc_brick_ke(c, mat_val(m, e, 1), mat_val(m, e, 2), Ke);
  }
  return AF_ERR_TYP;
}

int orc_elem_ke(void *mv, long e, double *Ke) { return elem_ke((orc_model *)mv, e, Ke); }

/* fem_dofs, fem/fem_sol.c:1263-1395 (femFastBC off) and femKhit, fem/fem_mloc.c:83 */
int orc_dofs(void *mv, long *nDOFAct_out)
{
  orc_model *m = (orc_model *)mv;
  long i, j, k, act = 0, sum = m->nLen * KNOWN_DOFS;
  free(m->nDOFfld);
  m->nDOFfld = (long *)calloc(sum, sizeof(long));
  for (i = 0; i < m->eLen; i++) {
    long t = m->eType[i];
    for (j = 0; j < elem_nodes(t); j++) {
      long np = m->eNodes[i * m->nn + j];
      if (np < 0 || np >= m->nLen) return AF_ERR_VAL;
      for (k = 0; k < elem_dofs(t); k++) {
        long d = np * KNOWN_DOFS + k;   /* ndof = {U_X,U_Y[,U_Z]} -> slots 0,1[,2] */
        if (m->nDOFfld[d] == 0) { m->nDOFfld[d] = 1; act++; }
      }
    }
  }
  if (act < 1) return AF_ERR_SIZ;
  m->nDOFAct = act;
  act = 1;
  for (i = 0; i < sum; i++) if (m->nDOFfld[i] != 0) m->nDOFfld[i] = act++;
  if (nDOFAct_out) *nDOFAct_out = m->nDOFAct;
  return AF_OK;
}

void orc_get_ndoffld(void *mv, long *out) { orc_model *m = (orc_model *)mv; memcpy(out, m->nDOFfld, m->nLen * KNOWN_DOFS * sizeof(long)); }

static long kpos(orc_model *m, long node, long dof)
{
  long pi = node * KNOWN_DOFS + (dof - 1);
  if (pi < 0 || pi >= m->nLen * KNOWN_DOFS) return 0;
  return m->nDOFfld[pi];
}

/* femMatPutAdd, fem/fem_math.c:185-236: linear search of the row, first
 * empty slot (pos==0) takes the new column; mode 1 = add, 0 = put */
static int mat_putadd(orc_model *m, long row, long col, double val, int add)
{
  long i;
  for (i = m->frompos[row - 1]; i < m->frompos[row - 1] + m->defpos[row - 1]; i++) {
    if (m->pos[i] == col) { if (add) m->Kdata[i] += val; else m->Kdata[i] = val; return AF_OK; }
    if (m->pos[i] == 0) { m->pos[i] = col; if (add) m->Kdata[i] += val; else m->Kdata[i] = val; return AF_OK; }
  }
  return AF_ERR_BIG;
}

static double mat_get(orc_model *m, long row, long col)
{
  long i;
  for (i = m->frompos[row - 1]; i < m->frompos[row - 1] + m->defpos[row - 1]; i++) {
    if (m->pos[i] == 0) break;
    if (m->pos[i] == col) return m->Kdata[i];
  }
  return 0.0;
}

static void loc_vec(orc_model *m, long e, long *lf)
{
  long t = m->eType[e];
  int n, d, p = 0;
  for (n = 0; n < elem_nodes(t); n++)
    for (d = 0; d < elem_dofs(t); d++) {
      lf[p] = kpos(m, m->eNodes[e * m->nn + n], d + 1);
      if (lf[p] < 1) lf[p] = 0;
      p++;
    }
}

/* allocation of the row-slot K (fem_sol_alloc fem/fem_sol.c:479 with
 * K_rows from femKhit) followed by fem_fill_K(AF_NO) in element order */
int orc_fill_K(void *mv)
{
  orc_model *m = (orc_model *)mv;
  long i, j, k, e, lf[24], *krows, sum = 0;
  double Ke[576];
  int rv, sz;
  m->rows = m->nDOFAct;
  krows = (long *)calloc(m->rows, sizeof(long));
  for (i = 0; i < m->eLen; i++) {
    long t = m->eType[i];
    for (j = 0; j < elem_nodes(t); j++)
      for (k = 0; k < elem_dofs(t); k++) {
        long p = kpos(m, m->eNodes[i * m->nn + j], k + 1);
        if (p < 1) continue;
        krows[p - 1] += elem_nodes(t) * elem_dofs(t);
      }
  }
  free(m->frompos); free(m->defpos); free(m->pos); free(m->Kdata);
  m->frompos = (long *)malloc(m->rows * sizeof(long));
  m->defpos = (long *)malloc(m->rows * sizeof(long));
  for (i = 0; i < m->rows; i++) { sum += krows[i]; m->defpos[i] = krows[i]; m->frompos[i] = sum - krows[i]; }
  free(krows);
  m->Klen = sum;
  m->pos = (long *)calloc(sum, sizeof(long));
  m->Kdata = (double *)calloc(sum, sizeof(double));
  free(m->F); free(m->u);
  m->F = (double *)calloc(m->rows, sizeof(double));
  m->u = (double *)calloc(m->rows, sizeof(double));
  for (e = 0; e < m->eLen; e++) {
    if ((rv = elem_ke(m, e, Ke)) != AF_OK) return rv;
    loc_vec(m, e, lf);
    sz = elem_nodes(m->eType[e]) * elem_dofs(m->eType[e]);
    for (i = 0; i < sz; i++)
      for (j = 0; j < sz; j++)
        if ((lf[i] * lf[j]) != 0)
          if ((rv = mat_putadd(m, lf[i], lf[j], Ke[i * sz + j], 1)) != AF_OK) return rv;
  }
  return AF_OK;
}

long orc_K_len(void *mv) { return ((orc_model *)mv)->Klen; }
long orc_rows(void *mv) { return ((orc_model *)mv)->rows; }
void orc_get_K(void *mv, long *frompos, long *defpos, long *pos, double *data)
{
  orc_model *m = (orc_model *)mv;
  if (frompos) memcpy(frompos, m->frompos, m->rows * sizeof(long));
  if (defpos) memcpy(defpos, m->defpos, m->rows * sizeof(long));
  if (pos) memcpy(pos, m->pos, m->Klen * sizeof(long));
  if (data) memcpy(data, m->Kdata, m->Klen * sizeof(double));
}
void orc_get_F(void *mv, double *F) { orc_model *m = (orc_model *)mv; memcpy(F, m->F, m->rows * sizeof(double)); }
void orc_get_u(void *mv, double *u) { orc_model *m = (orc_model *)mv; memcpy(u, m->u, m->rows * sizeof(double)); }
void orc_set_u(void *mv, const double *u) { orc_model *m = (orc_model *)mv; memcpy(m->u, u, m->rows * sizeof(double)); }

/* fem_add_loads(0) (fem/fem_sol.c:1119): type-3 nodal forces, F[pos] += val */
int orc_add_loads(void *mv)
{
  orc_model *m = (orc_model *)mv;
  long i, p;
  for (i = 0; i < m->nlLen; i++) {
    if (m->nlType[i] != 3) continue;
    p = kpos(m, m->nlNode[i], m->nlDir[i]);
    if (p <= 0) continue;
    m->F[p - 1] += m->nlVal[i];
  }
  return AF_OK;
}

/* reaction list, fem_sol_res_alloc fem/fem_sol.c:676-722 (type 1 with value 0) */
static void alloc_reac(orc_model *m)
{
  long i, s = 0;
  free(m->resRnode); free(m->resRdof); free(m->resRval);
  m->resRLen = 0;
  for (i = 0; i < m->nlLen; i++) if (m->nlType[i] == 1 && m->nlVal[i] == 0.0) m->resRLen++;
  m->resRnode = (long *)calloc(m->resRLen + 1, sizeof(long));
  m->resRdof = (long *)calloc(m->resRLen + 1, sizeof(long));
  m->resRval = (double *)calloc(m->resRLen + 1, sizeof(double));
  for (i = 0; i < m->nlLen; i++)
    if (m->nlType[i] == 1 && m->nlVal[i] == 0.0) { m->resRnode[s] = m->nlNode[i]; m->resRdof[s] = m->nlDir[i]; s++; }
}

/* fem_add_disps(AF_YES,0) fem/fem_sol.c:1195 -> femApplyDisp fem/fem_loads.c:116-262,
 * serial femMatSetZeroCol (whole-matrix scan, fem/fem_math.c:680) */
int orc_add_disps(void *mv)
{
  orc_model *m = (orc_model *)mv;
  long i, j, P, r;
  alloc_reac(m);
  for (i = 0; i < m->nlLen; i++) {
    double Val = m->nlVal[i], F_Val;
    if (m->nlType[i] != 1) continue;
    if ((P = kpos(m, m->nlNode[i], m->nlDir[i])) <= 0) return AF_ERR_VAL;
    F_Val = m->F[P - 1];
    if (Val == 0) {
      for (j = m->frompos[P - 1]; j < m->frompos[P - 1] + m->defpos[P - 1]; j++) { if (m->pos[j] == 0) break; m->Kdata[j] = 0; }
      for (j = 0; j < m->Klen; j++) if (m->pos[j] == P) m->Kdata[j] = 0;
      mat_putadd(m, P, P, 1, 0);
      m->u[P - 1] = Val; m->F[P - 1] = Val;
      for (r = 0; r < m->resRLen; r++)
        if (m->resRnode[r] == m->nlNode[i] && m->resRdof[r] == m->nlDir[i]) { m->resRval[r] -= F_Val; break; }
    } else {
      double u_Val = Val;
      for (r = 1; r <= m->rows; r++) m->F[r - 1] += (-1.0 * mat_get(m, r, P) * u_Val);
      for (j = m->frompos[P - 1]; j < m->frompos[P - 1] + m->defpos[P - 1]; j++) { if (m->pos[j] == 0) break; m->Kdata[j] = 0; }
      for (j = 0; j < m->Klen; j++) if (m->pos[j] == P) m->Kdata[j] = 0;
      m->u[P - 1] = Val;
      if (fabs(m->F[P - 1] / u_Val) > FEM_ZERO) mat_putadd(m, P, P, (m->F[P - 1] / u_Val), 0);
      else { mat_putadd(m, P, P, 1.0, 0); m->F[P - 1] = Val; }
    }
  }
  return AF_OK;
}

/* ------------------------------------------------------------------------ */
/* solvers on the row-slot matrix                                           */
/* ------------------------------------------------------------------------ */

typedef struct { long rows; const long *frompos, *defpos, *pos; const double *data; } rs_mat;

static void spmv(const rs_mat *a, const double *b, double *c)
{
  long i, j; double val;
  for (i = 0; i < a->rows; i++) {
    val = 0.0;
    for (j = a->frompos[i]; j < a->frompos[i] + a->defpos[i]; j++) {
      if (a->pos[j] <= 0) break;
      val += (a->data[j] * b[a->pos[j] - 1]);
    }
    c[i] = val;
  }
}
static double dot(long n, const double *a, const double *b) { long i; double s = 0.0; for (i = 0; i < n; i++) s += (a[i] * b[i]); return s; }
static double vnorm(long n, const double *a) { long i; double s = 0.0; for (i = 0; i < n; i++) s += (a[i] * a[i]); return sqrt(s); }
static double mnorm(const rs_mat *a)
{
  long i, j; double nr, mx = 0.0;
  for (i = 0; i < a->rows; i++) {
    nr = 0.0;
    for (j = a->frompos[i]; j < a->frompos[i] + a->defpos[i]; j++) { if (a->pos[j] <= 0) break; nr += (a->data[j] * a->data[j]); }
    nr = sqrt(nr);
    if (nr > mx) mx = nr;
  }
  return mx;
}
static double diag(const rs_mat *a, long i)
{
  long j;
  for (j = a->frompos[i]; j < a->frompos[i] + a->defpos[i]; j++) { if (a->pos[j] == 0) break; if (a->pos[j] == i + 1) return a->data[j]; }
  return 0.0;
}

/* femEqsCGwJ, fem/fem_eqs.c:88-247.  Test-infrastructure extension (not in
 * the reference): a negative eps selects the relative-residual rule
 * |r| <= |eps| |b| on the recursive residual, the CPU leg at the GPU solver's
 * tolerance (at 1e-8 the recursive and the true FP64 residual agree). */
int orc_eqs_cgwj(long rows, const long *frompos, const long *defpos, const long *pos, const double *data,
                 const double *b, double *x, double eps, long maxIt, long *iters)
{
  rs_mat A = {rows, frompos, defpos, pos, data};
  double *M, *r, *z, *p, *q, ro, alpha, beta, roro = 0.0, normRes, normX, normA, normB;
  long n = rows, i, j;
  int rv = AF_OK, conv = 0;
  if (iters) *iters = 0;
  normA = mnorm(&A);
  normB = vnorm(n, b);
  if (normB <= 0.0) { for (i = 0; i < n; i++) x[i] = 0.0; return AF_OK; }
  M = (double *)calloc(n, sizeof(double)); r = (double *)calloc(n, sizeof(double)); z = (double *)calloc(n, sizeof(double));
  p = (double *)calloc(n, sizeof(double)); q = (double *)calloc(n, sizeof(double));
  for (i = 0; i < n; i++) { M[i] = diag(&A, i); if (fabs(M[i]) < FEM_ZERO) { rv = AF_ERR_ZER; goto out; } }
  spmv(&A, x, r);
  for (i = 0; i < n; i++) r[i] = b[i] - r[i];
  for (i = 1; i <= maxIt; i++) {
    for (j = 0; j < n; j++) z[j] = (r[j] / M[j]);
    ro = dot(n, r, z);
    if (i == 1) { for (j = 0; j < n; j++) p[j] = z[j]; }
    else { beta = ro / roro; for (j = 0; j < n; j++) p[j] = (z[j] + (beta * p[j])); }
    spmv(&A, p, q);
    alpha = ro / dot(n, p, q);
    for (j = 0; j < n; j++) { x[j] = x[j] + (alpha * p[j]); r[j] = r[j] - (alpha * q[j]); }
    normRes = vnorm(n, r);
    normX = vnorm(n, x);
    if (iters) *iters = i;
    if (eps < 0.0 ? normRes <= -eps * normB : normRes <= (eps * ((normA * normX) + normB))) { conv = 1; break; }
    roro = ro;
  }
  if (!conv) rv = AF_ERR;
out:
  free(M); free(r); free(z); free(p); free(q);
  return rv;
}

/* femEqsCGwSSOR, fem/fem_eqs.c:1001-1217 (sparse branch of the sweeps) */
int orc_eqs_cgwssor(long rows, const long *frompos, const long *defpos, const long *pos, const double *data,
                    const double *b, double *x, double eps, long maxIt, long *iters)
{
  rs_mat A = {rows, frompos, defpos, pos, data};
  double *M, *r, *z, *zz, *p, *q, ro, alpha, beta, roro = 0.0, normRes, normX, normA, normB, val;
  long n = rows, i, ii, j, ip;
  int rv = AF_OK, conv = 0;
  if (iters) *iters = 0;
  normA = mnorm(&A);
  normB = vnorm(n, b);
  if (normB <= 0.0) { for (i = 0; i < n; i++) x[i] = 0.0; return AF_OK; }
  M = (double *)calloc(n, sizeof(double)); r = (double *)calloc(n, sizeof(double)); z = (double *)calloc(n, sizeof(double));
  zz = (double *)calloc(n, sizeof(double)); p = (double *)calloc(n, sizeof(double)); q = (double *)calloc(n, sizeof(double));
  for (i = 0; i < n; i++) { val = diag(&A, i); if (fabs(val) < FEM_ZERO) { rv = AF_ERR_ZER; goto out; } M[i] = 1.0 / val; }
  spmv(&A, x, r);
  for (i = 0; i < n; i++) r[i] = b[i] - r[i];
  for (i = 1; i <= maxIt; i++) {
    for (ii = 1; ii <= n; ii++) {
      val = 0.0;
      for (j = frompos[ii - 1]; j < frompos[ii - 1] + defpos[ii - 1]; j++) {
        ip = pos[j];
        if ((ip >= ii) || (ip < 1)) continue;
        val += data[j] * zz[ip - 1];
      }
      zz[ii - 1] = M[ii - 1] * (r[ii - 1] - val);
    }
    for (ii = n; ii >= 1; ii--) {
      val = 0.0;
      for (j = frompos[ii - 1]; j < frompos[ii - 1] + defpos[ii - 1]; j++) {
        ip = pos[j];
        if (ip > ii) val += data[j] * z[ip - 1];
      }
      z[ii - 1] = zz[ii - 1] - M[ii - 1] * val;
    }
    ro = dot(n, r, z);
    if (i == 1) { for (j = 0; j < n; j++) p[j] = z[j]; }
    else { beta = ro / roro; for (j = 0; j < n; j++) p[j] = (z[j] + (beta * p[j])); }
    spmv(&A, p, q);
    alpha = ro / dot(n, p, q);
    for (j = 0; j < n; j++) { x[j] = x[j] + (alpha * p[j]); r[j] = r[j] - (alpha * q[j]); }
    normRes = vnorm(n, r);
    normX = vnorm(n, x);
    if (iters) *iters = i;
    if (normRes <= (eps * ((normA * normX) + normB))) { conv = 1; break; }
    roro = ro;
  }
  if (!conv) rv = AF_ERR;
out:
  free(M); free(r); free(z); free(zz); free(p); free(q);
  return rv;
}

/* femEqsBiCCSwJ, fem/fem_eqs.c:262-468.  The reference's true-residual call
 * eqsCompResid(a, b, x, &res) passes b and x swapped against the prototype
 * (a, x, b, r) (fem/fem_eqs.c:37 vs :425), so its test measures |A b - x|;
 * restated as written.  Always returns AF_OK, as the reference does. */
int orc_eqs_bicgs(long rows, const long *frompos, const long *defpos, const long *pos, const double *data,
                  const double *b, double *x, double eps, long maxIt, long *iters)
{
  rs_mat A = {rows, frompos, defpos, pos, data};
  double *M, *r, *rr, *p, *pp, *s, *ss, *t, *v, *res;
  double ro, beta, roro = 0.0, alpha = 0.0, omega = 0.0, normRes, normX, normA, normB;
  long n = rows, i, j;
  if (iters) *iters = 0;
  normA = mnorm(&A);
  normX = vnorm(n, x);
  normB = vnorm(n, b);
  M = (double *)calloc(n, sizeof(double)); r = (double *)calloc(n, sizeof(double)); rr = (double *)calloc(n, sizeof(double));
  p = (double *)calloc(n, sizeof(double)); pp = (double *)calloc(n, sizeof(double)); s = (double *)calloc(n, sizeof(double));
  ss = (double *)calloc(n, sizeof(double)); t = (double *)calloc(n, sizeof(double)); v = (double *)calloc(n, sizeof(double));
  res = (double *)calloc(n, sizeof(double));
  for (i = 0; i < n; i++) { M[i] = diag(&A, i); if (fabs(M[i]) < FEM_ZERO) goto out; }
  spmv(&A, x, r);
  for (i = 0; i < n; i++) { r[i] = b[i] - r[i]; rr[i] = r[i]; }
  if (vnorm(n, r) <= FEM_ZERO) goto out;
  for (i = 1; i <= maxIt; i++) {
    if (iters) *iters = i;
    ro = dot(n, rr, r);
    if (fabs(ro) <= 0.0) goto out;
    if (i == 1) { for (j = 0; j < n; j++) p[j] = r[j]; }
    else {
      beta = (ro / roro) * (alpha / omega);
      for (j = 0; j < n; j++) p[j] = r[j] + beta * (p[j] - (omega * v[j]));
    }
    for (j = 0; j < n; j++) pp[j] = p[j] / M[j];
    spmv(&A, pp, v);
    alpha = (ro / dot(n, rr, v));
    for (j = 0; j < n; j++) s[j] = r[j] - (alpha * v[j]);
    if (vnorm(n, s) <= FEM_ZERO) { for (j = 0; j < n; j++) x[j] += alpha * pp[j]; break; }
    for (j = 0; j < n; j++) ss[j] = s[j] / M[j];
    spmv(&A, ss, t);
    omega = (dot(n, t, s) / dot(n, t, t));
    for (j = 0; j < n; j++) { x[j] += alpha * pp[j] + (omega * ss[j]); r[j] = s[j] - (omega * t[j]); }
    roro = ro;
    /* eqsCompResid(a, b, x, &res): res = A*b - x, fem/fem_eqs.c:37-60 */
    {
      long k, q;
      for (k = 0; k < n; k++) {
        res[k] = 0 - x[k];
        for (q = frompos[k]; q < frompos[k] + defpos[k]; q++) { if (pos[q] <= 0) break; res[k] += (data[q] * b[pos[q] - 1]); }
      }
    }
    normRes = vnorm(n, res);
    normX = vnorm(n, x);
    if (normRes < (eps * ((normA * normX) + normB))) break;
  }
out:
  free(M); free(r); free(rr); free(p); free(pp); free(s); free(ss); free(t); free(v); free(res);
  return AF_OK;
}

/* solver selection as femSolve (fem/fem_sol.c:1716-1730): 0 = CGwJ, 1 = SSOR, 2 = BiCGStab */
int orc_solve(void *mv, int solver, double eps, long maxIt, long *iters)
{
  orc_model *m = (orc_model *)mv;
  if (solver == 1) return orc_eqs_cgwssor(m->rows, m->frompos, m->defpos, m->pos, m->Kdata, m->F, m->u, eps, maxIt, iters);
  if (solver == 2) return orc_eqs_bicgs(m->rows, m->frompos, m->defpos, m->pos, m->Kdata, m->F, m->u, eps, maxIt, iters);
  return orc_eqs_cgwj(m->rows, m->frompos, m->defpos, m->pos, m->Kdata, m->F, m->u, eps, maxIt, iters);
}

/* ------------------------------------------------------------------------ */
/* result pass: stresses at every integration point, internal forces,       */
/* reactions (fem_fill_K(AF_YES), fem/fem_sol.c:748-880)                    */
/* ------------------------------------------------------------------------ */

/* stresses: quad 4 IPs x (SX,SY,SXY); brick 27 IPs x (SX,SY,SZ,SYZ,SZX,SXY).
 * sig must hold eLen*4*3 (quad) or eLen*27*6 (brick) doubles.
 * fint (length rows) receives the assembled internal forces sum_e F_e. */
int orc_results(void *mv, double *sig, double *fint, double *reac)
{
  orc_model *m = (orc_model *)mv;
  long e, i, j, lf[24], r;
  int rv;
  double *F = (double *)calloc(m->rows, sizeof(double));
  for (e = 0; e < m->eLen; e++) {
    long t = m->eType[e];
    double ue[24], Fe[24];
    int sz = elem_nodes(t) * elem_dofs(t), n;
    loc_vec(m, e, lf);
    for (i = 0; i < sz; i++) ue[i] = lf[i] ? m->u[lf[i] - 1] : 0.0;
    for (i = 0; i < sz; i++) Fe[i] = 0.0;
    if (t == 2) {
      double xy[8], posgp[2], cartd[2][4], B[3][8], D[3][3], djacb, dvolu, eps3[3], s3[3], si2[3][4];
      double thick = rs_val(m, e, 0);
      int ig, jg, ip = 0, problem = thick <= 0.0 ? 1 : 0;
      for (n = 0; n < 4; n++) { long q = m->eNodes[e * m->nn + n]; xy[2 * n] = m->xyz[3 * q]; xy[2 * n + 1] = m->xyz[3 * q + 1]; }
      posgp[0] = -QUAD_GP; posgp[1] = -1 * posgp[0];
      if ((rv = plane_D(mat_val(m, e, 1), mat_val(m, e, 2), problem, D)) != AF_OK) { free(F); return rv; }
      for (ig = 0; ig < 2; ig++)
        for (jg = 0; jg < 2; jg++, ip++) {
          if ((rv = quad_cartd(xy, posgp[ig], posgp[jg], cartd, &djacb)) != AF_OK) { free(F); return rv; }
          quad_B(cartd, B);
          for (i = 0; i < 3; i++) { eps3[i] = 0.0; for (j = 0; j < 8; j++) eps3[i] += (B[i][j] * ue[j]); }
          for (i = 0; i < 3; i++) { s3[i] = 0.0; for (j = 0; j < 3; j++) s3[i] += (eps3[j] * D[i][j]); }
          for (i = 0; i < 3; i++) { si2[i][ip] = s3[i]; if (sig) sig[(e * 4 + ip) * 3 + i] = s3[i]; }
        }
      ip = 0;
      for (ig = 0; ig < 2; ig++)
        for (jg = 0; jg < 2; jg++, ip++) {
          quad_cartd(xy, posgp[ig], posgp[jg], cartd, &djacb);
          dvolu = djacb * 1.0 * 1.0;
          if (thick > 0.0) dvolu = dvolu * thick;
          quad_B(cartd, B);
          for (i = 0; i < 8; i++) for (j = 0; j < 3; j++) Fe[i] += B[j][i] * si2[j][ip] * dvolu;
        }
    } else {
      double c[24], H[6][24], D[6][6], mult, ep[6], sg[6], F0[24];
      int a, b, k, ip = 0;
      for (n = 0; n < 8; n++) { long q = m->eNodes[e * m->nn + n]; c[3 * n] = m->xyz[3 * q]; c[3 * n + 1] = m->xyz[3 * q + 1]; c[3 * n + 2] = m->xyz[3 * q + 2]; }
      iso_D3(mat_val(m, e, 1), mat_val(m, e, 2), D);
      for (a = 0; a < 3; a++) for (b = 0; b < 3; b++) for (k = 0; k < 3; k++, ip++) {
        if ((rv = brick_H(c, a, b, k, H, &mult)) != AF_OK) { free(F); return rv; }
        for (i = 0; i < 6; i++) { ep[i] = 0.0; for (j = 0; j < 24; j++) ep[i] += (ue[j] * H[i][j]); }
        for (i = 0; i < 6; i++) { sg[i] = 0.0; for (j = 0; j < 6; j++) sg[i] += (ep[j] * D[i][j]); }
        if (sig) for (i = 0; i < 6; i++) sig[(e * 27 + ip) * 6 + i] = sg[i];
        for (i = 0; i < 24; i++) { F0[i] = 0.0; for (j = 0; j < 6; j++) F0[i] += (sg[j] * H[j][i]); }
        for (i = 0; i < 24; i++) Fe[i] += mult * F0[i];
      }
    }
    for (i = 0; i < sz; i++) if (lf[i] != 0) F[lf[i] - 1] += Fe[i];
  }
  if (fint) memcpy(fint, F, m->rows * sizeof(double));
  if (reac) {
    for (r = 0; r < m->resRLen; r++) {
      long p = kpos(m, m->resRnode[r], m->resRdof[r]);
      reac[r] = m->resRval[r] + (p > 0 ? F[p - 1] : 0.0);
    }
  }
  free(F);
  return AF_OK;
}

long orc_reac_len(void *mv) { return ((orc_model *)mv)->resRLen; }

/* strains eps = B u_e at every integration point, the values the result pass
 * stores as RES_EX.. (quad: EX, EY, EXY, fem/fem_e002.c:656-658; brick: EX,
 * EY, EZ, EYZ, EZX, EXY, fem/fem_e009.c:545-556); layout as orc_results' sig. */
int orc_strains(void *mv, double *eps)
{
  orc_model *m = (orc_model *)mv;
  long e, i, j, lf[24];
  int rv;
  for (e = 0; e < m->eLen; e++) {
    long t = m->eType[e];
    double ue[24];
    int sz = elem_nodes(t) * elem_dofs(t), n;
    loc_vec(m, e, lf);
    for (i = 0; i < sz; i++) ue[i] = lf[i] ? m->u[lf[i] - 1] : 0.0;
    if (t == 2) {
      double xy[8], posgp[2], cartd[2][4], B[3][8], djacb;
      int ig, jg, ip = 0;
      for (n = 0; n < 4; n++) { long q = m->eNodes[e * m->nn + n]; xy[2 * n] = m->xyz[3 * q]; xy[2 * n + 1] = m->xyz[3 * q + 1]; }
      posgp[0] = -QUAD_GP; posgp[1] = -1 * posgp[0];
      for (ig = 0; ig < 2; ig++)
        for (jg = 0; jg < 2; jg++, ip++) {
          if ((rv = quad_cartd(xy, posgp[ig], posgp[jg], cartd, &djacb)) != AF_OK) return rv;
          quad_B(cartd, B);
          for (i = 0; i < 3; i++) {
            double s = 0.0;
            for (j = 0; j < 8; j++) s += (B[i][j] * ue[j]);
            eps[(e * 4 + ip) * 3 + i] = s;
          }
        }
    } else {
      double c[24], H[6][24], mult;
      int a, b, k, ip = 0;
      for (n = 0; n < 8; n++) { long q = m->eNodes[e * m->nn + n]; c[3 * n] = m->xyz[3 * q]; c[3 * n + 1] = m->xyz[3 * q + 1]; c[3 * n + 2] = m->xyz[3 * q + 2]; }
      for (a = 0; a < 3; a++) for (b = 0; b < 3; b++) for (k = 0; k < 3; k++, ip++) {
        if ((rv = brick_H(c, a, b, k, H, &mult)) != AF_OK) return rv;
        for (i = 0; i < 6; i++) {
          double s = 0.0;
          for (j = 0; j < 24; j++) s += (ue[j] * H[i][j]);
          eps[(e * 27 + ip) * 6 + i] = s;
        }
      }
    }
  }
  return AF_OK;
}
