// Element-result outputs of the Monte Carlo table and the general failure
// function, as GPU passes over (element, sample):
//   * RES_E (one stored point of one element, fem/fem_mont.c:577-583);
//   * RES_SUM_E / RES_MAX_E / RES_MIN_E / RES_FAIL_E over every element and
//     result set (fem/fem_mont.c:585-650);
//   * RES_FAIL: fem_asse_max_disp_simple and fem_asse_fail_cond
//     (fem/fem_mont.c:661-676, fem/fem_asse.c:42-47, :271-374).
//
// What the reference reads (femGetEResVal -> femGetRepVal,
// fem/fem_accs.c:196-277): set 0 and every set past the element's stored
// points read 0, the linear result pass stores only stresses and strains, so
// sums and extremes run over the stored points of the stress and strain
// codes and every other code gives 0.  MAX/MIN start from the zeroed output
// (so they are max(0, ...) and min(0, ...)), FAIL_E is "some value > 0", i.e.
// MAX_E > 0.  The failure function fails an element whose F_YC reads 0
// (the zero stress of set 0 is not below it) or any stored point whose
// sqrt(3 J2) is not below |F_YC| (tested as 3 J2 against F_YC^2); the
// displacement test compares
// femVecMaxAbs(u), which returns sqrt(max |u_i|) (fem/fem_math.c:2136-2163),
// with MAX_D.
//
// Batches (S a multiple of 128 samples, sample-minor vectors x[row*S + s]):
// one block per (element range, 128 samples); the block computes the
// gradients of each element's stored points once in shared memory and every
// thread (sample) forms its strains and stresses from them, so geometry is
// paid per element, not per sample.  One sample (the plugin's
// monte_solution): one thread per element.  Both write one record per
// (element range, sample) -- sums, maxima, minima of the 2*ns stress/strain
// components and the strength flag -- and k_eo_final folds the ranges in
// order (run-to-run identical).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "elem_point.cuh"
#include "ufem_internal.h"

namespace ufem {

namespace {

constexpr int kEoThreads = 128;
constexpr int kUmaxChunks = 64;

template <int B>
struct EoRec {
  static constexpr int NN = (B == 3) ? 8 : 4;   // nodes
  static constexpr int NG = NN * B;             // gradient values per point
  static constexpr int NV = (B == 3) ? 12 : 6;  // stresses then strains
  static constexpr int NQ = 3 * NV + 1;         // sums, maxima, minima, flag
  double sum[NV], mx[NV], mn[NV];
  int fail;
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int c = 0; c < NV; c++) sum[c] = mx[c] = mn[c] = 0.0;
    fail = 0;
  }
  __device__ __forceinline__ void add(const double *v) {
#pragma unroll
    for (int c = 0; c < NV; c++) {
      sum[c] += v[c];
      mx[c] = (v[c] > mx[c]) ? v[c] : mx[c];
      mn[c] = (v[c] < mn[c]) ? v[c] : mn[c];
    }
  }
  __device__ __forceinline__ double get(int q) const {
    double r = 0.0;
#pragma unroll
    for (int c = 0; c < NV; c++) {
      if (q == c) r = sum[c];
      if (q == NV + c) r = mx[c];
      if (q == 2 * NV + c) r = mn[c];
    }
    return q == 3 * NV ? (double)fail : r;
  }
};

template <int B>
__device__ __forceinline__ void point_grad(const double *xyz, const int *en, int ip, double *G) {
  if (B == 3) ep::point_grad_brick(xyz, en, ip, G);
  else ep::point_grad_quad(xyz, en, ip, G);
}

// D per element and sample: 3 (solid) or 4 (plane) coefficients
template <int B>
__device__ __forceinline__ void elem_D(double Ee, double nu, double th, double *d) {
  if (B == 3) ep::elem_D_brick(Ee, nu, d);
  else ep::elem_D_quad(Ee, nu, th, d);
}

template <int B>
__device__ __forceinline__ void point_values(const double *G, const double *ue, const double *d, double *v) {
  if (B == 3) ep::point_values_brick(G, ue, d, v);
  else ep::point_values_quad(G, ue, d, v);
}

template <int B>
__device__ __forceinline__ double point_vmis2(const double *v) {
  return (B == 3) ? ep::vmis2_brick(v) : ep::vmis2_quad(v);
}

// |F_YC| of element e for sample s: the material's value, or the sample's
// input column when one randomises it
__device__ __forceinline__ double elem_fy(int e, int s, int nsamp, const double *fy0, const int *fycol,
                                          const double *ifld, long ilen) {
  double fy = fy0[e];
  const int c = fycol ? fycol[e] : -1;
  if (c >= 0 && s < nsamp) fy = ifld[(size_t)s * ilen + c];
  return fabs(fy);
}

// batches: block = (element range blockIdx.x, 128 samples blockIdx.y)
template <int B>
__global__ void __launch_bounds__(kEoThreads) k_eo_samples(int ne, int S, int nsamp, const int *__restrict__ enodes,
                                                           const int *__restrict__ node_rank,
                                                           const unsigned char *__restrict__ enpts,
                                                           const double *__restrict__ xyz, const double *__restrict__ E,
                                                           const double *__restrict__ eNu,
                                                           const double *__restrict__ eThick,
                                                           const double *__restrict__ u, int strength,
                                                           const double *__restrict__ fy0, const int *__restrict__ fycol,
                                                           const double *__restrict__ ifld, long ilen,
                                                           double *__restrict__ part) {
  using R = EoRec<B>;
  __shared__ double sG[ep::kMaxStored][R::NG];
  __shared__ int sEn[R::NN], sRow[R::NN];
  const int s = blockIdx.y * kEoThreads + threadIdx.x;
  const int per = (ne + gridDim.x - 1) / gridDim.x;
  const int e0 = blockIdx.x * per, e1 = min(ne, e0 + per);
  R a;
  a.init();
  for (int e = e0; e < e1; e++) {
    const int np = enpts[e];
    if (threadIdx.x < R::NN) {
      const int q = enodes[(size_t)e * R::NN + threadIdx.x];
      sEn[threadIdx.x] = q;
      sRow[threadIdx.x] = node_rank[q] * B;
    }
    __syncthreads();
    if (threadIdx.x < np) point_grad<B>(xyz, sEn, threadIdx.x, sG[threadIdx.x]);
    double ue[R::NG];
#pragma unroll
    for (int n = 0; n < R::NN; n++)
#pragma unroll
      for (int d = 0; d < B; d++) ue[n * B + d] = u[(size_t)(sRow[n] + d) * S + s];
    double d[4];
    elem_D<B>(E[(size_t)e * S + s], eNu[e], eThick[e], d);
    double fy2 = 0.0;
    if (strength) {
      const double fy = elem_fy(e, s, nsamp, fy0, fycol, ifld, ilen);
      if (!(0.0 < fy)) a.fail = 1;  // result set 0 (zero stress), fem/fem_asse.c:323-327
      fy2 = fy * fy;
    }
    __syncthreads();
    for (int p = 0; p < np; p++) {
      double v[R::NV];
      point_values<B>(sG[p], ue, d, v);
      a.add(v);
      if (strength && !(point_vmis2<B>(v) < fy2)) a.fail = 1;
    }
    __syncthreads();
  }
  for (int q = 0; q < R::NQ; q++) part[((size_t)blockIdx.x * R::NQ + q) * S + s] = a.get(q);
}

// one sample: thread per element, the block folds its 128 records in order
template <int B>
__global__ void __launch_bounds__(kEoThreads) k_eo_elements(int ne, const int *__restrict__ enodes,
                                                            const int *__restrict__ node_rank,
                                                            const unsigned char *__restrict__ enpts,
                                                            const double *__restrict__ xyz,
                                                            const double *__restrict__ E,
                                                            const double *__restrict__ eNu,
                                                            const double *__restrict__ eThick,
                                                            const double *__restrict__ u, int strength,
                                                            const double *__restrict__ fy0, double *__restrict__ part) {
  using R = EoRec<B>;
  __shared__ double sh[R::NQ][kEoThreads];
  const int e = blockIdx.x * kEoThreads + threadIdx.x;
  R a;
  a.init();
  if (e < ne) {
    int en[R::NN];
    double ue[R::NG];
#pragma unroll
    for (int n = 0; n < R::NN; n++) {
      en[n] = enodes[(size_t)e * R::NN + n];
      const int r0 = node_rank[en[n]] * B;
#pragma unroll
      for (int d = 0; d < B; d++) ue[n * B + d] = u[r0 + d];
    }
    double d[4];
    elem_D<B>(E[e], eNu[e], eThick[e], d);
    const double fy = strength ? fabs(fy0[e]) : 0.0, fy2 = fy * fy;
    if (strength && !(0.0 < fy)) a.fail = 1;
    const int np = enpts[e];
    for (int p = 0; p < np; p++) {
      double G[R::NG], v[R::NV];
      point_grad<B>(xyz, en, p, G);
      point_values<B>(G, ue, d, v);
      a.add(v);
      if (strength && !(point_vmis2<B>(v) < fy2)) a.fail = 1;
    }
  }
  for (int q = 0; q < R::NQ; q++) sh[q][threadIdx.x] = a.get(q);
  __syncthreads();
  for (int q = threadIdx.x; q < R::NQ; q += kEoThreads) {
    double r = 0.0;
    for (int t = 0; t < kEoThreads; t++) {
      const double x = sh[q][t];
      if (q < R::NV) r += x;
      else if (q < 2 * R::NV) r = (x > r) ? x : r;
      else if (q < 3 * R::NV) r = (x < r) ? x : r;
      else r = (x != 0.0) ? 1.0 : r;
    }
    part[(size_t)blockIdx.x * R::NQ + q] = r;
  }
}

// max |u_i| per sample over a chunk of rows (lane = sample)
__global__ void __launch_bounds__(256) k_eo_umax(long n, int S, const double *__restrict__ u,
                                                 double *__restrict__ part) {
  __shared__ double sh[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int s = blockIdx.x * 32 + lane;
  const long per = (n + gridDim.y - 1) / gridDim.y;
  const long i0 = (long)blockIdx.y * per, i1 = min(n, i0 + per);
  double m = 0.0;
  if (s < S)
    for (long i = i0 + w; i < i1; i += 8) {
      const double v = fabs(u[(size_t)i * S + s]);
      m = (m < v) ? v : m;
    }
  sh[w][lane] = m;
  __syncthreads();
  if (w == 0 && s < S) {
    double r = 0.0;
    for (int k = 0; k < 8; k++) r = (r < sh[k][lane]) ? sh[k][lane] : r;
    part[(size_t)blockIdx.y * S + s] = r;
  }
}

// aggregates: kind 11 sum, 12 max, 13 min, 14 max > 0, 19 failure function
template <int B>
__global__ void k_eo_final(int nch, int S, int nsamp, int nagg, const int *__restrict__ akind,
                           const int *__restrict__ acomp, const int *__restrict__ apos,
                           const double *__restrict__ part, int nchu, const double *__restrict__ upart, double md0,
                           int mdcol, const double *__restrict__ ifld, long ilen, long olen,
                           double *__restrict__ ofld) {
  using R = EoRec<B>;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsamp) return;
  for (int k = 0; k < nagg; k++) {
    const int kind = akind[k], c = acomp[k];
    double r = 0.0;
    if (kind == 11) {
      for (int ch = 0; ch < nch; ch++) r += part[((size_t)ch * R::NQ + c) * S + s];
    } else if (kind == 12 || kind == 14) {
      for (int ch = 0; ch < nch; ch++) {
        const double x = part[((size_t)ch * R::NQ + R::NV + c) * S + s];
        r = (x > r) ? x : r;
      }
      if (kind == 14) r = (r > 0.0) ? 1.0 : 0.0;
    } else if (kind == 13) {
      for (int ch = 0; ch < nch; ch++) {
        const double x = part[((size_t)ch * R::NQ + 2 * R::NV + c) * S + s];
        r = (x < r) ? x : r;
      }
    } else if (kind == 19) {
      for (int ch = 0; ch < nch; ch++)
        if (part[((size_t)ch * R::NQ + 3 * R::NV) * S + s] != 0.0) r = 1.0;
      const double md = (mdcol >= 0) ? fabs(ifld[(size_t)s * ilen + mdcol]) : md0;
      if (md > 0.0 && upart) {
        double um = 0.0;
        for (int ch = 0; ch < nchu; ch++) {
          const double x = upart[(size_t)ch * S + s];
          um = (um < x) ? x : um;
        }
        if (sqrt(um) >= md) r = 1.0;
      }
    }
    ofld[(size_t)s * olen + apos[k]] = r;
  }
}

// RES_E: thread per (point output, sample)
template <int B>
__global__ void k_eo_points(int npo, int S, int nsamp, const int *__restrict__ pel, const int *__restrict__ pip,
                            const int *__restrict__ pcomp, const int *__restrict__ ppos,
                            const int *__restrict__ enodes, const int *__restrict__ node_rank,
                            const double *__restrict__ xyz, const double *__restrict__ E,
                            const double *__restrict__ eNu, const double *__restrict__ eThick,
                            const double *__restrict__ u, long olen, double *__restrict__ ofld) {
  using R = EoRec<B>;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)npo * nsamp) return;
  const int o = (int)(t / nsamp), s = (int)(t % nsamp), e = pel[o];
  int en[R::NN];
  double ue[R::NG], G[R::NG], v[R::NV];
  for (int n = 0; n < R::NN; n++) {
    en[n] = enodes[(size_t)e * R::NN + n];
    const int r0 = node_rank[en[n]] * B;
    for (int d = 0; d < B; d++) ue[n * B + d] = u[(size_t)(r0 + d) * S + s];
  }
  double d[4];
  elem_D<B>(E[(size_t)e * S + s], eNu[e], eThick[e], d);
  point_grad<B>(xyz, en, pip[o], G);
  point_values<B>(G, ue, d, v);
  double r = 0.0;
  for (int c = 0; c < R::NV; c++)
    if (c == pcomp[o]) r = v[c];
  ofld[(size_t)s * olen + ppos[o]] = r;
}

// index of a result code in the point value vector (stresses, then strains),
// -1 for codes the linear result pass does not store
int value_index(int etype, long code) {
  static const int quad[6] = {7, 8, 10, 13, 14, 16};
  static const int brick[12] = {7, 8, 9, 11, 12, 10, 13, 14, 15, 17, 18, 16};
  const int *t = etype == 2 ? quad : brick;
  const int n = etype == 2 ? 6 : 12;
  for (int c = 0; c < n; c++)
    if (t[c] == code) return c;
  return -1;
}

}  // namespace

int stored_points(long eType) {
  return eType == 2 ? ep::kStoredQuad : (eType == 10 ? ep::kStoredBrickW : ep::kStoredBrick);
}

double mat_f_yc(const ufem_model *m, long mat) {
  // F_YC in the type's non-repeating list: type 5 position 4 (fem/fem_m005.c:39),
  // none in type 1 (fem/fem_m001.c:39); femGetMPValPos gives 0 when absent
  if (mat < 0 || mat >= (long)m->mpVals.size()) return 0.0;
  const long ty = m->mpTypeH[mat];
  const auto &v = m->mpVals[mat];
  if (ty == 5 && v.size() > 4) return v[4];
  return 0.0;
}

int build_elem_outputs(const ufem_model *m, ElemOutPlan &P, const std::vector<int> *fy_col_by_mat, int md_col) {
  std::vector<int> ak, ac, apos, pe, pi, pc, pp;
  P.strength = false;
  for (long i = m->mc_ilen; i < m->mc_ilen + m->mc_olen; i++) {
    const long ty = m->mc_type[i], item = m->mc_item[i], sub = m->mc_sub[i], it = m->mc_iter[i];
    const int pos = (int)m->mc_pos[i - m->mc_ilen];  // fem/fem_mont.c:522 and on
    if ((ty == 10 || (ty >= 11 && ty <= 14) || ty == 19) && (pos < 0 || pos >= m->mc_olen)) {
      set_error("Monte Carlo output position out of range");
      return UFEM_AF_ERR_VAL;
    }
    if (ty == 10) {
      const int c = value_index(m->etype, sub);
      if (c >= 0 && item >= 0 && item < m->eLen && it >= 1 && it <= stored_points(m->eType[item])) {
        pe.push_back((int)item); pi.push_back((int)it - 1); pc.push_back(c); pp.push_back(pos);
      }
    } else if (ty >= 11 && ty <= 14) {
      const int c = value_index(m->etype, sub);
      if (c >= 0) {
        ak.push_back((int)ty); ac.push_back(c); apos.push_back(pos);
      }
    } else if (ty == 19) {
      ak.push_back(19); ac.push_back(0); apos.push_back(pos);
      P.strength = true;
    }
  }
  P.nagg = (int)ak.size();
  P.npo = (int)pe.size();
  P.h_apos = apos;
  P.h_ppos = pp;
  P.md_col = md_col;
  if (P.nagg == 0 && P.npo == 0) return UFEM_AF_OK;
  int rv;
  if ((rv = P.akind.upload(ak.data(), ak.size())) || (rv = P.acomp.upload(ac.data(), ac.size())) ||
      (rv = P.apos.upload(apos.data(), apos.size())) || (rv = P.pel.upload(pe.data(), pe.size())) ||
      (rv = P.pip.upload(pi.data(), pi.size())) || (rv = P.pcomp.upload(pc.data(), pc.size())) ||
      (rv = P.ppos.upload(pp.data(), pp.size())))
    return rv;
  std::vector<unsigned char> np(m->eLen);
  for (long e = 0; e < m->eLen; e++) np[e] = (unsigned char)stored_points(m->eType[e]);
  if ((rv = P.enpts.upload(np.data(), np.size()))) return rv;
  if (P.strength) {
    std::vector<double> fy(m->eLen);
    std::vector<int> col(m->eLen, -1);
    for (long e = 0; e < m->eLen; e++) {
      fy[e] = mat_f_yc(m, m->eMat[e]);
      if (fy_col_by_mat && m->eMat[e] < (long)fy_col_by_mat->size()) col[e] = (*fy_col_by_mat)[m->eMat[e]];
    }
    if ((rv = P.fy0.upload(fy.data(), fy.size())) || (rv = P.fycol.upload(col.data(), col.size()))) return rv;
  }
  return UFEM_AF_OK;
}

int run_elem_outputs(const ufem_model *m, ElemOutPlan &P, int S, int nsamp, const double *u, const double *E,
                     const double *ifld, long ilen, double md0, double *ofld, long olen, int *launches) {
  if ((P.nagg == 0 && P.npo == 0) || nsamp <= 0) return UFEM_AF_OK;
  if (S != 1 && S % kEoThreads != 0) {
    set_error("element outputs: S must be 1 or a multiple of 128");
    return UFEM_AF_ERR_VAL;
  }
  const int B = m->b, ne = (int)m->eLen;
  const int NQ = (B == 3) ? EoRec<3>::NQ : EoRec<2>::NQ;
  int rv;
  if (P.npo > 0) {
    const long tot = (long)P.npo * nsamp;
    const unsigned g = (unsigned)((tot + 127) / 128);
    if (B == 3)
      k_eo_points<3><<<g, 128>>>(P.npo, S, nsamp, P.pel.p, P.pip.p, P.pcomp.p, P.ppos.p, m->d_enodes.p,
                                 m->d_noderank.p, m->d_xyz.p, E, m->d_eNu.p, m->d_eThick.p, u, olen, ofld);
    else
      k_eo_points<2><<<g, 128>>>(P.npo, S, nsamp, P.pel.p, P.pip.p, P.pcomp.p, P.ppos.p, m->d_enodes.p,
                                 m->d_noderank.p, m->d_xyz.p, E, m->d_eNu.p, m->d_eThick.p, u, olen, ofld);
    ++*launches;
  }
  if (P.nagg == 0 || ne == 0) {
    UFEM_CUDA_TRY(cudaGetLastError());
    return UFEM_AF_OK;
  }
  int nch;
  if (S == 1) {
    nch = (ne + kEoThreads - 1) / kEoThreads;
  } else {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int sblocks = S / kEoThreads;
    nch = std::max(1, std::min(ne, (4 * sms + sblocks - 1) / sblocks));
  }
  if ((rv = P.part.ensure((size_t)nch * NQ * S))) return rv;
  const int strength = P.strength ? 1 : 0;
  if (S == 1) {
    if (B == 3)
      k_eo_elements<3><<<nch, kEoThreads>>>(ne, m->d_enodes.p, m->d_noderank.p, P.enpts.p, m->d_xyz.p, E,
                                            m->d_eNu.p, m->d_eThick.p, u, strength, P.fy0.p, P.part.p);
    else
      k_eo_elements<2><<<nch, kEoThreads>>>(ne, m->d_enodes.p, m->d_noderank.p, P.enpts.p, m->d_xyz.p, E,
                                            m->d_eNu.p, m->d_eThick.p, u, strength, P.fy0.p, P.part.p);
  } else {
    const dim3 grid((unsigned)nch, (unsigned)(S / kEoThreads));
    if (B == 3)
      k_eo_samples<3><<<grid, kEoThreads>>>(ne, S, nsamp, m->d_enodes.p, m->d_noderank.p, P.enpts.p, m->d_xyz.p,
                                            E, m->d_eNu.p, m->d_eThick.p, u, strength, P.fy0.p, P.fycol.p, ifld,
                                            ilen, P.part.p);
    else
      k_eo_samples<2><<<grid, kEoThreads>>>(ne, S, nsamp, m->d_enodes.p, m->d_noderank.p, P.enpts.p, m->d_xyz.p,
                                            E, m->d_eNu.p, m->d_eThick.p, u, strength, P.fy0.p, P.fycol.p, ifld,
                                            ilen, P.part.p);
  }
  ++*launches;
  int nchu = 0;
  const bool disp = P.strength && (P.md_col >= 0 || md0 > 0.0);
  if (disp) {
    nchu = (int)std::max(1L, std::min((long)kUmaxChunks, (long)m->nDOFAct / 256));
    if ((rv = P.upart.ensure((size_t)nchu * S))) return rv;
    const dim3 grid((unsigned)((S + 31) / 32), (unsigned)nchu);
    k_eo_umax<<<grid, 256>>>((long)m->nDOFAct, S, u, P.upart.p);
    ++*launches;
  }
  const unsigned gf = (unsigned)((nsamp + 127) / 128);
  if (B == 3)
    k_eo_final<3><<<gf, 128>>>(nch, S, nsamp, P.nagg, P.akind.p, P.acomp.p, P.apos.p, P.part.p, nchu,
                               disp ? P.upart.p : nullptr, md0, P.md_col, ifld, ilen, olen, ofld);
  else
    k_eo_final<2><<<gf, 128>>>(nch, S, nsamp, P.nagg, P.akind.p, P.acomp.p, P.apos.p, P.part.p, nchu,
                               disp ? P.upart.p : nullptr, md0, P.md_col, ifld, ilen, olen, ofld);
  ++*launches;
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_AF_OK;
}

}  // namespace ufem
