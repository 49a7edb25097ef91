// Batched Monte Carlo solve: many samples of several meshes (uneven sizes) in
// one persistent launch.  Replaces the per-sample loop an external driver runs
// over monte_solution (fem/fem_mont.c:694) -> monte_linear_solver
// (fem/fem_mont.c:480-508), which zeroes K/F/u, re-assembles (fem_fill_K),
// re-applies loads and supports and solves, one sample at a time.
//
// Layout (per mesh, S samples padded to a multiple of the sample group GS):
//   values  V[(k*B*B + e)*S + s]   block k, entry e, sample s (sample fastest)
//   vectors x[i*S + s]             DOF i, sample s
// so a warp that owns one block row and GS samples reads every value and
// every gathered neighbour with full 128-byte transactions, and one read of
// the row's column indices serves GS samples.
//
// Assembly: the element matrices of one mesh are integrated once with E = 1
// (K_e is linear in E for the isotropic D of fem/fem_pl3d.c:32-57) and kept
// in FP64.  Per sample, K_s = sum_e E_{s,e} K_e is gathered block by block
// through per-block contribution lists in element order -- the order of the
// reference's femLocKM_e accumulation (fem/fem_mloc.c:163-221) -- so the FP64
// sums are deterministic without atomics.  Supports are applied in the same
// pass (rows/columns of fixed DOFs -> identity, fem/fem_loads.c:158-166).
//
// Solve: Jacobi PCG with the FP32 matrix and FP32 work vectors (FP64 when
// precision = 0), one persistent cooperative kernel over work tiles (mesh,
// sample group, block-row chunk) of every mesh.  The solution is kept in
// FP64 (x += alpha p in FP64), and the recursive residual is replaced by the
// true residual f - K x, computed in FP64 from the FP64 values, every
// replace_every iterations and whenever it has dropped by the factor
// replace_near since the last replacement: the CG keeps its search direction
// across replacements (no restart), so FP32 costs about the FP64 iteration
// count.  A sample converges only on a true residual, |f - K x| / |f| <=
// tol: once its recursive residual is below tol / 2 it is frozen until a
// true-residual pass of its group confirms it (or it resumes).  Two bounded
// grid barriers per iteration (three when a replacement runs, two more for
// the coarse correction); per-sample masks freeze converged samples, a
// group of GS samples drops out when all of its samples are done, the launch
// ends when no group is left or at the iteration cap.  Per-sample scalars
// come from per-tile partials reduced in a fixed order (run-to-run
// identical); partial buffers are double-buffered by iteration parity so no
// block overwrites what another still reads.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <sys/stat.h>
#include <memory>
#include <vector>

#include "device_util.cuh"
#include "tcgen05.cuh"
#include "ufem_internal.h"

namespace ufem {

// ---------------------------------------------------------------------------
// per-mesh plan (host + device), built once per model
// ---------------------------------------------------------------------------
struct McOut {
  int type;    // MONTE_VTYPE_RES_*
  int pos;     // ofld position
  int row;     // DOF row for RES_D / RES_R / RES_D_MAX / RES_D_MIN (0-based) or -1;
               // the constant of RES_D_SUM
  int reac;    // reaction index
};

// FP32 unit blocks of the implicit form: B*B values padded to 12 floats
// (three 16-byte loads per contribution)
constexpr int kW32Stride = 12;

struct McPlan {
  bool built = false;
  int s = 0;                       // element matrix size (8 or 24)
  DBuf<double> Khat;               // eLen*s*s, E = 1
  DBuf<int> gptr, gel, gpair;      // per-block contribution lists
  DBuf<int> elem_var;              // ifld column of each element's E, -1 = base
  DBuf<double> F0;                 // loads that no input variable overrides
  std::vector<int> ovr_row, ovr_var;
  DBuf<int> d_ovr_row, d_ovr_var;
  DBuf<int> d_ovr_ptr, d_ovr_rvar;  // the overrides by DOF row (input order within a row)
  std::vector<McOut> outs;
  DBuf<int> d_out_type, d_out_pos, d_out_row;
  DBuf<int> reac_rows;             // DOF rows of the reaction list
  long ilen = 0, olen = 0;
  // host copies for the implicit form
  std::vector<int> h_gptr, h_gel, h_gpair, h_elem_var;
  // implicit (matrix-free) form, precision 2: per block, the unit-E element
  // blocks summed per multiplier -- multiplier 0 is the constant 1 (elements
  // whose E is not random, pre-scaled by their E), multiplier j >= 1 is the
  // ifld column mult_col[j] -- with supported rows/columns zeroed
  bool imp_built = false;
  int nmult = 0, cstride = 0;
  std::vector<int> mult_col;
  DBuf<int> d_mult_col, cptr, crow;  // contributions of block k / of block row I
  DBuf<double> cval;               // [nc][cstride]: B*B values, then (multiplier << 32 | J)
  DBuf<float> w32;                 // [nc][12]: the B*B values in FP32 (precision 4's SpMV products)
  DBuf<int> sperm;                 // block rows in the order the gathering phases visit them
  long nc = 0;
  // coarse space of the preconditioner (ufem_mc_set_coarse): Wc [n][cmodes]
  // as BF16 tensor-core operand tiles, supported rows zero
  int cmodes = 0;
  DBuf<uint8_t> wt1, wt3;
  // element-result outputs and the failure function (mcout.cu)
  ElemOutPlan eo;
};

static std::vector<std::unique_ptr<McPlan>> g_plans;
static std::vector<const ufem_model *> g_plan_owner;

McPlan *get_plan(const ufem_model *m) {
  for (size_t i = 0; i < g_plan_owner.size(); i++)
    if (g_plan_owner[i] == m) return g_plans[i].get();
  g_plan_owner.push_back(m);
  g_plans.emplace_back(new McPlan());
  return g_plans.back().get();
}

void drop_work(const ufem_model *m);

void drop_plan(const ufem_model *m) {
  drop_work(m);
  for (size_t i = 0; i < g_plan_owner.size(); i++)
    if (g_plan_owner[i] == m) {
      g_plan_owner.erase(g_plan_owner.begin() + i);
      g_plans.erase(g_plans.begin() + i);
      return;
    }
}

int element_matrices_unitE(ufem_model *m, double *d_out);  // kernels.cu

// The order in which the gathering phases (q = A p, the true residual) visit
// block rows: by the Morton key of the row's node position (coordinates
// quantised to 1024 steps per axis over the model's bounding box), so that
// the rows a block works on at once, and one after another, are neighbours in
// space and their gathered neighbour vectors stay in the SM's L1.  On the
// 40x10x10 beam an LRU model of a 128 KB L1 fetches 2x (FP64) to 3x (FP32)
// fewer bytes from L2 per row than in the natural (x fastest) order.
static std::vector<int> morton_row_order(const ufem_model *m) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int I = 0; I < m->nbr; I++)
    for (int d = 0; d < 3; d++) {
      const double v = m->xyz[(size_t)m->rank_node[I] * 3 + d];
      lo[d] = std::min(lo[d], v);
      hi[d] = std::max(hi[d], v);
    }
  std::vector<std::pair<unsigned long long, int>> key(m->nbr);
  for (int I = 0; I < m->nbr; I++) {
    unsigned long long k = 0;
    unsigned q[3];
    for (int d = 0; d < 3; d++) {
      const double span = hi[d] - lo[d];
      const double t = span > 0 ? (m->xyz[(size_t)m->rank_node[I] * 3 + d] - lo[d]) / span : 0.0;
      q[d] = (unsigned)std::min(1023.0, std::max(0.0, t * 1023.0 + 0.5));
    }
    for (int b = 0; b < 10; b++)
      for (int d = 0; d < 3; d++) k |= (unsigned long long)((q[d] >> b) & 1u) << (3 * b + d);
    key[I] = {k, I};
  }
  std::stable_sort(key.begin(), key.end(),
                   [](const std::pair<unsigned long long, int> &a, const std::pair<unsigned long long, int> &b) {
                     return a.first < b.first;
                   });
  std::vector<int> order(m->nbr);
  for (int I = 0; I < m->nbr; I++) order[I] = key[I].second;
  return order;
}

static int build_plan(ufem_model *m, McPlan *P) {
  int rv;
  if ((rv = host_pattern(m)) != UFEM_AF_OK) return rv;
  {
    const std::vector<int> order = morton_row_order(m);
    if ((rv = P->sperm.upload(order.data(), order.size())) != UFEM_AF_OK) return rv;
  }
  const int nn = m->nn, B = m->b, s = nn * B;
  P->s = s;
  P->ilen = m->mc_ilen;
  P->olen = m->mc_olen;
  if ((rv = P->Khat.alloc((size_t)m->eLen * s * s)) != UFEM_AF_OK) return rv;
  if ((rv = element_matrices_unitE(m, P->Khat.p)) != UFEM_AF_OK) return rv;
  // contribution lists: element order within each block
  std::vector<int> cnt(m->nnzb + 1, 0);
  for (long e = 0; e < m->eLen; e++)
    for (int p = 0; p < nn * nn; p++) cnt[m->emap[(size_t)e * nn * nn + p] + 1]++;
  for (long k = 0; k < m->nnzb; k++) cnt[k + 1] += cnt[k];
  std::vector<int> gel(cnt[m->nnzb]), gpair(cnt[m->nnzb]), fill(cnt.begin(), cnt.end() - 1);
  for (long e = 0; e < m->eLen; e++)
    for (int p = 0; p < nn * nn; p++) {
      int k = m->emap[(size_t)e * nn * nn + p];
      gel[fill[k]] = (int)e;
      gpair[fill[k]] = p;
      fill[k]++;
    }
  P->h_gptr = cnt;
  P->h_gel = gel;
  P->h_gpair = gpair;
  if ((rv = P->gptr.upload(cnt.data(), cnt.size())) != UFEM_AF_OK) return rv;
  if ((rv = P->gel.upload(gel.data(), gel.size())) != UFEM_AF_OK) return rv;
  if ((rv = P->gpair.upload(gpair.data(), gpair.size())) != UFEM_AF_OK) return rv;
  // inputs: MONTE_VTYPE_MAT (E, F_YC), MONTE_VTYPE_NLD and MONTE_VTYPE_MAX_D (fem/fem_mont.c:721-797)
  std::vector<int> mat_var(m->mpVals.size(), -1), fy_var(m->mpVals.size(), -1);
  std::vector<int> load_var(m->loads.size(), -1);
  int md_col = -1;
  for (long i = 0; i < m->mc_ilen; i++) {
    long ty = m->mc_type[i], item = m->mc_item[i], sub = m->mc_sub[i], it = m->mc_iter[i];
    int col = (int)m->mc_pos[i];
    if (col < 0 || col >= m->mc_ilen) {
      set_error("Monte Carlo input position out of range");
      return UFEM_AF_ERR_VAL;
    }
    if (ty == 1 && sub == 12 && it == 0 && item >= 0 && item < (long)m->mpVals.size()) {
      // MAT_F_YC: read by the failure function only; a record without it
      // ignores the input (femGetRepValIndex gives -1, fem/fem_mont.c:722-735)
      if (m->mpTypeH[item] == 5 && m->mpVals[item].size() > 4) fy_var[item] = col;
    } else if (ty == 1) {  // MONTE_VTYPE_MAT
      if (sub != 2 || item < 0 || item >= (long)m->mpVals.size()) {
        set_error("batched Monte Carlo randomises material E (MAT_EX) and F_YC only");
        return UFEM_AF_ERR_TYP;
      }
      mat_var[item] = col;
    } else if (ty == 7) {  // MONTE_VTYPE_MAX_D, fem/fem_mont.c:795-797
      md_col = col;
    } else if (ty == 3) {  // MONTE_VTYPE_NLD: first load with node/type/dir (fem/fem_mont.c:757-768)
      for (size_t j = 0; j < m->loads.size(); j++)
        if (m->loads[j].node == item && m->loads[j].type == sub && m->loads[j].dir == it) {
          if (m->loads[j].type != 3) {
            set_error("batched Monte Carlo randomises nodal forces (type 3) only");
            return UFEM_AF_ERR_TYP;
          }
          load_var[j] = col;
          break;
        }
    } else {
      set_error("input variable type not on the batched path (MAT E / F_YC, NLD forces and MAX_D only)");
      return UFEM_AF_ERR_TYP;
    }
  }
  std::vector<int> ev(m->eLen);
  for (long e = 0; e < m->eLen; e++) ev[e] = mat_var[m->eMat[e]];
  P->h_elem_var = ev;
  if ((rv = P->elem_var.upload(ev.data(), ev.size())) != UFEM_AF_OK) return rv;
  std::vector<double> F0(m->nDOFAct, 0.0);
  P->ovr_row.clear();
  P->ovr_var.clear();
  for (size_t j = 0; j < m->loads.size(); j++) {
    const auto &l = m->loads[j];
    if (l.type == 1 && l.val != 0.0) {
      set_error("batched Monte Carlo needs zero-valued supports");
      return UFEM_AF_ERR_TYP;
    }
    if (l.type != 3) continue;
    long p = m->dof(l.node * KNOWN_DOFS + l.dir - 1);
    if (p <= 0) continue;
    if (load_var[j] >= 0) {
      P->ovr_row.push_back((int)(p - 1));
      P->ovr_var.push_back(load_var[j]);
    } else {
      F0[p - 1] += l.val;
    }
  }
  if ((rv = P->F0.upload(F0.data(), F0.size())) != UFEM_AF_OK) return rv;
  if ((rv = P->d_ovr_row.upload(P->ovr_row.data(), P->ovr_row.size())) != UFEM_AF_OK) return rv;
  if ((rv = P->d_ovr_var.upload(P->ovr_var.data(), P->ovr_var.size())) != UFEM_AF_OK) return rv;
  {
    std::vector<int> ptr(m->nDOFAct + 1, 0), rvar(P->ovr_row.size()), fill;
    for (int r : P->ovr_row) ptr[r + 1]++;
    for (long i = 0; i < m->nDOFAct; i++) ptr[i + 1] += ptr[i];
    fill.assign(ptr.begin(), ptr.end() - 1);
    for (size_t j = 0; j < P->ovr_row.size(); j++) rvar[fill[P->ovr_row[j]]++] = P->ovr_var[j];
    if ((rv = P->d_ovr_ptr.upload(ptr.data(), ptr.size())) != UFEM_AF_OK) return rv;
    if ((rv = P->d_ovr_rvar.upload(rvar.data(), rvar.size())) != UFEM_AF_OK) return rv;
  }
  // outputs (fem/fem_mont.c:514-686)
  P->outs.clear();
  std::vector<int> ot, op, orow;
  for (long i = m->mc_ilen; i < m->mc_ilen + m->mc_olen; i++) {
    McOut o{(int)m->mc_type[i], (int)m->mc_pos[i - m->mc_ilen], -1, -1};
    if (o.pos < 0 || o.pos >= m->mc_olen) {
      set_error("Monte Carlo output position out of range");
      return UFEM_AF_ERR_VAL;
    }
    long item = m->mc_item[i], sub = m->mc_sub[i], it = m->mc_iter[i];
    if (o.type == 8 || o.type == 15 || o.type == 16) {
      // RES_D, RES_D_MAX, RES_D_MIN: u at node item, DOF sub (fem/fem_mont.c:524-548;
      // max/min against the zeroed output)
      if (item >= 0 && item < m->nLen && sub >= 1 && sub <= KNOWN_DOFS)
        o.row = (int)m->dof(item * KNOWN_DOFS + sub - 1) - 1;
    } else if (o.type == 17) {
      // RES_D_SUM adds nDOFfld[nDOFfld[pos]], the DOF number of another slot
      // (fem/fem_mont.c:550-555); kept as a constant in `row`
      o.row = 0;
      if (item >= 0 && item < m->nLen && sub >= 1 && sub <= KNOWN_DOFS) {
        const long p = m->dof(item * KNOWN_DOFS + sub - 1);
        if (p >= 0 && p < m->dof_slots()) o.row = (int)m->dof(p);
      }
    } else if (o.type == 9) {  // RES_R: reaction of node item, DOF sub
      for (size_t r = 0; r < m->reacNode.size(); r++)
        if (m->reacNode[r] == item && m->reacDof[r] == sub) {
          o.reac = (int)r;
          o.row = m->reacRow[r];
          break;
        }
    } else {
      // RES_E, the element sums/extremes and RES_FAIL come from the element
      // pass (mcout.cu), which writes after this one; RES_A_MAX is 0 outside
      // dynamics (fem/fem_mont.c:557-563)
      o.type = -1;
    }
    P->outs.push_back(o);
    ot.push_back(o.type); op.push_back(o.pos); orow.push_back(o.row);
  }
  if ((rv = P->d_out_type.upload(ot.data(), ot.size())) != UFEM_AF_OK) return rv;
  if ((rv = P->d_out_pos.upload(op.data(), op.size())) != UFEM_AF_OK) return rv;
  if ((rv = P->d_out_row.upload(orow.data(), orow.size())) != UFEM_AF_OK) return rv;
  if ((rv = build_elem_outputs(m, P->eo, &fy_var, md_col)) != UFEM_AF_OK) return rv;
  P->built = true;
  return UFEM_AF_OK;
}

// The implicit form of K_s = sum_e E_{s,e} K_e: for every block, the
// element contributions (element order) summed per multiplier.  Rows and
// columns of supported DOFs are zeroed; the PCG kernel gives those rows the
// identity (fem/fem_loads.c:158-166).
static int build_implicit(ufem_model *m, McPlan *P) {
  int rv;
  if ((rv = host_pattern(m)) != UFEM_AF_OK) return rv;
  const int B = m->b, nn = m->nn, se = P->s, BB = B * B;
  const int stride = (BB + 2) & ~1;  // values + index, a multiple of 16 bytes
  std::vector<double> Kh((size_t)m->eLen * se * se);
  UFEM_CUDA_TRY(cudaMemcpy(Kh.data(), P->Khat.p, Kh.size() * sizeof(double), cudaMemcpyDeviceToHost));
  std::vector<int> col2mult(std::max<long>(1, m->mc_ilen), -1), emult(m->eLen);
  P->mult_col.assign(1, -1);
  for (long e = 0; e < m->eLen; e++) {
    const int v = P->h_elem_var[e];
    if (v < 0) {
      emult[e] = 0;
      continue;
    }
    if (col2mult[v] < 0) {
      col2mult[v] = (int)P->mult_col.size();
      P->mult_col.push_back(v);
    }
    emult[e] = col2mult[v];
  }
  std::vector<int> blkrow(m->nnzb);
  for (int r = 0; r < m->nbr; r++)
    for (int k = m->rowptr[r]; k < m->rowptr[r + 1]; k++) blkrow[k] = r;
  std::vector<int> cptr(m->nnzb + 1, 0);
  std::vector<double> cval;
  cval.reserve((size_t)m->nnzb * stride * 2);
  std::vector<int> slot_mult;
  std::vector<double> W;
  for (long k = 0; k < m->nnzb; k++) {
    slot_mult.clear();
    W.clear();
    for (int c = P->h_gptr[k]; c < P->h_gptr[k + 1]; c++) {
      const int e = P->h_gel[c], p = P->h_gpair[c], la = p / nn, lb = p % nn, mi = emult[e];
      const double scale = (mi == 0) ? m->eE[e] : 1.0;
      size_t sl = 0;
      while (sl < slot_mult.size() && slot_mult[sl] != mi) sl++;
      if (sl == slot_mult.size()) {
        slot_mult.push_back(mi);
        W.resize(W.size() + BB, 0.0);
      }
      const double *kh = Kh.data() + (size_t)e * se * se + (size_t)(la * B) * se + lb * B;
      for (int i = 0; i < B; i++)
        for (int j = 0; j < B; j++) W[sl * BB + i * B + j] += scale * kh[i * se + j];
    }
    const int I = blkrow[k], J = m->colind[k];
    for (size_t sl = 0; sl < slot_mult.size(); sl++) {
      bool any = false;
      for (int i = 0; i < B; i++)
        for (int j = 0; j < B; j++) {
          double &w = W[sl * BB + i * B + j];
          if (m->fixedMask[I * B + i] || m->fixedMask[J * B + j]) w = 0.0;
          any = any || (w != 0.0);
        }
      if (!any) continue;
      for (int t = 0; t < BB; t++) cval.push_back(W[sl * BB + t]);
      // the multiplier and the block column in one exactly representable integer
      cval.push_back((double)(((long long)slot_mult[sl] << 32) | (long long)J));
      for (int t = BB + 1; t < stride; t++) cval.push_back(0.0);
      cptr[k + 1]++;
    }
  }
  for (long k = 0; k < m->nnzb; k++) cptr[k + 1] += cptr[k];
  std::vector<int> crow(m->nbr + 1);
  for (int r = 0; r <= m->nbr; r++) crow[r] = cptr[m->rowptr[r]];
  P->nmult = (int)P->mult_col.size();
  P->cstride = stride;
  P->nc = cptr[m->nnzb];
  if (cval.empty()) cval.assign(stride, 0.0);
  {
    std::vector<float> w32((size_t)std::max<long>(1, P->nc) * kW32Stride, 0.0f);
    for (long c = 0; c < P->nc; c++)
      for (int t = 0; t < BB; t++) w32[(size_t)c * kW32Stride + t] = (float)cval[(size_t)c * stride + t];
    if ((rv = P->w32.upload(w32.data(), w32.size()))) return rv;
  }
  if ((rv = P->cptr.upload(cptr.data(), cptr.size())) || (rv = P->cval.upload(cval.data(), cval.size())) ||
      (rv = P->crow.upload(crow.data(), crow.size())) ||
      (rv = P->d_mult_col.upload(P->mult_col.data(), P->mult_col.size())))
    return rv;
  P->imp_built = true;
  return UFEM_AF_OK;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
namespace {

constexpr int kThreads = 256;

template <typename T>
struct VecOf;
template <>
struct VecOf<float> {
  static constexpr int N = 4;
  using V = float4;
};
template <>
struct VecOf<double> {
  static constexpr int N = 2;
  using V = double2;
};

// Which samples a lane holds.  FP32 kernels: 4 adjacent samples (one 16-byte
// load).  FP64 kernels: pairs of adjacent samples, one pair in every 64-sample
// half of the group (lane l: 2l, 2l+1 [, 64 + 2l, 64 + 2l + 1]), so that every
// 16-byte-per-lane load reads 512 contiguous bytes -- with 4 adjacent doubles
// per lane, the two loads would each fetch half of every sector from L2.
template <typename T, int VN>
__device__ __forceinline__ int lane_base(int lane) {
  return sizeof(T) == 8 ? lane * 2 : lane * VN;
}
template <typename T, int VN>
__device__ __forceinline__ int lane_sample(int lane, int v) {
  return sizeof(T) == 8 ? (v >> 1) * 64 + lane * 2 + (v & 1) : lane * VN + v;
}
// VN doubles of this lane's samples (p = row + group start + lane_base):
// FP64 kernels read pairs 64 samples apart, FP32 kernels VN adjacent ones
template <typename T, int VN>
__device__ __forceinline__ void ld64(const double *p, double (&o)[VN]) {
#pragma unroll
  for (int h = 0; h < VN / 2; h++) {
    const double2 v = __ldcg(reinterpret_cast<const double2 *>(p + (sizeof(T) == 8 ? h * 64 : h * 2)));
    o[2 * h] = v.x;
    o[2 * h + 1] = v.y;
  }
}
// the same through the non-coherent path, for data no block writes during
// the kernel (the per-sample multipliers of the implicit form)
template <typename T, int VN>
__device__ __forceinline__ void ld64_ro(const double *p, double (&o)[VN]) {
#pragma unroll
  for (int h = 0; h < VN / 2; h++) {
    const double2 v = __ldg(reinterpret_cast<const double2 *>(p + (sizeof(T) == 8 ? h * 64 : h * 2)));
    o[2 * h] = v.x;
    o[2 * h + 1] = v.y;
  }
}
template <typename T, int VN>
__device__ __forceinline__ void ld64_stream(const double *p, double (&o)[VN]) {
#pragma unroll
  for (int h = 0; h < VN / 2; h++) {
    const double2 v = __ldcs(reinterpret_cast<const double2 *>(p + (sizeof(T) == 8 ? h * 64 : h * 2)));
    o[2 * h] = v.x;
    o[2 * h + 1] = v.y;
  }
}
template <typename T, int VN>
__device__ __forceinline__ void st64(double *p, const double (&o)[VN]) {
#pragma unroll
  for (int h = 0; h < VN / 2; h++)
    *reinterpret_cast<double2 *>(p + (sizeof(T) == 8 ? h * 64 : h * 2)) = make_double2(o[2 * h], o[2 * h + 1]);
}

// Neighbour gathers through L1: VN values in the lane layout of T, read with
// default caching.  Only for vectors that no block writes during the phase
// that gathers them (z in the q = A p phase, x in the true-residual phase):
// the grid barrier before the phase (an atomic arrival, a gpu-scope fence
// after the wait, then the block barrier -- the pattern of a cooperative grid
// sync) orders every earlier write before these loads, so no L1 line can be
// stale, and the rows that a block gathers from its neighbourhood are reused
// from L1 instead of being fetched from L2 once per neighbour.
template <typename T, int VN>
__device__ __forceinline__ void ld64_l1(const double *p, double (&o)[VN]) {
#pragma unroll
  for (int h = 0; h < VN / 2; h++) {
    const double2 v = *reinterpret_cast<const double2 *>(p + (sizeof(T) == 8 ? h * 64 : h * 2));
    o[2 * h] = v.x;
    o[2 * h + 1] = v.y;
  }
}
template <typename T, int VN>
__device__ __forceinline__ void ldn_l1(const T *p, T (&o)[VN]) {
  if constexpr (sizeof(T) == 8) {
    ld64_l1<T, VN>(p, o);
  } else {
#pragma unroll
    for (int h = 0; h < VN / 4; h++) {
      const float4 v = reinterpret_cast<const float4 *>(p)[h];
      o[4 * h] = v.x;
      o[4 * h + 1] = v.y;
      o[4 * h + 2] = v.z;
      o[4 * h + 3] = v.w;
    }
  }
}

// VN values of type T at a 16-byte aligned address (double: VN = 2 or 4,
// float: VN = 4), read through L2 (other blocks write them during the kernel)
template <typename T, int VN>
__device__ __forceinline__ void ldn(const T *p, T (&o)[VN]) {
  if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int h = 0; h < VN / 2; h++) {
      const double2 v = __ldcg(reinterpret_cast<const double2 *>(p + h * 64));
      o[2 * h] = v.x;
      o[2 * h + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int h = 0; h < VN / 4; h++) {
      const float4 v = __ldcg(reinterpret_cast<const float4 *>(p) + h);
      o[4 * h] = v.x;
      o[4 * h + 1] = v.y;
      o[4 * h + 2] = v.z;
      o[4 * h + 3] = v.w;
    }
  }
}
template <typename T, int VN>
__device__ __forceinline__ void stn(T *p, const T (&o)[VN]) {
  if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int h = 0; h < VN / 2; h++) *reinterpret_cast<double2 *>(p + h * 64) = make_double2(o[2 * h], o[2 * h + 1]);
  } else {
#pragma unroll
    for (int h = 0; h < VN / 4; h++)
      reinterpret_cast<float4 *>(p)[h] = make_float4(o[4 * h], o[4 * h + 1], o[4 * h + 2], o[4 * h + 3]);
  }
}
// streaming (evict-first) loads for data read once per iteration: the
// matrix values, so that L2 keeps the gathered vectors instead
template <typename T, int VN>
__device__ __forceinline__ void ldn_stream(const T *p, T (&o)[VN]) {
  if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int h = 0; h < VN / 2; h++) {
      const double2 v = __ldcs(reinterpret_cast<const double2 *>(p + h * 64));
      o[2 * h] = v.x;
      o[2 * h + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int h = 0; h < VN / 4; h++) {
      const float4 v = __ldcs(reinterpret_cast<const float4 *>(p) + h);
      o[4 * h] = v.x;
      o[4 * h + 1] = v.y;
      o[4 * h + 2] = v.z;
      o[4 * h + 3] = v.w;
    }
  }
}
// E of every element for every sample: E[e*S + s]
__global__ void k_make_E(int eLen, int S, int nsamp, long ilen, const double *__restrict__ ifld,
                         const int *__restrict__ elem_var, const double *__restrict__ eE, double *__restrict__ E) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)eLen * S) return;
  int e = (int)(t / S), s = (int)(t % S);
  int v = elem_var[e];
  E[t] = (v >= 0 && s < nsamp) ? ifld[(size_t)s * ilen + v] : eE[e];
}

// F for every sample (fem_add_loads order: fixed part, then the overridden
// lines in input order); F at fixed DOFs is kept in Fval and zeroed.
__global__ void k_make_F(int n, int S, int nsamp, long ilen, const double *__restrict__ ifld,
                         const double *__restrict__ F0, const int *__restrict__ ovr_ptr,
                         const int *__restrict__ ovr_var, double *__restrict__ F) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)n * S) return;
  int i = (int)(t / S), s = (int)(t % S);
  double f = (s < nsamp) ? F0[i] : 0.0;
  if (s < nsamp)
    for (int j = ovr_ptr[i]; j < ovr_ptr[i + 1]; j++) f += ifld[(size_t)s * ilen + ovr_var[j]];
  F[t] = f;
}

__global__ void k_fix_F(int n, int S, const unsigned char *__restrict__ fixed, double *__restrict__ F) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)n * S) return;
  if (fixed[t / S]) F[t] = 0.0;
}

// K_s = sum_e E_{s,e} K_e gathered per block; supports; FP64 and FP32 copies;
// Jacobi diagonal.  grid (nnzb, S/128), block 128 threads = 128 samples.
template <int B>
__global__ void __launch_bounds__(128) k_assemble_batch(int S, int s_el, const int *__restrict__ blkrow,
                                                        const int *__restrict__ colind,
                                                        const int *__restrict__ gptr, const int *__restrict__ gel,
                                                        const int *__restrict__ gpair,
                                                        const double *__restrict__ Khat,
                                                        const double *__restrict__ E,
                                                        const unsigned char *__restrict__ fixed,
                                                        double *__restrict__ V64, float *__restrict__ V32,
                                                        double *__restrict__ M64, float *__restrict__ M32) {
  const long k = blockIdx.x;
  const int s = blockIdx.y * 128 + threadIdx.x;
  const int I = blkrow[k], J = colind[k];
  const int c0 = gptr[k], c1 = gptr[k + 1];
  const int nn = s_el / B;
  double acc[B * B];
#pragma unroll
  for (int t = 0; t < B * B; t++) acc[t] = 0.0;
  for (int c = c0; c < c1; c++) {
    const int e = __ldg(gel + c), p = __ldg(gpair + c);
    const int a = p / nn, b = p % nn;
    const double Ee = E[(size_t)e * S + s];
    const double *kh = Khat + (size_t)e * s_el * s_el + (size_t)(a * B) * s_el + b * B;
#pragma unroll
    for (int i = 0; i < B; i++)
#pragma unroll
      for (int j = 0; j < B; j++) acc[i * B + j] += Ee * __ldg(kh + i * s_el + j);
  }
#pragma unroll
  for (int i = 0; i < B; i++)
#pragma unroll
    for (int j = 0; j < B; j++) {
      const int row = I * B + i, col = J * B + j;
      double v = acc[i * B + j];
      if (fixed[row] | fixed[col]) v = (row == col) ? 1.0 : 0.0;
      const size_t o = ((size_t)k * B * B + i * B + j) * S + s;
      V64[o] = v;
      if (V32) V32[o] = (float)v;
      if (row == col) {
        if (M64) M64[(size_t)row * S + s] = v;
        if (M32) M32[(size_t)row * S + s] = (float)v;
      }
    }
}

// per-sample multipliers of the implicit form: mult[j][s] = 1 (j = 0) or the
// sample's ifld value of column mult_col[j]
__global__ void k_make_mult(int nmult, int S, int nsamp, long ilen, const double *__restrict__ ifld,
                            const int *__restrict__ mult_col, double *__restrict__ mult) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)nmult * S) return;
  const int j = (int)(t / S), s = (int)(t % S);
  mult[t] = (j == 0 || s >= nsamp) ? 1.0 : ifld[(size_t)s * ilen + mult_col[j]];
}

// FP32 copy of the Jacobi diagonal (the FP32 implicit form)
__global__ void k_diag_f32(long n, const double *__restrict__ M, float *__restrict__ M32) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) M32[i] = (float)M[i];
}

// Jacobi diagonal of the implicit K_s (supported rows: 1)
template <int B>
__global__ void k_diag_implicit(int nbr, int S, const int *__restrict__ diagblk, const int *__restrict__ cptr,
                                const double *__restrict__ cval, int cstride, const double *__restrict__ mult,
                                const unsigned char *__restrict__ fixed, double *__restrict__ M) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)nbr * S) return;
  const int I = (int)(t / S), s = (int)(t % S);
  const int k = diagblk[I];
#pragma unroll
  for (int a = 0; a < B; a++) {
    double d = 0.0;
    for (int c = cptr[k]; c < cptr[k + 1]; c++) {
      const double *w = cval + (size_t)c * cstride;
      d += mult[(size_t)((long long)w[B * B] >> 32) * S + s] * w[a * B + a];
    }
    const int row = I * B + a;
    M[(size_t)row * S + s] = fixed[row] ? 1.0 : d;
  }
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// the persistent masked PCG over all meshes, with residual replacement
// ---------------------------------------------------------------------------
// ST_CAND: the recursive residual is below tol; the sample is frozen until
// the group's next true-residual pass decides (converged, or resumed)
// ST_NAN: a non-finite residual or p.q (NaN or infinite inputs); the sample is frozen
enum { ST_ACTIVE = 0, ST_CONV = 1, ST_MAXIT = 2, ST_BREAK = 3, ST_SKIP = 4, ST_CAND = 5, ST_NAN = 6 };

template <typename T>
struct BMesh {
  int nbr, S, ngroups, ntpg, rows_per_tile, B;
  const int *rowptr, *colind;
  const T *V;           // inner-precision values [nnzb*B*B][S]
  const double *V64;    // FP64 values, for the true residual
  const T *M;           // diagonal [n][S]
  const double *F;      // right-hand side (supports applied) [n][S]
  double *x;            // solution, FP64 [n][S] (in: initial guess)
  T *r, *z, *p0, *p1, *q;
  double *part_pq;      // [ngroups*ntpg*GS] (dot products accumulate in FP64)
  double *part_rr, *part_rz;  // [2][ngroups*ntpg*GS] by iteration parity
  double *tot_pq;       // [S] group totals of the partials, written by the
  double *tot_rr, *tot_rz;  // [2][S] last tile of the group to finish
  int *gcnt;            // [ngroups][2] tiles finished (p.q; r.r and r.z)
  double *rho;          // [2][S]
  double *rrlast;       // [S] true |r|^2 at the last replacement
  const double *tol2;   // [S] (tol |F_s|)^2
  int *state, *iters;   // [S]
  int *gactive;         // [ngroups]
  int *gtrue;           // [ngroups] the group's latest rr partials are true residuals
  int *gneed;           // [ngroups] a replacement is due after this iteration
  int *glast;           // [ngroups] iteration of the last replacement
  // implicit form (precision 2): block k = sum over c in [cptr[k], cptr[k+1])
  // of mult[idx_c][s] * W_c, W_c and idx_c in cval[c*cstride ...]
  const int *cptr;
  const int *crow;      // contributions of block row I: [crow[I], crow[I+1])
  const int *sperm;     // block rows in the visiting order of the gathering phases
  const double *cval;
  const double *mult;
  const float *w32;     // FP32 copies of the unit blocks (precision 4)
  const unsigned char *fixed;
  int cstride;
  int nmult;            // multipliers (rows of mult)
  int smult;            // the tile's multipliers are staged in shared memory
  // coarse correction of the preconditioner (precision 2, 128-sample groups):
  // z = r / M + Wc c with c = Wc^T r, both products on the tensor cores
  int n;                // scalar rows (nbr * B)
  int cmodes;           // modes of Wc (0: Jacobi alone), a multiple of 16, at most 128
  int nsplit, rps;      // c = Wc^T r runs as nsplit row ranges of rps rows (a multiple of 64) per group
  const uint8_t *wt1;   // Wc^T, BF16 operand tiles of 64 rows: [ceil(n/64)][cmodes x 64]
  const uint8_t *wt3;   // Wc, BF16 operand tiles of 128 rows: [ceil(n/128)][128 x cmodes]
  uint8_t *cb;          // c of each group, BF16 operand tile: [ngroups][128 x cmodes]
  float *cpart;         // partial c of each row range: [ngroups][nsplit][cmodes][128]
  int *ccnt;            // [ngroups] row ranges finished
  int *gcz;             // [ngroups] z = r / M was written this iteration: add Wc c
};

template <typename T>
struct BArgs {
  const BMesh<T> *meshes;
  int nmesh;                // at most kMaxMeshes
  const int4 *tiles;  // (mesh, group, chunk, -)
  int ntiles;
  GridBar *bar;
  int *active_count;  // groups still iterating (changes only in phase S)
  int *rcount;        // groups due for replacement (changes only in phase U)
  long maxit;
  long rr_every;      // at most this many iterations between replacements
  double near2;       // recursive |r|^2 <= near2 * (true |r|^2 at the last replacement) asks for one
  long *iter_out;
  int coarse;          // some mesh has a coarse space (the launch holds TMEM and shared memory for it)
  const int4 *c1items;  // (mesh, group, row range) of c = Wc^T r
  int nc1;
  const int4 *c3items;  // (mesh, group, 128-row chunk) of z += Wc c
  int nc3;
  // phase profile (global timer, nanoseconds): [p] the blocks' summed time
  // inside phase p's work items, [kProfWall + p] block 0's time from the
  // start of phase p to the start of the next phase (its barrier wait
  // included), [2 kProfWall] true-residual passes run.  Phases: kPh*.
  unsigned long long *prof;
  int *wctr;            // [kPhN] next work item of each phase (zero before its first use)
  // Split iterations (the coarse-corrected FP32 kernels): kstep >= 0 runs
  // one iteration's phases U, R, C1, C3 (kstep = 0: the initial residual
  // and coarse correction), phase S runs in k_batch_s; -1: every iteration
  // in this launch.
  long kstep;
  int *done;            // split: set when the iterations end (later launches return at once)
};

enum { kPhInit = 0, kPhS = 1, kPhU = 2, kPhR = 3, kPhC1 = 4, kPhC3 = 5, kPhN = 6 };
constexpr int kRepAlign = 4;  // FP32: iterations on which drop-triggered replacements run
constexpr int kProfWall = 8;

// Per-block phase clocks, kept by thread 0 in shared memory.
__shared__ unsigned long long s_prof_busy[kPhN], s_prof_wall[kPhN], s_prof_t0, s_prof_w0;
__shared__ int s_prof_cur;

__device__ __forceinline__ void prof_init() {
  if (threadIdx.x == 0) {
    for (int p = 0; p < kPhN; p++) s_prof_busy[p] = s_prof_wall[p] = 0;
    s_prof_w0 = s_prof_t0 = global_ns();
    s_prof_cur = kPhInit;
  }
}
// a phase's work starts (after the barrier that ended the previous phase)
__device__ __forceinline__ void prof_begin(int ph) {
  if (threadIdx.x == 0) {
    const unsigned long long t = global_ns();
    s_prof_wall[s_prof_cur] += t - s_prof_w0;
    s_prof_w0 = s_prof_t0 = t;
    s_prof_cur = ph;
  }
}
// the block's work items of the current phase are done (before its barrier)
__device__ __forceinline__ void prof_end() {
  if (threadIdx.x == 0) s_prof_busy[s_prof_cur] += global_ns() - s_prof_t0;
}
// The next work item of the current phase for this block.  Items are handed
// out in order by one global counter per phase, so a block that finishes its
// items early takes more (the per-item results do not depend on which block
// computes them).  Block 0 zeroes a phase's counter after the grid barrier
// that ends the phase: every block has left the phase's loop by then, and the
// next use comes after further barriers.
__device__ __forceinline__ int claim(int *ctr) {
  __shared__ int s_claim;
  __syncthreads();  // every thread has read the previous claim
  if (threadIdx.x == 0) s_claim = atomicAdd(ctr, 1);
  __syncthreads();
  return s_claim;
}
__device__ __forceinline__ void release_counter(int *ctr) {
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(ctr, 0);
}

__device__ __forceinline__ void prof_flush(unsigned long long *prof) {
  if (threadIdx.x == 0 && prof) {
    const unsigned long long t = global_ns();
    s_prof_wall[s_prof_cur] += t - s_prof_w0;
    for (int p = 0; p < kPhN; p++) {
      atomicAdd(prof + p, s_prof_busy[p]);
      if (blockIdx.x == 0) prof[kProfWall + p] += s_prof_wall[p];
    }
  }
}

// Dynamic shared memory of the persistent PCG: the operand staging of the
// coarse phases, and during the other phases the multipliers of the tile's
// sample group (implicit form), never both at once.
extern __shared__ __align__(1024) uint8_t s_dyn_smem[];

// acc[a][v] += mult[var_c][s] * (W_c X_{J_c})[a] over the contributions
// [c0, c1) of one block row of the implicit form.  The row's contribution
// keys (multiplier << 32 | J) are fetched 32 at a time, one per lane, and
// broadcast; the gathers of U contributions are issued together so that U
// neighbour loads are in flight per warp.  W and the multipliers are
// read-only for the whole kernel (non-coherent loads); X is written by other
// blocks during the kernel (loads after the phase's grid barrier).  LT is the
// kernel's lane layout (double: sample pairs 64 apart; float: 4 adjacent
// samples), XT the type of X (the FP32 kernels gather FP32 z, and FP64 x for
// their true residuals), CT the type of the products and sums: FP64 (W and
// the multipliers in FP64) or FP32 (W from the FP32 copies, the multipliers
// rounded: precision 4).  SMULT: the multipliers come from the tile's
// shared-memory copy ([nmult][GS] of CT) instead of global memory.
template <typename LT, typename XT, typename CT, int B, int VN, int U, bool SMULT>
__device__ __forceinline__ void implicit_row(const double *__restrict__ cval, int cstride,
                                             const float *__restrict__ w32, const double *__restrict__ mult,
                                             const CT *s_mult, const XT *X, int S, int sb, int c0, int c1,
                                             CT (&acc)[B][VN]) {
  static_assert(sizeof(XT) == 8 || sizeof(LT) == 4, "FP32 vectors only in the FP32 lane layout");
  constexpr int GS = 32 * VN;
  const int lane = threadIdx.x & 31;
  for (int cb = c0; cb < c1; cb += 32) {
    const long long mykey = (cb + lane < c1) ? (long long)__ldg(cval + (size_t)(cb + lane) * cstride + B * B) : 0;
    const int cnt = min(32, c1 - cb);
    for (int j = 0; j < cnt; j += U) {
      XT xv[U][B][VN];
      double av[SMULT ? 1 : U][VN];
      int vars[SMULT ? U : 1];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const long long key = __shfl_sync(0xffffffffu, mykey, min(j + u, cnt - 1));
        const int J = (int)(key & 0xffffffffLL);
#pragma unroll
        for (int b = 0; b < B; b++) {
          if constexpr (sizeof(XT) == 8) ld64_l1<LT, VN>(X + (size_t)(J * B + b) * S + sb, xv[u][b]);
          else ldn_l1<XT, VN>(X + (size_t)(J * B + b) * S + sb, xv[u][b]);
        }
        if constexpr (SMULT) vars[u] = (int)(key >> 32);
        else ld64_ro<LT, VN>(mult + (size_t)(int)(key >> 32) * S + sb, av[u]);
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (j + u >= cnt) break;
        CT W[B * B];
        if constexpr (sizeof(CT) == 8) {
          const double *w = cval + (size_t)(cb + j + u) * cstride;
#pragma unroll
          for (int h = 0; h < (B * B) / 2; h++) {
            const double2 v = __ldg(reinterpret_cast<const double2 *>(w) + h);
            W[2 * h] = v.x;
            W[2 * h + 1] = v.y;
          }
          if ((B * B) & 1) W[B * B - 1] = __ldg(w + B * B - 1);
        } else {
          const float4 *w = reinterpret_cast<const float4 *>(w32 + (size_t)(cb + j + u) * kW32Stride);
#pragma unroll
          for (int h = 0; h < (B * B + 3) / 4; h++) {
            const float4 v = __ldg(w + h);
            const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int q = 0; q < 4; q++)
              if (4 * h + q < B * B) W[4 * h + q] = e[q];
          }
        }
        CT a[VN];
        if constexpr (SMULT) {
          const CT *sm = s_mult + vars[u] * GS;
#pragma unroll
          for (int v = 0; v < VN; v++) a[v] = sm[lane_sample<LT, VN>(lane, v)];
        } else {
#pragma unroll
          for (int v = 0; v < VN; v++) a[v] = (CT)av[u][v];
        }
#pragma unroll
        for (int r = 0; r < B; r++)
#pragma unroll
          for (int v = 0; v < VN; v++) {
            CT t = 0;
#pragma unroll
            for (int b = 0; b < B; b++) t = fma(W[r * B + b], (CT)xv[u][b][v], t);
            acc[r][v] = fma(a[v], t, acc[r][v]);
          }
      }
    }
  }
}

// The multipliers of group g, mult[v][g GS + i], into shared memory as CT
// (by every thread of the block; the caller synchronises before use).
template <typename CT, int GS>
__device__ __forceinline__ void stage_mult(const double *__restrict__ mult, int nmult, int S, int g, CT *s_mult) {
  for (int i = threadIdx.x; i < nmult * GS; i += blockDim.x)
    s_mult[i] = (CT)__ldg(mult + (size_t)(i / GS) * S + (size_t)g * GS + (i % GS));
}

// Called by every tile of group g after it wrote its partials: the last
// tile of the group to arrive adds the group's partials in tile order (the
// same order every run) into the per-sample totals, so no other tile has to.
template <int GS>
__device__ __forceinline__ void group_close(int *cnt, int ntpg, int g, const double *part, double *tot,
                                            const double *part2, double *tot2) {
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(cnt, 1) == ntpg - 1);
  __syncthreads();
  if (s_last) {
    __threadfence();
    if (threadIdx.x < GS) {
      double t = 0.0, t2 = 0.0;
      for (int c = 0; c < ntpg; c++) {
        const size_t o = ((size_t)g * ntpg + c) * GS + threadIdx.x;
        t += __ldcg(part + o);
        if (part2) t2 += __ldcg(part2 + o);
      }
      tot[(size_t)g * GS + threadIdx.x] = t;
      if (tot2) tot2[(size_t)g * GS + threadIdx.x] = t2;
    }
    if (threadIdx.x == 0) atomicExch(cnt, 0);  // next used after a grid barrier
  }
  __syncthreads();
}

// q = A p with p = z + beta p_old on the block rows of one tile for GS
// samples; pnew = p on the own rows; partial p.q per sample.  Explicit form:
// p is formed at every gathered neighbour.  Implicit form: q = A z + beta
// q_old (A p_old is the previous q), so only z is gathered.
template <typename T, int B, bool IMP, int UN, int VN, int NW, bool F32P = false>
__device__ __forceinline__ void tile_spmv(const BMesh<T> &M, int g, int chunk, const T *s_beta, bool first,
                                          const T *pold, T *pnew, double (*s_red)[32 * VN]) {
  // The implicit form forms every product and sum in FP64 (its unit blocks
  // and multipliers are FP64) whatever the vector precision T, except in
  // precision 4 (F32P: FP32 unit blocks, multipliers and sums, the inner FP32
  // matrix).  FP32 products lose the cancellation of K z for smooth z: from
  // zero on the 16-zone beam 565 instead of 289 Jacobi iterations, and no
  // convergence with the coarse correction; warm-started with the coarse
  // correction they keep the iteration count and are faster.
  using AT = typename std::conditional<IMP, typename std::conditional<F32P, float, double>::type, T>::type;
  constexpr int GS = 32 * VN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = M.S;
  const int sb = g * GS + lane_base<T, VN>(lane);
  const int row0 = chunk * M.rows_per_tile, row1 = min(M.nbr, row0 + M.rows_per_tile);
  T beta[VN];
#pragma unroll
  for (int v = 0; v < VN; v++) beta[v] = s_beta[lane_sample<T, VN>(lane, v)];
  AT *s_mult = nullptr;
  if constexpr (IMP) {
    if (M.smult) {
      s_mult = reinterpret_cast<AT *>(s_dyn_smem);
      stage_mult<AT, GS>(M.mult, M.nmult, S, g, s_mult);
      __syncthreads();
    }
  }
  double pq[VN];
#pragma unroll
  for (int v = 0; v < VN; v++) pq[v] = 0;
  for (int ri = row0 + warp; ri < row1; ri += NW) {
    const int I = __ldg(M.sperm + ri);  // rows in the gathering order (neighbours in space together)
    AT acc[B][VN];
#pragma unroll
    for (int a = 0; a < B; a++)
#pragma unroll
      for (int v = 0; v < VN; v++) acc[a][v] = 0;
    if constexpr (IMP) {
      if (s_mult)
        implicit_row<T, T, AT, B, VN, UN, true>(M.cval, M.cstride, M.w32, M.mult, s_mult, M.z, S, sb, __ldg(M.crow + I),
                                            __ldg(M.crow + I + 1), acc);
      else
        implicit_row<T, T, AT, B, VN, UN, false>(M.cval, M.cstride, M.w32, M.mult, nullptr, M.z, S, sb, __ldg(M.crow + I),
                                             __ldg(M.crow + I + 1), acc);
    } else {
      const int k0 = __ldg(M.rowptr + I), k1 = __ldg(M.rowptr + I + 1);
      for (int kb = k0; kb < k1; kb += 32) {
        // the row's column indices, one per lane, then broadcast by shuffle:
        // the neighbour gathers no longer wait on a dependent index load
        const int myJ = (kb + lane < k1) ? __ldg(M.colind + kb + lane) : 0;
        const int cnt = min(32, k1 - kb);
        for (int j = 0; j < cnt; j++) {
          const int k = kb + j;
          T vv[B * B][VN];
#pragma unroll
          for (int e = 0; e < B * B; e++) ldn_stream<T, VN>(M.V + ((size_t)k * B * B + e) * S + sb, vv[e]);
          const int J = __shfl_sync(0xffffffffu, myJ, j);
          T xv[B][VN];
#pragma unroll
          for (int c = 0; c < B; c++) {
            ldn_l1<T, VN>(M.z + (size_t)(J * B + c) * S + sb, xv[c]);
            if (!first) {
              T pv[VN];
              ldn_l1<T, VN>(pold + (size_t)(J * B + c) * S + sb, pv);
#pragma unroll
              for (int v = 0; v < VN; v++) xv[c][v] = xv[c][v] + beta[v] * pv[v];
            }
          }
#pragma unroll
          for (int a = 0; a < B; a++)
#pragma unroll
            for (int c = 0; c < B; c++)
#pragma unroll
              for (int v = 0; v < VN; v++) acc[a][v] += vv[a * B + c][v] * xv[c][v];
        }
      }
    }
#pragma unroll
    for (int a = 0; a < B; a++) {
      const size_t o = (size_t)(I * B + a) * S + sb;
      T zi[VN], pi[VN];
      ldn<T, VN>(M.z + o, zi);
      if (!first) {
        T po[VN];
        ldn<T, VN>(pold + o, po);
#pragma unroll
        for (int v = 0; v < VN; v++) pi[v] = zi[v] + beta[v] * po[v];
      } else {
#pragma unroll
        for (int v = 0; v < VN; v++) pi[v] = zi[v];
      }
      if constexpr (IMP) {
        if (!first) {
          T qo[VN];
          ldn<T, VN>(M.q + o, qo);
#pragma unroll
          for (int v = 0; v < VN; v++) acc[a][v] = fma((AT)beta[v], (AT)qo[v], acc[a][v]);
        }
        if (M.fixed[I * B + a]) {  // supported DOF: identity row
#pragma unroll
          for (int v = 0; v < VN; v++) acc[a][v] = pi[v];
        }
      }
      T qv[VN];
#pragma unroll
      for (int v = 0; v < VN; v++) qv[v] = (T)acc[a][v];
      stn<T, VN>(pnew + o, pi);
      stn<T, VN>(M.q + o, qv);
#pragma unroll
      for (int v = 0; v < VN; v++) pq[v] += (double)pi[v] * (double)qv[v];
    }
  }
#pragma unroll
  for (int v = 0; v < VN; v++) s_red[warp][lane_sample<T, VN>(lane, v)] = pq[v];
  __syncthreads();
  if (threadIdx.x < GS) {
    double t = 0;
    for (int w = 0; w < NW; w++) t += s_red[w][threadIdx.x];
    M.part_pq[((size_t)g * M.ntpg + chunk) * GS + threadIdx.x] = t;
  }
  group_close<GS>(M.gcnt + 2 * g, M.ntpg, g, M.part_pq, M.tot_pq, nullptr, nullptr);
}

// Writes the tile's r.r and r.z partials of parity slot `par`.
template <typename T, int VN, int NW>
__device__ __forceinline__ void tile_partials(const BMesh<T> &M, int g, int chunk, int par, const double (&rr)[VN],
                                              const double (&rz)[VN], double (*s_red)[32 * VN],
                                              double (*s_red2)[32 * VN]) {
  constexpr int GS = 32 * VN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int v = 0; v < VN; v++) {
    s_red[warp][lane_sample<T, VN>(lane, v)] = rr[v];
    s_red2[warp][lane_sample<T, VN>(lane, v)] = rz[v];
  }
  __syncthreads();
  if (threadIdx.x < GS) {
    double a = 0, b = 0;
    for (int w = 0; w < NW; w++) {
      a += s_red[w][threadIdx.x];
      b += s_red2[w][threadIdx.x];
    }
    const size_t slot = (size_t)par * M.ngroups * M.ntpg * GS + ((size_t)g * M.ntpg + chunk) * GS + threadIdx.x;
    M.part_rr[slot] = a;
    M.part_rz[slot] = b;
  }
  const size_t half = (size_t)M.ngroups * M.ntpg * GS;
  group_close<GS>(M.gcnt + 2 * g + 1, M.ntpg, g, M.part_rr + par * half, M.tot_rr + (size_t)par * M.S,
                  M.part_rz + par * half, M.tot_rz + (size_t)par * M.S);
}

// x += alpha p (FP64), r -= alpha q, z = r / M; partial r.r and r.z (the
// Jacobi part r.(r / M) when the mesh has a coarse space).
template <typename T, int B, int VN, int NW>
__device__ __forceinline__ void tile_update(const BMesh<T> &M, int g, int chunk, const T *s_alpha, const T *pnew,
                                            int par, double (*s_red)[32 * VN], double (*s_red2)[32 * VN]) {
  constexpr int GS = 32 * VN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = M.S;
  const int sb = g * GS + lane_base<T, VN>(lane);
  const int row0 = chunk * M.rows_per_tile, row1 = min(M.nbr, row0 + M.rows_per_tile);
  T alpha[VN];
#pragma unroll
  for (int v = 0; v < VN; v++) alpha[v] = s_alpha[lane_sample<T, VN>(lane, v)];
  double rr[VN], rz[VN];
#pragma unroll
  for (int v = 0; v < VN; v++) rr[v] = rz[v] = 0;
  // the vectors do not overlap: the loads of a row's next DOFs may be issued
  // ahead of the stores of its first (more loads in flight per warp)
  const T *__restrict__ Md = M.M;
  const T *__restrict__ pd = pnew;
  const T *__restrict__ qd = M.q;
  T *__restrict__ rd = M.r;
  T *__restrict__ zd = M.z;
  double *__restrict__ xd = M.x;
  for (int I = row0 + warp; I < row1; I += NW) {
#pragma unroll
    for (int a = 0; a < B; a++) {
      const size_t o = (size_t)(I * B + a) * S + sb;
      T ri[VN], mi[VN], pi[VN], qi[VN], zi[VN];
      double xi[VN];
      ldn<T, VN>(Md + o, mi);
      ldn<T, VN>(rd + o, ri);
      ldn<T, VN>(pd + o, pi);
      ldn<T, VN>(qd + o, qi);
      ld64<T, VN>(xd + o, xi);
#pragma unroll
      for (int v = 0; v < VN; v++) {
        xi[v] += (double)alpha[v] * (double)pi[v];
        ri[v] = ri[v] - alpha[v] * qi[v];
        zi[v] = ri[v] / mi[v];
        rr[v] += (double)ri[v] * (double)ri[v];
        rz[v] += (double)ri[v] * (double)zi[v];
      }
      st64<T, VN>(xd + o, xi);
      stn<T, VN>(rd + o, ri);
      stn<T, VN>(zd + o, zi);  // with a coarse space the C3 phase adds Wc c
    }
  }
  tile_partials<T, VN, NW>(M, g, chunk, par, rr, rz, s_red, s_red2);
}

// Residual replacement: r = F - K x in FP64 from the FP64 values, then
// r (inner precision), z = r / M and the partials of the true residual.
template <typename T, int B, bool IMP, int UN, int VN, int NW>
__device__ __forceinline__ void tile_true_residual(const BMesh<T> &M, int g, int chunk, int par,
                                                   double (*s_red)[32 * VN], double (*s_red2)[32 * VN]) {
  constexpr int GS = 32 * VN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = M.S;
  const int sb = g * GS + lane_base<T, VN>(lane);
  const int row0 = chunk * M.rows_per_tile, row1 = min(M.nbr, row0 + M.rows_per_tile);
  double rr[VN], rz[VN];
#pragma unroll
  for (int v = 0; v < VN; v++) rr[v] = rz[v] = 0;
  // the FP64 multipliers of the tile's group in shared memory
  const double *s_mult = nullptr;
  if constexpr (IMP) {
    if (M.smult) {
      double *sm = reinterpret_cast<double *>(s_dyn_smem);
      stage_mult<double, GS>(M.mult, M.nmult, S, g, sm);
      __syncthreads();
      s_mult = sm;
    }
  }
  for (int ri = row0 + warp; ri < row1; ri += NW) {
    const int I = __ldg(M.sperm + ri);  // rows in the gathering order (neighbours in space together)
    double acc[B][VN];
#pragma unroll
    for (int a = 0; a < B; a++)
#pragma unroll
      for (int v = 0; v < VN; v++) acc[a][v] = 0.0;
    if constexpr (IMP) {
      if (s_mult)
        implicit_row<T, double, double, B, VN, UN, true>(M.cval, M.cstride, M.w32, M.mult, s_mult, M.x, S, sb, __ldg(M.crow + I),
                                                 __ldg(M.crow + I + 1), acc);
      else
        implicit_row<T, double, double, B, VN, UN, false>(M.cval, M.cstride, M.w32, M.mult, nullptr, M.x, S, sb, __ldg(M.crow + I),
                                                  __ldg(M.crow + I + 1), acc);
    } else {
      const int k0 = __ldg(M.rowptr + I), k1 = __ldg(M.rowptr + I + 1);
      for (int kb = k0; kb < k1; kb += 32) {
        const int myJ = (kb + lane < k1) ? __ldg(M.colind + kb + lane) : 0;
        const int cnt = min(32, k1 - kb);
        for (int j = 0; j < cnt; j++) {
          const int k = kb + j;
          const int J = __shfl_sync(0xffffffffu, myJ, j);
          double xv[B][VN];
#pragma unroll
          for (int c = 0; c < B; c++) ld64_l1<T, VN>(M.x + (size_t)(J * B + c) * S + sb, xv[c]);
#pragma unroll
          for (int a = 0; a < B; a++)
#pragma unroll
            for (int c = 0; c < B; c++) {
              double vv[VN];
              ld64_stream<T, VN>(M.V64 + ((size_t)k * B * B + a * B + c) * S + sb, vv);
#pragma unroll
              for (int v = 0; v < VN; v++) acc[a][v] += vv[v] * xv[c][v];
            }
        }
      }
    }
#pragma unroll
    for (int a = 0; a < B; a++) {
      const size_t o = (size_t)(I * B + a) * S + sb;
      double f[VN];
      T ri[VN], mi[VN], zi[VN];
      ld64<T, VN>(M.F + o, f);
      ldn<T, VN>(M.M + o, mi);
      if constexpr (IMP) {
        if (M.fixed[I * B + a]) {  // supported DOF: identity row
          double xo[VN];
          ld64<T, VN>(M.x + o, xo);
#pragma unroll
          for (int v = 0; v < VN; v++) acc[a][v] = xo[v];
        }
      }
#pragma unroll
      for (int v = 0; v < VN; v++) {
        const double r64 = f[v] - acc[a][v];
        ri[v] = (T)r64;
        zi[v] = ri[v] / mi[v];
        rr[v] += r64 * r64;
        rz[v] += (double)ri[v] * (double)zi[v];
      }
      stn<T, VN>(M.r + o, ri);
      stn<T, VN>(M.z + o, zi);
    }
  }
  tile_partials<T, VN, NW>(M, g, chunk, par, rr, rz, s_red, s_red2);
}

// ---------------------------------------------------------------------------
// coarse correction of the preconditioner: M^-1 = D^-1 + Wc Wc^T
// ---------------------------------------------------------------------------
// Wc = Phi L^-T spans a coarse space (the POD basis of earlier solutions) and
// is scaled by the Cholesky factor L of a mean reduced operator Phi^T K Phi,
// so Wc Wc^T = Phi (Phi^T K Phi)^-1 Phi^T: the additive two-level
// preconditioner (the AD variant of Tang, Nabben, Vuik & Erlangga 2009).
// It removes the smooth modes that Jacobi PCG resolves last; symmetric
// positive definite, so plain PCG applies.  Both products run per group of
// 128 samples on the tensor cores (BF16 operands, FP32 accumulation): the
// preconditioner need not be exact, and the residual, x and every dot
// product stay FP64.  Per iteration:
//   C1  c = Wc^T r   D[128 samples x cmodes] = R^T . Wc over row ranges; the
//                    group's last range adds the partials in range order,
//                    writes c (BF16 operand tile) and adds c.c to r.z
//                    (r.z = r.(r / M) + |Wc^T r|^2 without reading z)
//   C3  z += Wc c    D[128 samples x 128 rows] = c^T . Wc^T per chunk, added
//                    to z = r / M as the U phase (or a true-residual pass)
//                    wrote it.  Only a group with no iterating sample left can
//                    see some of its tiles skip U; its z is not used again
//                    before a true-residual pass rewrites every row.
// TMEM lane = sample of the group, so every epilogue access of a warp covers
// 32 consecutive samples of one row (256 contiguous bytes).
constexpr int kCoarseMaxModes = 128;
constexpr int kCoarseThreads = 512;                 // threads per block of the coarse instance (1 block per SM)
constexpr int kCoarseCols = 128;                    // TMEM columns per block
constexpr int kCoarseStage = 32 * 1024;             // C1: A (128 x 64) + B (<= 128 x 64), BF16
constexpr size_t kCoarseSmem = 2 * kCoarseStage;    // C1 double-buffered; C3 A + B (2 x 128 x 128 BF16)
constexpr long kMmaSpinLimit = 1L << 24;
constexpr int kErrMma = 2;                          // GridBar::err: a tensor-core wait ran out

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}

// Per-block state of the coarse phases, in shared memory so that none of it
// stays live in registers through the PCG phases: the TMEM accumulator, the
// MMA completion barrier, the operand staging area (dynamic shared memory).
__shared__ uint32_t s_coarse_tmem;
__shared__ uint32_t s_coarse_phase;  // parity of the MMA barrier's next completion
__shared__ __align__(8) uint64_t s_coarse_mbar;
__shared__ uint32_t s_tile_phase;   // parity of the operand-tile barrier's next completion
__shared__ __align__(8) uint64_t s_tile_mbar;

// Bulk (non-tensor) copies global -> shared memory that complete on an
// mbarrier: one thread announces the bytes, then issues the copies.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   tc::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
               : "memory");
}

// Leaves the kernel at the next grid barrier: every block sees the error.
__device__ __forceinline__ void coarse_fail(GridBar *bar) { atomicExch(&bar->err, kErrMma); }

// c = Wc^T r over row range `range` of group g (GS = 128 samples), by the
// kCoarseThreads threads of the block.
template <typename T>
__device__ __noinline__ void coarse_c1(const BMesh<T> &M, int g, int range, int par, uint32_t &phase,
                                       GridBar *gb) {
  constexpr int kQ = kCoarseThreads / 128;  // threads per sample
  static_assert(8 % kQ == 0, "the 8 row groups of a chunk split evenly over the threads of a sample");
  __shared__ int s_last;
  __shared__ double s_cc[kCoarseThreads];
  const uint32_t tmem = s_coarse_tmem;
  uint64_t *bar = &s_coarse_mbar;
  uint8_t *sm = s_dyn_smem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nmod = M.cmodes, S = M.S;
  const int r0 = range * M.rps, r1 = min(M.n, r0 + M.rps);
  const int nch = (r1 - r0 + 63) / 64;
  const uint32_t idesc = tc::idesc_bf16(128, nmod);
  const int stage_b = nmod * 64 * 2;
  const int m = tid & 127, q = tid >> 7;  // sample of the group staged by this thread, and its share
  const T *rcol = M.r + (size_t)g * 128 + m;
  // this thread stages row groups kg = q + kQ j (8 rows each) of sample m
  auto load_chunk = [&](int ch, T (&v)[8 / kQ][8]) {
    const int rb = r0 + ch * 64;
#pragma unroll
    for (int j = 0; j < 8 / kQ; j++)
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int row = rb + (q + kQ * j) * 8 + e;
        v[j][e] = row < r1 ? __ldcg(rcol + (size_t)row * S) : T(0);
      }
  };
  // this thread's 16-byte pieces of a chunk's Wc^T tile (at most 2: the
  // tile is cmodes x 64 BF16 <= 16 KB)
  constexpr int kBp = (kCoarseMaxModes * 64 * 2 / 16 + kCoarseThreads - 1) / kCoarseThreads;
  auto load_tile = [&](int ch, uint4 (&b)[kBp]) {
    const uint4 *src = reinterpret_cast<const uint4 *>(M.wt1 + (size_t)(r0 / 64 + ch) * stage_b);
#pragma unroll
    for (int j = 0; j < kBp; j++) {
      const int i = tid + j * kCoarseThreads;
      if (i < stage_b / 16) b[j] = __ldg(src + i);
    }
  };
  T cur[8 / kQ][8], nxt[8 / kQ][8];
  uint4 bcur[kBp], bnxt[kBp];
  load_chunk(0, cur);
  load_tile(0, bcur);
  bool ok = true;
  for (int ch = 0; ch < nch; ch++) {
    uint8_t *sA = sm + (ch & 1) * kCoarseStage, *sB = sA + 128 * 64 * 2;
    // A = R^T (128 samples x 64 rows): 8 rows of one sample per 16-byte store
#pragma unroll
    for (int j = 0; j < 8 / kQ; j++) {
      uint4 pk;
      pk.x = pack_bf16x2((float)cur[j][0], (float)cur[j][1]);
      pk.y = pack_bf16x2((float)cur[j][2], (float)cur[j][3]);
      pk.z = pack_bf16x2((float)cur[j][4], (float)cur[j][5]);
      pk.w = pack_bf16x2((float)cur[j][6], (float)cur[j][7]);
      *reinterpret_cast<uint4 *>(sA + tc::cm_offset(m, (q + kQ * j) * 8, 64)) = pk;
    }
    // B = the chunk's Wc^T tile (cmodes x 64), stored in operand order; it
    // was loaded one chunk ahead
#pragma unroll
    for (int j = 0; j < kBp; j++) {
      const int i = tid + j * kCoarseThreads;
      if (i < stage_b / 16) reinterpret_cast<uint4 *>(sB)[i] = bcur[j];
    }
    // the next chunk's residuals and tile are in flight during the MMAs of this one
    if (ch + 1 < nch) {
      load_chunk(ch + 1, nxt);
      load_tile(ch + 1, bnxt);
    }
    tc::fence_proxy_async();
    // the MMAs of the previous chunk read the other buffer; wait for them
    // before the next staging round overwrites it
    if (ch > 0) {
      ok = ok && tc::mbar_wait(bar, phase, kMmaSpinLimit);
      phase ^= 1u;
    }
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < 4; ks++)
        tc::mma_bf16(tmem, tc::desc_kmajor(tc::smem_u32(sA) + ks * 256, 128, 1024),
                     tc::desc_kmajor(tc::smem_u32(sB) + ks * 256, 128, 1024), idesc, ch > 0 || ks > 0);
      tc::commit(bar);
    }
#pragma unroll
    for (int j = 0; j < 8 / kQ; j++)
#pragma unroll
      for (int e = 0; e < 8; e++) cur[j][e] = nxt[j][e];
#pragma unroll
    for (int j = 0; j < kBp; j++) bcur[j] = bnxt[j];
  }
  ok = ok && tc::mbar_wait(bar, phase, kMmaSpinLimit);
  phase ^= 1u;
  tc::fence_after_sync();
  if (!ok) coarse_fail(gb);
  // the modes in kQ parts of cw columns (a multiple of 8), the last one short
  const int cw = ((nmod / kQ) + 7) / 8 * 8;
  {
    // partial c -> cpart[g][range][mode][sample]: warp w reads TMEM lanes
    // 32 (w % 4) .. +31 (its samples), columns of part w / 4
    const int part = warp >> 2, ms = (warp & 3) * 32 + lane;
    const int k0 = part * cw, k1 = min(nmod, k0 + cw);
    float *dst = M.cpart + ((size_t)g * M.nsplit + range) * nmod * 128;
    for (int kk = k0; kk < k1; kk += 8) {
      uint32_t v[8];
      tc::tmem_ld8(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)kk, v);
#pragma unroll
      for (int e = 0; e < 8; e++) __stcg(dst + (size_t)(kk + e) * 128 + ms, __uint_as_float(v[e]));
    }
  }
  tc::fence_before_sync();
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = (atomicAdd(M.ccnt + g, 1) == M.nsplit - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // the group's last range: c = sum of the partials in range order; BF16
  // operand tile for C3; c.c into the group's r.z
  double cc = 0.0;
  for (int kk = q * cw; kk < min(nmod, (q + 1) * cw); kk += 8) {
    float c8[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int k = kk + e;
      float t = 0.0f;
      for (int sp = 0; sp < M.nsplit; sp++)
        t += __ldcg(M.cpart + (((size_t)g * M.nsplit + sp) * nmod + k) * 128 + m);
      c8[e] = t;
      cc += (double)t * (double)t;
    }
    uint4 pk;
    pk.x = pack_bf16x2(c8[0], c8[1]);
    pk.y = pack_bf16x2(c8[2], c8[3]);
    pk.z = pack_bf16x2(c8[4], c8[5]);
    pk.w = pack_bf16x2(c8[6], c8[7]);
    __stcg(reinterpret_cast<uint4 *>(M.cb + (size_t)g * 128 * nmod * 2 + tc::cm_offset(m, kk, nmod)), pk);
  }
  s_cc[tid] = cc;
  __syncthreads();
  if (tid < 128) {
    double t = 0.0;
    for (int j = 0; j < kQ; j++) t += s_cc[tid + 128 * j];
    double *rz = M.tot_rz + (size_t)par * S + (size_t)g * 128 + tid;
    __stcg(rz, __ldcg(rz) + t);
  }
  if (tid == 0) atomicExch(M.ccnt + g, 0);  // next used after a grid barrier
  __syncthreads();
}

// z += Wc c on the 128-row chunk `chunk` of group g.
template <typename T>
__device__ __noinline__ void coarse_c3(const BMesh<T> &M, int g, int chunk, uint32_t &phase, GridBar *gb) {
  constexpr int kRows = 128 / (kCoarseThreads / 128);  // rows of the chunk per thread
  const uint32_t tmem = s_coarse_tmem;
  uint64_t *bar = &s_coarse_mbar;
  uint8_t *sm = s_dyn_smem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nmod = M.cmodes, S = M.S;
  const int tbytes = 128 * nmod * 2;
  uint8_t *sA = sm, *sB = sm + tbytes;
  // A = c of the group, B = Wc rows of the chunk: both tiles lie contiguous
  // in global memory in operand order, so one bulk copy each brings them in
  // while the threads' z loads are in flight.  c was written in this launch
  // by other blocks (before the grid barrier that started the phase), and
  // shared memory by this block's threads in earlier phases: the proxy
  // fence orders both before the copies.
  if (tid == 0) {
    asm volatile("fence.proxy.async;" ::: "memory");
    mbar_expect_tx(&s_tile_mbar, 2u * (uint32_t)tbytes);
    bulk_g2s(sA, M.cb + (size_t)g * tbytes, (uint32_t)tbytes, &s_tile_mbar);
    bulk_g2s(sB, M.wt3 + (size_t)chunk * tbytes, (uint32_t)tbytes, &s_tile_mbar);
  }
  // lanes = samples, columns = rows of the chunk: warp w reads TMEM lanes
  // 32 (w % 4) .. +31 and rows kRows (w / 4) .. +kRows-1
  const int ms = (warp & 3) * 32 + lane, j0 = (warp >> 2) * kRows;
  T *zc = M.z + (size_t)g * 128 + ms;
  const int rbase = chunk * 128 + j0;
  const int nrow = min(kRows, M.n - rbase);  // rows of this thread's share in the mesh
  // all z loads of this thread are in flight during the copies and the MMAs
  T zv[kRows];
#pragma unroll
  for (int e = 0; e < kRows; e++) zv[e] = e < nrow ? __ldcg(zc + (size_t)(rbase + e) * S) : T(0);
  const uint32_t tph = s_tile_phase;
  const bool tok = tc::mbar_wait(&s_tile_mbar, tph, kMmaSpinLimit);
  __syncthreads();
  if (tid == 0) {
    s_tile_phase = tph ^ 1u;
    if (!tok) coarse_fail(gb);
    tc::fence_after_sync();
    const uint32_t idesc = tc::idesc_bf16(128, 128), sbo = (uint32_t)(nmod / 8) * 128;
    for (int ks = 0; ks < nmod / 16; ks++)
      tc::mma_bf16(tmem, tc::desc_kmajor(tc::smem_u32(sA) + ks * 256, 128, sbo),
                   tc::desc_kmajor(tc::smem_u32(sB) + ks * 256, 128, sbo), idesc, ks > 0);
    tc::commit(bar);
  }
  const bool ok = tc::mbar_wait(bar, phase, kMmaSpinLimit);
  phase ^= 1u;
  tc::fence_after_sync();
  if (!ok) coarse_fail(gb);
#pragma unroll
  for (int e0 = 0; e0 < kRows; e0 += 8) {
    uint32_t v[8];
    tc::tmem_ld8(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(j0 + e0), v);
#pragma unroll
    for (int e = 0; e < 8; e++)
      if (e0 + e < nrow) zc[(size_t)(rbase + e0 + e) * S] = (T)((double)zv[e0 + e] + (double)__uint_as_float(v[e]));
  }
  tc::fence_before_sync();
  __syncthreads();  // the next item restages the operand tiles and reuses the accumulator
}

// Wc [n][cm] (FP64, row-major) -> the two BF16 operand tilings; supported rows zero
__global__ void k_coarse_tiles(int n, int cm, const double *__restrict__ Wc, const unsigned char *__restrict__ fixed,
                               __nv_bfloat16 *__restrict__ wt1, __nv_bfloat16 *__restrict__ wt3, int n64, int n128) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long tot1 = (long)n64 * 64 * cm, tot3 = (long)n128 * 128 * cm;
  if (t < tot1) {
    // wt1: tile q holds rows 64q..64q+63 as a cm x 64 operand (mode, row)
    const int q = (int)(t / (64L * cm)), rem = (int)(t % (64L * cm));
    const int k = rem / 64, j = rem % 64, row = q * 64 + j;
    const double v = (row < n && !fixed[row]) ? Wc[(size_t)row * cm + k] : 0.0;
    wt1[((size_t)q * 64 * cm * 2 + tc::cm_offset(k, j, 64)) / 2] = __float2bfloat16((float)v);
  } else if (t < tot1 + tot3) {
    // wt3: tile q holds rows 128q..128q+127 as a 128 x cm operand (row, mode)
    const long u = t - tot1;
    const int q = (int)(u / (128L * cm)), rem = (int)(u % (128L * cm));
    const int j = rem / cm, k = rem % cm, row = q * 128 + j;
    const double v = (row < n && !fixed[row]) ? Wc[(size_t)row * cm + k] : 0.0;
    wt3[((size_t)q * 128 * cm * 2 + tc::cm_offset(j, k, cm)) / 2] = __float2bfloat16((float)v);
  }
}

constexpr int kMaxMeshes = 8;
constexpr size_t kMultSmem = 32 * 1024;  // largest staged multiplier table of a tile's group

#ifndef UFEM_PCG_MIN_BLOCKS
#define UFEM_PCG_MIN_BLOCKS 2
#endif
// The coarse phases (precisions 2 and 3, 128-sample groups): C1 then C3 over the
// groups whose z has to be formed from r; two grid barriers.  The parity of
// the MMA barrier is kept in shared memory between calls.
template <typename T>
__device__ __noinline__ bool coarse_phases(const BArgs<T> A, const BMesh<T> *s_meshes, int par) {
  __shared__ int s_go;
  uint32_t phase = s_coarse_phase;
  {
    prof_begin(kPhC1);
    for (int t = claim(A.wctr + kPhC1); t < A.nc1; t = claim(A.wctr + kPhC1)) {
      const int4 it = A.c1items[t];
      const BMesh<T> &M = s_meshes[it.x];
      if (threadIdx.x == 0) s_go = __ldcg(M.gcz + it.y);
      __syncthreads();
      const int go = s_go;
      __syncthreads();
      if (go) coarse_c1(M, it.y, it.z, par, phase, A.bar);
    }
    prof_end();
    if (!grid_barrier(A.bar)) return false;
    release_counter(A.wctr + kPhC1);
    prof_begin(kPhC3);
    for (int t = claim(A.wctr + kPhC3); t < A.nc3; t = claim(A.wctr + kPhC3)) {
      const int4 it = A.c3items[t];
      const BMesh<T> &M = s_meshes[it.x];
      if (threadIdx.x == 0) s_go = __ldcg(M.gcz + it.y);
      __syncthreads();
      const int go = s_go;
      __syncthreads();
      if (go) coarse_c3(M, it.y, it.z, phase, A.bar);
    }
    prof_end();
    if (!grid_barrier(A.bar)) return false;
    release_counter(A.wctr + kPhC3);
  }
  if (threadIdx.x == 0) s_coarse_phase = phase;  // every thread holds the same parity
  __syncthreads();
  return true;
}

// Phase S of iteration k: per-sample convergence on true residuals, beta,
// q = A p with p = z + beta p_old, p.q (the tiles' work items).
template <typename T, int B, bool IMP, int UN, int VN, int NW, bool F32P>
__device__ __forceinline__ void phase_S(const BArgs<T> &A, const BMesh<T> *s_meshes, long k,
                                        double (*s_red)[32 * VN], T *s_sc) {
  constexpr int GS = 32 * VN;
  __shared__ int s_flag;
  const int par = (int)(k & 1), parm1 = (int)((k - 1) & 1);
  const bool first = (k == 1);
  prof_begin(kPhS);
  for (int t = claim(A.wctr + kPhS); t < A.ntiles; t = claim(A.wctr + kPhS)) {
    const int4 ti = A.tiles[t];
    const BMesh<T> &M = s_meshes[ti.x];
    if (threadIdx.x == 0) s_flag = __ldcg(M.gtrue + ti.y);
    __syncthreads();
    const int g = ti.y;
    const bool is_true = s_flag != 0;
    int upd = 0, near = 0, wait = 0;
    if (threadIdx.x < GS) {
      const int sl = threadIdx.x, s = g * GS + sl;
      const double rr = __ldcg(M.tot_rr + (size_t)parm1 * M.S + s);
      const double rzn = __ldcg(M.tot_rz + (size_t)parm1 * M.S + s);
      const double rzo = first ? 1.0 : __ldcg(M.rho + (size_t)parm1 * M.S + s);
      const double tol2 = M.tol2[s];
      const int st = __ldcg(M.state + s);
      // A sample whose recursive residual reaches tol / 2 is frozen until
      // the group's next true-residual pass confirms it (or it resumes).
      // FP32 inner iterations too: the residual is replaced every time it
      // has dropped by replace_near, so the recursive residual's drift is
      // small against tol when it gets there.
      constexpr bool kFreeze = true;
      int nst = st;
      if (st == ST_ACTIVE || st == ST_CAND) {
        if (!(rr == rr) || isinf(rr)) nst = ST_NAN;
        else if (is_true && (double)rr <= tol2) nst = ST_CONV;
        else if (k > A.maxit) nst = ST_MAXIT;
        else if (is_true) nst = ST_ACTIVE;  // a candidate that failed its check resumes
        else if (kFreeze && rr <= 0.25 * tol2) nst = ST_CAND;
      }
      upd = (nst == ST_ACTIVE);
      wait = (nst == ST_CAND);
      // replace once the recursive residual has dropped by the factor
      // near since the last replacement (FP32: also to verify convergence)
      near = upd && !is_true &&
             (rr <= A.near2 * __ldcg(M.rrlast + s) || (!kFreeze && rr <= 0.25 * tol2));
      s_sc[sl] = upd ? (first ? T(0) : (T)(rzn / rzo)) : T(0);
      if (ti.z == 0) {  // the group's first tile records per-sample results
        if (sl == 0 && M.cmodes) M.gcz[g] = 0;  // z was formed in the last coarse phase
        if (nst != st) {
          M.state[s] = nst;
          // a verified candidate keeps the count of the iterate it froze at
          if (!(st == ST_CAND && nst == ST_CONV)) M.iters[s] = (int)(k - 1);
        }
        M.rho[(size_t)par * M.S + s] = rzn;
        if (is_true) M.rrlast[s] = rr;
      }
    }
    upd = __syncthreads_or(upd);
    near = __syncthreads_or(near);
    wait = __syncthreads_or(wait);
    if (ti.z == 0 && threadIdx.x == 0) {
      if (!upd && !wait && M.gactive[g]) {
        M.gactive[g] = 0;
        atomicSub(A.active_count, 1);
      }
      // a true-residual pass.  FP32: on the residual drop and every
      // rr_every iterations -- both only on every kRepAlign-th iteration,
      // so that the groups' replacements share passes (a pass over few
      // groups leaves most SMs idle) -- and at once to verify candidates
      // once no sample of the group still iterates.  FP64 (no drift to
      // correct): only to verify candidates, once no sample of the group
      // still iterates or rr_every iterations after the last pass.
      const bool due = (k - M.glast[g] >= A.rr_every);
      if (sizeof(T) == 8) M.gneed[g] = wait && (!upd || due);
      else M.gneed[g] = (upd && (near || due) && (k % kRepAlign) == 0) || (wait && !upd);
    }
    if (!upd) {
      __syncthreads();
      continue;
    }
    const T *pold = (k & 1) ? M.p0 : M.p1;
    T *pnew = (k & 1) ? M.p1 : M.p0;
    tile_spmv<T, B, IMP, UN, VN, NW, F32P>(M, g, ti.z, s_sc, first, pold, pnew, s_red);
  }
}

// Phase U of iteration k: alpha, x += alpha p, r -= alpha q, z = r / M, and
// the groups that asked for a true-residual pass counted in A.rcount.
template <typename T, int B, int VN, int NW>
__device__ __forceinline__ void phase_U(const BArgs<T> &A, const BMesh<T> *s_meshes, long k,
                                        double (*s_red)[32 * VN], double (*s_red2)[32 * VN], T *s_sc) {
  constexpr int GS = 32 * VN;
  const int par = (int)(k & 1);
  prof_begin(kPhU);
  for (int t = claim(A.wctr + kPhU); t < A.ntiles; t = claim(A.wctr + kPhU)) {
    const int4 ti = A.tiles[t];
    const BMesh<T> &M = s_meshes[ti.x];
    __syncthreads();
    const int g = ti.y;
    int upd = 0;
    if (threadIdx.x < GS) {
      const int sl = threadIdx.x, s = g * GS + sl;
      const int st = __ldcg(M.state + s);
      T alpha = 0;
      if (st == ST_ACTIVE) {
        const double pq = __ldcg(M.tot_pq + s);
        const double rho = __ldcg(M.rho + (size_t)par * M.S + s);
        if (pq > 0.0 && isfinite(pq)) {
          alpha = (T)(rho / pq);
          upd = 1;
        } else if (ti.z == 0) {
          M.state[s] = isfinite(pq) ? ST_BREAK : ST_NAN;  // p.q <= 0 or not finite: the sample is frozen
          M.iters[s] = (int)k;
        }
      }
      s_sc[sl] = alpha;
    }
    upd = __syncthreads_or(upd);
    int live = 0;
    if (threadIdx.x < GS) live = (__ldcg(M.state + g * GS + threadIdx.x) == ST_ACTIVE);
    live = __syncthreads_or(live) | upd;
    // groups due for a true-residual pass are counted whether or not they
    // update (a group of frozen candidates only waits for that pass)
    if (ti.z == 0 && threadIdx.x == 0 && __ldcg(M.gneed + g)) atomicAdd(A.rcount, 1);
    if (!live) continue;
    const T *pnew = (k & 1) ? M.p1 : M.p0;
    tile_update<T, B, VN, NW>(M, g, ti.z, s_sc, pnew, par, s_red, s_red2);
    if (ti.z == 0 && threadIdx.x == 0) M.gtrue[g] = 0;
    if (M.cmodes && threadIdx.x == 0) M.gcz[g] = 1;
  }
}

// Phase R of iteration k: the groups that asked replace their recursive
// residual by the true one.
template <typename T, int B, bool IMP, int UN, int VN, int NW>
__device__ __forceinline__ void phase_R(const BArgs<T> &A, const BMesh<T> *s_meshes, long k,
                                        double (*s_red)[32 * VN], double (*s_red2)[32 * VN]) {
  __shared__ int s_flag;
  const int par = (int)(k & 1);
  prof_begin(kPhR);
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.prof) A.prof[2 * kProfWall] += 1;
  for (int t = claim(A.wctr + kPhR); t < A.ntiles; t = claim(A.wctr + kPhR)) {
    const int4 ti = A.tiles[t];
    const BMesh<T> &M = s_meshes[ti.x];
    if (threadIdx.x == 0) s_flag = __ldcg(M.gneed + ti.y);
    __syncthreads();
    if (!s_flag) {
      __syncthreads();  // thread 0 rewrites s_flag for the next tile
      continue;
    }
    tile_true_residual<T, B, IMP, UN, VN, NW>(M, ti.y, ti.z, par, s_red, s_red2);
    if (ti.z == 0 && threadIdx.x == 0) {
      M.gtrue[ti.y] = 1;
      M.glast[ti.y] = (int)k;
    }
    if (M.cmodes && threadIdx.x == 0) M.gcz[ti.y] = 1;
  }
}

// The block's shared state of the PCG launches (declared once per kernel).
template <typename T, int NW, int GS>
struct PcgShared {
  double red[NW][GS];   // per-warp partial sums
  double red2[NW][GS];
  T sc[GS];             // per-sample scalars of the tile's group
  BMesh<T> meshes[kMaxMeshes];
};

template <typename T, int B, bool IMP, int UN, int VN, bool CO, int NW, bool F32P>
__device__ __forceinline__ void pcg_body(const BArgs<T> A, PcgShared<T, NW, 32 * VN> &sh) {
  constexpr int GS = 32 * VN;
  constexpr bool kCoarse = CO;
  static_assert(!CO || (IMP && VN == 4), "the coarse correction runs with the implicit form and 128-sample groups");
  double (*s_red)[GS] = sh.red;
  double (*s_red2)[GS] = sh.red2;
  T *s_sc = sh.sc;
  BMesh<T> *s_meshes = sh.meshes;
  // the mesh descriptors, once per launch
  for (int i = threadIdx.x; i < A.nmesh * (int)(sizeof(BMesh<T>) / sizeof(int)); i += blockDim.x)
    reinterpret_cast<int *>(s_meshes)[i] = reinterpret_cast<const int *>(A.meshes)[i];
  prof_init();
  __syncthreads();
  // phase 0: the true residual of the initial guess (parity slot 0)
  for (int t = claim(A.wctr + kPhInit); t < A.ntiles; t = claim(A.wctr + kPhInit)) {
    const int4 ti = A.tiles[t];
    const BMesh<T> &M = s_meshes[ti.x];
    int any = 0;
    if (threadIdx.x < GS) any = (M.state[ti.y * GS + threadIdx.x] == ST_ACTIVE);
    any = __syncthreads_or(any);
    if (any) {
      tile_true_residual<T, B, IMP, UN, VN, NW>(M, ti.y, ti.z, 0, s_red, s_red2);
      if (ti.z == 0 && threadIdx.x == 0) {
        M.gtrue[ti.y] = 1;
        M.glast[ti.y] = 0;
      }
      if (M.cmodes && threadIdx.x == 0) M.gcz[ti.y] = 1;
    }
    __syncthreads();
  }
  prof_end();
  if (!grid_barrier(A.bar)) return;
  release_counter(A.wctr + kPhInit);
  if constexpr (kCoarse) {
    if (A.coarse && !coarse_phases<T>(A, s_meshes, 0)) return;
  }
  long k;
  for (k = 1;; k++) {
    const int par = (int)(k & 1);
    // ---- phase S: convergence on true residuals, beta, q = A p -------------
    phase_S<T, B, IMP, UN, VN, NW, F32P>(A, s_meshes, k, s_red, s_sc);
    prof_end();
    if (!grid_barrier(A.bar)) return;
    release_counter(A.wctr + kPhS);
    // The group counter changes only in phase S: read between the barriers,
    // every block takes the same exit decision.
    const int remaining = atomicAdd(A.active_count, 0);
    // ---- phase U: alpha, x += alpha p, r -= alpha q, z = r / M --------------
    phase_U<T, B, VN, NW>(A, s_meshes, k, s_red, s_red2, s_sc);
    prof_end();
    if (!grid_barrier(A.bar)) return;
    release_counter(A.wctr + kPhU);
    // ---- phase R (when a group asked): replace the recursive residual -------
    const int nrep = atomicAdd(A.rcount, 0);  // changes only in phase U
    if (nrep > 0) {
      phase_R<T, B, IMP, UN, VN, NW>(A, s_meshes, k, s_red, s_red2);
      prof_end();
      if (!grid_barrier(A.bar)) return;
      release_counter(A.wctr + kPhR);
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(A.rcount, 0);  // read again only after the next U
    }
    if (remaining <= 0 || k > A.maxit + 1) break;
    // ---- phases C1, C3 (coarse space): z = r / M + Wc Wc^T r ----------------
    if constexpr (kCoarse) {
      if (A.coarse && !coarse_phases<T>(A, s_meshes, par)) return;
    }
  }
  prof_flush(A.prof);
  if (blockIdx.x == 0 && threadIdx.x == 0) *A.iter_out = k;
}

// One iteration of the split form (A.kstep = k >= 1): phases U, R, C1, C3
// after the k_batch_s launch that ran phase S; A.kstep = 0: the initial
// residual and coarse correction.  The grid barriers inside the launch are
// those of pcg_body; the launch boundaries replace the barrier after S.
template <typename T, int B, bool IMP, int UN, int VN, int NW, bool F32P>
__device__ __forceinline__ void pcg_step(const BArgs<T> A, PcgShared<T, NW, 32 * VN> &sh) {
  constexpr int GS = 32 * VN;
  double (*s_red)[GS] = sh.red;
  double (*s_red2)[GS] = sh.red2;
  T *s_sc = sh.sc;
  BMesh<T> *s_meshes = sh.meshes;
  // every block reads the flag before the first barrier; block 0 sets it
  // only after the launch's barriers
  if (__ldcg(A.done)) return;
  for (int i = threadIdx.x; i < A.nmesh * (int)(sizeof(BMesh<T>) / sizeof(int)); i += blockDim.x)
    reinterpret_cast<int *>(s_meshes)[i] = reinterpret_cast<const int *>(A.meshes)[i];
  prof_init();
  __syncthreads();
  const long k = A.kstep;
  if (k == 0) {
    for (int t = claim(A.wctr + kPhInit); t < A.ntiles; t = claim(A.wctr + kPhInit)) {
      const int4 ti = A.tiles[t];
      const BMesh<T> &M = s_meshes[ti.x];
      int any = 0;
      if (threadIdx.x < GS) any = (M.state[ti.y * GS + threadIdx.x] == ST_ACTIVE);
      any = __syncthreads_or(any);
      if (any) {
        tile_true_residual<T, B, IMP, UN, VN, NW>(M, ti.y, ti.z, 0, s_red, s_red2);
        if (ti.z == 0 && threadIdx.x == 0) {
          M.gtrue[ti.y] = 1;
          M.glast[ti.y] = 0;
        }
        if (M.cmodes && threadIdx.x == 0) M.gcz[ti.y] = 1;
      }
      __syncthreads();
    }
    prof_end();
    if (!grid_barrier(A.bar)) return;
    release_counter(A.wctr + kPhInit);
    if (A.coarse && !coarse_phases<T>(A, s_meshes, 0)) return;
    prof_flush(A.prof);
    return;
  }
  const int par = (int)(k & 1);
  release_counter(A.wctr + kPhS);  // k_batch_s has finished with it
  // the group counter changes only in phase S (the previous launch)
  const int remaining = atomicAdd(A.active_count, 0);
  phase_U<T, B, VN, NW>(A, s_meshes, k, s_red, s_red2, s_sc);
  prof_end();
  if (!grid_barrier(A.bar)) return;
  release_counter(A.wctr + kPhU);
  const int nrep = atomicAdd(A.rcount, 0);  // changes only in phase U
  if (nrep > 0) {
    phase_R<T, B, IMP, UN, VN, NW>(A, s_meshes, k, s_red, s_red2);
    prof_end();
    if (!grid_barrier(A.bar)) return;
    release_counter(A.wctr + kPhR);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(A.rcount, 0);
  }
  if (remaining <= 0 || k > A.maxit + 1) {
    prof_flush(A.prof);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      *A.iter_out = k;
      atomicExch(A.done, 1);
    }
    return;
  }
  if (A.coarse && !coarse_phases<T>(A, s_meshes, par)) return;
  prof_flush(A.prof);
  if (blockIdx.x == 0 && threadIdx.x == 0) *A.iter_out = k;
}

// Phase S of iteration k for the split form, with more warps per SM than
// the coarse instance's 16 (the gathers are latency-bound; the other phases
// keep their 128 registers a thread in k_batch_pcg).  Ordinary launch, one
// block per SM.  28 warps (72 registers) measured best: S 85.0 ms per step
// at 24 warps, 83.2 at 28, 84.8 at 32 (8,192 samples of the 40x10x10 beam).
constexpr int kSplitThreads = 896;
template <typename T, int B, int UN, int VN, bool F32P>
__global__ void __launch_bounds__(kSplitThreads, 1) k_batch_s(BArgs<T> A, long k) {
  constexpr int GS = 32 * VN, NW = kSplitThreads / 32;
  __shared__ double s_red[NW][GS];
  __shared__ T s_sc[GS];
  __shared__ BMesh<T> s_meshes[kMaxMeshes];
  if (__ldcg(A.done)) return;
  for (int i = threadIdx.x; i < A.nmesh * (int)(sizeof(BMesh<T>) / sizeof(int)); i += blockDim.x)
    reinterpret_cast<int *>(s_meshes)[i] = reinterpret_cast<const int *>(A.meshes)[i];
  prof_init();
  __syncthreads();
  phase_S<T, B, true, UN, VN, NW, F32P>(A, s_meshes, k, s_red, s_sc);
  prof_end();
  prof_flush(A.prof);
}

// UN: contributions whose gathers are issued together (implicit form);
// VN: samples per lane (a sample group is 32 VN samples); CO: the launch
// has a coarse space -- a separate instance, so that the Jacobi-only kernel
// keeps its own register allocation.  A kernel that uses tensor memory runs
// one block per SM, so the coarse instance has kCoarseThreads threads per
// block (the Jacobi instance: two blocks of kThreads); the block holds
// kCoarseCols TMEM columns and kCoarseSmem bytes of dynamic shared memory
// for the whole launch.
template <typename T, int B, bool IMP, int UN, int VN, bool CO = false, bool F32P = false>
__global__ void __launch_bounds__(CO ? kCoarseThreads : kThreads, CO ? 1 : (IMP ? UFEM_PCG_MIN_BLOCKS : 2))
    k_batch_pcg(BArgs<T> A) {
  constexpr bool kCoarse = CO;
  if constexpr (kCoarse) {
    if (A.coarse) {
      if (threadIdx.x == 0) {
        tc::mbar_init(&s_coarse_mbar, 1);
        s_coarse_phase = 0;
        tc::mbar_init(&s_tile_mbar, 1);
        s_tile_phase = 0;
      }
      if ((threadIdx.x >> 5) == 0) tc::tmem_alloc(&s_coarse_tmem, kCoarseCols);
      tc::fence_before_sync();
      __syncthreads();
      tc::fence_after_sync();
    }
  }
  constexpr int NW = (CO ? kCoarseThreads : kThreads) / 32;
  __shared__ PcgShared<T, NW, 32 * VN> sh;
  if constexpr (CO && sizeof(T) == 4 && B == 3 && F32P) {
    pcg_step<T, B, IMP, UN, VN, NW, F32P>(A, sh);  // always split (run_pcg)
  } else {
    pcg_body<T, B, IMP, UN, VN, CO, NW, F32P>(A, sh);
  }
  if constexpr (kCoarse) {
    if (A.coarse) {
      tc::fence_before_sync();
      __syncthreads();
      if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(s_coarse_tmem, kCoarseCols);
    }
  }
}

// outputs: RES_D (u), RES_R (reaction = internal force - F at the support),
// RES_D_MAX / RES_D_MIN / RES_D_SUM; thread per (output, sample).  Element
// results and RES_FAIL: mcout.cu.
template <int B>
__global__ void k_outputs(int nout, int S, int nsamp, long olen, const int *__restrict__ otype,
                          const int *__restrict__ opos, const int *__restrict__ orow, const double *__restrict__ u,
                          const int *__restrict__ rowptr, const int *__restrict__ colind,
                          const int *__restrict__ gptr, const int *__restrict__ gel, const int *__restrict__ gpair,
                          int s_el, const double *__restrict__ Khat, const double *__restrict__ E,
                          const double *__restrict__ Fraw, double *__restrict__ ofld) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)nout * nsamp) return;
  const int o = (int)(t / nsamp), s = (int)(t % nsamp);
  const int ty = otype[o];
  double val = 0.0;
  if (ty == 8) {
    const int row = orow[o];
    if (row >= 0) val = u[(size_t)row * S + s];
  } else if (ty == 9) {
    const int row = orow[o];
    if (row >= 0) {
      const int I = row / B, a = row % B, nn = s_el / B;
      double fint = 0.0;
      for (int k = rowptr[I]; k < rowptr[I + 1]; k++) {
        const int J = colind[k];
        for (int c = gptr[k]; c < gptr[k + 1]; c++) {
          const int e = gel[c], p = gpair[c], la = p / nn, lb = p % nn;
          const double *kh = Khat + (size_t)e * s_el * s_el + (size_t)(la * B + a) * s_el + lb * B;
          double acc = 0.0;
          for (int j = 0; j < B; j++) acc += kh[j] * u[(size_t)(J * B + j) * S + s];
          fint += E[(size_t)e * S + s] * acc;
        }
      }
      val = (0.0 - Fraw[(size_t)row * S + s]) + fint;
    }
  } else if (ty == 15 || ty == 16) {
    const int row = orow[o];
    if (row >= 0) {
      const double v = u[(size_t)row * S + s];
      val = (ty == 15) ? (v > 0.0 ? v : 0.0) : (v < 0.0 ? v : 0.0);
    }
  } else if (ty == 17) {
    val = (double)orow[o];
  }
  ofld[(size_t)s * olen + opos[o]] = val;
}

// |F_s|^2 per sample in two passes with a fixed summation order (run-to-run
// identical): k_ff_part sums one chunk of rows for 32 samples per block (the
// lane is the sample, so each row read is one 256-byte transaction; 8 warps
// stride the chunk and are combined in warp order), k_tol2 adds the chunks in
// order and forms (|F_s| tol)^2.
constexpr int kFfChunks = 64;

__global__ void __launch_bounds__(256) k_ff_part(long n, int S, const double *__restrict__ F,
                                                 double *__restrict__ part) {
  __shared__ double sh[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int s = blockIdx.x * 32 + lane;  // S is a multiple of 128
  const long per = (n + gridDim.y - 1) / gridDim.y;
  const long i0 = (long)blockIdx.y * per, i1 = min(n, i0 + per);
  double t = 0.0;
  for (long i = i0 + w; i < i1; i += 8) {
    const double f = F[(size_t)i * S + s];
    t += f * f;
  }
  sh[w][lane] = t;
  __syncthreads();
  if (w == 0) {
    double a = 0.0;
    for (int k = 0; k < 8; k++) a += sh[k][lane];
    part[(size_t)blockIdx.y * S + s] = a;
  }
}

__global__ void k_tol2(int nch, int S, const double *__restrict__ part, double tol, double *__restrict__ tol2,
                       double *__restrict__ ff) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  double t = 0.0;
  for (int c = 0; c < nch; c++) t += part[(size_t)c * S + s];
  ff[s] = t;
  tol2[s] = tol * tol * t;
}

}  // namespace

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
struct McWork {
  int S = 0, nsamp = 0;
  DBuf<double> E, F, Fraw, V64, M64, x64, tol2, ff, ffpart;
  DBuf<float> V32, M32;
  DBuf<double> mult;     // implicit form: per-sample multipliers [nmult][S]
  // inner vectors, FP32 or FP64
  DBuf<float> fr, fz, fp0, fp1, fq;
  DBuf<double> dr, dz, dp0, dp1, dq, pq, prr, prz, rho, rrlast;
  DBuf<int> state, iters, gactive, gtrue, gneed, glast, gcnt;
  DBuf<double> tpq, trr, trz;  // group totals of the PCG partials
  // coarse correction: c per group (BF16 operand tiles), partial c per row range
  DBuf<uint8_t> cb;
  DBuf<float> cpart;
  DBuf<int> ccnt, gcz;
  std::vector<double> h_ff;
};

static ufem_mc_stats g_stats;

// Per-launch tables of the persistent PCG (mesh descriptors, work lists,
// grid barrier, counters), kept per device for the life of the process and
// only grown: a cudaFree per solve would synchronise the device and cost a
// variable few milliseconds.
template <typename T>
struct LaunchBufs {
  DBuf<BMesh<T>> meshes;
  DBuf<int4> tiles, c1, c3;
  DBuf<GridBar> bar;
  DBuf<int> cnt, rcnt;
  DBuf<long> itout;
  DBuf<unsigned long long> prof;
  DBuf<int> wctr;
  DBuf<int> done;
};
template <typename T>
LaunchBufs<T> &launch_bufs() {
  static std::vector<std::pair<int, std::unique_ptr<LaunchBufs<T>>>> per_dev;
  int dev = 0;
  cudaGetDevice(&dev);
  for (auto &e : per_dev)
    if (e.first == dev) return *e.second;
  per_dev.emplace_back(dev, std::unique_ptr<LaunchBufs<T>>(new LaunchBufs<T>()));
  return *per_dev.back().second;
}

// ---------------------------------------------------------------------------
// autotuned launch shapes: (tiles per block, gather unroll) per batch shape,
// kept in memory and in a text cache file (one "key tpb unroll ms" per line)
// ---------------------------------------------------------------------------
struct TuneEntry {
  std::string key;
  int tpb, unroll, lanes;
  double ms;
};
static std::vector<TuneEntry> g_tune;
static bool g_tune_loaded = false;

static std::string tune_cache_path(const char *path) {
  if (path && *path) return path;
  const char *e = getenv("UFEM_TUNE_CACHE");
  if (e && *e) return e;
  const char *h = getenv("HOME");
  return std::string(h ? h : "/tmp") + "/.cache/ufem_b200_tune.txt";
}

static void tune_load(const std::string &path) {
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return;
  char key[512];
  int tpb, un, ln;
  double ms;
  while (fscanf(f, "%511s %d %d %d %lf", key, &tpb, &un, &ln, &ms) == 5) {
    bool found = false;
    for (auto &t : g_tune)
      if (t.key == key) {
        t.tpb = tpb; t.unroll = un; t.lanes = ln; t.ms = ms;
        found = true;
      }
    if (!found) g_tune.push_back({key, tpb, un, ln, ms});
  }
  fclose(f);
}

static void tune_save(const std::string &path) {
  const size_t slash = path.find_last_of('/');
  if (slash != std::string::npos) {
    std::string dir = path.substr(0, slash);
    for (size_t i = 1; i <= dir.size(); i++)  // mkdir -p
      if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
  }
  FILE *f = fopen(path.c_str(), "w");
  if (!f) return;
  for (auto &t : g_tune) fprintf(f, "%s %d %d %d %.4f\n", t.key.c_str(), t.tpb, t.unroll, t.lanes, t.ms);
  fclose(f);
}

// the batch shape a tuned choice is valid for: device, precision, element
// family, and per mesh its block rows and padded sample count
static bool implicit_form(int precision) { return precision >= 2 && precision <= 4; }

static int coarse_modes(int nmesh, ufem_model *const *models, const ufem_mc_options &opt) {
  if (!implicit_form(opt.precision) || !opt.coarse) return 0;
  int cm = 0;
  for (int i = 0; i < nmesh; i++) cm = std::max(cm, get_plan(models[i])->cmodes);
  return cm;
}

static std::string tune_key(int nmesh, ufem_model *const *models, const long *nsamp, int precision,
                            int cmodes = 0) {
  // the device part once per device: cudaGetDeviceProperties takes several
  // milliseconds, erratically, and this runs on every solve
  static std::vector<std::pair<int, std::string>> dev_names;
  int dev = 0;
  cudaGetDevice(&dev);
  std::string name, *cached = nullptr;
  for (auto &e : dev_names)
    if (e.first == dev) cached = &e.second;
  if (!cached) {
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, dev);
    std::string nm = prop.name;
    for (auto &c : nm)
      if (c == ' ') c = '_';
    dev_names.emplace_back(dev, nm + "/sm" + std::to_string(nsm));
    cached = &dev_names.back().second;
  }
  name = *cached;
  std::string k = name + "/p" + std::to_string(precision) + "/b" + std::to_string(models[0]->b);
  for (int i = 0; i < nmesh; i++)
    k += "/" + std::to_string(models[i]->nbr) + "x" +
         std::to_string(std::max<long>(128, (nsamp[i] + 127) / 128 * 128));
  if (cmodes) k += "/c" + std::to_string(cmodes);
  return k;
}

static const TuneEntry *tune_find(const std::string &key) {
  if (!g_tune_loaded) {
    tune_load(tune_cache_path(nullptr));
    g_tune_loaded = true;
  }
  for (auto &t : g_tune)
    if (t.key == key) return &t;
  return nullptr;
}

// Workspaces are kept per model between calls, so repeated batches reuse
// their device buffers instead of allocating gigabytes each time.
static std::vector<std::pair<const ufem_model *, std::unique_ptr<McWork>>> g_work;

McWork *get_work(const ufem_model *m) {
  for (auto &w : g_work)
    if (w.first == m) return w.second.get();
  g_work.emplace_back(m, std::unique_ptr<McWork>(new McWork()));
  return g_work.back().second.get();
}

void drop_work(const ufem_model *m) {
  for (size_t i = 0; i < g_work.size(); i++)
    if (g_work[i].first == m) {
      g_work.erase(g_work.begin() + i);
      return;
    }
}

extern "C" void ufem_mc_default_options(ufem_mc_options *o) {
  o->precision = 1;
  o->tol = 1e-8;
  o->max_iters = 20000;
  o->replace_every = 50;
  o->replace_near = 1e-2;
  o->use_graphs = 0;
  o->tiles_per_block = 0;
  o->unroll = 0;
  o->lane_samples = 0;
  o->coarse = 1;
}

extern "C" int ufem_mc_get_stats(ufem_mc_stats *s) {
  *s = g_stats;
  return UFEM_AF_OK;
}

namespace {

struct EvTimer {
  cudaEvent_t a, b;
  EvTimer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
  }
  double stop() {
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~EvTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

template <typename T, bool IMP, int VN, bool F32P = false>
int run_pcg(int nmesh, ufem_model *const *models, std::vector<McWork *> &W, const std::vector<McPlan *> &plans,
            const ufem_mc_options &opt, long *iters_run) {
  constexpr int GS = 32 * VN;
  int rv;
  std::vector<BMesh<T>> hm(nmesh);
  std::vector<int4> tiles;
  int dev = 0, nsm = 0, occ = 0;
  UFEM_CUDA_TRY(cudaGetDevice(&dev));
  UFEM_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int B = models[0]->b;
  // the coarse correction needs 128-sample groups (one UMMA M tile)
  bool coarse = false;
  if constexpr (IMP && VN == 4) coarse = coarse_modes(nmesh, models, opt) > 0;
  void (*kern)(BArgs<T>) = nullptr;
  if constexpr (!IMP) {
    kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 1, VN> : k_batch_pcg<T, 2, IMP, 1, VN>;
  } else if constexpr (F32P) {
    // FP32 products (precision 4): 2 or 4 contributions in flight
    const int un = opt.unroll > 0 ? opt.unroll : 2;
    if (un <= 2) kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 2, VN, false, true> : k_batch_pcg<T, 2, IMP, 2, VN, false, true>;
    else kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 4, VN, false, true> : k_batch_pcg<T, 2, IMP, 4, VN, false, true>;
    if (coarse) {
      if (un <= 2) kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 2, VN, true, true> : k_batch_pcg<T, 2, IMP, 2, VN, true, true>;
      else kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 4, VN, true, true> : k_batch_pcg<T, 2, IMP, 4, VN, true, true>;
    }
  } else {
    const int un = opt.unroll > 0 ? opt.unroll : 2;
    if (un <= 2) kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 2, VN> : k_batch_pcg<T, 2, IMP, 2, VN>;
    else if (un <= 4) kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 4, VN> : k_batch_pcg<T, 2, IMP, 4, VN>;
    else kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 8, VN> : k_batch_pcg<T, 2, IMP, 8, VN>;
    if constexpr (VN == 4) {
      if (coarse) {
        if (un <= 2) kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 2, VN, true> : k_batch_pcg<T, 2, IMP, 2, VN, true>;
        else if (un <= 4) kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 4, VN, true> : k_batch_pcg<T, 2, IMP, 4, VN, true>;
        else kern = (B == 3) ? k_batch_pcg<T, 3, IMP, 8, VN, true> : k_batch_pcg<T, 2, IMP, 8, VN, true>;
      }
    }
  }
  // The multipliers of a tile's sample group go to shared memory when the
  // largest mesh's fit in kMultSmem bytes (zone models; per-element E
  // models read them from global memory); the coarse phases reuse the space.
  int max_nmult = 0;
  if constexpr (IMP)
    for (int k = 0; k < nmesh; k++) max_nmult = std::max(max_nmult, plans[k]->nmult);
  const size_t mult_bytes = (size_t)max_nmult * GS * sizeof(double);  // the true residual stages FP64
  const bool smult = IMP && max_nmult > 0 && mult_bytes <= kMultSmem;
  const size_t dsmem = std::max(coarse ? kCoarseSmem : (size_t)0, smult ? mult_bytes : (size_t)0);
  // one block per SM either way (tensor memory): the rest of the unified
  // L1 / shared memory stays L1 for the contribution records
  if (dsmem) UFEM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem));
  const int nthreads = coarse ? kCoarseThreads : kThreads, nwarps = nthreads / 32;
  UFEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, nthreads, dsmem));
  if (occ < 1) {
    set_error("batched PCG kernel does not fit on an SM");
    return UFEM_AF_ERR;
  }
  // every resident block holds kCoarseCols of the SM's 512 TMEM columns
  if (coarse) occ = std::min(occ, 512 / kCoarseCols);
  const int G = nsm * occ;
  // rows per tile: about tiles_per_block tiles per block over the whole batch
  long total_rows = 0;
  for (int k = 0; k < nmesh; k++) total_rows += (long)models[k]->nbr * (W[k]->S / GS);
  // measured best on B200: 12 for both forms (2 x 256-thread blocks per SM)
  // and for the coarse-corrected precision-4 solve with its split launches
  // (8,192 samples of the 40x10x10 beam: 182.5 / 180.4 / 182.5 / 184.4 /
  // 184.9 ms per step at 8 / 10 / 12 / 16 / 20 tiles per block); 16 for the
  // one-kernel coarse-corrected instance (201.2 ms against 206.1 at 24 and
  // 202.7 at 12)
  const bool split_form = coarse && F32P && sizeof(T) == 4 && IMP && VN == 4 && B == 3;
  const long tpb = opt.tiles_per_block > 0 ? opt.tiles_per_block : (coarse && !split_form ? 16 : 12);
  g_stats.tiles_per_block = (int)tpb;
  g_stats.unroll = IMP ? (opt.unroll > 0 ? opt.unroll : 2) : 0;
  g_stats.lane_samples = VN;
  int rpt = (int)std::max<long>(nwarps, (total_rows + tpb * G - 1) / (tpb * G));
  rpt = (rpt + nwarps - 1) / nwarps * nwarps;
  int active_groups = 0;
  std::vector<std::vector<int>> act(nmesh);  // active groups of each mesh
  for (int k = 0; k < nmesh; k++) {
    ufem_model *m = models[k];
    McWork &w = *W[k];
    BMesh<T> &b = hm[k];
    b.n = (int)m->nDOFAct;
    b.cmodes = b.nsplit = b.rps = 0;
    b.wt1 = b.wt3 = nullptr;
    b.cb = nullptr;
    b.cpart = nullptr;
    b.ccnt = b.gcz = nullptr;
    b.nbr = m->nbr;
    b.S = w.S;
    b.ngroups = w.S / GS;
    b.rows_per_tile = rpt;
    b.ntpg = (m->nbr + rpt - 1) / rpt;
    b.B = m->b;
    b.rowptr = m->d_rowptr.p;
    b.colind = m->d_colind.p;
    b.V64 = w.V64.p;
    b.F = w.F.p;
    b.x = w.x64.p;
    b.tol2 = w.tol2.p;
    b.cptr = plans[k]->cptr.p;
    b.crow = plans[k]->crow.p;
    b.cval = plans[k]->cval.p;
    b.mult = w.mult.p;
    b.fixed = m->d_fixed.p;
    b.cstride = plans[k]->cstride;
    b.sperm = plans[k]->sperm.p;
    b.w32 = plans[k]->w32.p;
    b.nmult = plans[k]->nmult;
    b.smult = smult ? 1 : 0;
    const size_t n = (size_t)m->nDOFAct * w.S;
    const size_t np = (size_t)b.ngroups * b.ntpg * GS;
    if constexpr (sizeof(T) == 4) {
      b.V = w.V32.p;
      b.M = w.M32.p;
      if ((rv = w.fr.ensure(n)) || (rv = w.fz.ensure(n)) || (rv = w.fp0.ensure(n)) || (rv = w.fp1.ensure(n)) ||
          (rv = w.fq.ensure(n)))
        return rv;
      b.r = w.fr.p; b.z = w.fz.p; b.p0 = w.fp0.p; b.p1 = w.fp1.p; b.q = w.fq.p;
    } else {
      b.V = IMP ? nullptr : w.V64.p;
      b.M = w.M64.p;
      if ((rv = w.dr.ensure(n)) || (rv = w.dz.ensure(n)) || (rv = w.dp0.ensure(n)) || (rv = w.dp1.ensure(n)) ||
          (rv = w.dq.ensure(n)))
        return rv;
      b.r = w.dr.p; b.z = w.dz.p; b.p0 = w.dp0.p; b.p1 = w.dp1.p; b.q = w.dq.p;
    }
    if ((rv = w.pq.ensure(np)) || (rv = w.prr.ensure(2 * np)) || (rv = w.prz.ensure(2 * np)) ||
        (rv = w.rho.ensure(2 * w.S)) || (rv = w.rrlast.ensure(w.S)))
      return rv;
    b.part_pq = w.pq.p; b.part_rr = w.prr.p; b.part_rz = w.prz.p; b.rho = w.rho.p; b.rrlast = w.rrlast.p;
    if ((rv = w.tpq.ensure(w.S)) || (rv = w.trr.ensure(2 * (size_t)w.S)) || (rv = w.trz.ensure(2 * (size_t)w.S)) ||
        (rv = w.gcnt.ensure(2 * (size_t)b.ngroups)))
      return rv;
    UFEM_CUDA_TRY(cudaMemsetAsync(w.gcnt.p, 0, 2 * b.ngroups * sizeof(int)));
    b.tot_pq = w.tpq.p; b.tot_rr = w.trr.p; b.tot_rz = w.trz.p; b.gcnt = w.gcnt.p;
    UFEM_CUDA_TRY(cudaMemsetAsync(b.p0, 0, n * sizeof(T)));
    UFEM_CUDA_TRY(cudaMemsetAsync(b.p1, 0, n * sizeof(T)));
    if ((rv = w.gactive.ensure(b.ngroups)) || (rv = w.gtrue.ensure(b.ngroups)) || (rv = w.gneed.ensure(b.ngroups)) ||
        (rv = w.glast.ensure(b.ngroups)))
      return rv;
    b.state = w.state.p;
    b.iters = w.iters.p;
    b.gactive = w.gactive.p;
    b.gtrue = w.gtrue.p;
    b.gneed = w.gneed.p;
    b.glast = w.glast.p;
    UFEM_CUDA_TRY(cudaMemsetAsync(w.gtrue.p, 0, b.ngroups * sizeof(int)));
    UFEM_CUDA_TRY(cudaMemsetAsync(w.gneed.p, 0, b.ngroups * sizeof(int)));
    UFEM_CUDA_TRY(cudaMemsetAsync(w.glast.p, 0, b.ngroups * sizeof(int)));
    // per-sample state: solve the real samples with a nonzero load
    std::vector<int> st(w.S), ga(b.ngroups, 0);
    for (int s = 0; s < w.S; s++) {
      if (s >= w.nsamp) st[s] = ST_SKIP;
      else if (!std::isfinite(w.h_ff[s])) st[s] = ST_NAN;  // NaN or infinite loads
      else if (!(w.h_ff[s] > 0.0)) st[s] = ST_CONV;  // zero load: u = 0 at once
      else st[s] = ST_ACTIVE;
      if (st[s] == ST_ACTIVE) ga[s / GS] = 1;
    }
    for (int g = 0; g < b.ngroups; g++) active_groups += ga[g];
    UFEM_CUDA_TRY(cudaMemcpyAsync(w.state.p, st.data(), w.S * sizeof(int), cudaMemcpyHostToDevice));
    UFEM_CUDA_TRY(cudaMemsetAsync(w.iters.p, 0, w.S * sizeof(int)));
    UFEM_CUDA_TRY(cudaMemcpyAsync(w.gactive.p, ga.data(), b.ngroups * sizeof(int), cudaMemcpyHostToDevice));
    for (int g = 0; g < b.ngroups; g++)
      if (ga[g]) {
        act[k].push_back(g);
        for (int c = 0; c < b.ntpg; c++) tiles.push_back(make_int4(k, g, c, 0));
      }
  }
  if (active_groups == 0) {
    *iters_run = 0;
    return UFEM_AF_OK;
  }
  // coarse phases: C1 row ranges of every active group, C3 128-row chunks
  std::vector<int4> c1items, c3items;
  int max_cmodes = 0;
  if (coarse) {
    for (int k = 0; k < nmesh; k++) {
      McPlan *P = plans[k];
      BMesh<T> &b = hm[k];
      McWork &w = *W[k];
      if (P->cmodes <= 0) continue;
      const int n = b.n, n64 = (n + 63) / 64, n128 = (n + 127) / 128;
      // at most one wave of row ranges: finer ranges that do not fill whole
      // waves leave the phase waiting on its last blocks (measured)
      int nsplit = std::max(1, std::min(n64, G / active_groups));
      b.rps = (n64 + nsplit - 1) / nsplit * 64;
      b.nsplit = (n + b.rps - 1) / b.rps;
      b.cmodes = P->cmodes;
      b.wt1 = P->wt1.p;
      b.wt3 = P->wt3.p;
      if ((rv = w.cb.ensure((size_t)b.ngroups * 128 * b.cmodes * 2)) ||
          (rv = w.cpart.ensure((size_t)b.ngroups * b.nsplit * b.cmodes * 128)) ||
          (rv = w.ccnt.ensure(b.ngroups)) || (rv = w.gcz.ensure(b.ngroups)))
        return rv;
      UFEM_CUDA_TRY(cudaMemsetAsync(w.ccnt.p, 0, b.ngroups * sizeof(int)));
      UFEM_CUDA_TRY(cudaMemsetAsync(w.gcz.p, 0, b.ngroups * sizeof(int)));
      b.cb = w.cb.p;
      b.cpart = w.cpart.p;
      b.ccnt = w.ccnt.p;
      b.gcz = w.gcz.p;
      max_cmodes = std::max(max_cmodes, b.cmodes);
      for (int g : act[k]) {
        for (int sp = 0; sp < b.nsplit; sp++) c1items.push_back(make_int4(k, g, sp, 0));
        for (int c = 0; c < n128; c++) c3items.push_back(make_int4(k, g, c, 0));
      }
    }
  }
  g_stats.coarse_modes = max_cmodes;
  LaunchBufs<T> &LB = launch_bufs<T>();
  auto &d_meshes = LB.meshes;
  auto &d_tiles = LB.tiles, &d_c1 = LB.c1, &d_c3 = LB.c3;
  auto &bar = LB.bar;
  auto &cnt = LB.cnt, &rcnt = LB.rcnt;
  auto &itout = LB.itout;
  const int zero = 0;
  if ((rv = d_meshes.upload(hm.data(), hm.size())) || (rv = d_tiles.upload(tiles.data(), tiles.size())) ||
      (rv = bar.ensure(1)) || (rv = cnt.upload(&active_groups, 1)) || (rv = rcnt.upload(&zero, 1)) ||
      (rv = itout.ensure(1)) || (rv = LB.prof.ensure(2 * kProfWall + 1)) || (rv = LB.wctr.ensure(kPhN)) ||
      (rv = LB.done.ensure(1)))
    return rv;
  UFEM_CUDA_TRY(cudaMemsetAsync(LB.wctr.p, 0, kPhN * sizeof(int)));
  UFEM_CUDA_TRY(cudaMemsetAsync(LB.done.p, 0, sizeof(int)));
  UFEM_CUDA_TRY(cudaMemsetAsync(LB.prof.p, 0, (2 * kProfWall + 1) * sizeof(unsigned long long)));
  if (!c1items.empty() && ((rv = d_c1.upload(c1items.data(), c1items.size())) ||
                           (rv = d_c3.upload(c3items.data(), c3items.size()))))
    return rv;
  UFEM_CUDA_TRY(cudaMemset(bar.p, 0, sizeof(GridBar)));
  BArgs<T> a;
  a.meshes = d_meshes.p;
  a.nmesh = nmesh;
  a.tiles = d_tiles.p;
  a.ntiles = (int)tiles.size();
  a.bar = bar.p;
  a.active_count = cnt.p;
  a.rcount = rcnt.p;
  a.maxit = opt.max_iters;
  a.rr_every = std::max<long>(1, opt.replace_every);
  a.near2 = opt.replace_near * opt.replace_near;
  a.iter_out = itout.p;
  a.coarse = !c1items.empty();
  a.c1items = d_c1.p;
  a.nc1 = (int)c1items.size();
  a.c3items = d_c3.p;
  a.nc3 = (int)c3items.size();
  a.prof = LB.prof.p;
  a.wctr = LB.wctr.p;
  a.kstep = -1;
  a.done = LB.done.p;
  void *args[] = {&a};
  const int grid = std::min<int>(G, (int)tiles.size());
  // The coarse-corrected precision-4 kernels of the brick family run each
  // iteration as two launches: phase S in k_batch_s (28 warps per SM), the
  // other phases in this kernel; every 4 iterations the host reads whether
  // the iterations ended (later launches return at once).  (Precision 3's
  // FP64 products need more registers than 28 warps leave: 35,858 ->
  // 24,961 solves/s split, so it keeps the persistent kernel.)
  bool split = false;
  void (*skern)(BArgs<T>, long) = nullptr;
  int sgrid = 0;
  size_t sdsmem = 0;
  if constexpr (IMP && VN == 4 && sizeof(T) == 4 && F32P) {
    if (coarse && B == 3) {
      const int un = opt.unroll > 0 ? opt.unroll : 2;
      skern = un <= 2 ? k_batch_s<T, 3, 2, VN, F32P> : k_batch_s<T, 3, 4, VN, F32P>;
      sdsmem = smult ? mult_bytes : 0;
      if (sdsmem) UFEM_CUDA_TRY(cudaFuncSetAttribute(skern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sdsmem));
      int socc = 0;
      UFEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&socc, skern, kSplitThreads, sdsmem));
      if (socc < 1) {
        set_error("batched PCG: the q = A z kernel does not fit on an SM");
        return UFEM_AF_ERR;
      }
      split = true;
      sgrid = std::min<int>(nsm * socc, (int)tiles.size());
    }
  }
  cudaEvent_t ev0, ev1;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  cudaEventRecord(ev0);
  if (!split) {
    UFEM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(grid), dim3(nthreads), args, dsmem, 0));
    g_stats.kernel_launches += 1;
  } else {
    a.kstep = 0;
    UFEM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(grid), dim3(nthreads), args, dsmem, 0));
    g_stats.kernel_launches += 1;
    int hdone = 0;
    for (long k = 1; k <= opt.max_iters + 2; k++) {
      skern<<<sgrid, kSplitThreads, sdsmem>>>(a, k);
      UFEM_CUDA_TRY(cudaGetLastError());
      a.kstep = k;
      UFEM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(grid), dim3(nthreads), args, dsmem, 0));
      g_stats.kernel_launches += 2;
      if ((k & 3) == 0) {
        GridBar hb0;
        UFEM_CUDA_TRY(cudaMemcpy(&hdone, LB.done.p, sizeof(int), cudaMemcpyDeviceToHost));
        UFEM_CUDA_TRY(cudaMemcpy(&hb0, bar.p, sizeof(hb0), cudaMemcpyDeviceToHost));
        if (hdone || hb0.err) break;
      }
    }
  }
  cudaEventRecord(ev1);
  long its = 0;
  GridBar hb;
  UFEM_CUDA_TRY(cudaMemcpy(&its, itout.p, sizeof(long), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(&hb, bar.p, sizeof(hb), cudaMemcpyDeviceToHost));
  float kms = 0;
  cudaEventElapsedTime(&kms, ev0, ev1);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  g_stats.ms_pcg += kms;
  g_stats.pcg_launch_ms[std::min<long>(g_stats.pcg_launches, 15)] = kms;
  g_stats.pcg_launches += 1;
  if (hb.err) {
    set_error(hb.err == kErrMma ? "batched PCG: a tensor-core wait of the coarse correction timed out"
                                : "batched PCG: grid barrier timed out");
    return UFEM_AF_ERR;
  }
  {
    unsigned long long pr[2 * kProfWall + 1];
    UFEM_CUDA_TRY(cudaMemcpy(pr, LB.prof.p, sizeof(pr), cudaMemcpyDeviceToHost));
    for (int p = 0; p < kPhN; p++) {
      g_stats.phase_wall_ms[p] += pr[kProfWall + p] * 1e-6;
      g_stats.phase_busy_ms[p] += pr[p] * 1e-6 / grid;
    }
    g_stats.true_residual_passes += (long)pr[2 * kProfWall];
  }
  *iters_run = its;
  // Algorithmic bytes.  A group of GS samples moves data only while it is
  // live, so each group counts the iterations it ran; the index arrays count
  // once per mesh-iteration.
  for (int k = 0; k < nmesh; k++) {
    const ufem_model *m = models[k];
    const McWork &w = *W[k];
    std::vector<int> st(w.S), itv(w.S);
    UFEM_CUDA_TRY(cudaMemcpy(st.data(), w.state.p, w.S * sizeof(int), cudaMemcpyDeviceToHost));
    UFEM_CUDA_TRY(cudaMemcpy(itv.data(), w.iters.p, w.S * sizeof(int), cudaMemcpyDeviceToHost));
    const double n = (double)m->nDOFAct, bb = m->b * m->b;
    long mesh_its = 0;
    for (int g = 0; g < w.S / GS; g++) {
      long gi = 0;
      for (int s = g * GS; s < (g + 1) * GS; s++) {
        if (st[s] == ST_SKIP || s >= w.nsamp) continue;
        long si = (st[s] == ST_ACTIVE || st[s] == ST_MAXIT) ? its : itv[s];
        gi = std::max(gi, si);
      }
      mesh_its = std::max(mesh_its, gi);
      // explicit: every sample's values; implicit: every sample's multipliers
      const double vals = IMP ? (double)plans[k]->nmult * sizeof(double) * GS : m->nnzb * bb * sizeof(T) * GS;
      const double vec = n * GS * sizeof(T);
      g_stats.spmv_bytes += (vals + 2.0 * vec) * gi;
      // S phase: values, 2 gathered and 2 own vectors in, 2 out; U phase:
      // M, r, p, q in, r, z out, x (FP64) in and out
      g_stats.pcg_bytes += (vals + 11.0 * vec + 2.0 * n * GS * sizeof(double)) * gi;
      // coarse phases: C1 reads r, C3 reads and writes z; the partial and
      // BF16 c tiles of the group
      const int cm = hm[k].cmodes;
      if (cm) g_stats.pcg_bytes += (3.0 * vec + 2.0 * hm[k].nsplit * cm * 128 * 4.0 + 3.0 * 128 * cm * 2.0) * gi;
    }
    double idx = m->nnzb * 4.0 + 4.0 * (m->nbr + 1);
    // implicit: the shared contribution table, once per mesh-iteration
    if (IMP) idx += 4.0 * (m->nnzb + 1) + 8.0 * plans[k]->nc * plans[k]->cstride;
    g_stats.spmv_bytes += idx * mesh_its;
    g_stats.pcg_bytes += idx * mesh_its;
    // the Wc tiles, once per mesh-iteration (both tilings)
    if (hm[k].cmodes) g_stats.pcg_bytes += 2.0 * n * hm[k].cmodes * 2.0 * mesh_its;
  }
  return UFEM_AF_OK;
}

}  // namespace

// The implicit form and the load tables of a model's Monte Carlo plan, for
// the warm start's reduced (Galerkin) operators; builds them when needed.
int mc_implicit_view(ufem_model *m, McImplicitView *v) {
  int rv;
  McPlan *P = get_plan(m);
  if (!P->built && (rv = build_plan(m, P)) != UFEM_AF_OK) return rv;
  if (!P->imp_built && (rv = build_implicit(m, P)) != UFEM_AF_OK) return rv;
  v->B = m->b;
  v->nbr = m->nbr;
  v->nmult = P->nmult;
  v->cstride = P->cstride;
  v->crow = P->crow.p;
  v->cval = P->cval.p;
  v->mult_col = P->mult_col;
  v->F0 = P->F0.p;
  v->ovr_row = P->ovr_row;
  v->ovr_var = P->ovr_var;
  return UFEM_AF_OK;
}

int mc_solve_device(int nmesh, ufem_model *const *models, const long *nsamp, const double *const *d_ifld,
                    double *const *d_ofld, int *const *d_status, long *const *d_iters,
                    const double *const *d_u_guess, double *const *d_u_out, const ufem_mc_options *opt_in) {
  ufem_mc_options opt;
  if (opt_in) opt = *opt_in;
  else ufem_mc_default_options(&opt);
  std::memset(&g_stats, 0, sizeof(g_stats));
  int rv;
  if (opt.precision < 0 || opt.precision > 4) {
    set_error("batched Monte Carlo: precision 0 to 4");
    return UFEM_AF_ERR_VAL;
  }
  if (nmesh < 1 || nmesh > kMaxMeshes) {
    set_error("batched Monte Carlo: 1 to 8 meshes per launch");
    return UFEM_AF_ERR_SIZ;
  }
  // FP32 products need a starting guess: from zero they lose the cancellation
  // of K z for smooth z (about twice the iterations, and no convergence to
  // 1e-8 with the coarse space), so a launch with a mesh that has no guess
  // runs in precision 3
  if (opt.precision == 4)
    for (int k = 0; k < nmesh; k++)
      if (!d_u_guess || !d_u_guess[k]) opt.precision = 3;
  const int B = models[0]->b;
  for (int k = 0; k < nmesh; k++)
    if (models[k]->b != B) {
      set_error("all meshes of one batched launch must have the same element family");
      return UFEM_AF_ERR_TYP;
    }
  EvTimer total;
  std::vector<McWork *> W(nmesh);
  std::vector<McPlan *> plans(nmesh);
  // ---- plans, inputs, batched assembly, tolerances ------------------------
  {
    EvTimer t;
    for (int k = 0; k < nmesh; k++) {
      ufem_model *m = models[k];
      McPlan *P = get_plan(m);
      if (!P->built && (rv = build_plan(m, P)) != UFEM_AF_OK) return rv;
      const bool imp = implicit_form(opt.precision);
      if (imp && !P->imp_built && (rv = build_implicit(m, P)) != UFEM_AF_OK) return rv;
      plans[k] = P;
      W[k] = get_work(m);
      McWork &w = *W[k];
      w.nsamp = (int)nsamp[k];
      w.S = std::max(128, (int)((nsamp[k] + 127) / 128 * 128));
      const size_t n = (size_t)m->nDOFAct * w.S, nv = (size_t)m->nnzb * B * B * w.S;
      if ((rv = w.E.ensure((size_t)m->eLen * w.S)) || (rv = w.F.ensure(n)) || (rv = w.Fraw.ensure(n)) ||
          (rv = w.M64.ensure(n)) || (rv = w.x64.ensure(n)) || (rv = w.state.ensure(w.S)) ||
          (rv = w.iters.ensure(w.S)) || (rv = w.tol2.ensure(w.S)) || (rv = w.ff.ensure(w.S)) ||
          (rv = w.ffpart.ensure((size_t)kFfChunks * w.S)))
        return rv;
      if (imp) {
        // no per-sample matrix: the values are formed inside the PCG kernel
        w.V64.release();
        w.V32.release();
        if ((rv = w.mult.ensure((size_t)P->nmult * w.S))) return rv;
      } else if ((rv = w.V64.ensure(nv))) {
        return rv;
      }
      if (opt.precision == 1) {
        if ((rv = w.V32.ensure(nv)) || (rv = w.M32.ensure(n))) return rv;
      } else if (opt.precision >= 3) {
        if ((rv = w.M32.ensure(n))) return rv;
      }
      const long ne = (long)m->eLen * w.S;
      k_make_E<<<(unsigned)((ne + 255) / 256), 256>>>((int)m->eLen, w.S, w.nsamp, P->ilen, d_ifld[k],
                                                      P->elem_var.p, m->d_eE.p, w.E.p);
      k_make_F<<<(unsigned)((n + 255) / 256), 256>>>((int)m->nDOFAct, w.S, w.nsamp, P->ilen, d_ifld[k], P->F0.p,
                                                     P->d_ovr_ptr.p, P->d_ovr_rvar.p,
                                                     w.Fraw.p);
      UFEM_CUDA_TRY(cudaMemcpyAsync(w.F.p, w.Fraw.p, n * sizeof(double), cudaMemcpyDeviceToDevice));
      k_fix_F<<<(unsigned)((n + 255) / 256), 256>>>((int)m->nDOFAct, w.S, m->d_fixed.p, w.F.p);
      if (imp) {
        const long nm = (long)P->nmult * w.S, nd = (long)m->nbr * w.S;
        k_make_mult<<<(unsigned)((nm + 255) / 256), 256>>>(P->nmult, w.S, w.nsamp, P->ilen, d_ifld[k],
                                                           P->d_mult_col.p, w.mult.p);
        if (B == 3)
          k_diag_implicit<3><<<(unsigned)((nd + 255) / 256), 256>>>(m->nbr, w.S, m->d_diagblk.p, P->cptr.p,
                                                                    P->cval.p, P->cstride, w.mult.p,
                                                                    m->d_fixed.p, w.M64.p);
        else
          k_diag_implicit<2><<<(unsigned)((nd + 255) / 256), 256>>>(m->nbr, w.S, m->d_diagblk.p, P->cptr.p,
                                                                    P->cval.p, P->cstride, w.mult.p,
                                                                    m->d_fixed.p, w.M64.p);
        g_stats.kernel_launches += 1;  // two kernels here in place of the assembly
        if (opt.precision >= 3) {
          k_diag_f32<<<(unsigned)((n + 255) / 256), 256>>>((long)n, w.M64.p, w.M32.p);
          g_stats.kernel_launches += 1;
        }
      } else {
        dim3 ga((unsigned)m->nnzb, (unsigned)(w.S / 128));
        float *v32 = opt.precision == 1 ? w.V32.p : nullptr;
        float *m32 = opt.precision == 1 ? w.M32.p : nullptr;
        if (B == 3)
          k_assemble_batch<3><<<ga, 128>>>(w.S, P->s, m->d_blkrow.p, m->d_colind.p, P->gptr.p, P->gel.p,
                                           P->gpair.p, P->Khat.p, w.E.p, m->d_fixed.p, w.V64.p, v32, w.M64.p, m32);
        else
          k_assemble_batch<2><<<ga, 128>>>(w.S, P->s, m->d_blkrow.p, m->d_colind.p, P->gptr.p, P->gel.p,
                                           P->gpair.p, P->Khat.p, w.E.p, m->d_fixed.p, w.V64.p, v32, w.M64.p, m32);
      }
      k_ff_part<<<dim3((unsigned)(w.S / 32), kFfChunks), 256>>>((long)m->nDOFAct, w.S, w.F.p, w.ffpart.p);
      k_tol2<<<(w.S + 127) / 128, 128>>>(kFfChunks, w.S, w.ffpart.p, opt.tol, w.tol2.p, w.ff.p);
      g_stats.kernel_launches += 7;
      if (d_u_guess && d_u_guess[k]) {
        UFEM_CUDA_TRY(cudaMemcpyAsync(w.x64.p, d_u_guess[k], n * sizeof(double), cudaMemcpyDeviceToDevice));
      } else {
        UFEM_CUDA_TRY(cudaMemsetAsync(w.x64.p, 0, n * sizeof(double)));
      }
      w.h_ff.assign(w.S, 0.0);
      UFEM_CUDA_TRY(cudaMemcpy(w.h_ff.data(), w.ff.p, w.S * sizeof(double), cudaMemcpyDeviceToHost));
      // a sample without load has u = 0, whatever its guess (fem/fem_eqs.c:108-116)
      for (int s = 0; s < w.nsamp; s++)
        if (std::isfinite(w.h_ff[s]) && !(w.h_ff[s] > 0.0))
          UFEM_CUDA_TRY(cudaMemset2DAsync(w.x64.p + s, w.S * sizeof(double), 0, sizeof(double), m->nDOFAct));
    }
    UFEM_CUDA_TRY(cudaGetLastError());
    g_stats.ms_assemble = t.stop();
  }
  // ---- launch shape: the caller's, else the autotuned one for this batch --
  if (opt.tiles_per_block <= 0 || (implicit_form(opt.precision) && (opt.unroll <= 0 || opt.lane_samples <= 0))) {
    const TuneEntry *t = tune_find(tune_key(nmesh, models, nsamp, opt.precision, coarse_modes(nmesh, models, opt)));
    if (t) {
      if (opt.tiles_per_block <= 0) opt.tiles_per_block = t->tpb;
      if (opt.unroll <= 0) opt.unroll = t->unroll;
      if (opt.lane_samples <= 0) opt.lane_samples = t->lanes;
    }
  }
  // ---- one persistent launch over every mesh -----------------------------
  long its = 0;
  if (opt.precision == 1) rv = run_pcg<float, false, 4>(nmesh, models, W, plans, opt, &its);
  // FP32 implicit form: 4 adjacent samples per lane (one 16-byte load per row)
  else if (opt.precision == 3) rv = run_pcg<float, true, 4>(nmesh, models, W, plans, opt, &its);
  // FP32 vectors and FP32 SpMV products on the implicit form
  else if (opt.precision == 4) rv = run_pcg<float, true, 4, true>(nmesh, models, W, plans, opt, &its);
  // implicit form: 4 samples per lane unless 2 is asked for (measured best on B200)
  else if (opt.precision == 2 && (opt.lane_samples != 2 || coarse_modes(nmesh, models, opt) > 0))
    rv = run_pcg<double, true, 4>(nmesh, models, W, plans, opt, &its);
  else if (opt.precision == 2) rv = run_pcg<double, true, 2>(nmesh, models, W, plans, opt, &its);
  else rv = run_pcg<double, false, 2>(nmesh, models, W, plans, opt, &its);
  if (rv != UFEM_AF_OK) return rv;
  g_stats.pcg_iterations = its;
  // ---- outputs -------------------------------------------------------------
  {
    EvTimer t;
    for (int k = 0; k < nmesh; k++) {
      ufem_model *m = models[k];
      McWork &w = *W[k];
      McPlan *P = plans[k];
      const int nout = (int)P->outs.size();
      if (d_ofld && d_ofld[k] && nout > 0 && w.nsamp > 0) {
        const long tot = (long)nout * w.nsamp;
        if (B == 3)
          k_outputs<3><<<(unsigned)((tot + 127) / 128), 128>>>(
              nout, w.S, w.nsamp, P->olen, P->d_out_type.p, P->d_out_pos.p, P->d_out_row.p, w.x64.p,
              m->d_rowptr.p, m->d_colind.p, P->gptr.p, P->gel.p, P->gpair.p, P->s, P->Khat.p, w.E.p, w.Fraw.p,
              d_ofld[k]);
        else
          k_outputs<2><<<(unsigned)((tot + 127) / 128), 128>>>(
              nout, w.S, w.nsamp, P->olen, P->d_out_type.p, P->d_out_pos.p, P->d_out_row.p, w.x64.p,
              m->d_rowptr.p, m->d_colind.p, P->gptr.p, P->gel.p, P->gpair.p, P->s, P->Khat.p, w.E.p, w.Fraw.p,
              d_ofld[k]);
        g_stats.kernel_launches += 1;
        int eo_launches = 0;
        if ((rv = run_elem_outputs(m, P->eo, w.S, w.nsamp, w.x64.p, w.E.p, d_ifld[k], P->ilen, 0.0, d_ofld[k],
                                   P->olen, &eo_launches)) != UFEM_AF_OK)
          return rv;
        g_stats.kernel_launches += eo_launches;
      }
      if (d_u_out && d_u_out[k])
        UFEM_CUDA_TRY(cudaMemcpyAsync(d_u_out[k], w.x64.p, (size_t)m->nDOFAct * w.S * sizeof(double),
                                      cudaMemcpyDeviceToDevice));
      std::vector<int> st(w.S), itv(w.S);
      UFEM_CUDA_TRY(cudaMemcpy(st.data(), w.state.p, w.S * sizeof(int), cudaMemcpyDeviceToHost));
      UFEM_CUDA_TRY(cudaMemcpy(itv.data(), w.iters.p, w.S * sizeof(int), cudaMemcpyDeviceToHost));
      std::vector<int> hs(w.nsamp);
      std::vector<long> hi(w.nsamp);
      for (int s = 0; s < w.nsamp; s++) {
        switch (st[s]) {
          case ST_CONV: hs[s] = UFEM_ST_CONVERGED; break;
          case ST_BREAK: hs[s] = UFEM_ST_BREAKDOWN; break;
          case ST_NAN: hs[s] = UFEM_ST_NAN; break;
          default: hs[s] = UFEM_ST_MAXIT; break;
        }
        hi[s] = (st[s] == ST_ACTIVE || st[s] == ST_MAXIT) ? its : itv[s];
      }
      if (d_status && d_status[k] && w.nsamp > 0)
        UFEM_CUDA_TRY(cudaMemcpy(d_status[k], hs.data(), w.nsamp * sizeof(int), cudaMemcpyHostToDevice));
      if (d_iters && d_iters[k] && w.nsamp > 0)
        UFEM_CUDA_TRY(cudaMemcpy(d_iters[k], hi.data(), w.nsamp * sizeof(long), cudaMemcpyHostToDevice));
    }
    UFEM_CUDA_TRY(cudaGetLastError());
    g_stats.ms_outputs = t.stop();
  }
  g_stats.ms_total = total.stop();
  return UFEM_AF_OK;
}

}  // namespace ufem

using namespace ufem;

// Times bounded runs (30 PCG iterations) of every candidate launch shape on
// the caller's batch and keeps the fastest for batches of this shape.
extern "C" int ufem_mc_autotune(int nmesh, ufem_model *const *models, const long *nsamp,
                                const double *const *d_ifld, const ufem_mc_options *opt_in, const char *cache_path,
                                ufem_mc_options *best) {
  if (nmesh < 1 || !models || !nsamp || !d_ifld) return UFEM_AF_ERR_EMP;
  ufem_mc_options base;
  if (opt_in) base = *opt_in;
  else ufem_mc_default_options(&base);
  const std::string path = tune_cache_path(cache_path);
  if (!g_tune_loaded) {
    tune_load(path);
    g_tune_loaded = true;
  }
  const int tpbs[] = {3, 6, 12, 24, 48};
  std::vector<int> unrolls, lanes;
  if (implicit_form(base.precision)) {
    unrolls = {2, 4, 8};
    lanes = {2, 4};
    // the coarse correction needs 128-sample groups; the FP32 form holds 4 samples per lane
    if (coarse_modes(nmesh, models, base) > 0 || base.precision >= 3) lanes = {4};
    if (base.precision == 4) unrolls = {2, 4};
  } else {
    unrolls = {4};
    lanes = {0};
  }
  double best_ms = 1e300;
  int best_tpb = 12, best_un = unrolls[0], best_ln = lanes[0];
  for (int ln : lanes)
  for (int tpb : tpbs)
    for (int un : unrolls) {
      ufem_mc_options o = base;
      o.tiles_per_block = tpb;
      o.unroll = un;
      o.lane_samples = ln;
      o.max_iters = 30;
      double per_it = 0.0;
      for (int rep = 0; rep < 2; rep++) {  // the first run also builds the workspace
        int rv = mc_solve_device(nmesh, models, nsamp, d_ifld, nullptr, nullptr, nullptr, nullptr, nullptr, &o);
        if (rv != UFEM_AF_OK) return rv;
        per_it = g_stats.ms_pcg / (double)std::max<long>(1, g_stats.pcg_iterations);
      }
      if (per_it < best_ms) {
        best_ms = per_it;
        best_tpb = tpb;
        best_un = un;
        best_ln = ln;
      }
    }
  const std::string key = tune_key(nmesh, models, nsamp, base.precision, coarse_modes(nmesh, models, base));
  bool found = false;
  for (auto &t : g_tune)
    if (t.key == key) {
      t.tpb = best_tpb; t.unroll = best_un; t.lanes = best_ln; t.ms = best_ms;
      found = true;
    }
  if (!found) g_tune.push_back({key, best_tpb, best_un, best_ln, best_ms});
  tune_save(path);
  if (best) {
    *best = base;
    best->tiles_per_block = best_tpb;
    best->unroll = best_un;
    best->lane_samples = best_ln;
  }
  return UFEM_AF_OK;
}

extern "C" int ufem_mc_set_coarse(ufem_model *m, int nmodes, const double *d_Wc) {
  if (!m) return UFEM_AF_ERR_EMP;
  McPlan *P = get_plan(m);
  if (nmodes == 0) {
    P->cmodes = 0;
    return UFEM_AF_OK;
  }
  if (nmodes < 16 || nmodes > kCoarseMaxModes || nmodes % 16 || !d_Wc) {
    set_error("ufem_mc_set_coarse: nmodes a multiple of 16 up to 128 and a device array of nDOFAct x nmodes");
    return UFEM_AF_ERR_VAL;
  }
  int rv;
  const int n = (int)m->nDOFAct, n64 = (n + 63) / 64, n128 = (n + 127) / 128;
  if ((rv = P->wt1.ensure((size_t)n64 * 64 * nmodes * 2)) || (rv = P->wt3.ensure((size_t)n128 * 128 * nmodes * 2)))
    return rv;
  const long tot = (long)n64 * 64 * nmodes + (long)n128 * 128 * nmodes;
  k_coarse_tiles<<<(unsigned)((tot + 255) / 256), 256>>>(n, nmodes, d_Wc, m->d_fixed.p,
                                                         reinterpret_cast<__nv_bfloat16 *>(P->wt1.p),
                                                         reinterpret_cast<__nv_bfloat16 *>(P->wt3.p), n64, n128);
  UFEM_CUDA_TRY(cudaGetLastError());
  UFEM_CUDA_TRY(cudaDeviceSynchronize());
  P->cmodes = nmodes;
  return UFEM_AF_OK;
}

extern "C" int ufem_mc_solve_device(int nmesh, ufem_model *const *models, const long *nsamp,
                                    const double *const *d_ifld, double *const *d_ofld, int *const *d_status,
                                    long *const *d_iters, const double *const *d_u_guess,
                                    double *const *d_u_out, const ufem_mc_options *opt) {
  return mc_solve_device(nmesh, models, nsamp, d_ifld, d_ofld, d_status, d_iters, d_u_guess, d_u_out, opt);
}

extern "C" int ufem_mc_solve(int nmesh, ufem_model *const *models, const long *nsamp, const double *const *ifld,
                             double *const *ofld, int *const *status, long *const *iters,
                             const double *const *u_guess, const ufem_mc_options *opt) {
  int rv;
  std::vector<std::unique_ptr<DBuf<double>>> di, dof, dg;
  std::vector<std::unique_ptr<DBuf<int>>> ds;
  std::vector<std::unique_ptr<DBuf<long>>> dit;
  std::vector<const double *> pi(nmesh), pg(nmesh, nullptr);
  std::vector<double *> po(nmesh);
  std::vector<int *> ps(nmesh);
  std::vector<long *> pit(nmesh);
  for (int k = 0; k < nmesh; k++) {
    ufem_model *m = models[k];
    di.emplace_back(new DBuf<double>());
    dof.emplace_back(new DBuf<double>());
    dg.emplace_back(new DBuf<double>());
    ds.emplace_back(new DBuf<int>());
    dit.emplace_back(new DBuf<long>());
    if ((rv = di[k]->upload(ifld[k], (size_t)nsamp[k] * m->mc_ilen)) != UFEM_AF_OK) return rv;
    if ((rv = dof[k]->alloc((size_t)nsamp[k] * std::max<long>(1, m->mc_olen))) != UFEM_AF_OK) return rv;
    if ((rv = ds[k]->alloc(nsamp[k])) != UFEM_AF_OK) return rv;
    if ((rv = dit[k]->alloc(nsamp[k])) != UFEM_AF_OK) return rv;
    pi[k] = di[k]->p;
    po[k] = dof[k]->p;
    ps[k] = ds[k]->p;
    pit[k] = dit[k]->p;
    if (u_guess && u_guess[k]) {
      // host guesses are sample-major [nsamp][ndof]; the device layout is [ndof][S]
      const int S = (int)std::max<long>(128, (nsamp[k] + 127) / 128 * 128);
      std::vector<double> t((size_t)m->nDOFAct * S, 0.0);
      for (long s = 0; s < nsamp[k]; s++)
        for (long i = 0; i < m->nDOFAct; i++) t[(size_t)i * S + s] = u_guess[k][(size_t)s * m->nDOFAct + i];
      if ((rv = dg[k]->upload(t.data(), t.size())) != UFEM_AF_OK) return rv;
      pg[k] = dg[k]->p;
    }
  }
  rv = mc_solve_device(nmesh, models, nsamp, pi.data(), po.data(), ps.data(), pit.data(), pg.data(), nullptr, opt);
  if (rv != UFEM_AF_OK) return rv;
  for (int k = 0; k < nmesh; k++) {
    ufem_model *m = models[k];
    if (ofld && ofld[k] && m->mc_olen > 0)
      UFEM_CUDA_TRY(cudaMemcpy(ofld[k], po[k], (size_t)nsamp[k] * m->mc_olen * sizeof(double),
                               cudaMemcpyDeviceToHost));
    if (status && status[k]) UFEM_CUDA_TRY(cudaMemcpy(status[k], ps[k], nsamp[k] * sizeof(int), cudaMemcpyDeviceToHost));
    if (iters && iters[k]) UFEM_CUDA_TRY(cudaMemcpy(iters[k], pit[k], nsamp[k] * sizeof(long), cudaMemcpyDeviceToHost));
  }
  return UFEM_AF_OK;
}
