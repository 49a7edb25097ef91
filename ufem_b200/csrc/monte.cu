// The Monte Carlo plugin ABI of libfem.so (fem/fem_mont.c:137-866), served by
// the GPU path.  An external driver dlopen()s the library, calls
// monte_init_lib_stuff(input file), then monte_solution() per sample (or the
// batched extension monte_solution_batch()), and reads the outputs.
//
// Like the reference these functions act on one process-wide model and are
// not re-entrant; the variable-name functions return a static buffer.
//
// Behaviour kept from the reference:
//   * input variables (fem/fem_mont.c:715-800): RS (real set value), MAT
//     (material value by type), N (node coordinate), NLD (first nodal load
//     with the node/type/direction), NLPOS (load by position), MAX_D;
//   * outputs (fem/fem_mont.c:514-686): RES_D, RES_R, RES_E, RES_SUM_E,
//     RES_MAX_E, RES_MIN_E, RES_FAIL_E on the stress results;
//   * the solve: zero K/F/u, assemble, loads, supports, PCG, result pass
//     (monte_linear_solver, fem/fem_mont.c:480-508).
// Deliberate differences:
//   * the single-sample solve uses Jacobi PCG with the reference stopping
//     rule (femSolve's solver, fem/fem_sol.c:1722) instead of SSOR PCG;
//   * reactions are reported per sample; the reference never clears
//     resRval between samples (fem/fem_mont.c:483-486), so its RES_R outputs
//     accumulate across calls;
//   * an NLD input is named by its node ID; the reference's name function
//     indexes nlNode[] with the node position (fem/fem_mont.c:203);
//   * if_type 1 (price, which exit()s) and 2 (dynamics) are not on this path
//     and return AF_ERR_TYP.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ufem_internal.h"

namespace ufem {
void drop_plan(const ufem_model *m);
}

using namespace ufem;

namespace {

ufem_model *g_mc = nullptr;
char g_name[257];
double g_max_disp = 0.0;

ElemOutPlan g_eo;        // element outputs of the process-wide model (mcout.cu)
DBuf<double> g_dofld;    // their device output row

// position of value type `vt` in a material record of type `ty`: the type's
// non-repeating list (type 1 fem/fem_m001.c:39, type 5 fem/fem_m005.c:39)
int mat_index(long ty, long vt) {
  static const long t1[7] = {1 /*DENS*/, 2 /*EX*/, 5 /*NU*/, 38 /*ALPHA*/, 37 /*KXX*/, 39 /*C*/, 36 /*PRICE*/};
  static const long t5[8] = {1 /*DENS*/, 2 /*EX*/, 5 /*NU*/, 6 /*G*/, 12 /*F_YC*/, 14 /*F_YT*/, 15 /*F_UC*/,
                             17 /*F_UT*/};
  const long *order = ty == 5 ? t5 : t1;
  const int n = ty == 5 ? 8 : 7;
  for (int i = 0; i < n; i++)
    if (order[i] == vt) return i;
  return -1;
}

const char *dir_name(long sub, bool force) {
  static const char *u[] = {"__", "UX", "UY", "UZ", "RX", "RY", "RZ"};
  static const char *f[] = {"__", "FX", "FY", "FZ", "MX", "MY", "MZ"};
  if (sub < 1 || sub > 6) return "__";
  return force ? f[sub] : u[sub];
}

int apply_inputs(ufem_model *m, const double *ifld) {
  bool geom = false;
  for (long i = 0; i < m->mc_ilen; i++) {
    const long ty = m->mc_type[i], item = m->mc_item[i], sub = m->mc_sub[i], it = m->mc_iter[i];
    const double v = ifld[m->mc_pos[i]];
    switch (ty) {
      case 0:  // MONTE_VTYPE_RS: thickness (RS_HEIGHT = 3) of the elements of real set `item`
        if (sub == 3)
          for (long e = 0; e < m->eLen; e++)
            if (m->eRS[e] == item) m->eThick[e] = v;
        break;
      case 1: {  // MONTE_VTYPE_MAT
        if (item < 0 || item >= (long)m->mpVals.size() || it > 0) break;
        const int idx = mat_index(m->mpTypeH[item], sub);
        if (idx < 0 || idx >= (int)m->mpVals[item].size()) break;  // femGetRepValIndex -> -1
        m->mpVals[item][idx] = v;
        for (long e = 0; e < m->eLen; e++)
          if (m->eMat[e] == item) {
            m->eE[e] = m->mpVals[item].size() > 1 ? m->mpVals[item][1] : 0.0;
            m->eNu[e] = m->mpVals[item].size() > 2 ? m->mpVals[item][2] : 0.0;
          }
        break;
      }
      case 2:  // MONTE_VTYPE_N
        if (item >= 0 && item < m->nLen && sub >= 1 && sub <= 3) {
          m->xyz[3 * item + sub - 1] = v;
          geom = true;
        }
        break;
      case 3:  // MONTE_VTYPE_NLD
        for (auto &l : m->loads)
          if (l.node == item && l.type == sub && l.dir == it) {
            l.val = v;
            break;
          }
        break;
      case 5:  // MONTE_VTYPE_NLPOS
        if (item >= 0 && item < (long)m->loads.size() && m->loads[item].type == sub && m->loads[item].dir == it)
          m->loads[item].val = v;
        break;
      case 7:  // MONTE_VTYPE_MAX_D
        g_max_disp = std::fabs(v);
        break;
      default:
        break;
    }
  }
  int rv;
  if ((rv = setup_loads(m)) != UFEM_AF_OK) return rv;
  if ((rv = m->d_eE.upload(m->eE.data(), m->eE.size())) != UFEM_AF_OK) return rv;
  if ((rv = m->d_eNu.upload(m->eNu.data(), m->eNu.size())) != UFEM_AF_OK) return rv;
  if ((rv = m->d_eThick.upload(m->eThick.data(), m->eThick.size())) != UFEM_AF_OK) return rv;
  if ((rv = m->d_fixed.upload(m->fixedMask.data(), m->fixedMask.size())) != UFEM_AF_OK) return rv;
  if (geom && (rv = m->d_xyz.upload(m->xyz.data(), m->xyz.size())) != UFEM_AF_OK) return rv;
  drop_plan(m);  // the batched plan caches element matrices of the old tables
  return UFEM_AF_OK;
}

// The outputs of the sample just solved in m, as monte_fill_ofld_data writes
// them into the zeroed row `out` (fem/fem_mont.c:514-686): displacement and
// reaction outputs from the host copies, element results and RES_FAIL from
// the GPU element pass (mcout.cu).
int fill_outputs(ufem_model *m, const std::vector<double> &u, double *out) {
  for (long i = m->mc_ilen; i < m->mc_ilen + m->mc_olen; i++) {
    const long ty = m->mc_type[i], item = m->mc_item[i], sub = m->mc_sub[i];
    const long pos = m->mc_pos[i - m->mc_ilen];
    if (pos < 0 || pos >= m->mc_olen) continue;
    double &o = out[pos];
    const bool slot = item >= 0 && item < m->nLen && sub >= 1 && sub <= KNOWN_DOFS;
    const long p = slot ? m->dof(item * KNOWN_DOFS + sub - 1) : 0;
    const double v = p > 0 ? u[p - 1] : 0.0;
    switch (ty) {
      case 8: o = v; break;                                  // RES_D
      case 15: if (o < v) o = v; break;                      // RES_D_MAX
      case 16: if (o > v) o = v; break;                      // RES_D_MIN
      case 17:                                               // RES_D_SUM, fem/fem_mont.c:550-555
        if (slot && p >= 0 && p < m->dof_slots()) o += (double)m->dof(p);
        break;
      case 9:  // RES_R
        for (size_t r = 0; r < m->reacNode.size(); r++)
          if (m->reacNode[r] == item && m->reacDof[r] == sub) {
            o = m->reacVal[r];
            break;
          }
        break;
      default:
        break;  // element results and RES_FAIL below; dynamics outputs are 0
    }
  }
  int rv;
  if ((rv = build_elem_outputs(m, g_eo, nullptr, -1)) != UFEM_AF_OK) return rv;
  if (g_eo.nagg == 0 && g_eo.npo == 0) return UFEM_AF_OK;
  const long olen = m->mc_olen;
  if ((rv = g_dofld.ensure(olen))) return rv;
  UFEM_CUDA_TRY(cudaMemset(g_dofld.p, 0, olen * sizeof(double)));
  int launches = 0;
  if ((rv = run_elem_outputs(m, g_eo, 1, 1, m->d_u.p, m->d_eE.p, nullptr, 0, g_max_disp, g_dofld.p, olen,
                             &launches)) != UFEM_AF_OK)
    return rv;
  std::vector<double> row(olen);
  UFEM_CUDA_TRY(cudaMemcpy(row.data(), g_dofld.p, olen * sizeof(double), cudaMemcpyDeviceToHost));
  for (int q : g_eo.h_apos) out[q] = row[q];
  for (int q : g_eo.h_ppos) out[q] = row[q];
  return UFEM_AF_OK;
}

}  // namespace

extern "C" {

long monte_dlib_interface_type(void) { return 2; }

void monte_nums_of_vars(char *param, long *ilen, long *olen, long *ffunc) {
  (void)param;
  *ilen = g_mc ? g_mc->mc_ilen : 0;
  *olen = g_mc ? g_mc->mc_olen : 0;
  long ff = -1;
  if (g_mc)
    for (long i = 0; i < g_mc->mc_ilen + g_mc->mc_olen; i++)
      if (g_mc->mc_type[i] == 19) ff = i - g_mc->mc_ilen;  // fem/fem_mont.c:895-896
  *ffunc = ff;
}

char *monte_ivar_name(char *param, long pos) {
  (void)param;
  static char empty[] = "empty";
  if (!g_mc || pos < 0 || pos >= g_mc->mc_ilen) return empty;
  const long ty = g_mc->mc_type[pos], item = g_mc->mc_item[pos], sub = g_mc->mc_sub[pos],
             it = g_mc->mc_iter[pos];
  std::memset(g_name, 0, sizeof(g_name));
  switch (ty) {
    case 0:
      snprintf(g_name, 256, "RS_%li_P%li_I%li", item < (long)g_mc->rsID.size() ? g_mc->rsID[item] : item + 1, sub, it);
      break;
    case 1:
      snprintf(g_name, 256, "MAT_%li_P%li_I%li", item < (long)g_mc->mpID.size() ? g_mc->mpID[item] : item + 1, sub,
               it);
      break;
    case 2: {
      const char d = sub == 1 ? 'X' : sub == 2 ? 'Y' : sub == 3 ? 'Z' : '_';
      snprintf(g_name, 256, "N_%li_%c", g_mc->nID[item], d);
      break;
    }
    case 3:
      snprintf(g_name, 256, "NLD_N%li_T%li_D%li", (item >= 0 && item < g_mc->nLen) ? g_mc->nID[item] : item, sub, it);
      break;
    case 5:
      snprintf(g_name, 256, "NLP_%li_POS%li_T%li_D%li", pos + 1, item + 1, sub, it);
      break;
    case 6:
      snprintf(g_name, 256, item == 1 ? "DAMP_ALPHA" : "DAMP_BETA");
      break;
    case 7:
      snprintf(g_name, 256, "MAX_DISP");
      break;
    default:
      return empty;
  }
  return g_name;
}

char *monte_ovar_name(char *param, long pos) {
  (void)param;
  static char empty[] = "empty";
  if (!g_mc || pos < 0 || pos >= g_mc->mc_olen) return empty;
  const long p = pos + g_mc->mc_ilen;
  const long ty = g_mc->mc_type[p], item = g_mc->mc_item[p], sub = g_mc->mc_sub[p], it = g_mc->mc_iter[p];
  const long nid = (item >= 0 && item < g_mc->nLen) ? g_mc->nID[item] : item;
  const long eid = (item >= 0 && item < g_mc->eLen) ? g_mc->eID[item] : item;
  std::memset(g_name, 0, sizeof(g_name));
  switch (ty) {
    case 8: snprintf(g_name, 256, "DISP_%s_%li", dir_name(sub, false), nid); break;
    case 15: snprintf(g_name, 256, "DMAX_%s_%li", dir_name(sub, false), nid); break;
    case 16: snprintf(g_name, 256, "DMIN_%s_%li", dir_name(sub, false), nid); break;
    case 17: snprintf(g_name, 256, "DSUM_%s_%li", dir_name(sub, false), nid); break;
    case 18: snprintf(g_name, 256, "ACCMAX_%s_%li", dir_name(sub, false), nid); break;
    case 9: snprintf(g_name, 256, "REAC_%s_%li", dir_name(sub, true), nid); break;
    case 10: snprintf(g_name, 256, "ERES_E%li_T%li_I%li", eid, sub, it); break;
    case 11: snprintf(g_name, 256, "ERES_SUM_T%li", sub); break;
    case 12: snprintf(g_name, 256, "ERES_MAX_T%li", sub); break;
    case 13: snprintf(g_name, 256, "ERES_MIN_T%li", sub); break;
    case 14: snprintf(g_name, 256, "ERES_FAIL_T%li", sub); break;
    case 19: snprintf(g_name, 256, "RES_FAIL"); break;
    default: return empty;
  }
  return g_name;
}

int monte_init_lib_stuff(char *param) {
  if (param == nullptr || std::strlen(param) < 1) return -1;  // fem/fem_mont.c:443-444
  if (g_mc) {
    drop_plan(g_mc);
    delete g_mc;
    g_mc = nullptr;
  }
  ufem_model *m = nullptr;
  if (ufem_read_input(param, &m) != UFEM_AF_OK) return -1;
  g_mc = m;
  return 0;
}

int monte_clean_lib_stuff(char *param) {
  (void)param;
  if (g_mc) {
    drop_plan(g_mc);
    delete g_mc;
    g_mc = nullptr;
  }
  return 0;
}

int monte_solution(char *param, double *ifld, double *ofld, long if_type) {
  (void)param;
  if (!g_mc) return UFEM_AF_ERR;
  ufem_model *m = g_mc;
  // the reference zeroes the positions held by table rows 0..olen-1
  // (monte_io_var_pos[i-monte_i_len], fem/fem_mont.c:702-705)
  for (long i = 0; i < m->mc_olen; i++)
    if (m->mc_pos[i] >= 0 && m->mc_pos[i] < m->mc_olen) ofld[m->mc_pos[i]] = 0;
  if (if_type != 0) {
    set_error("only the linear static solution (if_type 0) is on this path");
    return UFEM_AF_ERR_TYP;
  }
  int rv;
  if ((rv = apply_inputs(m, ifld)) != UFEM_AF_OK) return rv;
  long iters = 0;
  if ((rv = ufem_fem_solve(m, UFEM_SOLVER_CGWJ, &iters)) != UFEM_AF_OK) return rv;
  std::vector<double> u(m->nDOFAct);
  if ((rv = ufem_get_u(m, u.data())) != UFEM_AF_OK) return rv;
  return fill_outputs(m, u, ofld);
}

int ufem_mc_solve_serial(ufem_model *m, long nsamp, const double *ifld, double *ofld, int *status, long *iters,
                         double tol) {
  if (!m) return UFEM_AF_ERR;
  int rv;
  std::vector<double> u(m->nDOFAct);
  for (long s = 0; s < nsamp; s++) {
    const double *in = ifld + s * m->mc_ilen;
    double *out = ofld + s * m->mc_olen;
    for (long i = 0; i < m->mc_olen; i++)
      if (m->mc_pos[i] >= 0 && m->mc_pos[i] < m->mc_olen) out[m->mc_pos[i]] = 0;
    if ((rv = apply_inputs(m, in)) != UFEM_AF_OK) return rv;
    long it = 0;
    if ((rv = ufem_fill_K(m, 0)) != UFEM_AF_OK) return rv;
    if ((rv = ufem_add_loads(m)) != UFEM_AF_OK) return rv;
    UFEM_CUDA_TRY(cudaMemset(m->d_u.p, 0, m->nDOFAct * sizeof(double)));
    if ((rv = ufem_add_disps(m)) != UFEM_AF_OK) return rv;
    int srv = ufem_solve(m, UFEM_SOLVER_CGWJ, UFEM_STOP_RELRES, tol, 10 * m->nDOFAct, &it);
    if (status) status[s] = srv == UFEM_AF_OK ? UFEM_ST_CONVERGED : UFEM_ST_MAXIT;
    if (iters) iters[s] = it;
    if ((rv = ufem_fill_K(m, 1)) != UFEM_AF_OK) return rv;
    if ((rv = ufem_get_u(m, u.data())) != UFEM_AF_OK) return rv;
    if ((rv = fill_outputs(m, u, out)) != UFEM_AF_OK) return rv;
  }
  return UFEM_AF_OK;
}

int monte_solution_batch(char *param, long nsamp, const double *ifld, double *ofld, long if_type, int *status) {
  (void)param;
  if (!g_mc) return UFEM_AF_ERR;
  if (if_type != 0) {
    set_error("only the linear static solution (if_type 0) is on this path");
    return UFEM_AF_ERR_TYP;
  }
  ufem_model *models[1] = {g_mc};
  const long ns[1] = {nsamp};
  const double *in[1] = {ifld};
  double *out[1] = {ofld};
  int *st[1] = {status};
  return ufem_mc_solve(1, models, ns, in, out, st, nullptr, nullptr, nullptr);
}

}  // extern "C"
