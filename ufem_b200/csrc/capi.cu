// extern "C" entry points of libufem_gpu.so (declared in include/ufem_gpu.h):
// model set-up, the static solve path and the level-1 drop-in solvers that
// take the reference's own row-slot matrix.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "ufem_internal.h"

namespace ufem {
const char *last_error();
double true_relres(const DevMatrix &A, const double *d_b, const double *d_x);
void drop_plan(const ufem_model *m);
}  // namespace ufem

using namespace ufem;

static DevMatrix model_matrix(const ufem_model *m) {
  DevMatrix A;
  A.B = m->b;
  A.nbr = m->nbr;
  A.nnzb = m->nnzb;
  A.rowptr = m->d_rowptr.p;
  A.colind = m->d_colind.p;
  A.val = m->d_val.p;
  return A;
}

static int check_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n < 1) {
    set_error("no CUDA device: libufem_gpu has no CPU fallback");
    return UFEM_AF_ERR;
  }
  return UFEM_AF_OK;
}

extern "C" {

const char *ufem_last_error(void) { return last_error(); }

int ufem_device_info(int *sm_count, int *cc_major, int *cc_minor, long *mem_bytes) {
  int rv = check_device();
  if (rv != UFEM_AF_OK) return rv;
  int dev = 0;
  cudaDeviceProp p;
  UFEM_CUDA_TRY(cudaGetDevice(&dev));
  UFEM_CUDA_TRY(cudaGetDeviceProperties(&p, dev));
  if (sm_count) *sm_count = p.multiProcessorCount;
  if (cc_major) *cc_major = p.major;
  if (cc_minor) *cc_minor = p.minor;
  if (mem_bytes) *mem_bytes = (long)p.totalGlobalMem;
  return UFEM_AF_OK;
}

int ufem_model_create(const ufem_tables *t, ufem_model **out) {
  int rv = check_device();
  if (rv != UFEM_AF_OK) return rv;
  ufem_model *m = new ufem_model();
  rv = model_from_tables(t, m);
  if (rv != UFEM_AF_OK) {
    delete m;
    return rv;
  }
  *out = m;
  return UFEM_AF_OK;
}

int ufem_read_input(const char *fname, ufem_model **out) {
  int rv = check_device();
  if (rv != UFEM_AF_OK) return rv;
  return read_input_file(fname, out);
}

int ufem_convert_input(const char *text_fname, const char *bin_fname) {
  if (!text_fname || !bin_fname) {
    set_error("ufem_convert_input: null file name");
    return UFEM_AF_ERR_VAL;
  }
  return convert_input_file(text_fname, bin_fname);
}

void ufem_model_free(ufem_model *m) {
  if (!m) return;
  drop_plan(m);
  delete m;
}

int ufem_model_set_mc_vars(ufem_model *m, long ilen, long olen, const long *vars) {
  if (!m || ilen < 0 || olen < 0) return UFEM_AF_ERR_VAL;
  m->mc_ilen = ilen;
  m->mc_olen = olen;
  m->mc_pos.clear();
  m->mc_type.clear();
  m->mc_item.clear();
  m->mc_sub.clear();
  m->mc_iter.clear();
  for (long i = 0; i < ilen + olen; i++) {
    m->mc_pos.push_back(vars[5 * i]);
    m->mc_type.push_back(vars[5 * i + 1]);
    m->mc_item.push_back(vars[5 * i + 2]);
    m->mc_sub.push_back(vars[5 * i + 3]);
    m->mc_iter.push_back(vars[5 * i + 4]);
  }
  drop_plan(m);
  return UFEM_AF_OK;
}

long ufem_ndof(const ufem_model *m) { return m ? m->nDOFAct : 0; }

int ufem_get_ndoffld(const ufem_model *m, long *nDOFfld) {
  for (long s = 0; s < m->dof_slots(); s++) nDOFfld[s] = m->dof(s);
  return UFEM_AF_OK;
}

int ufem_export_rowslot(const ufem_model *m, long *frompos, long *defpos, long *pos, long *len) {
  return export_rowslot(m, frompos, defpos, pos, len);
}

int ufem_bsr_shape(const ufem_model *m, long *b, long *nbr, long *nnzb) {
  if (b) *b = m->b;
  if (nbr) *nbr = m->nbr;
  if (nnzb) *nnzb = m->nnzb;
  return UFEM_AF_OK;
}

int ufem_get_bsr_pattern(const ufem_model *m, int *rowptr, int *colind) {
  const int rv = host_pattern(m);
  if (rv != UFEM_AF_OK) return rv;
  if (rowptr) std::memcpy(rowptr, m->rowptr.data(), m->rowptr.size() * sizeof(int));
  if (colind) std::memcpy(colind, m->colind.data(), m->colind.size() * sizeof(int));
  return UFEM_AF_OK;
}

long ufem_num_colours(const ufem_model *m) { return m->ncolours; }

int ufem_get_element_colours(const ufem_model *m, int *colour) {
  if (!colour) return UFEM_AF_OK;
  for (int c = 0; c < m->ncolours; c++)
    for (int k = m->colour_ptr[c]; k < m->colour_ptr[c + 1]; k++) colour[m->colour_elems[k]] = c;
  return UFEM_AF_OK;
}

int ufem_fill_K(ufem_model *m, long mode) {
  if (mode == 0) return gpu_fill_K(m);
  return gpu_results(m);
}

int ufem_add_loads(ufem_model *m) { return gpu_add_loads(m); }

int ufem_add_disps(ufem_model *m) { return gpu_add_disps(m); }

int ufem_solve(ufem_model *m, int solver, int stop_rule, double eps, long maxIt, long *iters) {
  if (!m->assembled) {
    set_error("solve before fill_K");
    return UFEM_AF_ERR;
  }
  if (maxIt <= 0) maxIt = m->nDOFAct;  // femSolve passes nDOFAct (fem/fem_sol.c:1722)
  DevMatrix A = model_matrix(m);
  float ms = 0;
  long it = 0;
  int rv;
  if (solver == UFEM_SOLVER_CGWJ_MIXED) {
    int outer = 0;
    // FP64 work vectors with the FP32 matrix copy: on the 80x20x20 beam 982
    // iterations against 1,112 with FP32 vectors (363 in FP64), on the
    // 128x128x64 block 661 against 689 (592), and faster per iteration
    rv = cg_jacobi_mixed(A, m->d_F.p, m->d_u.p, eps, maxIt, 1e-2, 50, false, &it, &outer, &ms);
  } else if (solver == UFEM_SOLVER_BICG) {
    rv = bicgstab_jacobi_fp64(A, m->d_F.p, m->d_u.p, eps, maxIt, stop_rule, &it, &ms);
  } else if (solver == UFEM_SOLVER_SSOR) {
    rv = cg_ssor_fp64(A, m->d_F.p, m->d_u.p, eps, maxIt, stop_rule, &it, &ms);
  } else {
    rv = cg_jacobi_fp64(A, m->d_F.p, m->d_u.p, eps, maxIt, stop_rule, &it, &ms);
    // the true-residual rule: restart from the current x while the FP64
    // residual |b - A x| / |b| is still above eps (recursive-residual drift)
    long total = it;
    for (int restart = 0; rv == UFEM_AF_OK && stop_rule == UFEM_STOP_RELRES && restart < 4; restart++) {
      double rr = true_relres(A, m->d_F.p, m->d_u.p);
      if (!(rr > eps)) break;
      float ms2 = 0;
      rv = cg_jacobi_fp64(A, m->d_F.p, m->d_u.p, eps, maxIt - total, stop_rule, &it, &ms2);
      total += it;
      ms += ms2;
    }
    it = total;
  }
  m->ms_solve = ms;
  if (iters) *iters = it;
  return rv;
}

int ufem_fem_solve(ufem_model *m, int solver, long *iters) {
  int rv;
  if ((rv = ufem_fill_K(m, 0)) != UFEM_AF_OK) return rv;
  if ((rv = ufem_add_loads(m)) != UFEM_AF_OK) return rv;
  // u starts at zero; the supports then write their prescribed values into
  // it (femApplyDisp, fem/fem_loads.c:170, :240), which is CG's initial guess
  UFEM_CUDA_TRY(cudaMemset(m->d_u.p, 0, m->nDOFAct * sizeof(double)));
  if ((rv = ufem_add_disps(m)) != UFEM_AF_OK) return rv;
  rv = ufem_solve(m, solver, UFEM_STOP_REFERENCE, FEM_ZERO / 10000.0, m->nDOFAct, iters);
  if (rv != UFEM_AF_OK) return rv;
  return ufem_fill_K(m, 1);
}

int ufem_get_u(const ufem_model *m, double *u) {
  UFEM_CUDA_TRY(cudaMemcpy(u, m->d_u.p, m->nDOFAct * sizeof(double), cudaMemcpyDeviceToHost));
  return UFEM_AF_OK;
}

int ufem_set_u(ufem_model *m, const double *u) {
  UFEM_CUDA_TRY(cudaMemcpy(m->d_u.p, u, m->nDOFAct * sizeof(double), cudaMemcpyHostToDevice));
  return UFEM_AF_OK;
}

int ufem_get_F(const ufem_model *m, double *F) {
  UFEM_CUDA_TRY(cudaMemcpy(F, m->d_F.p, m->nDOFAct * sizeof(double), cudaMemcpyDeviceToHost));
  return UFEM_AF_OK;
}

int ufem_get_K_values(const ufem_model *m, double *val) {
  UFEM_CUDA_TRY(cudaMemcpy(val, m->d_val.p, m->d_val.n * sizeof(double), cudaMemcpyDeviceToHost));
  return UFEM_AF_OK;
}

int ufem_get_element_matrices(ufem_model *m, double *Ke) { return gpu_element_matrices(m, Ke); }

int ufem_get_stresses(const ufem_model *m, double *sig, double *von_mises) {
  if (!m->d_sig.p) {
    set_error("no results: call ufem_fill_K(m, 1) first");
    return UFEM_AF_ERR;
  }
  if (sig) UFEM_CUDA_TRY(cudaMemcpy(sig, m->d_sig.p, m->d_sig.n * sizeof(double), cudaMemcpyDeviceToHost));
  if (von_mises) UFEM_CUDA_TRY(cudaMemcpy(von_mises, m->d_vm.p, m->d_vm.n * sizeof(double), cudaMemcpyDeviceToHost));
  return UFEM_AF_OK;
}

long ufem_num_reactions(const ufem_model *m) { return (long)m->reacNode.size(); }

int ufem_get_reactions(const ufem_model *m, long *node, long *dof, double *val) {
  for (size_t r = 0; r < m->reacNode.size(); r++) {
    if (node) node[r] = m->reacNode[r];
    if (dof) dof[r] = m->reacDof[r];
    if (val) val[r] = r < m->reacVal.size() ? m->reacVal[r] : 0.0;
  }
  return UFEM_AF_OK;
}

int ufem_get_ingest_ms(const ufem_model *m, double *ms) {
  if (ms) std::memcpy(ms, m->ms_ingest, sizeof(m->ms_ingest));
  return UFEM_AF_OK;
}

int ufem_get_phase_ms(const ufem_model *m, double *fill_ms, double *bc_ms, double *solve_ms, double *results_ms) {
  if (fill_ms) *fill_ms = m->ms_fill;
  if (bc_ms) *bc_ms = m->ms_bc;
  if (solve_ms) *solve_ms = m->ms_solve;
  if (results_ms) *results_ms = m->ms_results;
  return UFEM_AF_OK;
}

}  // extern "C"

// ---- level-1 drop-in solvers on the reference's row-slot matrix -------------

namespace {

// Row-slot tMatrix (fem/fem_math.h:47-57, 1-based columns, 0 ends a row) ->
// CSR on the device (B = 1).  Rows keep the reference's in-row order.
struct RowSlotCsr {
  DBuf<int> rowptr, colind;
  DBuf<double> val, b, x;
  DevMatrix A;
  int load(long rows, const long *frompos, const long *defpos, const long *pos, const double *data,
           const double *hb, const double *hx) {
    std::vector<int> rp(rows + 1, 0), ci;
    std::vector<double> v;
    for (long i = 0; i < rows; i++) {
      for (long j = frompos[i]; j < frompos[i] + defpos[i]; j++) {
        if (pos[j] <= 0) break;
        ci.push_back((int)(pos[j] - 1));
        v.push_back(data[j]);
      }
      rp[i + 1] = (int)ci.size();
    }
    int rv;
    if ((rv = rowptr.upload(rp.data(), rp.size())) != UFEM_AF_OK) return rv;
    if ((rv = colind.upload(ci.data(), ci.size())) != UFEM_AF_OK) return rv;
    if ((rv = val.upload(v.data(), v.size())) != UFEM_AF_OK) return rv;
    if ((rv = b.upload(hb, rows)) != UFEM_AF_OK) return rv;
    if ((rv = x.upload(hx, rows)) != UFEM_AF_OK) return rv;
    A.B = 1;
    A.nbr = (int)rows;
    A.nnzb = (long)ci.size();
    A.rowptr = rowptr.p;
    A.colind = colind.p;
    A.val = val.p;
    return UFEM_AF_OK;
  }
};

template <typename F>
int rowslot_solve(F solver, long rows, const long *frompos, const long *defpos, const long *pos,
                  const double *data, const double *b, double *x, double eps, long maxIt) {
  int rv = check_device();
  if (rv != UFEM_AF_OK) return rv;
  if (rows <= 0) return UFEM_AF_ERR_SIZ;
  RowSlotCsr m;
  if ((rv = m.load(rows, frompos, defpos, pos, data, b, x)) != UFEM_AF_OK) return rv;
  long it = 0;
  float ms = 0;
  rv = solver(m.A, m.b.p, m.x.p, eps, maxIt, UFEM_STOP_REFERENCE, &it, &ms);
  cudaError_t e = cudaMemcpy(x, m.x.p, rows * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    return UFEM_AF_ERR;
  }
  return rv;
}

}  // namespace

extern "C" {

int ufem_eqs_cgwj(long rows, const long *frompos, const long *defpos, const long *pos, const double *data,
                  const double *b, double *x, double eps, long maxIt) {
  return rowslot_solve(cg_jacobi_fp64, rows, frompos, defpos, pos, data, b, x, eps, maxIt);
}

int ufem_eqs_bicgs(long rows, const long *frompos, const long *defpos, const long *pos, const double *data,
                   const double *b, double *x, double eps, long maxIt) {
  return rowslot_solve(bicgstab_jacobi_fp64, rows, frompos, defpos, pos, data, b, x, eps, maxIt);
}

int ufem_eqs_cgwssor(long rows, const long *frompos, const long *defpos, const long *pos, const double *data,
                     const double *b, double *x, double eps, long maxIt) {
  return rowslot_solve(cg_ssor_fp64, rows, frompos, defpos, pos, data, b, x, eps, maxIt);
}

}  // extern "C"
