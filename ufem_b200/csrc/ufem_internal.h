// Internal definitions shared by the host model code and the CUDA kernels of
// libufem_gpu.so.  Not part of the public ABI (include/ufem_gpu.h is).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ufem_gpu.h"

namespace ufem {

constexpr int KNOWN_DOFS = 7;             // DOF slots per node, fem/fem_elem.h:43
constexpr double FEM_ZERO = 1e-17;        // fem/fem.h:59

void set_error(const std::string &msg);

#define UFEM_CUDA_TRY(call)                                                          \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      ::ufem::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));        \
      return (e_ == cudaErrorMemoryAllocation) ? UFEM_AF_ERR_MEM : UFEM_AF_ERR;      \
    }                                                                                \
  } while (0)

// A device allocation owned by the model.
template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  int alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return UFEM_AF_ERR_MEM;
    }
    n = count;
    return UFEM_AF_OK;
  }
  // keeps the allocation when it is already large enough (workspace reuse)
  int ensure(size_t count) {
    if (p && n >= count && count > 0) return UFEM_AF_OK;
    return alloc(count);
  }
  int upload(const T *h, size_t count) {
    int rv = ensure(count);
    if (rv != UFEM_AF_OK) return rv;
    if (count) {
      cudaError_t e = cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        set_error(std::string("cudaMemcpy H2D: ") + cudaGetErrorString(e));
        return UFEM_AF_ERR;
      }
    }
    return UFEM_AF_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { release(); }
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
};

// One support or nodal load line of the input (fem/fem_io.c:97-107).
struct NodalLoad {
  long node, type, dir;
  double val;
};

}  // namespace ufem

// The model: host copies of the reference tables, the derived GPU layout and
// the device state.  Block-sparse layout: block size b = DOFs per node (2 for
// quads, 3 for bricks); block row r = r-th node used by an element (the
// reference numbers DOFs node-major over used nodes, so DOF = b*r + d + 1).
struct ufem_model {
  // ---- host tables -------------------------------------------------------
  long nLen = 0, eLen = 0;
  std::vector<double> xyz;            // nLen*3
  std::vector<long> eType, eRS, eMP;  // eLen
  std::vector<int> enodes;            // eLen*nn node positions
  int nn = 0;                         // nodes per element (4 or 8)
  int b = 0;                          // DOFs per node (2 or 3)
  int etype = 0;                      // 2 = quad, 9 = brick
  std::vector<double> eE, eNu, eThick;  // per-element E, nu, thickness
  std::vector<long> eMat;             // material position per element (for MC)
  std::vector<std::vector<double>> mpVals;  // material records
  std::vector<long> mpTypeH;
  std::vector<long> nID, eID;         // identifiers (names), for MC variable names
  std::vector<long> mpID, rsID;
  std::vector<ufem::NodalLoad> loads;

  // ---- DOF map and pattern -------------------------------------------------
  long nDOFAct = 0;
  std::vector<int> node_rank;         // nLen, block row of a node or -1
  std::vector<int> rank_node;         // nbr
  // the reference's nDOFfld[s], s = node * KNOWN_DOFS + slot: 1-based DOF
  // number, 0 for an unused slot; slots 1..b of every used node, numbered
  // node by node (fem_dofs, fem/fem_sol.c:1263)
  long dof(long s) const {
    if (s < 0 || s >= nLen * ufem::KNOWN_DOFS) return 0;
    const long n = s / ufem::KNOWN_DOFS;
    const int d = (int)(s % ufem::KNOWN_DOFS);
    return (d < b && node_rank[n] >= 0) ? (long)b * node_rank[n] + d + 1 : 0;
  }
  long dof_slots() const { return nLen * ufem::KNOWN_DOFS; }
  int nbr = 0;                        // block rows
  long nnzb = 0;                      // blocks
  // the pattern and the scatter map are built on the device (pattern.cu);
  // these host copies are filled on first use by host_pattern()
  mutable std::vector<int> rowptr, colind, diagblk;
  mutable std::vector<int> emap;      // eLen*nn*nn block index per node pair
  mutable bool host_pattern_ok = false;
  int ncolours = 0;
  std::vector<int> colour_ptr, colour_elems;  // elements grouped by colour
  // wall-clock milliseconds of model set-up: file read, parse, tables,
  // DOF numbering + pattern + colouring, supports/loads, upload
  double ms_ingest[6] = {0, 0, 0, 0, 0, 0};

  // ---- supports / loads ----------------------------------------------------
  std::vector<double> F_loads;        // F after fem_add_loads (host, reference order)
  bool has_nonzero_bc = false;
  std::vector<long> reacNode, reacDof;  // fem_sol_res_alloc order
  std::vector<int> reacRow;           // 0-based DOF index or -1
  std::vector<double> reacFval;       // F value at the time each support was applied
  std::vector<unsigned char> fixedMask;  // nDOFAct, zero-valued supports

  // ---- Monte Carlo variable table (fem/fem_mont.c:866) ---------------------
  long mc_ilen = 0, mc_olen = 0;
  std::vector<long> mc_pos, mc_type, mc_item, mc_sub, mc_iter;

  // ---- device state --------------------------------------------------------
  int device = 0;
  ufem::DBuf<double> d_xyz;
  ufem::DBuf<int> d_enodes, d_emap, d_colour_elems, d_rowptr, d_colind, d_diagblk;
  ufem::DBuf<int> d_blkrow;           // block -> block row
  ufem::DBuf<int> d_noderank;         // node -> block row or -1
  ufem::DBuf<double> d_eE, d_eNu, d_eThick;
  ufem::DBuf<double> d_val;           // nnzb*b*b FP64 K
  ufem::DBuf<double> d_F, d_u;
  ufem::DBuf<unsigned char> d_fixed;
  ufem::DBuf<double> d_sig, d_vm, d_fint;
  bool assembled = false, bcs_applied = false;
  double ms_fill = 0, ms_bc = 0, ms_solve = 0, ms_results = 0;
  std::vector<double> reacVal;
};

namespace ufem {

// host model construction (model.cpp)
int build_model(ufem_model *m);
int setup_loads(ufem_model *m);
int read_input_file(const char *fname, ufem_model **out);
int convert_input_file(const char *text_fname, const char *bin_fname);
int model_from_tables(const ufem_tables *t, ufem_model *m);
int export_rowslot(const ufem_model *m, long *frompos, long *defpos, long *pos, long *len);

// device build of DOF numbering, pattern, scatter map, colouring (pattern.cu)
int gpu_build_pattern(ufem_model *m);
int host_pattern(const ufem_model *m);

// device work (kernels.cu)
int upload_model(ufem_model *m);
int gpu_fill_K(ufem_model *m);
int gpu_element_matrices(ufem_model *m, double *hKe);
int gpu_add_loads(ufem_model *m);
int gpu_add_disps(ufem_model *m);
int gpu_results(ufem_model *m);
int gpu_solve(ufem_model *m, int solver, int stop_rule, double eps, long maxIt, long *iters);

// generic solvers on a CSR matrix already on the device (solve.cu)
struct DevMatrix {
  int B;            // block size (1 = scalar CSR)
  int nbr;          // block rows
  long nnzb;
  const int *rowptr, *colind;
  const double *val;
};
int cg_jacobi_fp64(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt,
                   int stop_rule, long *iters, float *ms);
int bicgstab_jacobi_fp64(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt,
                         int stop_rule, long *iters, float *ms);
int cg_ssor_fp64(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt,
                 int stop_rule, long *iters, float *ms);
// the implicit form of a model's Monte Carlo plan (batch.cu): block row I has
// the contributions [crow[I], crow[I+1]) of cval ([cstride] each: B*B unit
// values, then (multiplier << 32 | block column)); multiplier 0 is the
// constant 1, j >= 1 the ifld column mult_col[j].  F0: loads that no input
// overrides; row ovr_row[j] adds ifld column ovr_var[j].
struct McImplicitView {
  int B = 0, nbr = 0, nmult = 0, cstride = 0;
  const int *crow = nullptr;
  const double *cval = nullptr;
  std::vector<int> mult_col;
  const double *F0 = nullptr;
  std::vector<int> ovr_row, ovr_var;
};
int mc_implicit_view(ufem_model *m, McImplicitView *v);

// MLP training with one step recorded as a CUDA graph (mlp.cu)
int mlp_train_graph(ufem_mlp *p, long ntrain, int bs, const float *d_X, const float *d_T,
                    const std::vector<float> &sched, int epochs, unsigned long long seed, float *loss_first,
                    float *loss_last, long *steps);
int cg_jacobi_mixed(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt, double replace_near,
                    long replace_every, bool fp32_vectors, long *iters, int *replacements, float *ms);

// Element-result outputs of a Monte Carlo table (RES_E, RES_SUM/MAX/MIN/FAIL_E)
// and the general failure function RES_FAIL, as GPU passes (mcout.cu)
struct ElemOutPlan {
  int nagg = 0, npo = 0;
  bool strength = false;  // a RES_FAIL output exists
  int md_col = -1;        // ifld column of MAX_D, -1: none
  std::vector<int> h_apos, h_ppos;
  DBuf<int> akind, acomp, apos;        // aggregates: kind 11..14 / 19, value index, ofld position
  DBuf<int> pel, pip, pcomp, ppos;     // RES_E: element, point, value index, ofld position
  DBuf<unsigned char> enpts;           // stored result points per element
  DBuf<double> fy0;                    // F_YC per element (0: the material holds none)
  DBuf<int> fycol;                     // ifld column that randomises it, -1: none
  DBuf<double> part, upart;            // per (element range, sample) records; max |u| per (row chunk, sample)
};
int stored_points(long eType);
double mat_f_yc(const ufem_model *m, long mat);
// fy_col_by_mat: ifld column of each material's F_YC (nullptr: none)
int build_elem_outputs(const ufem_model *m, ElemOutPlan &P, const std::vector<int> *fy_col_by_mat, int md_col);
// S == 1 (u, E per element) or S a multiple of 128 (x[row*S + s], E[e*S + s]);
// ofld[s*olen + pos]; ifld (device) is read only through the plan's columns
int run_elem_outputs(const ufem_model *m, ElemOutPlan &P, int S, int nsamp, const double *u, const double *E,
                     const double *ifld, long ilen, double md0, double *ofld, long olen, int *launches);

}  // namespace ufem
