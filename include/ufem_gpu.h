/*
 * ufem_gpu.h -- C ABI of libufem_gpu.so, the B200 (sm_100a) implementation of
 * uFEM's linear static solve path: element stiffness integration (4-node
 * plane quad, 8-node brick), assembly into a block-sparse K, supports and
 * nodal loads, Jacobi-preconditioned CG / BiCGStab / SSOR-CG, the result pass
 * (stresses, internal forces, reactions) and the Monte Carlo plugin ABI.
 *
 * Plain C types only: pointers, sizes, error codes.  Every function returns
 * the reference's AF_* codes (fem/fem.h:41-52).  There is no CPU fallback:
 * a missing or failing GPU gives AF_ERR / AF_ERR_MEM.
 *
 * Each entry point names the reference interface it replaces.
 */
#ifndef UFEM_GPU_H
#define UFEM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* return codes, identical to fem/fem.h:41-52 */
#define UFEM_AF_OK       0
#define UFEM_AF_ERR     (-1)
#define UFEM_AF_ERR_IO  (-2)
#define UFEM_AF_ERR_VAL (-3)
#define UFEM_AF_ERR_MEM (-4)
#define UFEM_AF_ERR_TYP (-5)
#define UFEM_AF_ERR_SIZ (-9)
#define UFEM_AF_ERR_SML (-10)
#define UFEM_AF_ERR_BIG (-11)
#define UFEM_AF_ERR_EMP (-12)
#define UFEM_AF_ERR_ZER (-13)

/* solver selection, as femSolve picks it (fem/fem_sol.c:1716-1730) */
#define UFEM_SOLVER_CGWJ  0   /* femEqsCGwJ    fem/fem_eqs.c:88   */
#define UFEM_SOLVER_SSOR  1   /* femEqsCGwSSOR fem/fem_eqs.c:1001 */
#define UFEM_SOLVER_BICG  2   /* femEqsBiCCSwJ fem/fem_eqs.c:262  */
#define UFEM_SOLVER_CGWJ_MIXED 3 /* Jacobi PCG on an FP32 copy of the matrix (FP64 vectors and
                                    sums), FP64 true-residual replacement without a Krylov
                                    restart (no reference counterpart); always stops on the
                                    FP64 true residual |b - Ax| <= eps |b| */

/* stopping rules */
#define UFEM_STOP_REFERENCE 0 /* |r| <= eps(|A||x| + |b|) with the recursive r
                                 and |A| = max row 2-norm, fem/fem_eqs.c:202-207 */
#define UFEM_STOP_RELRES    1 /* true residual |b - A x| / |b| <= eps (FP64)  */

/* per-sample status words of the batched Monte Carlo solve */
#define UFEM_ST_CONVERGED   0
#define UFEM_ST_MAXIT       1 /* iteration cap reached (the reference's AF_ERR) */
#define UFEM_ST_BREAKDOWN   2 /* p.q <= 0 or a zero pivot */
#define UFEM_ST_NAN         3 /* non-finite residual */
#define UFEM_ST_FALLBACK    4 /* warm start regressed; solved again from zero */

/*
 * Model tables.  Mirrors the flat global tables that femReadInput fills
 * (fem/fem_io.c:380-590; declarations fem/fem_data.c): every index is a
 * 0-based position, as in the reference's preparsed input.
 */
typedef struct ufem_tables {
  long nLen;                 /* nodes */
  const double *n_x, *n_y, *n_z;
  long eLen;                 /* elements */
  const long *eType;         /* element type: 2 (quad), 9 or 10 (brick) */
  const long *eRS;           /* real set position per element */
  const long *eMP;           /* material position per element */
  const long *eFrom;         /* start of the element's nodes in eNodesL */
  const long *eNodesL;       /* node positions */
  long rsLen;                /* real sets */
  const long *rsType, *rsFrom;
  long rsLenL;
  const double *rsValL;
  long mpLen;                /* materials (type 1, values DENS EX NU ...) */
  const long *mpType, *mpFrom;
  long mpLenL;
  const double *mpValL;
  long nlLen;                /* nodal loads and supports */
  const long *nlNode, *nlType, *nlDir;
  const double *nlVal;
} ufem_tables;

typedef struct ufem_model ufem_model;

/* ---- model set-up ------------------------------------------------------ */

/* Builds a model from the tables: DOF numbering (fem_dofs, fem/fem_sol.c:1263),
 * the block-sparse pattern, element colouring and the element->block scatter
 * map; uploads everything to the current CUDA device. */
int ufem_model_create(const ufem_tables *t, ufem_model **out);

/* Reads a preparsed uFEM input file (femReadInput, fem/fem_io.c:380, with
 * femPreparsedData = AF_YES) including its Monte Carlo section
 * (fem_monte_read_data, fem/fem_mont.c:866), then ufem_model_create.  A file
 * written by ufem_convert_input (it starts with "UFEMBIN1") is read in its
 * binary form: the same tables, no text parsing.  monte_init_lib_stuff reads
 * through this function, so it takes either form. */
int ufem_read_input(const char *fname, ufem_model **out);

/* Writes the tables of an input file (text or binary) to bin_fname in the
 * binary form: "UFEMBIN1", a uint32 byte-order mark 0x01020304, then 28
 * arrays (int64 count, then int64 or float64 items, little-endian): real
 * sets, materials, nodes, elements, nodal loads and the Monte Carlo table.
 * Host only; needs no GPU.  No counterpart in the reference (its reader is
 * text only, femReadInput fem/fem_io.c:380-635). */
int ufem_convert_input(const char *text_fname, const char *bin_fname);

void ufem_model_free(ufem_model *m);

/* Attaches a Monte Carlo variable table to a model built from tables: the
 * rows of the input file's Monte Carlo section (fem_monte_read_data,
 * fem/fem_mont.c:866-905), vars[(ilen+olen)*5] = (position, type, item,
 * subitem, subitem iteration) per variable, inputs first. */
int ufem_model_set_mc_vars(ufem_model *m, long ilen, long olen, const long *vars);

/* nDOFAct (fem/fem_sol.c:46) and nDOFfld[nLen*7] (fem/fem_sol.c:1263-1395) */
long ufem_ndof(const ufem_model *m);
int  ufem_get_ndoffld(const ufem_model *m, long *nDOFfld);

/* The reference's row-slot pattern (fem_sol_alloc + femKhit + the first-touch
 * column order of femMatPutAdd, fem/fem_math.c:185-236): frompos[rows],
 * defpos[rows], pos[len] with 1-based columns and 0 in unused slots.  Call
 * with pos == NULL to get *len. */
int ufem_export_rowslot(const ufem_model *m, long *frompos, long *defpos, long *pos, long *len);

/* Block-sparse pattern used on the GPU: block size b (2 quad, 3 brick),
 * nbr block rows (= used nodes), nnzb blocks; rowptr[nbr+1], colind[nnzb]. */
int ufem_bsr_shape(const ufem_model *m, long *b, long *nbr, long *nnzb);
int ufem_get_bsr_pattern(const ufem_model *m, int *rowptr, int *colind);
long ufem_num_colours(const ufem_model *m);
/* the colour of every element (eLen ints): elements of one colour share no
 * node, and the assembly adds the colours in order */
int ufem_get_element_colours(const ufem_model *m, int *colour);

/* ---- the static path (replaces femSolve's body, fem/fem_sol.c:1655-1760) -- */

/* fem_fill_K (fem/fem_sol.c:897).  mode 0: integrate every element and
 * assemble K on the GPU.  mode 1: the result pass -- integration-point
 * stresses, internal forces and reactions from the current u. */
int ufem_fill_K(ufem_model *m, long mode);

/* fem_add_loads(0) (fem/fem_sol.c:1119): type-3 nodal forces into F. */
int ufem_add_loads(ufem_model *m);

/* fem_add_disps(AF_YES,0) (fem/fem_sol.c:1195): type-1 supports; zero values
 * zero the row and column and put 1 on the diagonal (fem/fem_loads.c:158-166). */
int ufem_add_disps(ufem_model *m);

/* femEqsCGwJ / femEqsCGwSSOR / femEqsBiCCSwJ on the assembled K, F, u.
 * maxIt <= 0 means nDOFAct (femSolve's choice).  *iters gets the count. */
int ufem_solve(ufem_model *m, int solver, int stop_rule, double eps, long maxIt, long *iters);

/* The whole femSolve sequence: fill_K(0), loads, supports, solve with the
 * reference's stopping rule, fill_K(1). */
int ufem_fem_solve(ufem_model *m, int solver, long *iters);

/* results and intermediates (host copies) */
int ufem_get_u(const ufem_model *m, double *u);
int ufem_set_u(ufem_model *m, const double *u);
int ufem_get_F(const ufem_model *m, double *F);
int ufem_get_K_values(const ufem_model *m, double *val);  /* nnzb*b*b, BSR order */
/* every element matrix as the element kernel computes it, eLen*s*s
 * (s = 8 quad, 24 brick); debugging/parity aid */
int ufem_get_element_matrices(ufem_model *m, double *Ke);
/* integration-point stresses: quad eLen*4*3 (SX,SY,SXY), brick eLen*27*6
 * (SX,SY,SZ,SYZ,SZX,SXY); von Mises per point: eLen*4 or eLen*27 */
int ufem_get_stresses(const ufem_model *m, double *sig, double *von_mises);
/* reactions in the order of fem_sol_res_alloc (fem/fem_sol.c:676-722) */
long ufem_num_reactions(const ufem_model *m);
int ufem_get_reactions(const ufem_model *m, long *node, long *dof, double *val);
/* wall-clock milliseconds of the model's set-up by ufem_read_input or
 * ufem_model_from_tables, six stages: [0] file read, [1] parse, [2] host
 * tables, [3] DOF numbering + block pattern + scatter map + element colouring
 * (device kernels), [4] supports and loads, [5] upload of the rest */
int ufem_get_ingest_ms(const ufem_model *m, double *ms);
/* timing of the last call of each phase, milliseconds (CUDA events) */
int ufem_get_phase_ms(const ufem_model *m, double *fill_ms, double *bc_ms, double *solve_ms,
                      double *results_ms);

/* ---- level-1 drop-in on the reference's own matrix (fem/fem_math.h:150-152) --
 * a: the reference's MAT_SPAR tMatrix fields (rows, frompos[rows],
 * defpos[rows], pos[] 1-based with 0 ending a row, data[]); b, x: VEC_FULL
 * data of length rows; x is the initial guess and the result.  Same
 * semantics and return codes as the reference functions. */
int ufem_eqs_cgwj(long rows, const long *frompos, const long *defpos, const long *pos,
                  const double *data, const double *b, double *x, double eps, long maxIt);
int ufem_eqs_bicgs(long rows, const long *frompos, const long *defpos, const long *pos,
                   const double *data, const double *b, double *x, double eps, long maxIt);
int ufem_eqs_cgwssor(long rows, const long *frompos, const long *defpos, const long *pos,
                     const double *data, const double *b, double *x, double eps, long maxIt);

/* Jacobi PCG that allocates nothing.  No counterpart in the reference: it
 * serves callers that may not allocate device memory while they solve -- an
 * application whose own allocator owns the device pool, a solve issued from
 * inside another GPU library's callback, a loop that must avoid cudaMalloc's
 * implicit synchronisation.  Same algorithm, stopping rule and return codes
 * as ufem_eqs_cgwj, but the matrix is the GPU block-sparse form already in
 * device memory: block size B (1 = plain CSR), nbr block rows, d_rowptr
 * [nbr+1] and d_colind (0-based, int32), d_val (nnzb*B*B doubles, row-major
 * blocks); d_b and d_x (initial guess in, solution out) are device vectors
 * of nbr*B doubles.  All scratch lives in one array built into the library:
 * at most 131,072 rows (larger systems return AF_ERR_SIZ), about 6.3 MB held
 * on every GPU where the library's solver code is loaded -- the first use of
 * any of its solvers on a device (this function's first call included) loads
 * that code with the array, and both stay until the process exits; a caller
 * that must reserve nothing later makes one solve through any entry point at
 * set-up.  Every call shares the array, and two solves whose kernels
 * overlapped on the GPU would race on it; within one process an internal
 * lock serialises the calls and each call returns only after its kernels
 * have finished.  It runs on the legacy default stream with synchronous
 * copies.  The first call on each device looks the array's address up
 * (cudaGetSymbolAddress); make that first call before any stream capture
 * begins. */
int ufem_eqs_cgwj_noalloc(int B, int nbr, const int *d_rowptr, const int *d_colind, const double *d_val,
                          const double *d_b, double *d_x, double eps, long maxIt, long *iters);

/* ---- Monte Carlo plugin ABI (fem/fem_mont.c:137-866) --------------------- */
long  monte_dlib_interface_type(void);                                  /* :137 */
void  monte_nums_of_vars(char *param, long *ilen, long *olen, long *ffunc); /* :146 */
char *monte_ivar_name(char *param, long pos);                           /* :158 */
char *monte_ovar_name(char *param, long pos);                           /* :256 */
int   monte_init_lib_stuff(char *param);                                /* :424 */
int   monte_clean_lib_stuff(char *param);                               /* :471 */
int   monte_solution(char *param, double *ifld, double *ofld, long if_type); /* :694 */

/* Batched extension (no reference counterpart): nsamp samples of the model
 * loaded by monte_init_lib_stuff in one GPU launch.  ifld[nsamp*ilen],
 * ofld[nsamp*olen], status[nsamp] (UFEM_ST_*).  Solves to the relative
 * residual of ufem_mc_set_options (default 1e-8). */
int monte_solution_batch(char *param, long nsamp, const double *ifld, double *ofld,
                         long if_type, int *status);

/* Options of the batched solve.  precision 0: FP64 PCG on an explicit FP64
 * matrix per sample; 1: FP32 PCG (FP32 matrix and work vectors) with the
 * solution kept in FP64 and the residual replaced by the true FP64 residual
 * f - K u from time to time; 2: FP64 PCG with no per-sample matrix -- every
 * block is formed inside the PCG kernel from the mesh's unit-E element blocks
 * (summed per random E variable) times the sample's E values, which holds
 * because K_e is linear in E for the isotropic material; 3: the same implicit
 * form with FP32 work vectors (r, z, p, q, the diagonal) and FP64 products,
 * FP64 solution and FP64 true-residual replacement as in 1; 4: as 3 with the
 * SpMV's products and sums in FP32 (FP32 unit blocks and multipliers: the
 * inner FP32 matrix) -- fastest with a warm start and the coarse space; it
 * needs a starting guess for every mesh of the launch: without one the
 * launch runs in precision 3 (and the warm start's fallback re-solves in
 * precision 3).  A sample converges when its true relative residual
 * |f - K u| / |f| <= tol. */
typedef struct ufem_mc_options {
  int precision;
  double tol;
  long max_iters;            /* PCG iteration cap per sample */
  long replace_every;        /* at most this many iterations between FP64 residual replacements */
  double replace_near;       /* also replace once the recursive residual has dropped by this factor
                                since the last replacement, and when it reaches tol */
  int use_graphs;            /* reserved */
  int tiles_per_block;       /* work tiles per persistent block and phase (0: the autotuned or default choice) */
  int unroll;                /* precision 2: neighbour gathers issued together, 2, 4 or 8 (0: tuned or 2) */
  int lane_samples;          /* precision 2: samples per lane, 2 or 4 (a sample group is 32x that;
                                0: tuned or 4) */
  int coarse;                /* precision 2: apply the model's coarse space (ufem_mc_set_coarse)
                                when it has one (default 1); forces 4 samples per lane */
} ufem_mc_options;
void ufem_mc_default_options(ufem_mc_options *o);

/* Handle-based batched Monte Carlo over several meshes of uneven size in one
 * launch.  models[k] must carry a Monte Carlo variable table.  For mesh k:
 * ifld[k] is nsamp[k]*ilen_k, ofld[k] nsamp[k]*olen_k, status[k] nsamp[k],
 * iters[k] (may be NULL) nsamp[k] iteration counts.  u_guess[k] (may be NULL,
 * or NULL entries) gives nsamp[k]*nDOFAct initial guesses. */
int ufem_mc_solve(int nmesh, ufem_model *const *models, const long *nsamp,
                  const double *const *ifld, double *const *ofld, int *const *status,
                  long *const *iters, const double *const *u_guess, const ufem_mc_options *opt);

/* The plain method: the same samples solved one at a time, each by FP64
 * assembly (fem_fill_K), supports and the persistent FP64 Jacobi PCG to the
 * true relative residual tol -- what monte_solution does per call
 * (fem/fem_mont.c:694), kept as the comparison baseline of the batched
 * solve.  Arguments as ufem_mc_solve for one mesh. */
int ufem_mc_solve_serial(ufem_model *m, long nsamp, const double *ifld, double *ofld, int *status, long *iters,
                         double tol);

/* Same, with every input and output already in device memory (for timing the
 * kernels without host transfers).  d_u_guess[k] and d_u_out[k] (either may
 * be NULL) are [nDOFAct][S] with S = nsamp[k] rounded up to a multiple of
 * 128 -- DOF-major, sample fastest, the solver's own layout. */
int ufem_mc_solve_device(int nmesh, ufem_model *const *models, const long *nsamp,
                         const double *const *d_ifld, double *const *d_ofld, int *const *d_status,
                         long *const *d_iters, const double *const *d_u_guess,
                         double *const *d_u_out, const ufem_mc_options *opt);

/* Coarse space of the batched solve's preconditioner (no reference
 * counterpart): with d_Wc an nDOFAct x nmodes row-major FP64 device array,
 * precision-2 solves of this model use M^-1 = D^-1 + Wc Wc^T (D the Jacobi
 * diagonal of each sample) -- an additive two-level preconditioner; with
 * Wc = Phi L^-T, L L^T = Phi^T K Phi, it corrects the residual on span(Phi).
 * Both products run on the tensor cores (BF16 operands, FP32 accumulation);
 * the iterate, residual and stopping test stay FP64.  nmodes: a multiple of
 * 16, at most 128; 0 removes the coarse space.  Rows of supported DOFs are
 * ignored.  The warm start sets one from its POD basis after training. */
int ufem_mc_set_coarse(ufem_model *m, int nmodes, const double *d_Wc);

/* Autotuner of the batched solve's launch shape (no reference counterpart):
 * times bounded runs (30 PCG iterations) of every candidate -- work tiles per
 * persistent block 3..48 and, for precision 2, 2/4/8 neighbour gathers in
 * flight per warp and 2/4 samples per lane -- on the given batch (device inputs as for
 * ufem_mc_solve_device), keeps the fastest for batches of this shape (device,
 * precision, element family, block rows and padded sample count of every
 * mesh) in memory and in the text file cache_path (NULL: $UFEM_TUNE_CACHE,
 * else ~/.cache/ufem_b200_tune.txt), and returns it in *best.  Later solves
 * whose options leave tiles_per_block / unroll / lane_samples at 0 use the
 * cached choice. */
int ufem_mc_autotune(int nmesh, ufem_model *const *models, const long *nsamp, const double *const *d_ifld,
                     const ufem_mc_options *opt, const char *cache_path, ufem_mc_options *best);

/* Statistics of the last ufem_mc_solve*: kernel milliseconds of the inner
 * PCG, FP64 refinement, assembly and outputs, the number of inner PCG
 * iterations run, the algorithmic bytes moved by the PCG kernels, and the
 * number of kernels launched. */
typedef struct ufem_mc_stats {
  double ms_assemble, ms_pcg, ms_refine, ms_outputs, ms_total;
  long pcg_iterations;       /* inner iterations executed (max over samples) */
  double pcg_bytes;          /* algorithmic bytes of all PCG iterations */
  double spmv_bytes;         /* algorithmic bytes of the SpMV phases only */
  long kernel_launches;
  long pcg_launches;         /* PCG solves launched (one per refinement step; a precision-4
                                coarse-corrected solve runs as two kernel launches per
                                iteration and counts once here, each launch in kernel_launches) */
  double pcg_launch_ms[16];  /* their durations (CUDA events around each launch) */
  int tiles_per_block, unroll, lane_samples;  /* the launch shape used */
  int coarse_modes;          /* modes of the coarse correction applied (0: Jacobi alone) */
  /* phase profile of the persistent PCG launches (global timer): per phase
   * -- 0 initial true residual, 1 S (q = A p, p.q), 2 U (x, r, z updates),
   * 3 R (true-residual replacement), 4 C1 (c = Wc^T r), 5 C3 (z += Wc c) --
   * the wall time from the phase's start to the next phase's start (grid
   * barrier included) and the mean time a block spent on its work items */
  double phase_wall_ms[6], phase_busy_ms[6];
  long true_residual_passes; /* R phases run */
} ufem_mc_stats;
int ufem_mc_get_stats(ufem_mc_stats *s);

/* ---- learned warm start: the MLP (no counterpart in the reference; the
 * closest hook is the disabled warm start of monte_linear_solver,
 * fem/fem_mont.c:493-504) ---------------------------------------------------
 * n_in -> n_hidden -> n_hidden -> n_out, GELU, mean-squared-error training
 * with Adam.  Every product runs on the tensor cores (tcgen05, BF16 operands,
 * FP32 accumulation); master weights FP32.  Parameters flat: W1 [n_hidden]
 * [32] (inputs zero-padded to 32), b1, W2 [n_hidden][n_hidden], b2,
 * W3 [n_out][n_hidden], b3.  d_* are device pointers, row-major FP32. */
typedef struct ufem_mlp ufem_mlp;
int  ufem_mlp_create(int n_in, int n_hidden, int n_out, unsigned long long seed, ufem_mlp **out);
void ufem_mlp_free(ufem_mlp *p);
long ufem_mlp_num_params(const ufem_mlp *p);
int  ufem_mlp_get_params(const ufem_mlp *p, float *h_params);
int  ufem_mlp_set_params(ufem_mlp *p, const float *h_params);
int  ufem_mlp_forward(ufem_mlp *p, long nbatch, const float *d_x, float *d_y);
int  ufem_mlp_gradients(ufem_mlp *p, long nbatch, const float *d_x, const float *d_t, float *h_grad, float *loss);
int  ufem_mlp_train_step(ufem_mlp *p, long nbatch, const float *d_x, const float *d_t, float lr, float *loss);
/* C [M x N] = A [M x K] . B [N x K]^T, BF16 in, FP32 out, on the tensor
 * cores (the GEMM of the MLP, exposed for its tests); N a multiple of 16,
 * at most 256. */
int  ufem_tc_gemm_bf16(int M, int N, int K, const void *d_A, const void *d_B, float *d_C);

/* ---- learned warm start of the batched Monte Carlo solve (no counterpart in
 * the reference; its only hook is the disabled warm start of
 * monte_linear_solver, fem/fem_mont.c:493-504) ------------------------------
 * Training: the batched solver solves ntrain samples from zero; a POD basis
 * of n_modes modes is built from the first n_snapshots solutions (FP64,
 * randomised subspace iteration + Rayleigh-Ritz); the solutions' POD
 * coefficients (divided by the sample's value in scale_col: the solution is
 * linear in the load) are modelled as a least-squares quadratic polynomial
 * of the standardised inputs (FP64, fitted by normal equations; linear
 * terms only below 4 training samples per quadratic term) plus the MLP
 * above, trained on that polynomial's residual over one common scale, so
 * the network's squared error is the coefficients' squared error.
 * Solving: u0 = scale * Phi * (poly + MLP)(inputs) is the initial guess of the
 * batched PCG, which still iterates to the same tolerance; its iteration cap
 * is the largest cold iteration count seen in training (when solving at the
 * training's precision), and a sample that does not converge within it is
 * solved again from zero (UFEM_ST_FALLBACK).
 * d_ifld: device, nsamp*ilen (the model's Monte Carlo inputs). */
typedef struct ufem_warm_options {
  int n_modes;               /* POD modes: a multiple of 16, at most 128 */
  int n_hidden;              /* MLP width: a multiple of 16, at most 256 */
  int n_feat;                /* network inputs, 1..32 */
  long feat_cols[32];        /* ifld column of each input */
  int feat_log[32];          /* 1: the input enters as log|value|; 2: as 1/value (a compliance:
                                for a modulus E, displacements are close to linear in 1/E);
                                0: as is */
  long scale_col;            /* ifld column the solution is proportional to, or -1 */
  long n_snapshots;          /* solutions the basis is built from (>= n_modes + 16) */
  int power_iters;           /* subspace iterations of the POD */
  int epochs, batch;         /* MLP training: passes over the set, minibatch size */
  float lr;                  /* Adam learning rate (cosine decay to 2 %) */
  unsigned long long seed;
  int guess_mode;            /* 0: the MLP's coefficients; 1: each sample's POD-Galerkin
                                coefficients (Phi^T K Phi c = Phi^T f, assembled from the
                                per-variable operators Phi^T K_v Phi; models with at most
                                64 E variables, else the MLP's) */
  int n_coarse;              /* the leading POD modes that become the coarse space of the
                                PCG preconditioner after training (ufem_mc_set_coarse; at
                                most n_modes, a multiple of 16; 0: none; default 64; models
                                with at most 64 E variables); modes with energy below 1e-20
                                of the first are left out (rounded down to a multiple of 16) */
  double snap_tol;           /* relative residual of the snapshot solves (the first n_snapshots
                                training samples; default 1e-11, 0: the training tolerance) */
  int order_samples;         /* ufem_warm_solve groups samples of similar spread of log(E / mean E)
                                into the same 128-sample groups (outputs in the caller's order;
                                default 1) */
} ufem_warm_options;

typedef struct ufem_warm_train_stats {
  long cold_iters_max;       /* largest PCG iteration count of the cold solves */
  double cold_iters_mean;
  double ms_solve, ms_basis, ms_train;
  double sigma2[80];         /* energy (squared singular value) of each POD mode (the first 80) */
  float loss_first, loss_last;  /* mean training loss of the first / last epoch */
  int epochs;
  long steps;
  int coarse_modes;          /* modes of the coarse space set on the model (0: none) */
} ufem_warm_train_stats;

typedef struct ufem_warm_stats {
  long nsamp, fallbacks;     /* samples solved; of them solved again from zero */
  double guess_err_mean, guess_err_max;  /* |u0 - u| / |u| against the converged u */
  double iters_mean;
  long iters_max;
  long cold_cap;             /* the iteration cap of the warm-started run */
  double ms_guess, ms_solve, ms_fallback, ms_total;
  long kernel_launches;      /* kernels launched by the call */
  double pcg_ms, pcg_bytes;  /* persistent PCG kernel time and algorithmic bytes (warm run) */
  long pcg_launches;
} ufem_warm_stats;

typedef struct ufem_warm ufem_warm;
void ufem_warm_default_options(ufem_warm_options *o);
int  ufem_warm_create(ufem_model *m, const ufem_warm_options *o, ufem_warm **out);
void ufem_warm_free(ufem_warm *w);
int  ufem_warm_train(ufem_warm *w, long ntrain, const double *d_ifld, const ufem_mc_options *opt,
                     ufem_warm_train_stats *st);
/* the guesses alone, d_u0: device, nsamp*nDOFAct (sample-major) */
int  ufem_warm_guess(ufem_warm *w, long nsamp, const double *d_ifld, double *d_u0);
/* warm-started batched solve; d_ofld nsamp*olen, d_status, d_iters nsamp (device; may be NULL) */
int  ufem_warm_solve(ufem_warm *w, long nsamp, const double *d_ifld, double *d_ofld, int *d_status, long *d_iters,
                     const ufem_mc_options *opt, ufem_warm_stats *st);
/* switches the guess between the MLP (0: the least-squares quadratic model
 * of the coefficients plus the network's correction), the POD-Galerkin
 * system (1) and, as a diagnostic of what the network adds, the
 * least-squares model alone (2) */
int  ufem_warm_set_guess_mode(ufem_warm *w, int mode);
/* multiplies every guess by factor (1 by default): a diagnostic that makes the
 * guesses bad on purpose, to exercise the fallback */
int  ufem_warm_set_guess_scale(ufem_warm *w, double factor);
/* the basis [nDOFAct][n_modes] and the mode energies (host; either may be NULL) */
int  ufem_warm_get_basis(const ufem_warm *w, double *h_phi, double *h_sigma2);
/* the warm start's FP64 kernels, exposed for their tests: C [M x N] = A [M x K]
 * B [K x N] (row-major, device); symmetric eigen-decomposition of A [l x l]
 * (l even, <= 96; host arrays; V columns = eigenvectors, unsorted) */
int  ufem_dgemm_f64(int M, int N, long K, const double *d_A, const double *d_B, double *d_C);
int  ufem_sym_eig(int l, const double *h_A, double *h_V, double *h_lam, int *sweeps);

/* ---- device / diagnostics ------------------------------------------------ */
int ufem_device_info(int *sm_count, int *cc_major, int *cc_minor, long *mem_bytes);

/* Self-tests of the bounded device waits (no reference counterpart).  Every
 * spin-wait of the library's kernels ends after a limit with an error the
 * host reads, so the CUDA context stays usable.  The first makes the grid
 * barrier of the persistent solvers run out: nblocks co-resident blocks, one
 * of which leaves without arriving, the others waiting limit_ms (1 to 2000)
 * before they give up; it returns AF_ERR ("grid barrier timed out") with the
 * number of blocks that timed out and the kernel's duration.  The second
 * waits on a tensor-core completion barrier that nothing signals, for
 * spin_limit polls (the coarse phases and the MLP use 2^24); it returns
 * AF_ERR with *timed_out = 1. */
int ufem_selftest_barrier_timeout(int nblocks, int limit_ms, int *blocks_timed_out, double *ms);
int ufem_selftest_mma_wait_timeout(long spin_limit, int *timed_out);
const char *ufem_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* UFEM_GPU_H */
