// Single-system FP64 solvers on the GPU block-sparse K (block size B = 1, 2
// or 3; B = 1 is plain CSR), each one persistent cooperative kernel:
//
//   Jacobi PCG      femEqsCGwJ    fem/fem_eqs.c:88-247
//   Jacobi BiCGStab femEqsBiCCSwJ fem/fem_eqs.c:262-468
//   SSOR PCG        femEqsCGwSSOR fem/fem_eqs.c:1001-1217 (multicolour sweeps)
//
// Jacobi PCG: one cooperative launch runs every iteration; the grid meets at
// a bounded barrier twice per iteration.  Phase S computes q = A p with
// p = z + beta p_old formed on the fly from the gathered neighbours (p needs
// no pass of its own) and the partial p.q; phase U updates x and r, forms
// z = r / diag(A) and the partials of r.r, x.x and r.z.  Every block sums the
// per-block partials in the same fixed order, so all blocks take the same
// convergence decision and results are identical run to run.  Vectors that
// other blocks write during the kernel are read with ld.global.cg (L2), never
// from the non-coherent L1.
//
// SpMV mapping: one warp per block row; L = 32 - 32 % B lanes walk the row's
// (block, row-in-block) items with stride L, so a lane's row-in-block
// a = lane % B is fixed; each lane reads the B consecutive values of its block
// row (contiguous across the warp) and the B gathered neighbour values; the B
// sums are combined by warp shuffles in a fixed order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "device_util.cuh"
#include "ufem_internal.h"

namespace ufem {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

struct CgResult {
  long iters;
  int status;
  int pad;
  double normRes, normX;
};

// TV: the type of the matrix values and of every vector (double, or float
// for the inner solves of the mixed-precision PCG); products and dot
// products accumulate in double either way.
template <typename TV>
struct CgArgsT {
  int nbr;
  long nnzb;
  const int *rowptr, *colind;
  const TV *val;  // [nnzb][B][B]
  const TV *b;
  TV *x;
  const TV *M;
  TV *r, *z, *p0, *p1, *q;
  double *part;  // [grid][4]: slots 0..2 = r.r, x.x, r.z ; slot 3 = p.q
  GridBar *bar;
  CgResult *res;
  double eps, normA, normB;
  long maxIt;
  int stop_rule;
};
using CgArgs = CgArgsT<double>;

// B = 3 (L = 30 lanes): lane l holds a partial of row l % 3 (lanes 30, 31
// hold 0).  Lanes l, l + 15, l + 6, l + 3 and l + 12 share a row (the
// offsets are multiples of 3), so four shuffles leave each row's sum of its
// 10 lanes on lanes 0..2, in a fixed order (identical run to run).
__device__ __forceinline__ double row_sums3(double acc) {
  const double t1 = acc + __shfl_down_sync(0xffffffffu, acc, 15);  // lanes 0..14: l, l + 15
  double t = t1 + __shfl_down_sync(0xffffffffu, t1, 6);            // lanes 0..8: + l + 6, l + 21
  t += __shfl_down_sync(0xffffffffu, t, 3);                        // lanes 0..5: + l + 3, 9, 18, 24
  t += __shfl_down_sync(0xffffffffu, t1, 12);                      // lanes 0..2: + l + 12, l + 27
  return t;
}

// The items [k0, k1) of one block row of y = A (z + beta p) (use_p) or
// y = A z: the B row sums come back on lanes < B.  Jf >= 0: the column index
// of the lane's first item, already loaded by the caller.
template <int B, typename TV>
__device__ __forceinline__ double warp_items_spmv(int k0, int k1, int Jf, const int *__restrict__ colind,
                                                  const TV *__restrict__ val, const TV *z, const TV *p,
                                                  double beta, bool use_p, double *s_acc) {
  constexpr int L = 32 - (32 % B);
  const int lane = threadIdx.x & 31;
  const int nitems = (k1 - k0) * B;
  double acc = 0.0;
  if (lane < L) {
    const int a = lane % B;
    for (int t = lane; t < nitems; t += L) {
      const int k = k0 + t / B;
      const int J = (t == lane && Jf >= 0) ? Jf : __ldg(colind + k);
      const TV *v = val + (size_t)k * B * B + a * B;
#pragma unroll
      for (int c = 0; c < B; c++) {
        double xj = (double)__ldcg(z + (size_t)J * B + c);
        if (use_p) xj = xj + beta * (double)__ldcg(p + (size_t)J * B + c);
        acc += (double)__ldg(v + c) * xj;
      }
    }
  }
  if (B == 1) {
    return warp_sum(acc);
  } else if (B == 2) {
#pragma unroll
    for (int o = 16; o >= 2; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    return acc;
  } else {
    (void)s_acc;
    return row_sums3(acc);
  }
}

// One block row I (bounds read from rowptr).
template <int B, typename TV>
__device__ __forceinline__ double warp_row_spmv(int I, const int *__restrict__ rowptr,
                                                const int *__restrict__ colind, const TV *__restrict__ val,
                                                const TV *z, const TV *p, double beta, bool use_p,
                                                double *s_acc) {
  return warp_items_spmv<B, TV>(__ldg(rowptr + I), __ldg(rowptr + I + 1), -1, colind, val, z, p, beta, use_p,
                                s_acc);
}

// A warp's consecutive block rows [I0, I1) with the next row's bounds and
// first column indices loaded while the current row computes, and the row's
// own epilogue operands loaded before its SpMV: the loads that only depend on
// the row number leave the per-row chain (row bounds -> column index ->
// neighbour gathers -> epilogue).  pre(I) loads the epilogue operands (lanes
// < B) and returns them; post(I, y, ops) consumes them.
template <int B, typename TV, typename Pre, typename Post>
__device__ __forceinline__ void warp_rows_spmv(int I0, int I1, const int *__restrict__ rowptr,
                                               const int *__restrict__ colind, const TV *__restrict__ val,
                                               const TV *z, const TV *p, double beta, bool use_p, double *s_acc,
                                               Pre pre, Post post) {
  constexpr int L = 32 - (32 % B);
  const int lane = threadIdx.x & 31;
  if (I0 >= I1) return;
  const int kend = __ldg(rowptr + I1);
  int k0 = __ldg(rowptr + I0), k1 = __ldg(rowptr + I0 + 1);
  int Jf = (lane < L && k0 + lane / B < kend) ? __ldg(colind + k0 + lane / B) : 0;
  for (int I = I0; I < I1; I++) {
    const int k1n = (I + 1 < I1) ? __ldg(rowptr + I + 2) : k1;
    const int Jfn = (lane < L && k1 + lane / B < kend) ? __ldg(colind + k1 + lane / B) : 0;
    const auto ops = pre(I);
    const double y = warp_items_spmv<B, TV>(k0, k1, Jf, colind, val, z, p, beta, use_p, s_acc);
    post(I, y, ops);
    k0 = k1;
    k1 = k1n;
    Jf = Jfn;
  }
}

// Fixed-order sum of slot `off` of the per-block partials (all blocks agree).
__device__ __forceinline__ double part_total(const double *part, int G, int off) {
  __shared__ double s_t;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32) {
    double t = 0.0;
    for (int g = lane; g < G; g += 32) t += __ldcg(part + (size_t)g * 4 + off);
    t = warp_sum(t);
    if (lane == 0) s_t = t;
  }
  __syncthreads();
  double v = s_t;
  __syncthreads();
  return v;
}

// Four 256-thread blocks per SM (64 registers a thread): the SpMV's
// index -> gather chains are latency-bound, and 32 warps per SM hide them
// (128x128x64 block, FP64 PCG to 1e-8: 764 ms with 2 blocks per SM, 535 with
// 3, 450 with 4; 5 and 6 spill and gain nothing).
constexpr int kCgBlocksPerSm = 4;

template <typename TV, int B>
__global__ void __launch_bounds__(kThreads, kCgBlocksPerSm) k_cg(CgArgsT<TV> A) {
  __shared__ double s_acc[kWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gw = blockIdx.x * kWarps + warp, nw = gridDim.x * kWarps;
  const int rpw = (A.nbr + nw - 1) / nw;
  const int I0 = min(A.nbr, gw * rpw), I1 = min(A.nbr, I0 + rpw);
  const int G = gridDim.x;
  double *mypart = A.part + (size_t)blockIdx.x * 4;
  // phase 0: r = b - A x; z = r / M (fem/fem_eqs.c:150-162)
  {
    double rr = 0.0, xx = 0.0, rz = 0.0;
    auto pre = [&](int I) {
      double3 o = make_double3(0.0, 0.0, 1.0);
      if (lane < B) {
        const size_t i = (size_t)I * B + lane;
        o = make_double3((double)A.b[i], (double)A.x[i], (double)A.M[i]);
      }
      return o;
    };
    auto post = [&](int I, double y, double3 o) {
      if (lane < B) {
        size_t i = (size_t)I * B + lane;
        const TV ri = (TV)(o.x - y);
        const TV zi = (TV)((double)ri / o.z);
        A.r[i] = ri;
        A.z[i] = zi;
        rr += (double)ri * (double)ri;
        xx += o.y * o.y;
        rz += (double)ri * (double)zi;
      }
    };
    warp_rows_spmv<B, TV>(I0, I1, A.rowptr, A.colind, A.val, A.x, (const TV *)nullptr, 0.0, false, s_acc[warp], pre,
                          post);
    double v[3] = {rr, xx, rz};
    block_partials<3>(v, mypart);
  }
  if (!grid_barrier(A.bar)) return;
  double rho = part_total(A.part, G, 2), rhoold = 1.0;
  double normRes = sqrt(part_total(A.part, G, 0)), normX = sqrt(part_total(A.part, G, 1));
  int status = UFEM_AF_ERR;
  long it = 0;
  for (it = 1; it <= A.maxIt; it++) {
    const bool first = (it == 1);
    const double beta = first ? 0.0 : rho / rhoold;  // fem/fem_eqs.c:172
    const TV *pold = (it & 1) ? A.p0 : A.p1;
    TV *pnew = (it & 1) ? A.p1 : A.p0;
    // phase S: q = A p, p = z + beta p_old (fem/fem_eqs.c:168-186), partial p.q
    {
      double pq = 0.0;
      auto pre = [&](int I) {
        double2 o = make_double2(0.0, 0.0);
        if (lane < B) {
          const size_t i = (size_t)I * B + lane;
          o = make_double2((double)A.z[i], first ? 0.0 : (double)pold[i]);
        }
        return o;
      };
      auto post = [&](int I, double y, double2 o) {
        if (lane < B) {
          size_t i = (size_t)I * B + lane;
          const TV pi = (TV)(first ? o.x : (o.x + (beta * o.y)));
          const TV qi = (TV)y;
          pnew[i] = pi;
          A.q[i] = qi;
          pq += (double)pi * (double)qi;
        }
      };
      warp_rows_spmv<B, TV>(I0, I1, A.rowptr, A.colind, A.val, A.z, pold, beta, !first, s_acc[warp], pre, post);
      double v[1] = {pq};
      block_partials<1>(v, mypart + 3);
    }
    if (!grid_barrier(A.bar)) return;
    const double pq = part_total(A.part, G, 3);
    if (!(pq > 0.0) || !isfinite(pq)) {  // breakdown: p.q <= 0 or not finite
      status = UFEM_AF_ERR;
      it = -it;
      break;
    }
    const double alpha = rho / pq;  // fem/fem_eqs.c:188
    // phase U: x += alpha p, r -= alpha q (fem/fem_eqs.c:194-198), z = r / M
    {
      double rr = 0.0, xx = 0.0, rz = 0.0;
      const size_t i0 = (size_t)I0 * B, i1 = (size_t)I1 * B;
      for (size_t i = i0 + lane; i < i1; i += 32) {
        const TV xi = (TV)((double)A.x[i] + (alpha * (double)pnew[i]));
        const TV ri = (TV)((double)A.r[i] - (alpha * (double)A.q[i]));
        const TV zi = (TV)((double)ri / (double)A.M[i]);
        A.x[i] = xi;
        A.r[i] = ri;
        A.z[i] = zi;
        rr += (double)ri * (double)ri;
        xx += (double)xi * (double)xi;
        rz += (double)ri * (double)zi;
      }
      double v[3] = {rr, xx, rz};
      block_partials<3>(v, mypart);
    }
    if (!grid_barrier(A.bar)) return;
    normRes = sqrt(part_total(A.part, G, 0));
    normX = sqrt(part_total(A.part, G, 1));
    const double rhonew = part_total(A.part, G, 2);
    bool conv;
    if (A.stop_rule == UFEM_STOP_REFERENCE)
      conv = normRes <= (A.eps * ((A.normA * normX) + A.normB));  // fem/fem_eqs.c:207
    else
      conv = normRes <= A.eps * A.normB;
    if (!isfinite(normRes)) {
      status = UFEM_AF_ERR;
      break;
    }
    if (conv) {
      status = UFEM_AF_OK;
      break;
    }
    rhoold = rho;
    rho = rhonew;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    A.res->iters = it > A.maxIt ? A.maxIt : it;
    A.res->status = status;
    A.res->normRes = normRes;
    A.res->normX = normX;
  }
}

// ---- small kernels shared by the host-driven solvers ------------------------

template <int B>
__global__ void __launch_bounds__(kThreads) k_spmv(int nbr, const int *__restrict__ rowptr,
                                                   const int *__restrict__ colind, const double *__restrict__ val,
                                                   const double *__restrict__ x, double *__restrict__ y) {
  __shared__ double s_acc[kWarps][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int I = blockIdx.x * kWarps + warp;
  if (I >= nbr) return;
  double v = warp_row_spmv<B, double>(I, rowptr, colind, val, x, nullptr, 0.0, false, s_acc[warp]);
  if (lane < B) y[(size_t)I * B + lane] = v;
}

// Diagonal of A and its smallest magnitude check (fem/fem_eqs.c:134-145).
template <int B>
__global__ void k_diag(int nbr, const int *__restrict__ rowptr, const int *__restrict__ colind,
                       const double *__restrict__ val, double *__restrict__ M, int *__restrict__ zero_row) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbr * B) return;
  int I = t / B, a = t % B;
  double d = 0.0;
  for (int k = rowptr[I]; k < rowptr[I + 1]; k++)
    if (colind[k] == I) d = val[(size_t)k * B * B + a * B + a];
  M[t] = d;
  if (fabs(d) < FEM_ZERO) atomicMin(zero_row, t);
}

// max over rows of the row 2-norm (femMatNormBig, fem/fem_math.c:1856-1952)
template <int B>
__global__ void k_row_norm_max(int nbr, const int *__restrict__ rowptr, const double *__restrict__ val,
                               unsigned long long *__restrict__ out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbr * B) return;
  int I = t / B, a = t % B;
  double s = 0.0;
  for (int k = rowptr[I]; k < rowptr[I + 1]; k++)
    for (int c = 0; c < B; c++) {
      double v = val[(size_t)k * B * B + a * B + c];
      s += v * v;
    }
  s = sqrt(s);
  atomicMax(out, (unsigned long long)__double_as_longlong(s));  // order-free for s >= 0
}

// deterministic two-stage dot products
constexpr int kDotBlocks = 296;
__global__ void __launch_bounds__(kThreads) k_dot_part(long n, const double *__restrict__ a,
                                                       const double *__restrict__ b, double *__restrict__ part) {
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    s += a[i] * b[i];
  double v[1] = {s};
  block_partials<1>(v, part + blockIdx.x);
}
__global__ void k_dot_final(const double *__restrict__ part, int nb, double *__restrict__ out) {
  double t = 0.0;
  for (int g = threadIdx.x; g < nb; g += 32) t += part[g];
  t = warp_sum(t);
  if (threadIdx.x == 0) *out = t;
}

struct Dots {
  DBuf<double> part, vals;
  int init(int nslots) {
    int rv = part.alloc(kDotBlocks);
    if (rv != UFEM_AF_OK) return rv;
    return vals.alloc(nslots);
  }
  void dot(long n, const double *a, const double *b, int slot, cudaStream_t s = 0) {
    k_dot_part<<<kDotBlocks, kThreads, 0, s>>>(n, a, b, part.p);
    k_dot_final<<<1, 32, 0, s>>>(part.p, kDotBlocks, vals.p + slot);
  }
};

int setup_common(const DevMatrix &A, DBuf<double> &M, double *normA, int *zero_row_out) {
  const long n = (long)A.nbr * A.B;
  int rv;
  if ((rv = M.alloc(n)) != UFEM_AF_OK) return rv;
  DBuf<int> zr;
  DBuf<unsigned long long> nm;
  if ((rv = zr.alloc(1)) != UFEM_AF_OK) return rv;
  if ((rv = nm.alloc(1)) != UFEM_AF_OK) return rv;
  int big = 0x7fffffff;
  UFEM_CUDA_TRY(cudaMemcpy(zr.p, &big, sizeof(int), cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemset(nm.p, 0, sizeof(unsigned long long)));
  unsigned g = (unsigned)((n + 255) / 256);
  switch (A.B) {
    case 1: k_diag<1><<<g, 256>>>(A.nbr, A.rowptr, A.colind, A.val, M.p, zr.p);
            k_row_norm_max<1><<<g, 256>>>(A.nbr, A.rowptr, A.val, nm.p); break;
    case 2: k_diag<2><<<g, 256>>>(A.nbr, A.rowptr, A.colind, A.val, M.p, zr.p);
            k_row_norm_max<2><<<g, 256>>>(A.nbr, A.rowptr, A.val, nm.p); break;
    default: k_diag<3><<<g, 256>>>(A.nbr, A.rowptr, A.colind, A.val, M.p, zr.p);
             k_row_norm_max<3><<<g, 256>>>(A.nbr, A.rowptr, A.val, nm.p); break;
  }
  UFEM_CUDA_TRY(cudaGetLastError());
  unsigned long long nb = 0;
  UFEM_CUDA_TRY(cudaMemcpy(&nb, nm.p, sizeof(nb), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(zero_row_out, zr.p, sizeof(int), cudaMemcpyDeviceToHost));
  double d;
  memcpy(&d, &nb, sizeof(d));
  *normA = d;
  return UFEM_AF_OK;
}

double host_norm(long n, const double *d_v) {
  Dots d;
  if (d.init(1) != UFEM_AF_OK) return NAN;
  d.dot(n, d_v, d_v, 0);
  double h = 0;
  cudaMemcpy(&h, d.vals.p, sizeof(double), cudaMemcpyDeviceToHost);
  return std::sqrt(h);
}

void spmv_launch(const DevMatrix &A, const double *x, double *y, cudaStream_t s = 0) {
  unsigned g = (unsigned)((A.nbr + kWarps - 1) / kWarps);
  switch (A.B) {
    case 1: k_spmv<1><<<g, kThreads, 0, s>>>(A.nbr, A.rowptr, A.colind, A.val, x, y); break;
    case 2: k_spmv<2><<<g, kThreads, 0, s>>>(A.nbr, A.rowptr, A.colind, A.val, x, y); break;
    default: k_spmv<3><<<g, kThreads, 0, s>>>(A.nbr, A.rowptr, A.colind, A.val, x, y); break;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
int cg_jacobi_fp64(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt, int stop_rule,
                   long *iters, float *ms) {
  const long n = (long)A.nbr * A.B;
  int rv;
  if (iters) *iters = 0;
  double normA = 0.0;
  int zero_row = 0;
  DBuf<double> M;
  if ((rv = setup_common(A, M, &normA, &zero_row)) != UFEM_AF_OK) return rv;
  double normB = host_norm(n, d_b);
  if (!(normB > 0.0)) {  // zero load: x = 0 without iterating (fem/fem_eqs.c:108-116)
    UFEM_CUDA_TRY(cudaMemset(d_x, 0, n * sizeof(double)));
    return UFEM_AF_OK;
  }
  if (zero_row != 0x7fffffff) {
    set_error("matrix member on the diagonal has zero size");  // fem/fem_eqs.c:134-145
    return UFEM_AF_ERR_ZER;
  }
  DBuf<double> r, z, p0, p1, q, part;
  DBuf<GridBar> bar;
  DBuf<CgResult> res;
  if ((rv = r.alloc(n)) || (rv = z.alloc(n)) || (rv = p0.alloc(n)) || (rv = p1.alloc(n)) || (rv = q.alloc(n)))
    return rv;
  UFEM_CUDA_TRY(cudaMemset(p0.p, 0, n * sizeof(double)));
  UFEM_CUDA_TRY(cudaMemset(p1.p, 0, n * sizeof(double)));
  int dev = 0, nsm = 0, occ = 0;
  UFEM_CUDA_TRY(cudaGetDevice(&dev));
  UFEM_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  void (*kern)(CgArgs) = A.B == 1 ? k_cg<double, 1> : (A.B == 2 ? k_cg<double, 2> : k_cg<double, 3>);
  UFEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, 0));
  if (occ < 1) {
    set_error("persistent CG kernel does not fit on an SM");
    return UFEM_AF_ERR;
  }
  // at least two block rows per warp; never more blocks than are co-resident
  int G = (int)std::min<long>((long)nsm * std::min(occ, kCgBlocksPerSm), (A.nbr + 2 * kWarps - 1) / (2 * kWarps));
  G = std::max(G, 1);
  if ((rv = part.alloc((size_t)G * 4)) != UFEM_AF_OK) return rv;
  if ((rv = bar.alloc(1)) != UFEM_AF_OK) return rv;
  if ((rv = res.alloc(1)) != UFEM_AF_OK) return rv;
  UFEM_CUDA_TRY(cudaMemset(bar.p, 0, sizeof(GridBar)));
  UFEM_CUDA_TRY(cudaMemset(res.p, 0, sizeof(CgResult)));
  CgArgs a{};
  a.nbr = A.nbr; a.nnzb = A.nnzb; a.rowptr = A.rowptr; a.colind = A.colind; a.val = A.val; a.b = d_b; a.x = d_x;
  a.M = M.p; a.r = r.p; a.z = z.p; a.p0 = p0.p; a.p1 = p1.p; a.q = q.p; a.part = part.p;
  a.bar = bar.p; a.res = res.p; a.eps = eps; a.normA = normA; a.normB = normB;
  a.maxIt = maxIt; a.stop_rule = stop_rule;
  void *args[] = {&a};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  UFEM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(G), dim3(kThreads), args, 0, 0));
  cudaEventRecord(e1);
  UFEM_CUDA_TRY(cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  if (ms) *ms = t;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  GridBar hb;
  CgResult hr;
  UFEM_CUDA_TRY(cudaMemcpy(&hb, bar.p, sizeof(hb), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(&hr, res.p, sizeof(hr), cudaMemcpyDeviceToHost));
  if (hb.err) {
    set_error("persistent CG: grid barrier timed out");
    return UFEM_AF_ERR;
  }
  if (iters) *iters = hr.iters < 0 ? -hr.iters : hr.iters;
  if (hr.status != UFEM_AF_OK) set_error("unconverged solution");  // fem/fem_eqs.c:230-236
  return hr.status;
}

// ---- BiCGStab (femEqsBiCCSwJ) ------------------------------------------------
//
// One persistent cooperative launch runs every iteration of the reference's
// Jacobi BiCGStab (fem/fem_eqs.c:262-468): scalars stay on the device, every
// block sums the per-block partials in the same fixed order, and the grid
// meets at a bounded barrier after each of the five phases of an iteration
// (p and pp = p / M; v = A pp with rr.v; s and ss = s / M with s.s;
// t = A ss with t.s and t.t; x, r with the next rr.r and the stopping
// sums), plus one for the true residual under the relative-residual rule.
namespace {

__global__ void k_sub(long n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ c) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) c[i] = a[i] - b[i];
}

struct BiArgs {
  int nbr;
  const int *rowptr, *colind;
  const double *val, *b, *M;
  double *x, *r, *rr, *p, *pp, *s, *ss, *t, *v, *Ab;
  double *part;  // [grid][4]
  GridBar *bar;
  CgResult *res;
  double eps, normA, normB;
  long maxIt;
  int stop_rule;
};

template <int B>
__global__ void __launch_bounds__(kThreads, kCgBlocksPerSm) k_bicgstab(BiArgs A) {
  __shared__ double s_acc[kWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gw = blockIdx.x * kWarps + warp, nw = gridDim.x * kWarps;
  const int rpw = (A.nbr + nw - 1) / nw;
  const int I0 = min(A.nbr, gw * rpw), I1 = min(A.nbr, I0 + rpw);
  const size_t i0 = (size_t)I0 * B, i1 = (size_t)I1 * B;
  const int G = gridDim.x;
  double *mypart = A.part + (size_t)blockIdx.x * 4;
  // phase 0: r = b - A x, rr = r (fem/fem_eqs.c:340-350); A b for the
  // reference's stopping test
  {
    double r2 = 0.0;
    for (int I = I0; I < I1; I++) {
      const double y = warp_row_spmv<B, double>(I, A.rowptr, A.colind, A.val, A.x, nullptr, 0.0, false, s_acc[warp]);
      double yb = 0.0;
      if (A.stop_rule == UFEM_STOP_REFERENCE)
        yb = warp_row_spmv<B, double>(I, A.rowptr, A.colind, A.val, A.b, nullptr, 0.0, false, s_acc[warp]);
      if (lane < B) {
        const size_t i = (size_t)I * B + lane;
        const double ri = A.b[i] - y;
        A.r[i] = ri;
        A.rr[i] = ri;
        if (A.stop_rule == UFEM_STOP_REFERENCE) A.Ab[i] = yb;
        r2 += ri * ri;
      }
    }
    double v3[1] = {r2};
    block_partials<1>(v3, mypart);
  }
  if (!grid_barrier(A.bar)) return;
  double ro = part_total(A.part, G, 0);  // rr.r = r.r at the start
  long it = 0;
  double normRes = sqrt(ro), normX = 0.0;
  if (!(sqrt(ro) <= FEM_ZERO)) {
    double roro = 1.0, alpha = 0.0, omega = 1.0;
    for (it = 1; it <= A.maxIt; it++) {
      if (fabs(ro) <= 0.0) break;  // fem/fem_eqs.c:373-379
      // p = r + beta (p - omega v) (fem/fem_eqs.c:381-392), pp = p / M
      {
        const double beta = (it == 1) ? 0.0 : (ro / roro) * (alpha / omega);
        for (size_t i = i0 + lane; i < i1; i += 32) {
          const double pi = (it == 1) ? A.r[i] : A.r[i] + beta * (A.p[i] - (omega * A.v[i]));
          A.p[i] = pi;
          A.pp[i] = pi / A.M[i];
        }
      }
      if (!grid_barrier(A.bar)) return;
      // v = A pp, rr.v
      {
        double rv = 0.0;
        for (int I = I0; I < I1; I++) {
          const double y = warp_row_spmv<B, double>(I, A.rowptr, A.colind, A.val, A.pp, nullptr, 0.0, false,
                                                    s_acc[warp]);
          if (lane < B) {
            const size_t i = (size_t)I * B + lane;
            A.v[i] = y;
            rv += A.rr[i] * y;
          }
        }
        double v1[1] = {rv};
        block_partials<1>(v1, mypart);
      }
      if (!grid_barrier(A.bar)) return;
      alpha = ro / part_total(A.part, G, 0);
      // s = r - alpha v, ss = s / M, s.s
      {
        double s2 = 0.0;
        for (size_t i = i0 + lane; i < i1; i += 32) {
          const double si = A.r[i] - (alpha * A.v[i]);
          A.s[i] = si;
          A.ss[i] = si / A.M[i];
          s2 += si * si;
        }
        double v1[1] = {s2};
        block_partials<1>(v1, mypart + 1);
      }
      if (!grid_barrier(A.bar)) return;
      if (sqrt(part_total(A.part, G, 1)) <= FEM_ZERO) {  // fem/fem_eqs.c:407-417
        for (size_t i = i0 + lane; i < i1; i += 32) A.x[i] += alpha * A.pp[i];
        break;
      }
      // t = A ss, t.s and t.t
      {
        double ts = 0.0, tt = 0.0;
        for (int I = I0; I < I1; I++) {
          const double y = warp_row_spmv<B, double>(I, A.rowptr, A.colind, A.val, A.ss, nullptr, 0.0, false,
                                                    s_acc[warp]);
          if (lane < B) {
            const size_t i = (size_t)I * B + lane;
            A.t[i] = y;
            ts += y * A.s[i];
            tt += y * y;
          }
        }
        double v2[2] = {ts, tt};
        block_partials<2>(v2, mypart + 2);
      }
      if (!grid_barrier(A.bar)) return;
      omega = part_total(A.part, G, 2) / part_total(A.part, G, 3);
      // x += alpha pp + omega ss, r = s - omega t; the next rr.r and the
      // reference's stopping sums |A b - x|^2 and |x|^2 (its residual call
      // at fem/fem_eqs.c:425 swaps the arguments: res = A b - x)
      {
        double rr_r = 0.0, res2 = 0.0, x2 = 0.0;
        for (size_t i = i0 + lane; i < i1; i += 32) {
          const double xi = A.x[i] + (alpha * A.pp[i] + (omega * A.ss[i]));
          const double ri = A.s[i] - (omega * A.t[i]);
          A.x[i] = xi;
          A.r[i] = ri;
          rr_r += A.rr[i] * ri;
          if (A.stop_rule == UFEM_STOP_REFERENCE) {
            const double d = A.Ab[i] - xi;
            res2 += d * d;
          }
          x2 += xi * xi;
        }
        double v3[3] = {rr_r, res2, x2};
        block_partials<3>(v3, mypart);
      }
      if (!grid_barrier(A.bar)) return;
      roro = ro;
      ro = part_total(A.part, G, 0);
      normX = sqrt(part_total(A.part, G, 2));
      bool conv;
      if (A.stop_rule == UFEM_STOP_REFERENCE) {
        normRes = sqrt(part_total(A.part, G, 1));
        conv = normRes < (A.eps * ((A.normA * normX) + A.normB));
      } else {
        // the true residual b - A x
        double r2 = 0.0;
        for (int I = I0; I < I1; I++) {
          const double y = warp_row_spmv<B, double>(I, A.rowptr, A.colind, A.val, A.x, nullptr, 0.0, false,
                                                    s_acc[warp]);
          if (lane < B) {
            const double d = A.b[(size_t)I * B + lane] - y;
            r2 += d * d;
          }
        }
        double v1[1] = {r2};
        block_partials<1>(v1, mypart + 3);
        if (!grid_barrier(A.bar)) return;
        normRes = sqrt(part_total(A.part, G, 3));
        conv = normRes <= A.eps * A.normB;
      }
      if (!isfinite(normRes)) break;
      if (conv) break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    A.res->iters = it > A.maxIt ? A.maxIt : it;
    A.res->status = UFEM_AF_OK;
    A.res->normRes = normRes;
    A.res->normX = normX;
  }
}

// Launches a persistent cooperative solver kernel over the matrix rows with
// the grid of k_cg (at least two block rows per warp, never more blocks than
// are co-resident); returns the kernel's milliseconds.
template <typename Args>
int launch_persistent(void (*kern)(Args), const DevMatrix &A, Args &a, DBuf<double> &part, DBuf<GridBar> &bar,
                      float *ms) {
  int dev = 0, nsm = 0, occ = 0, rv;
  UFEM_CUDA_TRY(cudaGetDevice(&dev));
  UFEM_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  UFEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, 0));
  if (occ < 1) {
    set_error("persistent solver kernel does not fit on an SM");
    return UFEM_AF_ERR;
  }
  int G = (int)std::min<long>((long)nsm * std::min(occ, kCgBlocksPerSm), (A.nbr + 2 * kWarps - 1) / (2 * kWarps));
  G = std::max(G, 1);
  if ((rv = part.alloc((size_t)G * 4)) || (rv = bar.alloc(1))) return rv;
  UFEM_CUDA_TRY(cudaMemset(bar.p, 0, sizeof(GridBar)));
  a.part = part.p;
  a.bar = bar.p;
  void *args[] = {&a};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  UFEM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(G), dim3(kThreads), args, 0, 0));
  cudaEventRecord(e1);
  UFEM_CUDA_TRY(cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms) *ms = t;
  GridBar hb;
  UFEM_CUDA_TRY(cudaMemcpy(&hb, bar.p, sizeof(hb), cudaMemcpyDeviceToHost));
  if (hb.err) {
    set_error("persistent solver: grid barrier timed out");
    return UFEM_AF_ERR;
  }
  return UFEM_AF_OK;
}
}  // namespace

int bicgstab_jacobi_fp64(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt, int stop_rule,
                         long *iters, float *ms) {
  const long n = (long)A.nbr * A.B;
  int rv;
  if (iters) *iters = 0;
  double normA = 0.0;
  int zero_row = 0;
  DBuf<double> M;
  if ((rv = setup_common(A, M, &normA, &zero_row)) != UFEM_AF_OK) return rv;
  const double normB = host_norm(n, d_b);
  // the reference leaves through memFree and still returns AF_OK (fem/fem_eqs.c:352-360, :467)
  if (zero_row != 0x7fffffff) return UFEM_AF_OK;
  DBuf<double> r, rr, p, pp, s, ss, t, v, Ab, part;
  DBuf<GridBar> bar;
  DBuf<CgResult> res;
  if ((rv = r.alloc(n)) || (rv = rr.alloc(n)) || (rv = p.alloc(n)) || (rv = pp.alloc(n)) || (rv = s.alloc(n)) ||
      (rv = ss.alloc(n)) || (rv = t.alloc(n)) || (rv = v.alloc(n)) || (rv = Ab.alloc(n)) || (rv = res.alloc(1)))
    return rv;
  UFEM_CUDA_TRY(cudaMemset(res.p, 0, sizeof(CgResult)));
  UFEM_CUDA_TRY(cudaMemset(p.p, 0, n * sizeof(double)));
  UFEM_CUDA_TRY(cudaMemset(v.p, 0, n * sizeof(double)));
  BiArgs a{};
  a.nbr = A.nbr; a.rowptr = A.rowptr; a.colind = A.colind; a.val = A.val; a.b = d_b; a.M = M.p; a.x = d_x;
  a.r = r.p; a.rr = rr.p; a.p = p.p; a.pp = pp.p; a.s = s.p; a.ss = ss.p; a.t = t.p; a.v = v.p; a.Ab = Ab.p;
  a.res = res.p; a.eps = eps; a.normA = normA; a.normB = normB; a.maxIt = maxIt; a.stop_rule = stop_rule;
  void (*kern)(BiArgs) = A.B == 1 ? k_bicgstab<1> : (A.B == 2 ? k_bicgstab<2> : k_bicgstab<3>);
  if ((rv = launch_persistent(kern, A, a, part, bar, ms)) != UFEM_AF_OK) return rv;
  CgResult hr;
  UFEM_CUDA_TRY(cudaMemcpy(&hr, res.p, sizeof(hr), cudaMemcpyDeviceToHost));
  if (iters) *iters = hr.iters;
  return UFEM_AF_OK;  // the reference always returns AF_OK (fem/fem_eqs.c:467)
}

// ---- SSOR PCG (femEqsCGwSSOR) with multicolour Gauss-Seidel sweeps -----------
//
// The reference sweeps rows in natural order (fem/fem_eqs.c:1077-1129), a
// sequential recurrence.  Here block rows are coloured so that no two rows
// of a colour are coupled; the forward sweep visits colours in order and the
// backward sweep in reverse, rows of a colour in parallel, the B DOFs of a
// node in order.  This is symmetric Gauss-Seidel for a permuted ordering: an
// SPD preconditioner like the reference's, with different iterates.  One
// persistent cooperative launch runs every iteration: a bounded grid barrier
// after each colour of each sweep (r.z accumulates as the backward sweep
// finalises each row's z), after q = A p with p = z + beta p_old formed on
// the fly, and after the x, r update.
namespace {

__global__ void k_recip(long n, const double *__restrict__ M, double *__restrict__ Minv) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) Minv[i] = 1.0 / M[i];
}

struct SsorArgs {
  int nbr, ncol;
  const int *rowptr, *colind, *colour_of, *cptr, *crow;  // cptr [ncol+1], crow: rows by colour
  const double *val, *b, *Minv;
  double *x, *r, *zz, *z, *p0, *p1, *q;
  double *part;  // [grid][4]
  GridBar *bar;
  CgResult *res;
  double eps, normA, normB;
  long maxIt;
  int stop_rule;
};

// one block row of a sweep (the row's thread): FWD, out = zz from rhs = r;
// backward, out = z from rhs = zz (returns the row's r.z contribution)
template <int B, bool FWD>
__device__ __forceinline__ double sgs_row(const SsorArgs &A, int I, int colour, const double *rhs, double *out) {
  double loc[B];
#pragma unroll
  for (int a = 0; a < B; a++) loc[a] = 0.0;
  const int k0 = A.rowptr[I], k1 = A.rowptr[I + 1];
  int kd = k0;
  for (int k = k0; k < k1; k++) {
    const int J = A.colind[k];
    if (J == I) {
      kd = k;
      continue;
    }
    const int cj = A.colour_of[J];
    if (FWD ? (cj < colour) : (cj > colour)) {
#pragma unroll
      for (int a = 0; a < B; a++)
#pragma unroll
        for (int c = 0; c < B; c++) loc[a] += A.val[(size_t)k * B * B + a * B + c] * __ldcg(out + (size_t)J * B + c);
    }
  }
  const double *D = A.val + (size_t)kd * B * B;
  double rz = 0.0;
  if (FWD) {
#pragma unroll
    for (int a = 0; a < B; a++) {
      double s = loc[a];
      for (int c = 0; c < a; c++) s += D[a * B + c] * out[(size_t)I * B + c];
      out[(size_t)I * B + a] = A.Minv[(size_t)I * B + a] * (__ldcg(rhs + (size_t)I * B + a) - s);
    }
  } else {
#pragma unroll
    for (int a = B - 1; a >= 0; a--) {
      double s = loc[a];
      for (int c = a + 1; c < B; c++) s += D[a * B + c] * out[(size_t)I * B + c];
      const double zi = __ldcg(rhs + (size_t)I * B + a) - A.Minv[(size_t)I * B + a] * s;
      out[(size_t)I * B + a] = zi;
      rz += __ldcg(A.r + (size_t)I * B + a) * zi;
    }
  }
  return rz;
}

template <int B>
__global__ void __launch_bounds__(kThreads, kCgBlocksPerSm) k_cg_ssor(SsorArgs A) {
  __shared__ double s_acc[kWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gw = blockIdx.x * kWarps + warp, nw = gridDim.x * kWarps;
  const int rpw = (A.nbr + nw - 1) / nw;
  const int I0 = min(A.nbr, gw * rpw), I1 = min(A.nbr, I0 + rpw);
  const size_t i0 = (size_t)I0 * B, i1 = (size_t)I1 * B;
  const int G = gridDim.x;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
  double *mypart = A.part + (size_t)blockIdx.x * 4;
  // r = b - A x
  for (int I = I0; I < I1; I++) {
    const double y = warp_row_spmv<B, double>(I, A.rowptr, A.colind, A.val, A.x, nullptr, 0.0, false, s_acc[warp]);
    if (lane < B) A.r[(size_t)I * B + lane] = A.b[(size_t)I * B + lane] - y;
  }
  if (!grid_barrier(A.bar)) return;
  int status = UFEM_AF_ERR;
  double rho = 0.0, rhoold = 1.0, normRes = 0.0, normX = 0.0;
  long it;
  for (it = 1; it <= A.maxIt; it++) {
    // z = (symmetric multicolour Gauss-Seidel)^-1 r
    for (int c = 0; c < A.ncol; c++) {
      const int r0 = __ldg(A.cptr + c), nr = __ldg(A.cptr + c + 1) - r0;
      for (int t = gtid; t < nr; t += nthr) sgs_row<B, true>(A, __ldg(A.crow + r0 + t), c, A.r, A.zz);
      if (!grid_barrier(A.bar)) return;
    }
    double rz = 0.0;
    for (int c = A.ncol - 1; c >= 0; c--) {
      const int r0 = __ldg(A.cptr + c), nr = __ldg(A.cptr + c + 1) - r0;
      for (int t = gtid; t < nr; t += nthr) rz += sgs_row<B, false>(A, __ldg(A.crow + r0 + t), c, A.zz, A.z);
      if (c > 0 && !grid_barrier(A.bar)) return;
    }
    {
      double v1[1] = {rz};
      block_partials<1>(v1, mypart + 2);
    }
    if (!grid_barrier(A.bar)) return;
    rho = part_total(A.part, G, 2);
    const bool first = (it == 1);
    const double beta = first ? 0.0 : rho / rhoold;
    const double *pold = (it & 1) ? A.p0 : A.p1;
    double *pnew = (it & 1) ? A.p1 : A.p0;
    // q = A p with p = z + beta p_old, p.q
    {
      double pq = 0.0;
      for (int I = I0; I < I1; I++) {
        const double y = warp_row_spmv<B, double>(I, A.rowptr, A.colind, A.val, A.z, pold, beta, !first, s_acc[warp]);
        if (lane < B) {
          const size_t i = (size_t)I * B + lane;
          const double zi = __ldcg(A.z + i);  // written by the sweeps' row mapping
          const double pi = first ? zi : (zi + (beta * pold[i]));
          pnew[i] = pi;
          A.q[i] = y;
          pq += pi * y;
        }
      }
      double v1[1] = {pq};
      block_partials<1>(v1, mypart + 3);
    }
    if (!grid_barrier(A.bar)) return;
    const double alpha = rho / part_total(A.part, G, 3);
    // x += alpha p, r -= alpha q, |r|^2 and |x|^2
    {
      double rr = 0.0, xx = 0.0;
      for (size_t i = i0 + lane; i < i1; i += 32) {
        const double xi = A.x[i] + (alpha * pnew[i]);
        const double ri = A.r[i] - (alpha * A.q[i]);
        A.x[i] = xi;
        A.r[i] = ri;
        rr += ri * ri;
        xx += xi * xi;
      }
      double v2[2] = {rr, xx};
      block_partials<2>(v2, mypart);
    }
    if (!grid_barrier(A.bar)) return;
    normRes = sqrt(part_total(A.part, G, 0));
    normX = sqrt(part_total(A.part, G, 1));
    const bool conv = A.stop_rule == UFEM_STOP_REFERENCE ? normRes <= (A.eps * ((A.normA * normX) + A.normB))
                                                         : normRes <= A.eps * A.normB;
    if (!isfinite(normRes)) break;
    if (conv) {
      status = UFEM_AF_OK;
      break;
    }
    rhoold = rho;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    A.res->iters = it > A.maxIt ? A.maxIt : it;
    A.res->status = status;
    A.res->normRes = normRes;
    A.res->normX = normX;
  }
}
}  // namespace

int cg_ssor_fp64(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt, int stop_rule,
                 long *iters, float *ms) {
  const long n = (long)A.nbr * A.B;
  int rv;
  if (iters) *iters = 0;
  double normA = 0.0;
  int zero_row = 0;
  DBuf<double> M;
  if ((rv = setup_common(A, M, &normA, &zero_row)) != UFEM_AF_OK) return rv;
  double normB = host_norm(n, d_b);
  if (!(normB > 0.0)) {
    UFEM_CUDA_TRY(cudaMemset(d_x, 0, n * sizeof(double)));
    return UFEM_AF_OK;
  }
  if (zero_row != 0x7fffffff) {
    set_error("matrix member on the diagonal has zero size");
    return UFEM_AF_ERR_ZER;
  }
  // greedy colouring of block rows on the host
  std::vector<int> rp(A.nbr + 1), ci(A.nnzb);
  UFEM_CUDA_TRY(cudaMemcpy(rp.data(), A.rowptr, (A.nbr + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(ci.data(), A.colind, A.nnzb * sizeof(int), cudaMemcpyDeviceToHost));
  std::vector<int> col(A.nbr, -1);
  int ncol = 0;
  std::vector<char> used;
  for (int I = 0; I < A.nbr; I++) {
    used.assign(ncol + 1, 0);
    for (int k = rp[I]; k < rp[I + 1]; k++)
      if (ci[k] != I && col[ci[k]] >= 0) used[col[ci[k]]] = 1;
    int c = 0;
    while (used[c]) c++;
    col[I] = c;
    ncol = std::max(ncol, c + 1);
  }
  std::vector<int> cptr(ncol + 1, 0), crow(A.nbr);
  for (int I = 0; I < A.nbr; I++) cptr[col[I] + 1]++;
  for (int c = 0; c < ncol; c++) cptr[c + 1] += cptr[c];
  {
    std::vector<int> f(cptr.begin(), cptr.end() - 1);
    for (int I = 0; I < A.nbr; I++) crow[f[col[I]]++] = I;
  }
  DBuf<int> d_col, d_crow, d_cptr;
  DBuf<double> Minv, r, z, zz, p0, p1, q, part;
  DBuf<GridBar> bar;
  DBuf<CgResult> res;
  if ((rv = d_col.upload(col.data(), col.size())) || (rv = d_crow.upload(crow.data(), crow.size())) ||
      (rv = d_cptr.upload(cptr.data(), cptr.size())))
    return rv;
  if ((rv = Minv.alloc(n)) || (rv = r.alloc(n)) || (rv = z.alloc(n)) || (rv = zz.alloc(n)) || (rv = p0.alloc(n)) ||
      (rv = p1.alloc(n)) || (rv = q.alloc(n)) || (rv = res.alloc(1)))
    return rv;
  UFEM_CUDA_TRY(cudaMemset(res.p, 0, sizeof(CgResult)));
  UFEM_CUDA_TRY(cudaMemset(p0.p, 0, n * sizeof(double)));
  UFEM_CUDA_TRY(cudaMemset(p1.p, 0, n * sizeof(double)));
  k_recip<<<(unsigned)((n + 255) / 256), 256>>>(n, M.p, Minv.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  SsorArgs a{};
  a.nbr = A.nbr; a.ncol = ncol; a.rowptr = A.rowptr; a.colind = A.colind; a.colour_of = d_col.p;
  a.cptr = d_cptr.p; a.crow = d_crow.p; a.val = A.val; a.b = d_b; a.Minv = Minv.p; a.x = d_x; a.r = r.p;
  a.zz = zz.p; a.z = z.p; a.p0 = p0.p; a.p1 = p1.p; a.q = q.p; a.res = res.p; a.eps = eps; a.normA = normA;
  a.normB = normB; a.maxIt = maxIt; a.stop_rule = stop_rule;
  void (*kern)(SsorArgs) = A.B == 1 ? k_cg_ssor<1> : (A.B == 2 ? k_cg_ssor<2> : k_cg_ssor<3>);
  if ((rv = launch_persistent(kern, A, a, part, bar, ms)) != UFEM_AF_OK) return rv;
  CgResult hr;
  UFEM_CUDA_TRY(cudaMemcpy(&hr, res.p, sizeof(hr), cudaMemcpyDeviceToHost));
  if (iters) *iters = hr.iters;
  if (hr.status != UFEM_AF_OK) set_error("unconverged solution");
  return hr.status;
}

// true residual |b - A x| / |b| in FP64 (host helper for the RELRES rule)
double true_relres(const DevMatrix &A, const double *d_b, const double *d_x) {
  const long n = (long)A.nbr * A.B;
  DBuf<double> t;
  if (t.alloc(n) != UFEM_AF_OK) return NAN;
  spmv_launch(A, d_x, t.p);
  unsigned g = (unsigned)((n + 255) / 256);
  k_sub<<<g, 256>>>(n, d_b, t.p, t.p);
  return host_norm(n, t.p) / host_norm(n, d_b);
}

// ---------------------------------------------------------------------------
// Mixed precision: Jacobi PCG on an FP32 copy of the matrix (half the value
// bytes of the SpMV) with an FP64 solution and FP64 true-residual
// replacement, in one persistent launch.  The work vectors r, z, p, q are
// FP32 or FP64 (VT), products and dot products accumulate in FP64, x +=
// alpha p in FP64.  The recursive
// residual r is replaced by the true residual b - A x (FP64 matrix, FP64 x)
// whenever it has dropped by `near` since the last replacement, every
// `every` iterations, and when it reaches eps |b|; the search direction is
// kept across replacements (no Krylov restart), so the count stays close to
// the FP64 one.  Converged only on a true residual: |b - A x| <= eps |b|.
namespace {
__global__ void k_to_f32(long n, const double *__restrict__ a, float *__restrict__ b) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// One block row of y = A (z + beta p) with an FP32 matrix copy and VT
// vectors (the mapping of warp_row_spmv); products and sums in FP64.
template <int B, typename VT>
__device__ __forceinline__ double warp_row_spmv_mix(int I, const int *__restrict__ rowptr,
                                                    const int *__restrict__ colind, const float *__restrict__ val,
                                                    const VT *z, const VT *p, double beta, bool use_p,
                                                    double *s_acc) {
  constexpr int L = 32 - (32 % B);
  const int lane = threadIdx.x & 31;
  const int k0 = __ldg(rowptr + I), k1 = __ldg(rowptr + I + 1);
  const int nitems = (k1 - k0) * B;
  double acc = 0.0;
  if (lane < L) {
    const int a = lane % B;
    for (int t = lane; t < nitems; t += L) {
      const int k = k0 + t / B;
      const int J = __ldg(colind + k);
      const float *v = val + (size_t)k * B * B + a * B;
#pragma unroll
      for (int c = 0; c < B; c++) {
        double xj = (double)__ldcg(z + (size_t)J * B + c);
        if (use_p) xj = xj + beta * (double)__ldcg(p + (size_t)J * B + c);
        acc += (double)__ldg(v + c) * xj;
      }
    }
  }
  if (B == 1) {
    return warp_sum(acc);
  } else if (B == 2) {
#pragma unroll
    for (int o = 16; o >= 2; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    return acc;
  } else {
    (void)s_acc;
    return row_sums3(acc);
  }
}

// VT: the type of the work vectors r, z, p, q and of the diagonal (FP32, or
// FP64 with only the matrix copy in FP32)
template <typename VT>
struct CgMixArgs {
  int nbr;
  const int *rowptr, *colind;
  const float *val;      // FP32 copy of K [nnzb][B][B]
  const double *val64;   // FP64 K, for the true residuals
  const double *b;       // right-hand side
  double *x;             // solution (in: the initial guess)
  const VT *M;           // diagonal
  VT *r, *z, *p0, *p1, *q;
  double *part;          // [grid][4]: r.r, -, r.z, p.q
  GridBar *bar;
  CgResult *res;
  double eps, normB, near2;
  long maxIt, every;
  long *replacements;
};

// r = b - A x in FP64 (true residual), r (FP32), z = r / M and the partials
// of the true r.r and of r.z, over the warp's block rows
template <int B, typename VT>
__device__ __forceinline__ void mix_true_residual(const CgMixArgs<VT> &A, int I0, int I1, double *s_acc,
                                                  double *mypart) {
  const int lane = threadIdx.x & 31;
  double rr = 0.0, rz = 0.0;
  for (int I = I0; I < I1; I++) {
    const double y = warp_row_spmv<B, double>(I, A.rowptr, A.colind, A.val64, A.x, nullptr, 0.0, false, s_acc);
    if (lane < B) {
      const size_t i = (size_t)I * B + lane;
      const double r64 = A.b[i] - y;
      const VT ri = (VT)r64, zi = ri / A.M[i];
      A.r[i] = ri;
      A.z[i] = zi;
      rr += r64 * r64;
      rz += (double)ri * (double)zi;
    }
  }
  double v[3] = {rr, 0.0, rz};
  block_partials<3>(v, mypart);
}

template <int B, typename VT>
__global__ void __launch_bounds__(kThreads, kCgBlocksPerSm) k_cg_mixed(CgMixArgs<VT> A) {
  __shared__ double s_acc[kWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gw = blockIdx.x * kWarps + warp, nw = gridDim.x * kWarps;
  const int rpw = (A.nbr + nw - 1) / nw;
  const int I0 = min(A.nbr, gw * rpw), I1 = min(A.nbr, I0 + rpw);
  const int G = gridDim.x;
  double *mypart = A.part + (size_t)blockIdx.x * 4;
  const double tol2 = (A.eps * A.normB) * (A.eps * A.normB);
  mix_true_residual<B, VT>(A, I0, I1, s_acc[warp], mypart);
  if (!grid_barrier(A.bar)) return;
  double rr_true = part_total(A.part, G, 0), rho = part_total(A.part, G, 2), rhoold = 1.0, rr_last = rr_true;
  long it = 0, it_last = 0, nrep = 0;
  int status = UFEM_AF_ERR;
  if (rr_true <= tol2) status = UFEM_AF_OK;
  for (it = 1; status != UFEM_AF_OK && it <= A.maxIt; it++) {
    const bool first = (it == 1);
    const double beta = first ? 0.0 : rho / rhoold;
    const VT *pold = (it & 1) ? A.p0 : A.p1;
    VT *pnew = (it & 1) ? A.p1 : A.p0;
    // phase S: q = A p with p = z + beta p_old, partial p.q
    {
      double pq = 0.0;
      for (int I = I0; I < I1; I++) {
        const double y = warp_row_spmv_mix<B, VT>(I, A.rowptr, A.colind, A.val, A.z, pold, beta, !first, s_acc[warp]);
        if (lane < B) {
          const size_t i = (size_t)I * B + lane;
          const VT pi = (VT)(first ? (double)A.z[i] : ((double)A.z[i] + beta * (double)pold[i]));
          const VT qi = (VT)y;
          pnew[i] = pi;
          A.q[i] = qi;
          pq += (double)pi * (double)qi;
        }
      }
      double v[1] = {pq};
      block_partials<1>(v, mypart + 3);
    }
    if (!grid_barrier(A.bar)) return;
    const double pq = part_total(A.part, G, 3);
    if (!(pq > 0.0) || !isfinite(pq)) break;  // breakdown
    const double alpha = rho / pq;
    // phase U: x += alpha p (FP64), r -= alpha q, z = r / M
    {
      double rr = 0.0, rz = 0.0;
      const size_t i0 = (size_t)I0 * B, i1 = (size_t)I1 * B;
      for (size_t i = i0 + lane; i < i1; i += 32) {
        A.x[i] += alpha * (double)pnew[i];
        const VT ri = (VT)((double)A.r[i] - alpha * (double)A.q[i]);
        const VT zi = ri / A.M[i];
        A.r[i] = ri;
        A.z[i] = zi;
        rr += (double)ri * (double)ri;
        rz += (double)ri * (double)zi;
      }
      double v[3] = {rr, 0.0, rz};
      block_partials<3>(v, mypart);
    }
    if (!grid_barrier(A.bar)) return;
    const double rr_rec = part_total(A.part, G, 0);
    double rz_new = part_total(A.part, G, 2);
    if (!isfinite(rr_rec)) break;
    // a true-residual pass: on the residual drop, every `every` iterations,
    // and to verify convergence (every block takes the same decision)
    if (rr_rec <= tol2 || rr_rec <= A.near2 * rr_last || it - it_last >= A.every) {
      mix_true_residual<B, VT>(A, I0, I1, s_acc[warp], mypart);
      if (!grid_barrier(A.bar)) return;
      rr_true = part_total(A.part, G, 0);
      rz_new = part_total(A.part, G, 2);
      nrep++;
      if (rr_true <= tol2) {
        status = UFEM_AF_OK;
        break;
      }
      rr_last = rr_true;
      it_last = it;
    }
    rhoold = rho;
    rho = rz_new;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    A.res->iters = it > A.maxIt ? A.maxIt : it;
    A.res->status = status;
    A.res->normRes = sqrt(rr_true);
    *A.replacements = nrep;
  }
}
}  // namespace

namespace {
template <typename VT>
int run_cg_mixed(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt, double replace_near,
                 long replace_every, long *iters, int *replacements, float *ms) {
  const long n = (long)A.nbr * A.B, nv = A.nnzb * A.B * A.B;
  int rv;
  if (iters) *iters = 0;
  if (replacements) *replacements = 0;
  double normA = 0.0;
  int zero_row = 0;
  DBuf<double> M;
  if ((rv = setup_common(A, M, &normA, &zero_row)) != UFEM_AF_OK) return rv;
  const double normB = host_norm(n, d_b);
  if (!(normB > 0.0)) {
    UFEM_CUDA_TRY(cudaMemset(d_x, 0, n * sizeof(double)));
    return UFEM_AF_OK;
  }
  if (zero_row != 0x7fffffff) {
    set_error("matrix member on the diagonal has zero size");  // fem/fem_eqs.c:134-145
    return UFEM_AF_ERR_ZER;
  }
  DBuf<float> V32;
  DBuf<VT> M32, r, z, p0, p1, q;
  DBuf<double> part;
  DBuf<GridBar> bar;
  DBuf<CgResult> res;
  DBuf<long> nrep;
  if ((rv = V32.alloc(nv)) || (rv = M32.alloc(n)) || (rv = r.alloc(n)) || (rv = z.alloc(n)) || (rv = p0.alloc(n)) ||
      (rv = p1.alloc(n)) || (rv = q.alloc(n)) || (rv = nrep.alloc(1)))
    return rv;
  const unsigned gv = (unsigned)((nv + 255) / 256), gn = (unsigned)((n + 255) / 256);
  k_to_f32<<<gv, 256>>>(nv, A.val, V32.p);
  if constexpr (sizeof(VT) == 4) k_to_f32<<<gn, 256>>>(n, M.p, M32.p);
  else UFEM_CUDA_TRY(cudaMemcpy(M32.p, M.p, n * sizeof(double), cudaMemcpyDeviceToDevice));
  UFEM_CUDA_TRY(cudaMemset(p0.p, 0, n * sizeof(VT)));
  UFEM_CUDA_TRY(cudaMemset(p1.p, 0, n * sizeof(VT)));
  int dev = 0, nsm = 0, occ = 0;
  UFEM_CUDA_TRY(cudaGetDevice(&dev));
  UFEM_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  void (*kern)(CgMixArgs<VT>) = A.B == 1 ? k_cg_mixed<1, VT> : (A.B == 2 ? k_cg_mixed<2, VT> : k_cg_mixed<3, VT>);
  UFEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, 0));
  if (occ < 1) {
    set_error("persistent CG kernel does not fit on an SM");
    return UFEM_AF_ERR;
  }
  int G = (int)std::min<long>((long)nsm * std::min(occ, kCgBlocksPerSm), (A.nbr + 2 * kWarps - 1) / (2 * kWarps));
  G = std::max(G, 1);
  if ((rv = part.alloc((size_t)G * 4)) || (rv = bar.alloc(1)) || (rv = res.alloc(1))) return rv;
  UFEM_CUDA_TRY(cudaMemset(bar.p, 0, sizeof(GridBar)));
  UFEM_CUDA_TRY(cudaMemset(res.p, 0, sizeof(CgResult)));
  CgMixArgs<VT> a{};
  a.nbr = A.nbr; a.rowptr = A.rowptr; a.colind = A.colind; a.val = V32.p; a.val64 = A.val; a.b = d_b; a.x = d_x;
  a.M = M32.p; a.r = r.p; a.z = z.p; a.p0 = p0.p; a.p1 = p1.p; a.q = q.p; a.part = part.p; a.bar = bar.p;
  a.res = res.p; a.eps = eps; a.normB = normB; a.near2 = replace_near * replace_near; a.maxIt = maxIt;
  a.every = std::max<long>(1, replace_every); a.replacements = nrep.p;
  void *args[] = {&a};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  UFEM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(G), dim3(kThreads), args, 0, 0));
  cudaEventRecord(e1);
  UFEM_CUDA_TRY(cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  if (ms) *ms = t;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  GridBar hb;
  CgResult hr;
  long hrep = 0;
  UFEM_CUDA_TRY(cudaMemcpy(&hb, bar.p, sizeof(hb), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(&hr, res.p, sizeof(hr), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(&hrep, nrep.p, sizeof(hrep), cudaMemcpyDeviceToHost));
  if (hb.err) {
    set_error("persistent CG: grid barrier timed out");
    return UFEM_AF_ERR;
  }
  if (iters) *iters = hr.iters;
  if (replacements) *replacements = (int)hrep;
  if (hr.status != UFEM_AF_OK) set_error("unconverged solution");
  return hr.status;
}
}  // namespace

// fp32_vectors: the work vectors in FP32 as well (else FP64, only the matrix
// copy in FP32)
int cg_jacobi_mixed(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt, double replace_near,
                    long replace_every, bool fp32_vectors, long *iters, int *replacements, float *ms) {
  return fp32_vectors ? run_cg_mixed<float>(A, d_b, d_x, eps, maxIt, replace_near, replace_every, iters, replacements, ms)
                      : run_cg_mixed<double>(A, d_b, d_x, eps, maxIt, replace_near, replace_every, iters, replacements,
                                             ms);
}

// ---------------------------------------------------------------------------
// Jacobi PCG without any allocation (ufem_eqs_cgwj_noalloc)
//
// Some callers cannot allocate device memory at solve time: code running
// inside a framework that owns the whole device pool (an embedding
// application with its own allocator, a solver called from a callback of
// another GPU library), or a real-time loop that must not hit cudaMalloc's
// implicit device synchronisation.  For them the persistent Jacobi PCG above
// runs with all of its scratch -- the diagonal, the five work vectors, the
// per-block partial sums, the grid barrier and the result words -- placed in
// one fixed array compiled into this library.  The caller passes the matrix,
// the right-hand side and the solution in device memory.
//
// Limits: at most kNoallocMaxRows scalar rows (131,072) and kNoallocMaxGrid
// blocks; the array takes about 6.3 MB on every GPU where the library's
// solver code is loaded (the first use of any of its solvers on a device
// loads it, this entry point's first call included), until the process
// exits.  All calls share the one array, so two solves whose kernels
// overlapped on the GPU would race on it; this function prevents that in one
// process: a lock serialises calls, and each call returns only once its
// kernels have finished.  It runs on the legacy default stream with
// synchronous copies.  The first call on a device looks the array's device
// address up (once per device, with that device current); make that first
// call before any stream capture begins.
// ---------------------------------------------------------------------------
namespace {

constexpr long kNoallocMaxRows = 131072;
constexpr int kNoallocMaxGrid = 1024;
constexpr int kNoallocHeader = 64;  // doubles: barrier, result, norms, flags
constexpr long kNoallocDoubles = kNoallocHeader + (long)kDotBlocks + 4L * kNoallocMaxGrid + 6L * kNoallocMaxRows;

static __device__ __align__(256) double g_noalloc_scratch[kNoallocDoubles];

struct NoallocHeader {  // overlays the first kNoallocHeader doubles
  GridBar bar;
  CgResult res;
  unsigned long long normA_bits;
  int zero_row;
  int pad;
  double normB2;
};
static_assert(sizeof(NoallocHeader) <= kNoallocHeader * sizeof(double), "scratch header too large");

std::mutex g_noalloc_mu;
double *g_noalloc_addr[64] = {nullptr};

}  // namespace

int cg_jacobi_fp64_noalloc(const DevMatrix &A, const double *d_b, double *d_x, double eps, long maxIt,
                           long *iters) {
  const long n = (long)A.nbr * A.B;
  if (iters) *iters = 0;
  if (A.B < 1 || A.B > 3 || A.nbr < 1) {
    set_error("ufem_eqs_cgwj_noalloc: block size must be 1, 2 or 3 and the matrix non-empty");
    return UFEM_AF_ERR_SIZ;
  }
  if (n > kNoallocMaxRows) {
    set_error("ufem_eqs_cgwj_noalloc: more than 131072 rows; use ufem_eqs_cgwj or ufem_solve");
    return UFEM_AF_ERR_SIZ;
  }
  int dev = 0, nsm = 0, occ = 0;
  UFEM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("ufem_eqs_cgwj_noalloc: device index out of range");
    return UFEM_AF_ERR;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("ufem_eqs_cgwj_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return UFEM_AF_ERR;
    }
    g_noalloc_addr[dev] = static_cast<double *>(p);
  }
  double *base = g_noalloc_addr[dev];
  NoallocHeader *hdr = reinterpret_cast<NoallocHeader *>(base);
  double *dots = base + kNoallocHeader;
  double *part = dots + kDotBlocks;
  double *M = part + 4L * kNoallocMaxGrid;
  double *r = M + kNoallocMaxRows, *z = r + kNoallocMaxRows, *p0 = z + kNoallocMaxRows;
  double *p1 = p0 + kNoallocMaxRows, *q = p1 + kNoallocMaxRows;
  // what must start at zero: the barrier, the result, the norm maximum;
  // the zero-diagonal flag starts at INT_MAX (atomicMin target)
  UFEM_CUDA_TRY(cudaMemset(base, 0, kNoallocHeader * sizeof(double)));
  const int big = 0x7fffffff;
  UFEM_CUDA_TRY(cudaMemcpy(&hdr->zero_row, &big, sizeof(int), cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemset(p0, 0, n * sizeof(double)));
  UFEM_CUDA_TRY(cudaMemset(p1, 0, n * sizeof(double)));
  const unsigned g = (unsigned)((n + 255) / 256);
  switch (A.B) {
    case 1: k_diag<1><<<g, 256>>>(A.nbr, A.rowptr, A.colind, A.val, M, &hdr->zero_row);
            k_row_norm_max<1><<<g, 256>>>(A.nbr, A.rowptr, A.val, &hdr->normA_bits); break;
    case 2: k_diag<2><<<g, 256>>>(A.nbr, A.rowptr, A.colind, A.val, M, &hdr->zero_row);
            k_row_norm_max<2><<<g, 256>>>(A.nbr, A.rowptr, A.val, &hdr->normA_bits); break;
    default: k_diag<3><<<g, 256>>>(A.nbr, A.rowptr, A.colind, A.val, M, &hdr->zero_row);
             k_row_norm_max<3><<<g, 256>>>(A.nbr, A.rowptr, A.val, &hdr->normA_bits); break;
  }
  k_dot_part<<<kDotBlocks, kThreads>>>(n, d_b, d_b, dots);
  k_dot_final<<<1, 32>>>(dots, kDotBlocks, &hdr->normB2);
  UFEM_CUDA_TRY(cudaGetLastError());
  NoallocHeader h;
  UFEM_CUDA_TRY(cudaMemcpy(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost));
  double normA;
  memcpy(&normA, &h.normA_bits, sizeof(normA));
  const double normB = std::sqrt(h.normB2);
  if (!(normB > 0.0)) {  // zero load: x = 0 (fem/fem_eqs.c:108-116)
    UFEM_CUDA_TRY(cudaMemset(d_x, 0, n * sizeof(double)));
    return UFEM_AF_OK;
  }
  if (h.zero_row != big) {
    set_error("matrix member on the diagonal has zero size");
    return UFEM_AF_ERR_ZER;
  }
  UFEM_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  void (*kern)(CgArgs) = A.B == 1 ? k_cg<double, 1> : (A.B == 2 ? k_cg<double, 2> : k_cg<double, 3>);
  UFEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, 0));
  if (occ < 1) {
    set_error("persistent CG kernel does not fit on an SM");
    return UFEM_AF_ERR;
  }
  int G = (int)std::min<long>((long)nsm * std::min(occ, kCgBlocksPerSm), (A.nbr + 2 * kWarps - 1) / (2 * kWarps));
  G = std::max(1, std::min(G, kNoallocMaxGrid));
  CgArgs a{};
  a.nbr = A.nbr; a.nnzb = A.nnzb; a.rowptr = A.rowptr; a.colind = A.colind; a.val = A.val; a.b = d_b; a.x = d_x;
  a.M = M; a.r = r; a.z = z; a.p0 = p0; a.p1 = p1; a.q = q; a.part = part;
  a.bar = &hdr->bar; a.res = &hdr->res; a.eps = eps; a.normA = normA; a.normB = normB;
  a.maxIt = maxIt; a.stop_rule = UFEM_STOP_REFERENCE;
  void *args[] = {&a};
  UFEM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(G), dim3(kThreads), args, 0, 0));
  UFEM_CUDA_TRY(cudaMemcpy(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost));
  if (h.bar.err) {
    set_error("persistent CG: grid barrier timed out");
    return UFEM_AF_ERR;
  }
  if (iters) *iters = h.res.iters < 0 ? -h.res.iters : h.res.iters;
  if (h.res.status != UFEM_AF_OK) set_error("unconverged solution");
  return h.res.status;
}

}  // namespace ufem

// The allocation-free Jacobi PCG (declared in include/ufem_gpu.h).
extern "C" int ufem_eqs_cgwj_noalloc(int B, int nbr, const int *d_rowptr, const int *d_colind, const double *d_val,
                                     const double *d_b, double *d_x, double eps, long maxIt, long *iters) {
  ufem::DevMatrix A;
  A.B = B;
  A.nbr = nbr;
  A.nnzb = 0;
  A.rowptr = d_rowptr;
  A.colind = d_colind;
  A.val = d_val;
  return ufem::cg_jacobi_fp64_noalloc(A, d_b, d_x, eps, maxIt, iters);
}
