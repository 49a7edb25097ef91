// GPU build of the model's DOF numbering, block-sparse pattern, element ->
// block scatter map and element colouring (fem_dofs, fem/fem_sol.c:1263-1395;
// femKhit, fem/fem_mloc.c:83-116; the insertion pattern of femLocKM_e,
// fem/fem_mloc.c:163-221).
//
//   1. used nodes (any element's node) -> block row = rank of the node among
//      used nodes (an exclusive scan): DOF = b rank + d + 1 reproduces the
//      reference's slot-order numbering for a uniform element family;
//   2. node -> element incidence lists (counting sort by block row);
//   3. per block row, one warp gathers the block rows of every incident
//      element's nodes into shared memory, sorts them (bitonic) and keeps the
//      distinct ones: the row's block columns, sorted, and the diagonal block;
//      a count pass, a scan for rowptr, then a write pass;
//   4. the scatter map: for every (element, node a, node c), the block index
//      of (row a, column c) by binary search in row a;
//   5. a node-disjoint element colouring by Jones-Plassmann rounds: an
//      uncoloured element whose (hash, index) priority is above every
//      uncoloured element sharing a node with it takes the smallest colour
//      none of its coloured neighbours holds; each round reads the previous
//      round's colours only, so the colouring is the same every run.
//
// Everything stays in the model's device buffers.  The host keeps the block
// row of each node, the DOF numbers and the colour groups; the pattern and
// the scatter map are copied to the host on first use (host_pattern: the
// BSR pattern export and the Monte Carlo plans read them there).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include "ufem_internal.h"

namespace ufem {
namespace {

constexpr int kScanBlock = 1024;  // items per block of the scan (256 threads x 4)
constexpr int kMaxCand = 1024;    // element-node incidences gathered per block row (shared memory)
constexpr int kRowWarps = 8;

// ---- exclusive scan of ints ------------------------------------------------
__global__ void k_scan_block(long n, const int *__restrict__ in, int *__restrict__ out, int *__restrict__ sums) {
  __shared__ int s[256];
  const long base = (long)blockIdx.x * kScanBlock;
  int v[4], t = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const long i = base + threadIdx.x * 4 + q;
    v[q] = i < n ? in[i] : 0;
    t += v[q];
  }
  s[threadIdx.x] = t;
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {  // Hillis-Steele inclusive scan of the thread sums
    const int a = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += a;
    __syncthreads();
  }
  int run = s[threadIdx.x] - t;  // exclusive prefix of this thread
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const long i = base + threadIdx.x * 4 + q;
    if (i < n) out[i] = run;
    run += v[q];
  }
  if (threadIdx.x == 255) sums[blockIdx.x] = s[255];
}
__global__ void k_scan_add(long n, int *__restrict__ out, const int *__restrict__ offs) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += offs[i / kScanBlock];
}

// out[i] = sum_{j<i} in[i]; returns the total.  in and out may alias.
int scan_exclusive(long n, const int *d_in, int *d_out, long *total) {
  const long nb = (n + kScanBlock - 1) / kScanBlock;
  DBuf<int> sums;
  int rv;
  if ((rv = sums.alloc(nb + 1))) return rv;
  k_scan_block<<<(unsigned)nb, 256>>>(n, d_in, d_out, sums.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  std::vector<int> h(nb);
  UFEM_CUDA_TRY(cudaMemcpy(h.data(), sums.p, nb * sizeof(int), cudaMemcpyDeviceToHost));
  long run = 0;
  for (long b = 0; b < nb; b++) {
    const long t = h[b];
    h[b] = (int)run;
    run += t;
  }
  if (run > INT_MAX) {
    set_error("pattern build: more than 2^31 - 1 entries");
    return UFEM_AF_ERR_BIG;
  }
  UFEM_CUDA_TRY(cudaMemcpy(sums.p, h.data(), nb * sizeof(int), cudaMemcpyHostToDevice));
  k_scan_add<<<(unsigned)((n + 255) / 256), 256>>>(n, d_out, sums.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  *total = run;
  return UFEM_AF_OK;
}

// ---- 1. used nodes and block rows -----------------------------------------
__global__ void k_mark_used(long nent, const int *__restrict__ enodes, int *__restrict__ used) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nent) used[enodes[i]] = 1;
}
__global__ void k_node_rank(long nLen, const int *__restrict__ used, const int *__restrict__ scan,
                            int *__restrict__ node_rank, int *__restrict__ rank_node) {
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nLen) return;
  if (used[n]) {
    node_rank[n] = scan[n];
    rank_node[scan[n]] = (int)n;
  } else {
    node_rank[n] = -1;
  }
}

// ---- 2. node -> element incidence --------------------------------------------
__global__ void k_inc_count(long eLen, int nn, const int *__restrict__ enodes, const int *__restrict__ node_rank,
                            int *__restrict__ cnt) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < eLen * nn) atomicAdd(cnt + node_rank[enodes[i]], 1);
}
__global__ void k_inc_fill(long eLen, int nn, const int *__restrict__ enodes, const int *__restrict__ node_rank,
                           int *__restrict__ fill, int *__restrict__ n2e) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < eLen * nn) n2e[atomicAdd(fill + node_rank[enodes[i]], 1)] = (int)(i / nn);
}

// ---- 3. block columns of each row ---------------------------------------------
// WRITE = false: counts[r] = distinct columns; WRITE = true: colind and diagblk.
template <bool WRITE>
__global__ void __launch_bounds__(kRowWarps * 32) k_row_cols(int nbr, int nn, const int *__restrict__ enodes,
                                                             const int *__restrict__ node_rank,
                                                             const int *__restrict__ n2e_ptr,
                                                             const int *__restrict__ n2e, int *__restrict__ counts,
                                                             const int *__restrict__ rowptr, int *__restrict__ colind,
                                                             int *__restrict__ diagblk, int *__restrict__ err) {
  __shared__ int s_c[kRowWarps][kMaxCand];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * kRowWarps + warp;
  if (r >= nbr) return;
  int *c = s_c[warp];
  const int q0 = n2e_ptr[r], q1 = n2e_ptr[r + 1];
  const int ncand = (q1 - q0) * nn;
  if (ncand > kMaxCand) {
    if (lane == 0) atomicExch(err, 1);
    return;
  }
  int m = 32;  // sort width: a power of two >= ncand
  while (m < ncand) m <<= 1;
  for (int t = lane; t < m; t += 32) c[t] = t < ncand ? node_rank[enodes[(size_t)n2e[q0 + t / nn] * nn + t % nn]] : INT_MAX;
  __syncwarp();
  // bitonic sort of c[0, m)
  for (int k = 2; k <= m; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = lane; t < m; t += 32) {
        const int p = t ^ j;
        if (p > t) {
          const int a = c[t], b = c[p];
          const bool up = (t & k) == 0;
          if ((a > b) == up) {
            c[t] = b;
            c[p] = a;
          }
        }
      }
      __syncwarp();
    }
  // distinct values: c[t] != c[t-1], below INT_MAX
  int base = 0;
  for (int t0 = 0; t0 < m; t0 += 32) {
    const int t = t0 + lane;
    const bool keep = t < ncand && c[t] != INT_MAX && (t == 0 || c[t] != c[t - 1]);
    const unsigned mask = __ballot_sync(0xffffffffu, keep);
    if (WRITE && keep) {
      const int pos = rowptr[r] + base + __popc(mask & ((1u << lane) - 1u));
      colind[pos] = c[t];
      if (c[t] == r) diagblk[r] = pos;
    }
    base += __popc(mask);
  }
  if (!WRITE && lane == 0) counts[r] = base;
}

// ---- 4. element -> block scatter map -------------------------------------------
__global__ void k_emap(long eLen, int nn, const int *__restrict__ enodes, const int *__restrict__ node_rank,
                       const int *__restrict__ rowptr, const int *__restrict__ colind, int *__restrict__ emap) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;  // (element, node a)
  if (i >= eLen * nn) return;
  const long e = i / nn;
  const int ra = node_rank[enodes[i]];
  const int k0 = rowptr[ra], k1 = rowptr[ra + 1];
  for (int cc = 0; cc < nn; cc++) {
    const int rc = node_rank[enodes[e * nn + cc]];
    int lo = k0, hi = k1;  // first position with colind >= rc
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (colind[mid] < rc) lo = mid + 1;
      else hi = mid;
    }
    emap[i * nn + cc] = lo;
  }
}

// ---- 5. Jones-Plassmann element colouring -----------------------------------------
__device__ __forceinline__ unsigned prio_hash(unsigned x) {  // a 32-bit integer mix (xorshift-multiply)
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// one round: an uncoloured element that comes before all its uncoloured
// neighbours takes a colour; every element's colour is carried into col_new.
// state[0] counts the elements left uncoloured, state[1] is an error flag.
__global__ void k_jp_round(long eLen, int nn, const int *__restrict__ enodes, const int *__restrict__ node_rank,
                           const int *__restrict__ n2e_ptr, const int *__restrict__ n2e,
                           const int *__restrict__ col_old, int *__restrict__ col_new, int *__restrict__ state) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= eLen) return;
  int c = col_old[e];
  if (c < 0) {
    const unsigned pe = prio_hash((unsigned)e);
    unsigned long long used = 0;
    bool first = true;
    for (int a = 0; a < nn && first; a++) {
      const int r = node_rank[enodes[e * nn + a]];
      for (int q = n2e_ptr[r]; q < n2e_ptr[r + 1]; q++) {
        const int f = n2e[q];
        if (f == e) continue;
        const int cf = col_old[f];
        if (cf >= 0) {
          used |= 1ull << cf;
        } else {
          const unsigned pf = prio_hash((unsigned)f);
          if (pf > pe || (pf == pe && f > e)) {  // an uncoloured neighbour comes first
            first = false;
            break;
          }
        }
      }
    }
    if (!first) {
      atomicAdd(state, 1);
    } else if (used == ~0ull) {
      atomicExch(state + 1, 2);
    } else {
      c = __ffsll((long long)~used) - 1;
    }
  }
  col_new[e] = c;
}

__global__ void k_blkrow(int nbr, const int *__restrict__ rowptr, int *__restrict__ blkrow) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nbr) return;
  for (int k = rowptr[r]; k < rowptr[r + 1]; k++) blkrow[k] = r;
}

}  // namespace

int gpu_build_pattern(ufem_model *m) {
  const int nn = m->nn, b = m->b;
  const long nLen = m->nLen, eLen = m->eLen, nent = eLen * nn;
  int rv;
  UFEM_CUDA_TRY(cudaGetDevice(&m->device));
  auto grid = [](long n) { return (unsigned)((n + 255) / 256); };
  if ((rv = m->d_enodes.upload(m->enodes.data(), m->enodes.size()))) return rv;
  DBuf<int> used, scan, err;
  if ((rv = used.alloc(nLen)) || (rv = scan.alloc(nLen)) || (rv = err.alloc(1))) return rv;
  UFEM_CUDA_TRY(cudaMemset(used.p, 0, nLen * sizeof(int)));
  UFEM_CUDA_TRY(cudaMemset(err.p, 0, sizeof(int)));
  k_mark_used<<<grid(nent), 256>>>(nent, m->d_enodes.p, used.p);
  long nbr = 0;
  if ((rv = scan_exclusive(nLen, used.p, scan.p, &nbr))) return rv;
  if (nbr < 1) {
    set_error("no degrees of freedom found");
    return UFEM_AF_ERR_SIZ;
  }
  DBuf<int> rank_node;
  if ((rv = m->d_noderank.alloc(nLen)) || (rv = rank_node.alloc(nbr))) return rv;
  k_node_rank<<<grid(nLen), 256>>>(nLen, used.p, scan.p, m->d_noderank.p, rank_node.p);
  // node -> element incidence
  DBuf<int> n2e_ptr, fill, n2e;
  if ((rv = n2e_ptr.alloc(nbr + 1)) || (rv = fill.alloc(nbr + 1)) || (rv = n2e.alloc(nent))) return rv;
  UFEM_CUDA_TRY(cudaMemset(n2e_ptr.p, 0, (nbr + 1) * sizeof(int)));
  k_inc_count<<<grid(nent), 256>>>(eLen, nn, m->d_enodes.p, m->d_noderank.p, n2e_ptr.p);
  long tot = 0;
  if ((rv = scan_exclusive(nbr + 1, n2e_ptr.p, n2e_ptr.p, &tot))) return rv;
  UFEM_CUDA_TRY(cudaMemcpy(fill.p, n2e_ptr.p, (nbr + 1) * sizeof(int), cudaMemcpyDeviceToDevice));
  k_inc_fill<<<grid(nent), 256>>>(eLen, nn, m->d_enodes.p, m->d_noderank.p, fill.p, n2e.p);
  // block columns: counts, rowptr, colind, diagblk
  const unsigned grow = (unsigned)((nbr + kRowWarps - 1) / kRowWarps);
  if ((rv = m->d_rowptr.alloc(nbr + 1)) || (rv = m->d_diagblk.alloc(nbr))) return rv;
  UFEM_CUDA_TRY(cudaMemset(m->d_rowptr.p, 0, (nbr + 1) * sizeof(int)));
  k_row_cols<false><<<grow, kRowWarps * 32>>>((int)nbr, nn, m->d_enodes.p, m->d_noderank.p, n2e_ptr.p, n2e.p,
                                              m->d_rowptr.p, nullptr, nullptr, nullptr, err.p);
  int herr = 0;
  UFEM_CUDA_TRY(cudaMemcpy(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (herr) {
    set_error("pattern build: a node is shared by more element-node incidences than the row gather holds (1024)");
    return UFEM_AF_ERR_BIG;
  }
  long nnzb = 0;
  if ((rv = scan_exclusive(nbr + 1, m->d_rowptr.p, m->d_rowptr.p, &nnzb))) return rv;
  if ((rv = m->d_colind.alloc(nnzb))) return rv;
  k_row_cols<true><<<grow, kRowWarps * 32>>>((int)nbr, nn, m->d_enodes.p, m->d_noderank.p, n2e_ptr.p, n2e.p,
                                             nullptr, m->d_rowptr.p, m->d_colind.p, m->d_diagblk.p, err.p);
  // scatter map
  if ((rv = m->d_emap.alloc((size_t)nent * nn))) return rv;
  k_emap<<<grid(nent), 256>>>(eLen, nn, m->d_enodes.p, m->d_noderank.p, m->d_rowptr.p, m->d_colind.p, m->d_emap.p);
  // colouring
  DBuf<int> col_a, col_b, state;
  if ((rv = col_a.alloc(eLen)) || (rv = col_b.alloc(eLen)) || (rv = state.alloc(2))) return rv;
  UFEM_CUDA_TRY(cudaMemset(col_a.p, 0xff, eLen * sizeof(int)));
  int hstate[2] = {1, 0};
  for (int round = 0; hstate[0] > 0; round++) {
    if (round == 100000) {  // each round colours at least the first uncoloured element
      set_error("element colouring did not finish");
      return UFEM_AF_ERR;
    }
    UFEM_CUDA_TRY(cudaMemset(state.p, 0, 2 * sizeof(int)));
    k_jp_round<<<grid(eLen), 256>>>(eLen, nn, m->d_enodes.p, m->d_noderank.p, n2e_ptr.p, n2e.p, col_a.p, col_b.p,
                                    state.p);
    std::swap(col_a.p, col_b.p);
    UFEM_CUDA_TRY(cudaMemcpy(hstate, state.p, 2 * sizeof(int), cudaMemcpyDeviceToHost));
    if (hstate[1] == 2) {
      set_error("element colouring needs more than 64 colours");
      return UFEM_AF_ERR_BIG;
    }
  }
  if ((rv = m->d_blkrow.alloc(nnzb))) return rv;
  k_blkrow<<<grid(nbr), 256>>>((int)nbr, m->d_rowptr.p, m->d_blkrow.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  // host copies: block rows and colours now, the pattern on first use
  m->nbr = (int)nbr;
  m->nnzb = nnzb;
  m->host_pattern_ok = false;
  m->node_rank.resize(nLen);
  m->rank_node.resize(nbr);
  std::vector<int> ecol(eLen);
  UFEM_CUDA_TRY(cudaMemcpy(m->node_rank.data(), m->d_noderank.p, nLen * sizeof(int), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(m->rank_node.data(), rank_node.p, nbr * sizeof(int), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(ecol.data(), col_a.p, eLen * sizeof(int), cudaMemcpyDeviceToHost));
  // DOF numbers follow from the block rows (ufem_model::dof)
  m->nDOFAct = (long)b * nbr;
  // elements grouped by colour, in element order within a colour
  int ncol = 0;
  for (long e = 0; e < eLen; e++) ncol = std::max(ncol, ecol[e] + 1);
  m->ncolours = ncol;
  m->colour_ptr.assign(ncol + 1, 0);
  for (long e = 0; e < eLen; e++) m->colour_ptr[ecol[e] + 1]++;
  for (int c = 0; c < ncol; c++) m->colour_ptr[c + 1] += m->colour_ptr[c];
  m->colour_elems.resize(eLen);
  {
    std::vector<int> f(m->colour_ptr.begin(), m->colour_ptr.end() - 1);
    for (long e = 0; e < eLen; e++) m->colour_elems[f[ecol[e]]++] = (int)e;
  }
  return m->d_colour_elems.upload(m->colour_elems.data(), m->colour_elems.size());
}

int host_pattern(const ufem_model *m) {
  if (m->host_pattern_ok) return UFEM_AF_OK;
  m->rowptr.resize(m->nbr + 1);
  m->colind.resize(m->nnzb);
  m->diagblk.resize(m->nbr);
  m->emap.resize((size_t)m->eLen * m->nn * m->nn);
  UFEM_CUDA_TRY(cudaMemcpy(m->rowptr.data(), m->d_rowptr.p, (m->nbr + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(m->colind.data(), m->d_colind.p, m->nnzb * sizeof(int), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(m->diagblk.data(), m->d_diagblk.p, m->nbr * sizeof(int), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(m->emap.data(), m->d_emap.p, m->emap.size() * sizeof(int), cudaMemcpyDeviceToHost));
  m->host_pattern_ok = true;
  return UFEM_AF_OK;
}

}  // namespace ufem
