// Self-tests of the bounded device waits (no reference counterpart).
//
// Every spin-wait in the library's kernels has a limit after which the
// kernel records an error and returns, so a wait that cannot end -- a block
// that never reaches a grid barrier, an MMA completion that never arrives --
// becomes an AF_ERR on the host and the CUDA context stays usable.  These
// entry points make each kind of wait run out on purpose, with nothing in
// flight that could fault: the grid barrier of the persistent solvers with one
// block that leaves without arriving, and the mbarrier wait of the tensor-core
// phases on a barrier that nothing signals.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_util.cuh"
#include "tcgen05.cuh"
#include "ufem_internal.h"

namespace ufem {
namespace {

// Block `skip` returns without arriving; every other block waits at the
// barrier until its limit, then records that it timed out.
__global__ void k_barrier_selftest(GridBar *bar, int skip, int *timed_out) {
  if ((int)blockIdx.x == skip) return;
  const bool ok = grid_barrier(bar);
  if (threadIdx.x == 0 && !ok) atomicAdd(timed_out, 1);
}

// One thread waits on an mbarrier that expects one arrival nobody makes.
__global__ void k_mbar_selftest(long spin_limit, int *timed_out) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) *timed_out = tc::mbar_wait(&bar, 0, spin_limit) ? 0 : 1;
}

}  // namespace
}  // namespace ufem

using namespace ufem;

extern "C" {

int ufem_selftest_barrier_timeout(int nblocks, int limit_ms, int *blocks_timed_out, double *ms) {
  if (nblocks < 2 || limit_ms < 1 || limit_ms > 2000) {
    set_error("ufem_selftest_barrier_timeout: at least 2 blocks and a limit of 1 to 2000 ms");
    return UFEM_AF_ERR_VAL;
  }
  int dev = 0, nsm = 0, occ = 0;
  UFEM_CUDA_TRY(cudaGetDevice(&dev));
  UFEM_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  UFEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_barrier_selftest, 128, 0));
  if (nblocks > nsm * occ) {
    set_error("ufem_selftest_barrier_timeout: more blocks than are co-resident");
    return UFEM_AF_ERR_VAL;
  }
  DBuf<GridBar> bar;
  DBuf<int> to;
  int rv;
  if ((rv = bar.alloc(1)) || (rv = to.alloc(1))) return rv;
  GridBar hb{0u, 0u, 0, limit_ms};
  UFEM_CUDA_TRY(cudaMemcpy(bar.p, &hb, sizeof(hb), cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemset(to.p, 0, sizeof(int)));
  int skip = 0;
  void *args[] = {&bar.p, &skip, &to.p};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  UFEM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)k_barrier_selftest, dim3(nblocks), dim3(128), args, 0, 0));
  cudaEventRecord(e1);
  UFEM_CUDA_TRY(cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms) *ms = t;
  int nto = 0;
  UFEM_CUDA_TRY(cudaMemcpy(&hb, bar.p, sizeof(hb), cudaMemcpyDeviceToHost));
  UFEM_CUDA_TRY(cudaMemcpy(&nto, to.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (blocks_timed_out) *blocks_timed_out = nto;
  if (hb.err) {
    set_error("persistent kernel: grid barrier timed out");
    return UFEM_AF_ERR;
  }
  return UFEM_AF_OK;
}

int ufem_selftest_mma_wait_timeout(long spin_limit, int *timed_out) {
  if (spin_limit < 1 || spin_limit > (1L << 24)) {
    set_error("ufem_selftest_mma_wait_timeout: a spin limit of 1 to 2^24");
    return UFEM_AF_ERR_VAL;
  }
  DBuf<int> to;
  int rv;
  if ((rv = to.alloc(1))) return rv;
  UFEM_CUDA_TRY(cudaMemset(to.p, 0, sizeof(int)));
  k_mbar_selftest<<<1, 32>>>(spin_limit, to.p);
  UFEM_CUDA_TRY(cudaGetLastError());
  UFEM_CUDA_TRY(cudaDeviceSynchronize());
  int h = 0;
  UFEM_CUDA_TRY(cudaMemcpy(&h, to.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (timed_out) *timed_out = h;
  if (h) {
    set_error("tensor-core completion wait timed out");
    return UFEM_AF_ERR;
  }
  return UFEM_AF_OK;
}

}  // extern "C"
