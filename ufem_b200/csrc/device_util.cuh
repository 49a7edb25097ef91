// Device helpers shared by the solver kernels: a bounded grid barrier for
// persistent (cooperatively launched) kernels and deterministic reductions.
#pragma once

#include <cuda_runtime.h>

namespace ufem {

// Generation-counting grid barrier.  Every wait is bounded: after
// kBarrierTimeoutNs of global time (or limit_ms, when set) the waiting block
// records an error, leaves the barrier and the kernel returns; the host turns
// the flag into AF_ERR.
struct GridBar {
  unsigned int count;
  unsigned int gen;
  int err;
  int limit_ms;  // 0: kBarrierTimeoutNs; set shorter by the self-test of the wait
};

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool grid_barrier(GridBar *gb) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int *vgen = &gb->gen;
    volatile int *verr = &gb->err;
    unsigned int g = *vgen;
    __threadfence();
    unsigned int arrived = atomicAdd(&gb->count, 1u);
    int ok = 1;
    if (arrived == gridDim.x - 1) {
      atomicExch(&gb->count, 0u);
      __threadfence();
      atomicAdd(&gb->gen, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      const int lim = gb->limit_ms;
      const unsigned long long limit_ns = lim > 0 ? (unsigned long long)lim * 1000000ull : kBarrierTimeoutNs;
      while (*vgen == g) {
        if (*verr) {
          ok = 0;
          break;
        }
        if (global_ns() - t0 > limit_ns) {
          atomicExch(&gb->err, 1);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    if (*verr) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-level partial sums of NV values, written by thread 0 to out[0..NV).
// Fixed combination order: lanes by xor-tree, warps in index order.
template <int NV>
__device__ __forceinline__ void block_partials(const double (&v)[NV], double *out) {
  __shared__ double s_w[32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double t = warp_sum(v[k]);
    if (lane == 0) s_w[warp][k] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = 0.0;
      for (int w = 0; w < nw; w++) t += s_w[w][k];
      out[k] = t;
    }
  }
  __syncthreads();
}

// Sum of part[g*NV + k] over g < G, identical in every block (fixed order).
template <int NV>
__device__ __forceinline__ void grid_total(const double *part, int G, double (&tot)[NV]) {
  __shared__ double s_t[NV];
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = 0.0;
      for (int g = lane; g < G; g += 32) t += __ldcg(part + (size_t)g * NV + k);
      t = warp_sum(t);
      if (lane == 0) s_t[k] = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; k++) tot[k] = s_t[k];
  __syncthreads();
}

}  // namespace ufem
