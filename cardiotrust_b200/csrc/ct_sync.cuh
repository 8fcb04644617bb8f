// Bounded device-side waits.
#pragma once

#include "ct_internal.cuh"

namespace ct {

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_gpu(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier for a cooperative launch (all CTAs co-resident) on a
// monotone arrival counter: barrier number n (0, 1, ...) completes when the
// counter reaches (n + 1) * gridDim.x. Thread 0 arrives with a release
// reduction and polls with acquire loads; the CTA barriers on either side
// extend the ordering to the whole CTA. The wait is bounded (~2 s of
// globaltimer): on expiry the CTA records CT_ERR_TIMEOUT in *status and
// returns false; CTAs also leave once another CTA has recorded an error.
// Callers must stop issuing work when this returns false.
__device__ __forceinline__ bool grid_barrier(GridBarrier* bar, unsigned int number, int32_t* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int target = (number + 1u) * gridDim.x;
    red_release_gpu(&bar->count, 1u);
    if (ld_acquire_gpu(&bar->count) < target) {
      const unsigned long long t0 = global_ns();
      while (ld_acquire_gpu(&bar->count) < target) {
        if (*(volatile int32_t*)status != 0) {
          ok = 0;
          break;
        }
        if (global_ns() - t0 > 2000000000ull) {
          atomicCAS(status, 0, (int32_t)CT_ERR_TIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Cooperative launch (all CTAs co-resident, required by grid_barrier) through cudaLaunchKernelExC with
// the cooperative attribute, which stream capture records as a cooperative kernel node.
inline cudaError_t launch_cooperative(const void* func, int grid, int block, void** args, size_t smem,
                                      cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, func, args);
}

}  // namespace ct
