// Bounded device-side waits.
#pragma once

#include "ct_internal.cuh"

namespace ct {

// Grid-wide barrier for a cooperative launch (all CTAs co-resident).
// Every wait is bounded: after kSpinLimit polls the CTA records CT_ERR_TIMEOUT
// in *status and returns false; CTAs also leave early once another CTA has
// recorded an error. Callers must stop issuing work when this returns false.
__device__ __forceinline__ bool grid_barrier(GridBarrier* bar, int32_t* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned int* vgen = &bar->generation;
    const unsigned int gen = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(&bar->count, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(&bar->count, 0u);
      __threadfence();
      atomicAdd(&bar->generation, 1u);
    } else {
      long long spins = 0;
      while (*vgen == gen) {
        if (*(volatile int32_t*)status != 0) {
          ok = 0;
          break;
        }
        if (++spins > kSpinLimit) {
          atomicCAS(status, 0, (int32_t)CT_ERR_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

}  // namespace ct
