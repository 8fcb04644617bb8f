// Forward propagation of one beat (system prediction without the measurement
// product): innovate_system_states_v1 + add_control_function,
// src/core/algorithm/estimation/prediction.rs:40-106.
//
// Compiled with -fmad=false: every `a + b * c` below rounds the product and
// the sum separately, as the reference does; fmaf() appears exactly where the
// reference calls mul_add. The state values are therefore bit-identical to the
// reference CPU loop.
//
// Layout and schedule
//   * Voxels are cut into tiles of kTileVoxels consecutive voxel numbers; a
//     persistent cooperative grid walks the tiles.
//   * Every read of the recurrence is of x[t-d] or x[t-d-1] with d >= 1, so
//     the states of steps t .. t+L-1 are independent when L <= min delay.
//     The kernel advances L = min(dmin, kMaxStepBlock) steps between two grid
//     barriers.
//   * The all-pass state is deduplicated: ap_outputs[3v+a, 3n+b] does not
//     depend on the row component a (same input state, coefficient and zero
//     start, prediction.rs:56-79), so it is kept as [V, 26*3].
//   * Phase A: one thread per (voxel, offset, component) runs the L-step
//     all-pass chain and stages the L outputs in shared memory.
//     Phase B: one thread per (voxel, row component, step parity) sums the 78
//     gain-weighted outputs in column order k = 0..77 for its steps.
//   * History reads go through L1: within one launch a history row is read
//     only after the grid barrier that completes it, so no SM can hold a
//     stale line of it (L1 holds no global data across launches).
#include <cuda_runtime.h>

#include "ct_internal.cuh"
#include "ct_sync.cuh"

namespace ct {
namespace {

constexpr int kTileVoxels = 32;
constexpr int kThreads = 256;
constexpr int kParity = 2;  // phase-B step groups per state

struct FwdArgs {
  int64_t V, S, T;
  const int32_t* nbr;
  const float* coefs;
  const int32_t* delays;
  const float* gains;
  const float* ctrl;
  const float* u;
  float* X;
  float* ap;
  float* ap_last;
  float* stepsum_part;
  const int32_t* dmin;
  float threshold;
  int32_t* status;
  GridBarrier* barrier;
};

constexpr size_t kSmemAp = sizeof(float) * kMaxStepBlock * kTileVoxels * kGainCols;
constexpr size_t kSmemX = sizeof(float) * kMaxStepBlock * kTileVoxels * 3;
constexpr size_t kSmemPart = sizeof(float) * kMaxStepBlock;
constexpr size_t kSmemBytes = kSmemAp + kSmemX + kSmemPart;

__global__ void __launch_bounds__(kThreads) forward_kernel(FwdArgs p) {
  extern __shared__ float smem[];
  float* sm_ap = smem;                                       // [L][TV*78]
  float* sm_x = smem + kMaxStepBlock * kTileVoxels * kGainCols;  // [L][TV*3]
  float* sm_part = sm_x + kMaxStepBlock * kTileVoxels * 3;   // [L]

  const int64_t V = p.V, S = p.S, T = p.T;
  const int64_t num_tiles = (V + kTileVoxels - 1) / kTileVoxels;
  int dmin = *p.dmin;
  if (dmin < 1) dmin = 1;
  const int Lmax = dmin < kMaxStepBlock ? dmin : kMaxStepBlock;

  for (int64_t t0 = 0; t0 < T; t0 += Lmax) {
    const int L = (T - t0) < Lmax ? (int)(T - t0) : Lmax;
    if (threadIdx.x < kMaxStepBlock) sm_part[threadIdx.x] = 0.0f;

    for (int64_t tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
      const int64_t v0 = tile * kTileVoxels;
      // ---- phase A: all-pass chains
      for (int item = threadIdx.x; item < kTileVoxels * kGainCols; item += blockDim.x) {
        const int vl = item / kGainCols;
        const int kk = item - vl * kGainCols;
        const int64_t v = v0 + vl;
        if (v >= V) continue;
        const int n = kk / 3, b = kk - 3 * (kk / 3);
        const int32_t nb = p.nbr[v * kOffsets + n];
        float a = p.ap[v * kGainCols + kk];
        if (nb >= 0) {
          const int64_t j = 3 * (int64_t)nb + b;
          const int64_t d = p.delays[v * kOffsets + n];
          const float c = p.coefs[v * kOffsets + n];
          // h[q] = x[t0 - d - 1 + q, j]: in(t0+s) = h[s+1], in_delayed(t0+s) = h[s]; rows before
          // t = 0 read as zero (prediction.rs:68-77). All loads are independent and issued together.
          float h[kMaxStepBlock + 1];
#pragma unroll
          for (int q = 0; q <= kMaxStepBlock; ++q) {
            const int64_t tr = t0 - d - 1 + q;
            h[q] = (q <= L && tr >= 0) ? p.X[tr * S + j] : 0.0f;
          }
#pragma unroll
          for (int s = 0; s < kMaxStepBlock; ++s) {
            if (s < L) {
              a = fmaf(c, h[s + 1] - a, h[s]);
              sm_ap[s * (kTileVoxels * kGainCols) + item] = a;
              if (t0 + s == T - 2) p.ap_last[v * kGainCols + kk] = a;
            }
          }
        } else {
          for (int s = 0; s < L; ++s) sm_ap[s * (kTileVoxels * kGainCols) + item] = 0.0f;
          if (T - 2 >= t0 && T - 2 < t0 + L) p.ap_last[v * kGainCols + kk] = a;
        }
        p.ap[v * kGainCols + kk] = a;
      }
      __syncthreads();
      // ---- phase B: gain-weighted sums in column order, plus the control input
      for (int item = threadIdx.x; item < kTileVoxels * 3 * kParity; item += blockDim.x) {
        const int par = item / (kTileVoxels * 3);
        const int st = item - par * (kTileVoxels * 3);
        const int vl = st / 3;
        const int64_t v = v0 + vl;
        if (v >= V) continue;
        const int64_t i = 3 * v + (st - 3 * vl);
        float acc[kMaxStepBlock / kParity];
#pragma unroll
        for (int q = 0; q < kMaxStepBlock / kParity; ++q) acc[q] = 0.0f;
        const float* grow = p.gains + i * kGainCols;
        const int32_t* nrow = p.nbr + v * kOffsets;
        for (int n = 0; n < kOffsets; ++n) {
          const bool valid = nrow[n] >= 0;
#pragma unroll
          for (int b = 0; b < 3; ++b) {
            const int k = 3 * n + b;
            const float g = valid ? __ldg(grow + k) : 0.0f;
#pragma unroll
            for (int q = 0; q < kMaxStepBlock / kParity; ++q) {
              const int s = par + kParity * q;
              if (s < L) acc[q] = acc[q] + g * sm_ap[s * (kTileVoxels * kGainCols) + vl * kGainCols + k];
            }
          }
        }
        const float cm = p.ctrl[i];
#pragma unroll
        for (int q = 0; q < kMaxStepBlock / kParity; ++q) {
          const int s = par + kParity * q;
          if (s < L) {
            const float x = acc[q] + p.u[t0 + s] * cm;
            p.X[(t0 + s) * S + i] = x;
            sm_x[s * (kTileVoxels * 3) + st] = x;
          }
        }
      }
      __syncthreads();
      // ---- maximum-regularisation contribution of this tile, per step (fixed-order tree)
      if (threadIdx.x < 32) {
        const int vl = threadIdx.x;
        for (int s = 0; s < L; ++s) {
          float f2 = 0.0f;
          if (v0 + vl < V) {
            const float* xs = sm_x + s * (kTileVoxels * 3) + 3 * vl;
            const float sum = fabsf(xs[0]) + fabsf(xs[1]) + fabsf(xs[2]);
            if (sum > p.threshold) {
              const float f = sum - p.threshold;
              f2 = f * f;
            }
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) f2 = f2 + __shfl_down_sync(0xffffffffu, f2, off);
          if (vl == 0) sm_part[s] = sm_part[s] + f2;
        }
      }
      __syncthreads();
    }
    if (threadIdx.x < L) p.stepsum_part[(t0 + threadIdx.x) * gridDim.x + blockIdx.x] = sm_part[threadIdx.x];
    if (t0 + L < T) {
      if (!grid_barrier(p.barrier, p.status)) return;
    }
  }
}

}  // namespace

int forward_grid_size(int64_t V, int device) {
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    configured = true;
  }
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, forward_kernel, kThreads, kSmemBytes);
  if (per_sm < 1) per_sm = 1;
  const int64_t tiles = (V + kTileVoxels - 1) / kTileVoxels;
  int64_t grid = (int64_t)sms * per_sm;
  if (tiles < grid) grid = tiles;
  if (grid < 1) grid = 1;
  return (int)grid;
}

cudaError_t launch_forward(DeviceScenario& d, float threshold, cudaStream_t stream) {
  FwdArgs a;
  a.V = d.V;
  a.S = d.S;
  a.T = d.T;
  a.nbr = d.nbr;
  a.coefs = d.coefs;
  a.delays = d.delays;
  a.gains = d.gains;
  a.ctrl = d.ctrl;
  a.u = d.u;
  a.X = d.X;
  a.ap = d.ap;
  a.ap_last = d.ap_last;
  a.stepsum_part = d.stepsum_part;
  a.dmin = d.dmin;
  a.threshold = threshold;
  a.status = d.status;
  a.barrier = d.barrier;
  cudaError_t err = cudaMemsetAsync(d.ap, 0, sizeof(float) * d.V * kGainCols, stream);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(d.ap_last, 0, sizeof(float) * d.V * kGainCols, stream);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(d.barrier, 0, sizeof(GridBarrier), stream);
  if (err != cudaSuccess) return err;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)forward_kernel, dim3(d.fwd_grid), dim3(kThreads), args,
                                     kSmemBytes, stream);
}

}  // namespace ct
