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
//   * Voxels are in device order (4x4x2 bricks, see ct_api.cu), cut into
//     tiles of kTileVoxels consecutive device voxels; a persistent
//     cooperative grid walks the tiles.
//   * Every read of the recurrence is of x[t-d] or x[t-d-1] with d >= 1, so
//     the states of steps t .. t+L-1 are independent when L <= min delay.
//     The kernel advances L = min(dmin, kMaxStepBlock) steps between two grid
//     barriers.
//   * The all-pass state is deduplicated: ap_outputs[3v+a, 3n+b] does not
//     depend on the row component a (same input state, coefficient and zero
//     start, prediction.rs:56-79), so it is kept as [V, 26*3].
//   * Shared memory holds, per tile: the gains transposed to [k][state]
//     (entries of absent neighbours zeroed, which adds exact zeros where the
//     reference skips), the (neighbour, delay, coefficient) of each
//     (voxel, offset) pair, the all-pass state, and the all-pass outputs of
//     one round of steps. A CTA that owns one tile stages it once per launch.
//   * A block of L steps runs in rounds of kSlots steps. Phase A: one thread
//     per (voxel, offset) runs the three all-pass chains for the round's steps;
//     its 3 (kSlots + 1) history loads are independent and issued together.
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
constexpr int kTileStates = 3 * kTileVoxels;
constexpr int kTileItems = kTileVoxels * kOffsets;  // (voxel, offset) pairs
constexpr int kThreads = 256;
constexpr int kParity = 2;  // phase-B step groups per state
constexpr int kItemsPerThread = (kTileItems + kThreads - 1) / kThreads;
constexpr int kSlots = 4;   // steps per round: a block of L steps runs in ceil(L / kSlots) rounds

struct FwdArgs {
  int V, S, T;
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

struct Smem {
  float gT[kGainCols][kTileStates];           // gains, transposed, absent neighbours zeroed
  float ap_out[kSlots][kTileVoxels * kGainCols];
  float ap_state[kTileVoxels * kGainCols];
  float x[kMaxStepBlock][kTileStates];
  int32_t j[kTileItems];                       // 3 * neighbour, -1 if absent
  int32_t d[kTileItems];
  float c[kTileItems];
  float ctrl[kTileStates];
  float part[kMaxStepBlock];
};

// Stage one tile: metadata first (the gain mask needs it), then the gains and the chain state.
__device__ __forceinline__ void stage_tile(Smem& sm, const FwdArgs& p, int v0) {
  const int nv = min(kTileVoxels, p.V - v0);
  for (int e = threadIdx.x; e < kTileItems; e += blockDim.x) {
    const int vl = e / kOffsets;
    if (vl < nv) {
      const int g = v0 * kOffsets + e;
      const int32_t nb = p.nbr[g];
      sm.j[e] = nb < 0 ? -1 : 3 * nb;
      sm.d[e] = p.delays[g];
      sm.c[e] = p.coefs[g];
    } else {
      sm.j[e] = -1;
      sm.d[e] = 1;
      sm.c[e] = 0.0f;
    }
  }
  for (int e = threadIdx.x; e < kTileStates; e += blockDim.x)
    sm.ctrl[e] = (e < 3 * nv) ? p.ctrl[3 * v0 + e] : 0.0f;
  __syncthreads();
  // gains: coalesced along each row, written transposed
  const float* g0 = p.gains + (size_t)3 * v0 * kGainCols;
  for (int e = threadIdx.x; e < kTileStates * kGainCols; e += blockDim.x) {
    const int st = e / kGainCols, k = e - st * kGainCols;
    float g = 0.0f;
    if (st < 3 * nv && sm.j[(st / 3) * kOffsets + k / 3] >= 0) g = g0[e];
    sm.gT[k][st] = g;
  }
  const float* a0 = p.ap + (size_t)v0 * kGainCols;
  for (int e = threadIdx.x; e < kTileVoxels * kGainCols; e += blockDim.x)
    sm.ap_state[e] = (e < nv * kGainCols) ? a0[e] : 0.0f;
  __syncthreads();
}

__device__ __forceinline__ void unstage_tile(Smem& sm, const FwdArgs& p, int v0) {
  const int nv = min(kTileVoxels, p.V - v0);
  float* a0 = p.ap + (size_t)v0 * kGainCols;
  for (int e = threadIdx.x; e < nv * kGainCols; e += blockDim.x) a0[e] = sm.ap_state[e];
}

__global__ void __launch_bounds__(kThreads, 1) forward_kernel(FwdArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);

  const int V = p.V, S = p.S, T = p.T;
  const int num_tiles = (V + kTileVoxels - 1) / kTileVoxels;
  const bool resident = num_tiles <= (int)gridDim.x;  // this CTA owns at most one tile
  int dmin = *p.dmin;
  if (dmin < 1) dmin = 1;
  const int Lmax = dmin < kMaxStepBlock ? dmin : kMaxStepBlock;

  if (resident && (int)blockIdx.x < num_tiles) stage_tile(sm, p, blockIdx.x * kTileVoxels);

  for (int t0 = 0; t0 < T; t0 += Lmax) {
    const int L = (T - t0) < Lmax ? (T - t0) : Lmax;
    if (threadIdx.x < kMaxStepBlock) sm.part[threadIdx.x] = 0.0f;

    for (int tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
      const int v0 = tile * kTileVoxels;
      const int nv = min(kTileVoxels, V - v0);
      if (!resident) stage_tile(sm, p, v0);

      for (int r0 = 0; r0 < L; r0 += kSlots) {
        const int R = (L - r0) < kSlots ? (L - r0) : kSlots;  // steps in this round
        const int tr0 = t0 + r0;                                // first step of the round
        // ---- phase A: three all-pass chains per (voxel, offset)
#pragma unroll
        for (int r = 0; r < kItemsPerThread; ++r) {
          const int e = threadIdx.x + r * kThreads;
          if (e >= kTileItems) break;
          const int vl = e / kOffsets;
          const int n = e - vl * kOffsets;
          const int jb = sm.j[e];
          float* st = sm.ap_state + vl * kGainCols + 3 * n;
          if (jb >= 0) {
            const int d = sm.d[e];
            const float c = sm.c[e];
            // h[q][b] = x[tr0 - d - 1 + q, jb + b]; in(tr0+s) = h[s+1], in_delayed(tr0+s) = h[s];
            // rows before t = 0 read as zero (prediction.rs:68-77)
            float h[kSlots + 1][3];
#pragma unroll
            for (int q = 0; q <= kSlots; ++q) {
              const int tr = tr0 - d - 1 + q;
              const bool ok = q <= R && tr >= 0;
              const float* row = p.X + (size_t)(ok ? tr : 0) * S + jb;
#pragma unroll
              for (int b = 0; b < 3; ++b) h[q][b] = ok ? row[b] : 0.0f;
            }
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              float a = st[b];
#pragma unroll
              for (int s = 0; s < kSlots; ++s) {
                if (s < R) {
                  a = fmaf(c, h[s + 1][b] - a, h[s][b]);
                  sm.ap_out[s][vl * kGainCols + 3 * n + b] = a;
                  if (tr0 + s == T - 2) p.ap_last[(size_t)(v0 + vl) * kGainCols + 3 * n + b] = a;
                }
              }
              st[b] = a;
            }
          } else {
#pragma unroll
            for (int s = 0; s < kSlots; ++s)
              if (s < R)
#pragma unroll
                for (int b = 0; b < 3; ++b) sm.ap_out[s][vl * kGainCols + 3 * n + b] = 0.0f;
            if (vl < nv && T - 2 >= tr0 && T - 2 < tr0 + R)
#pragma unroll
              for (int b = 0; b < 3; ++b) p.ap_last[(size_t)(v0 + vl) * kGainCols + 3 * n + b] = st[b];
          }
        }
        __syncthreads();

        // ---- phase B: gain-weighted sums in column order, plus the control input
        if (threadIdx.x < kTileStates * kParity) {
          const int par = threadIdx.x / kTileStates;
          const int st = threadIdx.x - par * kTileStates;
          const int vl = st / 3;
          if (vl < nv) {
            constexpr int Q = kSlots / kParity;
            float acc[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) acc[q] = 0.0f;
#pragma unroll 6
            for (int k = 0; k < kGainCols; ++k) {
              const float g = sm.gT[k][st];
#pragma unroll
              for (int q = 0; q < Q; ++q) {
                const int s = par + kParity * q;
                if (s < R) acc[q] = acc[q] + g * sm.ap_out[s][vl * kGainCols + k];
              }
            }
            const float cm = sm.ctrl[st];
            float* xcol = p.X + 3 * v0 + st;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
              const int s = par + kParity * q;
              if (s < R) {
                const float x = acc[q] + p.u[tr0 + s] * cm;
                xcol[(size_t)(tr0 + s) * S] = x;
                sm.x[r0 + s][st] = x;
              }
            }
          }
        }
        __syncthreads();
      }

      // ---- maximum-regularisation contribution of this tile, per step (fixed-order tree)
      if (threadIdx.x < 32) {
        const int vl = threadIdx.x;
        for (int s = 0; s < L; ++s) {
          float f2 = 0.0f;
          if (vl < nv) {
            const float sum = fabsf(sm.x[s][3 * vl]) + fabsf(sm.x[s][3 * vl + 1]) + fabsf(sm.x[s][3 * vl + 2]);
            if (sum > p.threshold) {
              const float f = sum - p.threshold;
              f2 = f * f;
            }
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) f2 = f2 + __shfl_down_sync(0xffffffffu, f2, off);
          if (vl == 0) sm.part[s] = sm.part[s] + f2;
        }
      }
      if (!resident) {
        __syncthreads();
        unstage_tile(sm, p, v0);
      }
      __syncthreads();
    }
    if ((int)threadIdx.x < L) p.stepsum_part[(size_t)(t0 + threadIdx.x) * gridDim.x + blockIdx.x] = sm.part[threadIdx.x];
    if (t0 + L < T) {
      if (!grid_barrier(p.barrier, p.status)) return;
    }
  }
  if (resident && (int)blockIdx.x < num_tiles) unstage_tile(sm, p, blockIdx.x * kTileVoxels);
}

}  // namespace

int forward_grid_size(int64_t V, int device) {
  static bool configured[128] = {};
  if (device >= 0 && device < 128 && !configured[device]) {
    cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
    configured[device] = true;
  }
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, forward_kernel, kThreads, sizeof(Smem));
  if (per_sm < 1) per_sm = 1;
  const int64_t tiles = (V + kTileVoxels - 1) / kTileVoxels;
  int64_t grid = (int64_t)sms * per_sm;
  if (tiles < grid) grid = tiles;
  if (grid < 1) grid = 1;
  return (int)grid;
}

cudaError_t launch_forward(DeviceScenario& d, float threshold, cudaStream_t stream) {
  FwdArgs a;
  a.V = (int)d.V;
  a.S = (int)d.S;
  a.T = (int)d.T;
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
                                     sizeof(Smem), stream);
}

}  // namespace ct
