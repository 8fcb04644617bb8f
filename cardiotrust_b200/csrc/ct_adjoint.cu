// Adjoint (back-propagation through time) of one beat: the exact gradient of
// the stated loss
//   L = sum_t (mse/M)/2 |H x_t - z_t|^2 + reg/2 sum_v relu(|x_v|_1 - thr)^2
// with respect to the gains and all-pass coefficients, through the forward
// recursion of innovate_system_states_v1 (prediction.rs:40-86):
//   ap[t] = c (in_t - ap[t-1]) + in1_t,   in_t = x[t-d, j] (t >= d), in1_t = x[t-d-1, j] (t > d)
//   x[t, 3v+a] = sum_k g[3v+a, k] ap[t][v, k] + u[t] B[3v+a]          (k = 3n + b).
// The reference crate has no counterpart: its derivation (derivation.rs:173-
// 229) keeps only the per-step terms. The adjoint recursions are
//   lx[t, i]    = (mse/M) (H^T r_t)[i] + reg f_v sign(x_i)
//                 + sum over items (v', n') whose neighbour is i's voxel of
//                   c' lap[t + d'] + lap[t + d' + 1]                (0 beyond T-1)
//   lap[t][v,k] = sum_a g[3v+a, k] lx[t, 3v+a] - c lap[t+1][v,k]
//   dG[3v+a, k] += lx[t, 3v+a] ap[t][v,k]
//   dC[v, n]    += sum_b lap[t][v, 3n+b] (in_t - ap[t-1])
//
// Schedule (one cooperative launch per beat):
//   * Checkpoints: the forward kernel stores the all-pass state every
//     kCkptSteps steps. Segments of kCkptSteps steps are visited from the
//     last to the first; each CTA first recomputes, from the checkpoint and
//     the stored states, the all-pass outputs ap[t] and the differences
//     q[t] = in_t - ap[t-1] of its own tiles for the segment (the same fmaf
//     as the forward, so bit-identical), then steps the segment backwards.
//   * The coupling between voxels is a gather, not a scatter: voxel j pulls
//     the adjoint all-pass values of the items that read it from a ring of
//     recent steps, lap[t mod ring][v', k]. Those reads are of steps at least
//     dmin ahead, so L = min(dmin, kMaxStepBlock) steps run between grid
//     barriers, as in the forward. The sums run in a fixed order, so results
//     are deterministic.
//   * Thread (tile column) e = (voxel, k) owns 3 gain-gradient and 1
//     coefficient-gradient accumulators; a CTA that owns one tile keeps them
//     in registers for the whole launch, otherwise they are added to global
//     memory after every block of steps.
#include <cuda_runtime.h>

#include "ct_internal.cuh"
#include "ct_sync.cuh"

namespace ct {
namespace {

constexpr int kTileVoxels = kFwdTileVoxels;
constexpr int kTileStates = 3 * kTileVoxels;
constexpr int kTileItems = kTileVoxels * kOffsets;
constexpr int kTileCols = kTileVoxels * kGainCols;
constexpr int kAdjThreads = 256;
constexpr int kColsPerThread = (kTileCols + kAdjThreads - 1) / kAdjThreads;  // 10

struct AdjArgs {
  int V, S, T, ring;
  const int32_t* nbr;
  const int32_t* rev;  // [V,26] voxel v' whose offset n' points at this voxel, -1 if none
  const float* coefs;
  const int32_t* delays;
  const float* init_delays;
  const float* gains;
  const float* X;
  const float* MR;
  const float* ckpt;  // [ceil(T / kCkptSteps), V, 78]; slot s = state before step s * kCkptSteps
  float* seg_ap;      // [kCkptSteps, V, 78]
  float* seg_q;       // [kCkptSteps, V, 78]
  float* lam;         // [ring, V, 78]
  float* dG;
  float* dC;
  float* dCk;  // [V,78] coefficient-gradient partials per column (zero on entry, zero on exit)
  const int32_t* dmin;
  float mse_scaling, reg_scaling, threshold, diffreg;
  int freeze_gains, freeze_delays, ap_derivative;
  int32_t* status;
  GridBarrier* barrier;
};

struct AdjSmem {
  float lx[kTileStates];
  float pull[kTileCols];  // [voxel][n'][b]
  int32_t src[kTileItems];
  int32_t sd[kTileItems];
  float sc[kTileItems];
};

__device__ __forceinline__ float signum_f(float x) { return copysignf(1.0f, x); }

__device__ __forceinline__ float powi5_f(float x) {
  const float x2 = x * x;
  const float x4 = x2 * x2;
  return x * x4;
}

// In-items of a tile: (voxel j, offset n') -> source voxel, its delay and coefficient.
__device__ __forceinline__ void stage_in_items(AdjSmem& sm, const AdjArgs& p, int v0, int nv) {
  for (int e = threadIdx.x; e < kTileItems; e += blockDim.x) {
    const int vl = e / kOffsets, n = e - vl * kOffsets;
    int32_t src = -1;
    if (vl < nv) src = p.rev[(size_t)(v0 + vl) * kOffsets + n];
    sm.src[e] = src;
    sm.sd[e] = src >= 0 ? p.delays[(size_t)src * kOffsets + n] : 0;
    sm.sc[e] = src >= 0 ? p.coefs[(size_t)src * kOffsets + n] : 0.0f;
  }
}

// ap[t] and q[t] = in_t - ap[t-1] of the tile's columns for steps [t_lo, t_hi).
__device__ __forceinline__ void recompute_segment(const AdjArgs& p, int v0, int nv, int seg, int t_lo, int t_hi) {
  const size_t plane = (size_t)p.V * kGainCols;
  for (int e = threadIdx.x; e < nv * kGainCols; e += blockDim.x) {
    const int vl = e / kGainCols, k = e - vl * kGainCols;
    const int v = v0 + vl, n = k / 3, b = k - 3 * n;
    const size_t col = (size_t)v * kGainCols + k;
    const int32_t nb = p.nbr[(size_t)v * kOffsets + n];
    if (nb < 0) {
      for (int t = t_lo; t < t_hi; ++t) {
        p.seg_ap[(size_t)(t - t_lo) * plane + col] = 0.0f;
        p.seg_q[(size_t)(t - t_lo) * plane + col] = 0.0f;
      }
      continue;
    }
    const int d = p.delays[(size_t)v * kOffsets + n];
    const float c = p.coefs[(size_t)v * kOffsets + n];
    const float* xs = p.X + 3 * nb + b;
    float a = p.ckpt[(size_t)seg * plane + col];
    float in_prev = (t_lo - d - 1 >= 0) ? xs[(size_t)(t_lo - d - 1) * p.S] : 0.0f;
    constexpr int kU = 8;
    for (int t0 = t_lo; t0 < t_hi; t0 += kU) {
      float in[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int t = t0 + u;
        in[u] = (t < t_hi && t - d >= 0) ? xs[(size_t)(t - d) * p.S] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int t = t0 + u;
        if (t < t_hi) {
          const float q = in[u] - a;
          a = fmaf(c, q, in_prev);
          p.seg_ap[(size_t)(t - t_lo) * plane + col] = a;
          p.seg_q[(size_t)(t - t_lo) * plane + col] = q;
          in_prev = in[u];
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kAdjThreads) adjoint_kernel(AdjArgs p) {
  __shared__ AdjSmem sm;
  const int V = p.V, T = p.T, S = p.S;
  const int num_tiles = (V + kTileVoxels - 1) / kTileVoxels;
  const bool resident = num_tiles <= (int)gridDim.x;
  const size_t plane = (size_t)V * kGainCols;
  const int rmask = p.ring - 1;
  int dmin = p.dmin[0], dmax = p.dmin[1];
  if (dmin < 1) dmin = 1;
  if (dmax < dmin) dmax = dmin;
  const int Lmax = dmin < kMaxStepBlock ? dmin : kMaxStepBlock;
  if (dmax + Lmax + 1 > p.ring) {  // the ring cannot hold the delay spread (all CTAs leave here)
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(p.status, 0, (int32_t)CT_ERR_NOT_SUPPORTED);
    return;
  }

  float dg[kColsPerThread][3], dc[kColsPerThread];
#pragma unroll
  for (int i = 0; i < kColsPerThread; ++i) {
    dg[i][0] = dg[i][1] = dg[i][2] = 0.0f;
    dc[i] = 0.0f;
  }
  if (resident && (int)blockIdx.x < num_tiles) {
    const int v0 = blockIdx.x * kTileVoxels;
    stage_in_items(sm, p, v0, min(kTileVoxels, V - v0));
  }

  unsigned int barrier_number = 0;
  const int nseg = (T + kCkptSteps - 1) / kCkptSteps;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int t_lo = seg * kCkptSteps;
    const int t_hi = min(T, t_lo + kCkptSteps);
    for (int tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
      const int v0 = tile * kTileVoxels;
      recompute_segment(p, v0, min(kTileVoxels, V - v0), seg, t_lo, t_hi);
    }
    for (int tb = t_hi - 1; tb >= t_lo; tb -= Lmax) {
      const int t_end = max(t_lo, tb - Lmax + 1);
      for (int tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
        const int v0 = tile * kTileVoxels;
        const int nv = min(kTileVoxels, V - v0);
        if (!resident) {
          __syncthreads();
          stage_in_items(sm, p, v0, nv);
        }
        __syncthreads();
        for (int t = tb; t >= t_end; --t) {
          // 1) pulls: c' lap[t+d'] + lap[t+d'+1] of every in-item component (steps >= t + dmin)
          for (int e = threadIdx.x; e < kTileCols; e += kAdjThreads) {
            const int vl = e / kGainCols, r = e - vl * kGainCols;
            const int n = r / 3;
            const int ii = vl * kOffsets + n;
            const int src = sm.src[ii];
            float val = 0.0f;
            if (src >= 0) {
              const int t1 = t + sm.sd[ii];
              const size_t col = (size_t)src * kGainCols + r;
              const float a1 = t1 < T ? p.lam[(size_t)(t1 & rmask) * plane + col] : 0.0f;
              const float a2 = t1 + 1 < T ? p.lam[(size_t)((t1 + 1) & rmask) * plane + col] : 0.0f;
              val = sm.sc[ii] * a1 + a2;
            }
            sm.pull[e] = val;
          }
          __syncthreads();
          // 2) lx[t] of the tile's states
          if (threadIdx.x < kTileStates) {
            const int vl = threadIdx.x / 3, b = threadIdx.x - 3 * (threadIdx.x / 3);
            float lx = 0.0f;
            if (vl < nv) {
              const float* x = p.X + (size_t)t * S + 3 * (v0 + vl);
              const float x0 = x[0], x1 = x[1], x2 = x[2];
              const float sum = fabsf(x0) + fabsf(x1) + fabsf(x2);
              const float f = sum > p.threshold ? sum - p.threshold : 0.0f;
              const float xb = b == 0 ? x0 : (b == 1 ? x1 : x2);
              const float mreg = f > 0.0f ? f * signum_f(xb) : 0.0f;
              float acc = 0.0f;
              const float* pl = sm.pull + vl * kGainCols + b;
#pragma unroll 2
              for (int n = 0; n < kOffsets; ++n) acc = acc + pl[3 * n];
              lx = p.mse_scaling * p.MR[(size_t)t * S + 3 * (v0 + vl) + b] + p.reg_scaling * mreg + acc;
            }
            sm.lx[threadIdx.x] = lx;
          }
          __syncthreads();
          // 3) items: lap[t], gradient accumulation, ring store
          const float* seg_ap_t = p.seg_ap + (size_t)(t - t_lo) * plane;
          const float* seg_q_t = p.seg_q + (size_t)(t - t_lo) * plane;
          float* lam_t = p.lam + (size_t)(t & rmask) * plane;
          const float* lam_n = p.lam + (size_t)((t + 1) & rmask) * plane;
#pragma unroll
          for (int i = 0; i < kColsPerThread; ++i) {
            const int e = threadIdx.x + i * kAdjThreads;
            if (e < nv * kGainCols) {
              const int vl = e / kGainCols, k = e - vl * kGainCols;
              const int v = v0 + vl, n = k / 3;
              const size_t col = (size_t)v * kGainCols + k;
              if (p.nbr[(size_t)v * kOffsets + n] >= 0) {
                const float l0 = sm.lx[3 * vl], l1 = sm.lx[3 * vl + 1], l2 = sm.lx[3 * vl + 2];
                const float* g = p.gains + (size_t)3 * v * kGainCols + k;
                const float G = g[0] * l0 + g[kGainCols] * l1 + g[2 * kGainCols] * l2;
                const float lprev = t + 1 < T ? lam_n[col] : 0.0f;
                const float lap = G - p.coefs[(size_t)v * kOffsets + n] * lprev;
                const float ap_t = seg_ap_t[col];
                dg[i][0] = dg[i][0] + l0 * ap_t;
                dg[i][1] = dg[i][1] + l1 * ap_t;
                dg[i][2] = dg[i][2] + l2 * ap_t;
                dc[i] = dc[i] + lap * seg_q_t[col];
                lam_t[col] = lap;
              }
            }
          }
        }
        if (!resident) {  // add this block's sums for the tile
#pragma unroll
          for (int i = 0; i < kColsPerThread; ++i) {
            const int e = threadIdx.x + i * kAdjThreads;
            if (e < nv * kGainCols) {
              const int vl = e / kGainCols, k = e - vl * kGainCols;
              const int v = v0 + vl;
              if (!p.freeze_gains) {
                float* g = p.dG + (size_t)3 * v * kGainCols + k;
                g[0] = g[0] + dg[i][0];
                g[kGainCols] = g[kGainCols] + dg[i][1];
                g[2 * kGainCols] = g[2 * kGainCols] + dg[i][2];
              }
              float* ck = p.dCk + (size_t)v * kGainCols + k;
              *ck = *ck + dc[i];
            }
            dg[i][0] = dg[i][1] = dg[i][2] = 0.0f;
            dc[i] = 0.0f;
          }
        }
      }
      if (!(seg == 0 && t_end == t_lo)) {
        if (!grid_barrier(p.barrier, barrier_number++, p.status)) return;
      }
    }
  }

  // per-tile epilogue: resident accumulators, then dC[v,n] += sum_b dCk + difference regularisation
  for (int tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    const int v0 = tile * kTileVoxels;
    const int nv = min(kTileVoxels, V - v0);
    if (resident) {
#pragma unroll
      for (int i = 0; i < kColsPerThread; ++i) {
        const int e = threadIdx.x + i * kAdjThreads;
        if (e < nv * kGainCols) {
          const int vl = e / kGainCols, k = e - vl * kGainCols;
          const int v = v0 + vl;
          if (!p.freeze_gains) {
            float* g = p.dG + (size_t)3 * v * kGainCols + k;
            g[0] = g[0] + dg[i][0];
            g[kGainCols] = g[kGainCols] + dg[i][1];
            g[2 * kGainCols] = g[2 * kGainCols] + dg[i][2];
          }
          p.dCk[(size_t)v * kGainCols + k] = dc[i];
        }
      }
    }
    __syncthreads();
    if (!p.freeze_delays) {
      for (int e = threadIdx.x; e < nv * kOffsets; e += blockDim.x) {
        const int v = v0 + e / kOffsets, n = e - (e / kOffsets) * kOffsets;
        const size_t ci = (size_t)v * kOffsets + n;
        float* ck = p.dCk + (size_t)v * kGainCols + 3 * n;
        float sum = (ck[0] + ck[1]) + ck[2];
        const int d = p.delays[ci];
        const float c = p.coefs[ci];
        const float delta = p.init_delays[ci] - ((float)d + (1.0f - c) / (c + 1.0f));
        float count = 9.0f * (float)T;
        if (p.ap_derivative == CT_AP_SIMPLE) count = p.nbr[ci] >= 0 ? 9.0f * (float)max(0, T - d) : 0.0f;
        sum = sum + count * (p.diffreg * powi5_f(delta));
        p.dC[ci] = p.dC[ci] + sum;
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nv * kGainCols; e += blockDim.x) p.dCk[(size_t)v0 * kGainCols + e] = 0.0f;
  }
}

}  // namespace

int adjoint_capacity(int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel, kAdjThreads, 0);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

cudaError_t launch_adjoint(DeviceScenario& d, const AdjointScalars& s, cudaStream_t stream) {
  AdjArgs a;
  a.V = (int)d.V;
  a.S = (int)d.S;
  a.T = (int)d.T;
  a.ring = d.adj_ring;
  a.nbr = d.nbr;
  a.rev = d.rev;
  a.coefs = d.coefs;
  a.delays = d.delays;
  a.init_delays = d.init_delays;
  a.gains = d.gains;
  a.X = d.X;
  a.MR = d.MR;
  a.ckpt = d.ckpt;
  a.seg_ap = d.seg_ap;
  a.seg_q = d.seg_q;
  a.lam = d.lam;
  a.dG = d.dG;
  a.dC = d.dC;
  a.dCk = d.dCk;
  a.dmin = d.dmin;
  a.mse_scaling = s.mse_scaling;
  a.reg_scaling = s.reg_scaling;
  a.threshold = s.threshold;
  a.diffreg = s.diffreg;
  a.freeze_gains = s.freeze_gains;
  a.freeze_delays = s.freeze_delays;
  a.ap_derivative = s.ap_derivative;
  a.status = d.status;
  a.barrier = d.barrier;
  cudaError_t err = cudaMemsetAsync(d.barrier, 0, sizeof(GridBarrier), stream);
  if (err != cudaSuccess) return err;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)adjoint_kernel, dim3(d.adj_grid), dim3(kAdjThreads), args, 0, stream);
}

}  // namespace ct
