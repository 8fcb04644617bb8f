// Adjoint (back-propagation through time) of one beat: the exact gradient of
// the stated loss
//   L = sum_t (mse/M)/2 |H x_t - z_t|^2 + reg/2 sum_v relu(|x_v|_1 - thr)^2
// with respect to the gains and all-pass coefficients, through the forward
// recursion of innovate_system_states_v1 (prediction.rs:40-86):
//   ap[t] = c (in_t - ap[t-1]) + in1_t,   in_t = x[t-d, j] (t >= d), in1_t = x[t-d-1, j] (t > d)
//   x[t, 3v+a] = sum_k g[3v+a, k] ap[t][v, k] + u[t] B[3v+a]          (k = 3n + b).
// The reference crate has no counterpart: its derivation (derivation.rs:173-
// 229) keeps only the per-step terms. With lap = dL/dap and lx = dL/dx:
//   lap[t][v,k] = sum_a g[3v+a, k] lx[t, 3v+a] - c lap[t+1][v,k]
//   lx[s, 3j+b] = (mse/M) (H^T r_s)[3j+b] + reg f_j sign(x_{3j+b})
//                 + sum over the items (v, n) with neighbour j of w_vn[s],
//   w_vn[s]     = c lap[s+d][v,3n+b] + lap[s+d+1][v,3n+b]         (lap = 0 from T on)
//   dG[3v+a, k] += lx[t, 3v+a] ap[t][v,k],   dC[v,n] += sum_b lap[t][v,3n+b] (in_t - ap[t-1]).
//
// Schedule (one cooperative launch per beat, or per beat of a batch of
// scenarios: every tile names its scenario):
//   * Checkpoints. The forward stores the all-pass state every kCkptSteps
//     steps. Segments are visited from the last to the first; a CTA first
//     recomputes, from the checkpoint and the stored states, ap[t] and
//     q[t] = in_t - ap[t-1] of its own tiles for the segment (the forward's
//     fmaf, so bit-identical), then steps the segment backwards.
//   * Inbox. At step t item (v, n) knows lap[t] and lap[t+1], so it writes
//     w_vn[t-d] into the inbox row of its neighbour j, column 3n+b, slot
//     (t-d) mod ring. Each inbox cell has exactly one writer and is read at
//     step t-d, in a later block: steps advance L = min(dmin, kMaxStepBlock)
//     at a time between grid barriers, as in the forward. A voxel's 78 inbox
//     cells are contiguous and summed in column order, so results are
//     deterministic (no atomics).
//   * Pipeline. Thread e owns tile columns e, e+256, ... A step's inbox row
//     and recomputed ap/q rows (contiguous per tile; plane pitch padded to 16
//     bytes) arrive by TMA bulk copies into a ring of kStages shared-memory
//     stages, issued kStages steps ahead by one thread and completed on an
//     mbarrier per stage (every wait bounded); gains sit in shared memory.
//   * A CTA that owns one tile keeps its columns' state and gradient sums in
//     registers for the launch; otherwise both go through global memory at
//     the end of every block of steps.
#include <cuda_runtime.h>

#include "ct_internal.cuh"
#include "ct_sync.cuh"

namespace ct {
namespace {

constexpr int kTileVoxels = kFwdTileVoxels;
constexpr int kTileStates = 3 * kTileVoxels;
constexpr int kTileCols = kTileVoxels * kGainCols;
constexpr int kAdjThreads = 256;
constexpr int kCols = (kTileCols + kAdjThreads - 1) / kAdjThreads;  // 10 columns per thread
constexpr int kStages = 4;
constexpr unsigned long long kWaitNs = 2000000000ull;  // bound of every mbarrier wait

struct AdjSmem {
  float g3[3][kTileCols];              // gains of the voxel's rows a = 0, 1, 2 at each column
  float stage[kStages][3][kTileCols];  // [stage][inbox | ap | q][column]
  float lx[kTileStates];
  uint64_t bar[kStages];
  uint32_t phase;                      // bit s: parity of the next completion of stage s
  uint32_t pending;                    // bit s: a copy into stage s is in flight
  int abort;
  AdjScn sp;                           // scenario of the current tile
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false (and CT_ERR_TIMEOUT recorded) if the phase does not complete in kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int32_t* status) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try(bar, parity)) {
    if (global_ns() - t0 > kWaitNs) {
      atomicCAS(status, 0, (int32_t)CT_ERR_TIMEOUT);
      return false;
    }
  }
  return true;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void red_add(float* p, float v) {
  asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

__device__ __forceinline__ float powi5_f(float x) {
  const float x2 = x * x;
  const float x4 = x2 * x2;
  return x * x4;
}

__device__ __forceinline__ void tile_of(const AdjLaunch& L, int tile, int* scn, int* v0) {
  if (L.tiles) {
    const int2 t = L.tiles[tile];
    *scn = t.x;
    *v0 = t.y;
  } else {
    *scn = 0;
    *v0 = tile * kTileVoxels;
  }
}

__device__ __forceinline__ void load_scn(AdjSmem& sm, const AdjLaunch& L, int scn) {
  __syncthreads();
  if (threadIdx.x == 0) sm.sp = L.scns ? L.scns[scn] : L.single;
  __syncthreads();
}

// ap[t] and q[t] = in_t - ap[t-1] of the tile's columns for steps [t_lo, t_hi) (own columns only).
__device__ __forceinline__ void recompute_segment(const AdjScn& p, int v0, int nv, int seg, int t_lo, int t_hi) {
  const size_t plane = (size_t)p.V * kGainCols;  // checkpoint planes are unpadded
  const size_t pitch = (size_t)p.pitch;
  float a[kCols], inp[kCols], c[kCols];
  const float* xs[kCols];
  int d[kCols];
#pragma unroll
  for (int i = 0; i < kCols; ++i) {
    const int e = threadIdx.x + i * kAdjThreads;
    a[i] = inp[i] = c[i] = 0.0f;
    d[i] = 1 << 30;  // absent: every input reads as zero
    xs[i] = p.X;
    if (e < nv * kGainCols) {
      const int vl = e / kGainCols, k = e - vl * kGainCols, n = k / 3, b = k - 3 * n;
      const int v = v0 + vl;
      const int32_t nb = p.nbr[(size_t)v * kOffsets + n];
      if (nb >= 0) {
        d[i] = p.delays[(size_t)v * kOffsets + n];
        c[i] = p.coefs[(size_t)v * kOffsets + n];
        xs[i] = p.X + 3 * nb + b;
        a[i] = p.ckpt[(size_t)seg * plane + (size_t)v0 * kGainCols + e];
        inp[i] = (t_lo - d[i] - 1 >= 0) ? xs[i][(size_t)(t_lo - d[i] - 1) * p.S] : 0.0f;
      }
    }
  }
  constexpr int kU = 4;
  for (int t0 = t_lo; t0 < t_hi; t0 += kU) {
    float in[kU][kCols];
#pragma unroll
    for (int u = 0; u < kU; ++u)
#pragma unroll
      for (int i = 0; i < kCols; ++i) {
        const int t = t0 + u;
        in[u][i] = (t < t_hi && t - d[i] >= 0) ? xs[i][(size_t)(t - d[i]) * p.S] : 0.0f;
      }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int t = t0 + u;
      if (t < t_hi) {
        float* sa = p.seg_ap + (size_t)(t - t_lo) * pitch + (size_t)v0 * kGainCols;
        float* sq = p.seg_q + (size_t)(t - t_lo) * pitch + (size_t)v0 * kGainCols;
#pragma unroll
        for (int i = 0; i < kCols; ++i) {
          const int e = threadIdx.x + i * kAdjThreads;
          const float q = in[u][i] - a[i];
          a[i] = fmaf(c[i], q, inp[i]);
          inp[i] = in[u][i];
          if (e < nv * kGainCols) {
            sa[e] = a[i];
            sq[e] = q;
          }
        }
      }
    }
  }
}

// Per-column registers of the tile a thread works on.
struct Cols {
  float c[kCols], lprev[kCols], dg[kCols][3], dc[kCols];
  int d[kCols], jw[kCols];  // delay; inbox cell neighbour * 78 + column, -1 if unconnected
};

__device__ __forceinline__ void load_cols(Cols& cs, AdjSmem& sm, const AdjScn& p, int v0, int nv, bool state) {
#pragma unroll
  for (int i = 0; i < kCols; ++i) {
    const int e = threadIdx.x + i * kAdjThreads;
    cs.c[i] = 0.0f;
    cs.d[i] = 1 << 30;
    cs.jw[i] = -1;
    cs.lprev[i] = 0.0f;
    float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
    if (e < nv * kGainCols) {
      const int vl = e / kGainCols, k = e - vl * kGainCols, n = k / 3;
      const int v = v0 + vl;
      const int32_t nb = p.nbr[(size_t)v * kOffsets + n];
      if (nb >= 0) {
        cs.c[i] = p.coefs[(size_t)v * kOffsets + n];
        cs.d[i] = p.delays[(size_t)v * kOffsets + n];
        cs.jw[i] = nb * kGainCols + k;
        const float* g = p.gains + (size_t)3 * v * kGainCols + k;
        g0 = g[0];
        g1 = g[kGainCols];
        g2 = g[2 * kGainCols];
      }
      if (state) cs.lprev[i] = p.lam_state[(size_t)v0 * kGainCols + e];
    }
    if (e < kTileCols) {
      sm.g3[0][e] = g0;
      sm.g3[1][e] = g1;
      sm.g3[2][e] = g2;
    }
    cs.dg[i][0] = cs.dg[i][1] = cs.dg[i][2] = 0.0f;
    cs.dc[i] = 0.0f;
  }
}

// Add the columns' gradient sums to dG / dCk (and keep their adjoint state for the next block).
__device__ __forceinline__ void flush_cols(Cols& cs, const AdjScn& p, int v0, int nv, bool keep_state) {
#pragma unroll
  for (int i = 0; i < kCols; ++i) {
    const int e = threadIdx.x + i * kAdjThreads;
    if (e < nv * kGainCols) {
      const int vl = e / kGainCols, k = e - vl * kGainCols;
      const int v = v0 + vl;
      // one owner per element, adds ordered by the grid barriers: a deterministic sum
      if (!p.freeze_gains) {
        float* g = p.dG + (size_t)3 * v * kGainCols + k;
        red_add(g, cs.dg[i][0]);
        red_add(g + kGainCols, cs.dg[i][1]);
        red_add(g + 2 * kGainCols, cs.dg[i][2]);
      }
      red_add(p.dCk + (size_t)v0 * kGainCols + e, cs.dc[i]);
      if (keep_state) p.lam_state[(size_t)v0 * kGainCols + e] = cs.lprev[i];
    }
    cs.dg[i][0] = cs.dg[i][1] = cs.dg[i][2] = 0.0f;
    cs.dc[i] = 0.0f;
  }
}

// Thread 0: bulk copies of step t's inbox, ap and q rows of the tile into stage `st`.
__device__ __forceinline__ void issue_stage(AdjSmem& sm, const AdjScn& p, int st, int v0, int nv, int t, int t_lo) {
  const size_t pitch = (size_t)p.pitch;
  const uint32_t bytes = (uint32_t)(((nv * kGainCols * 4) + 15) & ~15);  // stays inside the padded row
  mbar_expect_tx(&sm.bar[st], 3 * bytes);
  bulk_load(sm.stage[st][0], p.inbox + (size_t)(t & (p.ring - 1)) * pitch + (size_t)v0 * kGainCols, bytes,
            &sm.bar[st]);
  bulk_load(sm.stage[st][1], p.seg_ap + (size_t)(t - t_lo) * pitch + (size_t)v0 * kGainCols, bytes, &sm.bar[st]);
  bulk_load(sm.stage[st][2], p.seg_q + (size_t)(t - t_lo) * pitch + (size_t)v0 * kGainCols, bytes, &sm.bar[st]);
  sm.pending |= 1u << st;
}

// After a timed-out wait: let every copy still in flight land (bounded) before the CTA leaves.
__device__ __forceinline__ void drain_stages(AdjSmem& sm, int32_t* status) {
  if (threadIdx.x == 0)
    for (int st = 0; st < kStages; ++st)
      if (sm.pending & (1u << st)) mbar_wait(&sm.bar[st], (sm.phase >> st) & 1u, status);
}

// Steps ta down to t_end (inclusive) of one tile; t_lo is the segment's first step (row 0 of seg_ap/seg_q).
// Returns false if a wait timed out (the CTA must leave).
__device__ __forceinline__ bool backward_block(Cols& cs, AdjSmem& sm, const AdjScn& p, int v0, int nv, int ta,
                                               int t_end, int t_lo, int32_t* status) {
  const size_t pitch = (size_t)p.pitch;
  const int rmask = p.ring - 1;
  const int S = p.S;
  const bool lxt = (int)threadIdx.x < 3 * nv;  // implies < kTileStates
  const int vlx = threadIdx.x / 3;
  // every generic write this CTA's copies read (recomputed rows, inbox cells of earlier blocks,
  // made visible by the grid barrier) is ordered before the async-proxy reads
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async;" ::: "memory");
    for (int s = 0; s < kStages && ta - s >= t_end; ++s) issue_stage(sm, p, s, v0, nv, ta - s, t_lo);
  }
  float mr_n = 0.0f, x0_n = 0.0f, x1_n = 0.0f, x2_n = 0.0f;
  if (lxt) {
    const float* x = p.X + (size_t)ta * S + 3 * (v0 + vlx);
    mr_n = p.MR[(size_t)ta * S + 3 * v0 + threadIdx.x];
    x0_n = x[0];
    x1_n = x[1];
    x2_n = x[2];
  }
  for (int t = ta; t >= t_end; --t) {
    const int st = (ta - t) % kStages;
    const float mr = mr_n, x0 = x0_n, x1 = x1_n, x2 = x2_n;
    if (lxt && t - 1 >= t_end) {
      const float* x = p.X + (size_t)(t - 1) * S + 3 * (v0 + vlx);
      mr_n = p.MR[(size_t)(t - 1) * S + 3 * v0 + threadIdx.x];
      x0_n = x[0];
      x1_n = x[1];
      x2_n = x[2];
    }
    const uint32_t par = (sm.phase >> st) & 1u;
    if (!mbar_wait(&sm.bar[st], par, status)) sm.abort = 1;
    __syncthreads();  // (A) every thread past the wait; abort visible
    if (sm.abort) return false;
    // lx[t] of the tile's states: instantaneous terms + inbox, summed in column order
    if (threadIdx.x < kTileStates) {
      const int b = threadIdx.x - 3 * vlx;
      float lx = 0.0f;
      if (lxt) {
        const float sum = fabsf(x0) + fabsf(x1) + fabsf(x2);
        const float f = sum > p.threshold ? sum - p.threshold : 0.0f;
        const float xb = b == 0 ? x0 : (b == 1 ? x1 : x2);
        const float mreg = f > 0.0f ? f * copysignf(1.0f, xb) : 0.0f;
        const float* pl = sm.stage[st][0] + vlx * kGainCols + b;
        float acc = 0.0f;
#pragma unroll
        for (int n = 0; n < kOffsets; ++n) acc = acc + pl[3 * n];
        lx = p.mse_scaling * mr + p.reg_scaling * mreg + acc;
      }
      sm.lx[threadIdx.x] = lx;
    }
    __syncthreads();  // (B)
    if (threadIdx.x == 0) sm.phase ^= 1u << st;
    // the tile's columns: lap[t], gradient sums, inbox cell of the neighbour at step t - d
#pragma unroll
    for (int i = 0; i < kCols; ++i) {
      const int e = threadIdx.x + i * kAdjThreads;
      if (cs.jw[i] >= 0) {
        const int vl = e / kGainCols;
        const float l0 = sm.lx[3 * vl], l1 = sm.lx[3 * vl + 1], l2 = sm.lx[3 * vl + 2];
        const float G = sm.g3[0][e] * l0 + sm.g3[1][e] * l1 + sm.g3[2][e] * l2;
        const float lap = G - cs.c[i] * cs.lprev[i];
        const float ap_t = sm.stage[st][1][e];
        cs.dg[i][0] = cs.dg[i][0] + l0 * ap_t;
        cs.dg[i][1] = cs.dg[i][1] + l1 * ap_t;
        cs.dg[i][2] = cs.dg[i][2] + l2 * ap_t;
        cs.dc[i] = cs.dc[i] + lap * sm.stage[st][2][e];
        const int ts = t - cs.d[i];
        if (ts >= 0) p.inbox[(size_t)(ts & rmask) * pitch + cs.jw[i]] = cs.c[i] * lap + cs.lprev[i];
        cs.lprev[i] = lap;
      }
    }
    __syncthreads();  // (C) stage st and lx free again
    if (threadIdx.x == 0) {
      sm.pending &= ~(1u << st);
      if (t - kStages >= t_end) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_stage(sm, p, st, v0, nv, t - kStages, t_lo);
      }
    }
  }
  return true;
}

__global__ void __launch_bounds__(kAdjThreads, 1) adjoint_kernel(AdjLaunch L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  AdjSmem& sm = *reinterpret_cast<AdjSmem*>(smem_raw);
  const int ntiles = L.ntiles;
  const bool resident = ntiles <= (int)gridDim.x;
  // steps per block: the smallest delay of any scenario (capped); every inbox must span the delays
  int Lmax = kMaxStepBlock;
  bool ring_ok = true;
  for (int s = 0; s < L.nscn; ++s) {
    const int32_t* dm = L.scns ? L.scns[s].dmin : L.single.dmin;
    const int ring = L.scns ? L.scns[s].ring : L.single.ring;
    int dmin = dm[0], dmax = dm[1];
    if (dmin < 1) dmin = 1;
    if (dmax < dmin) dmax = dmin;
    if (dmin < Lmax) Lmax = dmin;
    if (dmax + kMaxStepBlock + 1 > ring) ring_ok = false;
  }
  if (!ring_ok) {  // every CTA leaves here, before any grid barrier
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(L.status, 0, (int32_t)CT_ERR_NOT_SUPPORTED);
    return;
  }

  if (threadIdx.x == 0) {
    for (int st = 0; st < kStages; ++st) mbar_init(&sm.bar[st], 1);
    sm.phase = 0;
    sm.pending = 0;
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  Cols cs;
  int cur_scn = -1, v0 = 0, nv = 0;
  if (resident && (int)blockIdx.x < ntiles) {
    tile_of(L, blockIdx.x, &cur_scn, &v0);
    load_scn(sm, L, cur_scn);
    nv = min(kTileVoxels, sm.sp.V - v0);
    load_cols(cs, sm, sm.sp, v0, nv, false);
  }

  unsigned int barrier_number = 0;
  const int K = L.ckpt_steps;
  const int nseg = (L.Tmax + K - 1) / K;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int t_lo = seg * K;
    const int t_hi = min(L.Tmax, t_lo + K);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      int scn;
      tile_of(L, tile, &scn, &v0);
      if (scn != cur_scn) {
        load_scn(sm, L, scn);
        cur_scn = scn;
      }
      nv = min(kTileVoxels, sm.sp.V - v0);
      if (t_lo < sm.sp.T) recompute_segment(sm.sp, v0, nv, seg, t_lo, min(sm.sp.T, t_lo + K));
    }
    for (int tb = t_hi - 1; tb >= t_lo; tb -= Lmax) {
      const int t_end = max(t_lo, tb - Lmax + 1);
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if (!resident) {
          int scn;
          tile_of(L, tile, &scn, &v0);
          if (scn != cur_scn) {
            load_scn(sm, L, scn);
            cur_scn = scn;
          }
          nv = min(kTileVoxels, sm.sp.V - v0);
        }
        const int ta = min(tb, sm.sp.T - 1);
        if (ta < t_end) continue;  // this tile's scenario ends before the block (uniform per CTA)
        if (!resident) {
          __syncthreads();
          load_cols(cs, sm, sm.sp, v0, nv, true);
        }
        __syncthreads();
        if (!backward_block(cs, sm, sm.sp, v0, nv, ta, t_end, t_lo, L.status)) {
          drain_stages(sm, L.status);
          return;
        }
        if (!resident) flush_cols(cs, sm.sp, v0, nv, true);
      }
      if (!(seg == 0 && t_end == t_lo)) {
        if (!grid_barrier(L.barrier, barrier_number++, L.status)) return;
      }
    }
  }

  // per-tile epilogue: dC[v,n] += sum_b dCk + difference regularisation; dCk back to zero
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int scn;
    tile_of(L, tile, &scn, &v0);
    if (scn != cur_scn) {
      load_scn(sm, L, scn);
      cur_scn = scn;
    }
    const AdjScn& p = sm.sp;
    nv = min(kTileVoxels, p.V - v0);
    if (resident) flush_cols(cs, p, v0, nv, false);
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
        float count = 9.0f * (float)p.T;
        if (p.ap_derivative == CT_AP_SIMPLE) count = p.nbr[ci] >= 0 ? 9.0f * (float)max(0, p.T - d) : 0.0f;
        sum = sum + count * (p.diffreg * powi5_f(delta));
        p.dC[ci] = p.dC[ci] + sum;
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nv * kGainCols; e += blockDim.x) p.dCk[(size_t)v0 * kGainCols + e] = 0.0f;
  }
}

bool configure(int device) {
  static bool done[128] = {};
  if (device < 0 || device >= 128) return false;
  if (!done[device]) {
    if (cudaFuncSetAttribute(adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(AdjSmem)) !=
        cudaSuccess)
      return false;
    done[device] = true;
  }
  return true;
}

}  // namespace

int adjoint_capacity(int device) {
  configure(device);
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel, kAdjThreads, sizeof(AdjSmem));
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

AdjScn adjoint_scenario(const DeviceScenario& d, const AdjointScalars& s) {
  AdjScn a;
  a.V = (int)d.V;
  a.S = (int)d.S;
  a.T = (int)d.T;
  a.ring = d.adj_ring;
  a.pitch = d.adj_pitch;
  a.nbr = d.nbr;
  a.coefs = d.coefs;
  a.delays = d.delays;
  a.init_delays = d.init_delays;
  a.gains = d.gains;
  a.X = d.X;
  a.MR = d.MR;
  a.ckpt = d.ckpt;
  a.seg_ap = d.seg_ap;
  a.seg_q = d.seg_q;
  a.inbox = d.inbox;
  a.lam_state = d.lam_state;
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
  return a;
}

cudaError_t launch_adjoint_tiles(const AdjLaunch& launch, int grid, cudaStream_t stream) {
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) return err;
  if (!configure(device)) return cudaErrorInvalidValue;
  err = cudaMemsetAsync(launch.barrier, 0, sizeof(GridBarrier), stream);
  if (err != cudaSuccess) return err;
  AdjLaunch l = launch;
  void* args[] = {&l};
  return launch_cooperative((const void*)adjoint_kernel, grid, kAdjThreads, args, sizeof(AdjSmem), stream);
}

cudaError_t launch_adjoint(DeviceScenario& d, const AdjointScalars& s, cudaStream_t stream) {
  const size_t plane = (size_t)d.V * kGainCols;
  cudaError_t err = cudaMemsetAsync(d.inbox, 0, sizeof(float) * d.adj_ring * (size_t)d.adj_pitch, stream);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(d.lam_state, 0, sizeof(float) * plane, stream);
  if (err != cudaSuccess) return err;
  AdjLaunch l;
  l.scns = nullptr;
  l.single = adjoint_scenario(d, s);
  l.nscn = 1;
  l.tiles = nullptr;
  l.ntiles = (int)((d.V + kTileVoxels - 1) / kTileVoxels);
  l.Tmax = (int)d.T;
  l.ckpt_steps = kCkptSteps;
  l.status = d.status;
  l.barrier = d.barrier;
  return launch_adjoint_tiles(l, d.adj_grid, stream);
}

}  // namespace ct
