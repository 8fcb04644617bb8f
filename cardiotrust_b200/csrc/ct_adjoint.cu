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
//   * Checkpoints. The forward stores the all-pass state every K steps
//     (K a power of two, 256 by default). Segments are visited from the last
//     to the first; a CTA first recomputes, from the checkpoint and the
//     stored states, q[t] = in_t - ap[t-1] of its own tiles for the segment,
//     then steps the segment backwards, rebuilding ap[t] = fmaf(c, q[t], in1_t)
//     (the forward's own expression, so bit-identical) from a gather of
//     in1_t = x[t-d-1, j]: one stored row per step instead of two.
//   * Inbox. At step t item (v, n) knows lap[t] and lap[t+1], so it writes
//     w_vn[t-d] into the inbox row of its neighbour j, column 3n+b, slot
//     (t-d) mod ring. Each inbox cell has exactly one writer and is read at
//     step t-d, in a later block: steps advance L = min(dmin, kMaxStepBlock)
//     at a time between grid barriers, as in the forward. A voxel's 78 inbox
//     cells are contiguous and summed in column order, so results are
//     deterministic (no atomics).
//   * Pipeline. Sixteen threads (half a warp) own one voxel of the tile, five
//     of its 78 columns each. A step's inbox row and q row (contiguous per
//     tile; plane pitch padded to 16 bytes) arrive by TMA bulk copies into a
//     ring of NS shared-memory stages (3, or 4 for a batch), issued NS steps
//     ahead by one thread and completed on a `full` mbarrier per stage; the states, mapped
//     residuals and in1 gathers of the step arrive by cp.async. Warps run
//     decoupled: each releases a stage on an `empty` mbarrier, and no CTA
//     barrier separates steps. Every wait is bounded.
//   * A CTA that owns one tile keeps its columns' state and gradient sums in
//     registers for the launch; otherwise both go through global memory at
//     the end of every block of steps.
#include <cuda_runtime.h>

#include "ct_internal.cuh"
#include "ct_sync.cuh"

namespace ct {
namespace {

constexpr int kTileVoxels = kFwdTileVoxels;
constexpr int kTileCols = kTileVoxels * kGainCols;
constexpr int kTileItems = kTileVoxels * kOffsets;
constexpr int kAdjThreads = 512;
constexpr int kGroup = 16;                 // threads per voxel (a half warp)
constexpr int kCols = 5;                   // columns per thread: k = lane + 16 i, k < 78
constexpr int kWarps = kAdjThreads / 32;
// Stages of the copy ring: 3 for one scenario's tiles (more L1 left for the gathers: cuboid20
// adjoint 11.8 ms against 12.4 ms with 4), 4 for a batch's tile list (each CTA walks many tiles,
// whose pipelines start cold: 64-scenario batched adjoint 3.40 s against 3.50 s with 3).
constexpr int kStagesSingle = 3;
constexpr int kStagesBatch = 4;
constexpr unsigned long long kWaitNs = 2000000000ull;  // bound of every mbarrier wait
static_assert(kTileVoxels * kGroup == kAdjThreads, "one voxel group per 16 threads");
static_assert(kCols * kGroup >= kGainCols, "columns per voxel");
static_assert(kGroup == 16 && kCols == 5 && 4 * kGroup < kGainCols, "the inbox sum's column grouping");

template <int NS>
struct AdjSmem {
  float g[kTileVoxels * 3 * kGainCols];  // the tile's gain rows, [voxel][row a][column k] as in HBM
  float stage[NS][3][kTileCols];         // [stage][inbox | q | in1][voxel * 78 + column]
  float xm[NS][kTileVoxels][8];          // [stage][voxel][x0 x1 x2 mr0 mr1 mr2 - -]
  float coef[kTileItems];                // per (voxel, offset) of the tile
  int32_t del[kTileItems];
  int32_t nbr[kTileItems];
  float lam[kTileCols];                  // adjoint state carried between blocks (tiles that are not resident)
  uint64_t full[NS];                     // the stage's rows have landed
  uint64_t empty[NS];                    // every warp is done with the stage
  uint64_t meta_bar;
  int abort;
  AdjScn sp;                             // scenario of the current tile
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
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

template <int NS>
__device__ __forceinline__ void load_scn(AdjSmem<NS>& sm, const AdjLaunch& L, int scn) {
  __syncthreads();
  if (threadIdx.x == 0) sm.sp = L.scns ? L.scns[scn] : L.single;
  __syncthreads();
}

// The thread's voxel in the tile and its column i (valid when < 78).
__device__ __forceinline__ int my_voxel() { return threadIdx.x / kGroup; }
__device__ __forceinline__ int my_col(int i) { return (int)(threadIdx.x % kGroup) + kGroup * i; }

// q[t] = in_t - ap[t-1] of the thread's columns for steps [t_lo, t_hi).
__device__ __forceinline__ void recompute_segment(const AdjScn& p, int v0, int nv, int seg, int t_lo, int t_hi) {
  const size_t plane = (size_t)p.V * kGainCols;  // checkpoint planes are unpadded
  const size_t pitch = (size_t)p.pitch;
  const int vl = my_voxel();
  float a[kCols], inp[kCols], c[kCols];
  const float* xs[kCols];
  int d[kCols];
#pragma unroll
  for (int i = 0; i < kCols; ++i) {
    const int k = my_col(i);
    a[i] = inp[i] = c[i] = 0.0f;
    d[i] = 1 << 30;  // absent: every input reads as zero
    xs[i] = p.X;
    if (vl < nv && k < kGainCols) {
      const int n = k / 3, b = k - 3 * n;
      const int v = v0 + vl;
      const int32_t nb = p.nbr[(size_t)v * kOffsets + n];
      if (nb >= 0) {
        d[i] = p.delays[(size_t)v * kOffsets + n];
        c[i] = p.coefs[(size_t)v * kOffsets + n];
        xs[i] = p.X + 3 * nb + b;
        a[i] = p.ckpt[(size_t)seg * plane + (size_t)v * kGainCols + k];
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
        float* sq = p.seg_q + (size_t)(t - t_lo) * pitch + (size_t)(v0 + vl) * kGainCols;
#pragma unroll
        for (int i = 0; i < kCols; ++i) {
          const int k = my_col(i);
          const float q = in[u][i] - a[i];
          a[i] = fmaf(c[i], q, inp[i]);
          inp[i] = in[u][i];
          if (vl < nv && k < kGainCols) sq[k] = q;
        }
      }
    }
  }
}

// Per-column registers of the tile a thread works on, and the thread's stage-barrier phases.
struct Cols {
  float c[kCols], lprev[kCols], dg[kCols][3], dc[kCols];
  int d[kCols], jw[kCols];  // delay; inbox cell neighbour * 78 + column, -1 if unconnected
  int xo[kCols];            // offset of the column's input x[t-d-1, 3 * neighbour + b] from row t: state - (d+1) S
  uint32_t full_ph;         // bit s: parity of the next completion of full[s]
  uint32_t empty_ph;        // thread 0: parity of the next completion of empty[s]
  uint32_t empty_wait;      // thread 0: bit s: a use of stage s has not been waited empty yet
  uint32_t inflight;        // thread 0: bit s: copies into stage s issued and not yet waited full
  uint32_t meta_ph;
};

// Per-tile tables into shared memory by bulk copies (gains, coefficients, delays, neighbours and,
// with `state`, the adjoint state of the previous block), then each thread's column registers.
// Called by all threads after a CTA barrier.
template <int NS>
__device__ __forceinline__ bool load_cols(Cols& cs, AdjSmem<NS>& sm, const AdjScn& p, int v0, int nv, bool state,
                                          int32_t* status) {
  if (threadIdx.x == 0) {
    const uint32_t gb = (uint32_t)((nv * 3 * kGainCols * 4 + 15) & ~15);
    const uint32_t ib = (uint32_t)((nv * kOffsets * 4 + 15) & ~15);
    const uint32_t lb = (uint32_t)((nv * kGainCols * 4 + 15) & ~15);
    asm volatile("fence.proxy.async;" ::: "memory");
    mbar_expect_tx(&sm.meta_bar, gb + 3 * ib + (state ? lb : 0));
    bulk_load(sm.g, p.gains + (size_t)3 * v0 * kGainCols, gb, &sm.meta_bar);
    bulk_load(sm.coef, p.coefs + (size_t)v0 * kOffsets, ib, &sm.meta_bar);
    bulk_load(sm.del, p.delays + (size_t)v0 * kOffsets, ib, &sm.meta_bar);
    bulk_load(sm.nbr, p.nbr + (size_t)v0 * kOffsets, ib, &sm.meta_bar);
    if (state) bulk_load(sm.lam, p.lam_state + (size_t)v0 * kGainCols, lb, &sm.meta_bar);
  }
  const bool ok = mbar_wait(&sm.meta_bar, cs.meta_ph, status);
  cs.meta_ph ^= 1u;
  const int vl = my_voxel();
#pragma unroll
  for (int i = 0; i < kCols; ++i) {
    const int k = my_col(i);
    cs.c[i] = 0.0f;
    cs.d[i] = 1 << 30;
    cs.jw[i] = -1;
    cs.xo[i] = 0;
    cs.lprev[i] = 0.0f;
    if (ok && vl < nv && k < kGainCols) {
      const int it = vl * kOffsets + k / 3;
      const int32_t nb = sm.nbr[it];
      if (nb >= 0) {
        cs.c[i] = sm.coef[it];
        cs.d[i] = sm.del[it];
        cs.jw[i] = nb * kGainCols + k;
        // fits 32 bits: (d + 1) S < 2^31 whenever the inbox ring of at least d + 9 planes of 26 S
        // floats fits in device memory
        cs.xo[i] = 3 * nb + k % 3 - (cs.d[i] + 1) * p.S;
      }
      if (state) cs.lprev[i] = sm.lam[vl * kGainCols + k];
    }
    cs.dg[i][0] = cs.dg[i][1] = cs.dg[i][2] = 0.0f;
    cs.dc[i] = 0.0f;
  }
  return ok;
}

// Add the columns' gradient sums to dG / dCk (and keep their adjoint state for the next block).
__device__ __forceinline__ void flush_cols(Cols& cs, const AdjScn& p, int v0, int nv, bool keep_state) {
  const int vl = my_voxel();
#pragma unroll
  for (int i = 0; i < kCols; ++i) {
    const int k = my_col(i);
    if (vl < nv && k < kGainCols) {
      const int v = v0 + vl;
      // one owner per element, adds ordered by the grid barriers: a deterministic sum
      if (!p.freeze_gains) {
        float* g = p.dG + (size_t)3 * v * kGainCols + k;
        red_add(g, cs.dg[i][0]);
        red_add(g + kGainCols, cs.dg[i][1]);
        red_add(g + 2 * kGainCols, cs.dg[i][2]);
      }
      red_add(p.dCk + (size_t)v * kGainCols + k, cs.dc[i]);
      if (keep_state) p.lam_state[(size_t)v * kGainCols + k] = cs.lprev[i];
    }
    cs.dg[i][0] = cs.dg[i][1] = cs.dg[i][2] = 0.0f;
    cs.dc[i] = 0.0f;
  }
}

// Thread 0: bulk copies of step t's inbox and q rows of the tile into stage `st`, once every
// warp has released the stage's previous use.
template <int NS>
__device__ __forceinline__ bool issue_stage(Cols& cs, AdjSmem<NS>& sm, const AdjScn& p, int st, int v0, int nv, int t,
                                           int t_lo, int32_t* status) {
  if (cs.empty_wait & (1u << st)) {
    if (!mbar_wait(&sm.empty[st], (cs.empty_ph >> st) & 1u, status)) return false;
    cs.empty_ph ^= 1u << st;
    cs.empty_wait &= ~(1u << st);
  }
  const size_t pitch = (size_t)p.pitch;
  const uint32_t bytes = (uint32_t)(((nv * kGainCols * 4) + 15) & ~15);  // stays inside the padded row
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(&sm.full[st], 2 * bytes);
  bulk_load(sm.stage[st][0], p.inbox + (size_t)(t & (p.ring - 1)) * pitch + (size_t)v0 * kGainCols, bytes,
            &sm.full[st]);
  bulk_load(sm.stage[st][1], p.seg_q + (size_t)(t - t_lo) * pitch + (size_t)v0 * kGainCols, bytes, &sm.full[st]);
  cs.empty_wait |= 1u << st;
  cs.inflight |= 1u << st;
  return true;
}

// Per thread, into stage `st` for step t: threads 0-5 of each voxel group copy the voxel's states
// and mapped residuals; every thread gathers in1_t = x[t-d-1, j] of its connected columns. One
// cp.async group per stage and thread, committed even when empty.
template <int NS>
__device__ __forceinline__ void issue_xm(const Cols& cs, AdjSmem<NS>& sm, const AdjScn& p, int st, int v0, int nv, int t,
                                         bool real) {
  const int vl = my_voxel(), q = threadIdx.x % kGroup;
  if (real && vl < nv) {
    if (q < 6) {
      const size_t off = (size_t)t * p.S + 3 * (v0 + vl) + (q % 3);
      cp_async4(&sm.xm[st][vl][q], (q < 3 ? p.X : p.MR) + off);
    }
    const float* xrow = p.X + (size_t)t * p.S;
#pragma unroll
    for (int i = 0; i < kCols; ++i) {
      const int t1 = t - cs.d[i] - 1;
      if (cs.jw[i] >= 0 && t1 >= 0)
        cp_async4(&sm.stage[st][2][vl * kGainCols + my_col(i)], xrow + cs.xo[i]);
    }
  }
  cp_async_commit();
}

// Steps ta down to t_end (inclusive) of one tile; t_lo is the segment's first step (row 0 of seg_q).
// Warps run decoupled: a step's rows arrive on full[st], each warp releases them on empty[st].
// Returns false if a wait timed out (the CTA must leave).
template <int NS>
__device__ __forceinline__ bool backward_block(Cols& cs, AdjSmem<NS>& sm, const AdjScn& p, int v0, int nv, int ta,
                                               int t_end, int t_lo, int32_t* status) {
  const size_t pitch = (size_t)p.pitch;
  const int rmask = p.ring - 1;
  const int vl = my_voxel();
  const int lane = threadIdx.x & 31;
  const bool live = vl < nv;
  // thread 0 orders every generic write these copies read (recomputed rows, inbox cells of earlier
  // blocks, made visible by the grid barrier) before the async-proxy reads, in issue_stage
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async;" ::: "memory");
    for (int s = 0; s < NS && ta - s >= t_end; ++s)
      if (!issue_stage(cs, sm, p, s, v0, nv, ta - s, t_lo, status)) sm.abort = 1;
  }
  for (int s = 0; s < NS; ++s) issue_xm(cs, sm, p, s, v0, nv, ta - s, ta - s >= t_end);
  for (int t = ta; t >= t_end; --t) {
    const int st = (ta - t) % NS;
    if (*(volatile int*)&sm.abort) return false;
    if (!mbar_wait(&sm.full[st], (cs.full_ph >> st) & 1u, status)) {
      sm.abort = 1;
      return false;
    }
    cs.full_ph ^= 1u << st;
    cs.inflight &= ~(1u << st);
    cp_async_wait<NS - 1>();  // this thread's copies of step t
    __syncwarp();             // the voxel group's copies of step t
    // lx[t] of the voxel: instantaneous terms + its 78 inbox cells (partial sums per component,
    // reduced over the 16-thread group in a fixed order)
    // column k = q + 16 i has component b = (q + i) mod 3 (16 = 1 mod 3): sum the columns i = j,
    // j + 3 (in order) into r[j], then rotate by q mod 3 so that pb[b] holds component b
    const float* in_row = sm.stage[st][0] + vl * kGainCols;
    const int q16 = threadIdx.x % kGroup;
    float r[3];
    r[0] = in_row[q16] + in_row[q16 + 3 * kGroup];
    r[1] = in_row[q16 + kGroup] + (q16 + 4 * kGroup < kGainCols ? in_row[q16 + 4 * kGroup] : 0.0f);
    r[2] = in_row[q16 + 2 * kGroup];
    const int rot = q16 % 3;
    float pb[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      // pb[b] = r[(b - rot) mod 3]
      const int j = b - rot;
      pb[b] = j == 0 ? r[0] : ((j == 1 || j == -2) ? r[1] : r[2]);
    }
#pragma unroll
    for (int off = kGroup / 2; off > 0; off >>= 1)
#pragma unroll
      for (int b = 0; b < 3; ++b) pb[b] = pb[b] + __shfl_xor_sync(0xffffffffu, pb[b], off);
    float lx[3] = {0.0f, 0.0f, 0.0f};
    if (live) {
      const float* xm = sm.xm[st][vl];
      const float x0 = xm[0], x1 = xm[1], x2 = xm[2];
      const float sum = fabsf(x0) + fabsf(x1) + fabsf(x2);
      const float f = sum > p.threshold ? sum - p.threshold : 0.0f;
      const float xs[3] = {x0, x1, x2};
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const float mreg = f > 0.0f ? f * copysignf(1.0f, xs[b]) : 0.0f;
        lx[b] = p.mse_scaling * xm[3 + b] + p.reg_scaling * mreg + pb[b];
      }
    }
    // the thread's columns: lap[t], gradient sums, inbox cell of the neighbour at step t - d
    const float* g = sm.g + vl * (3 * kGainCols);
#pragma unroll
    for (int i = 0; i < kCols; ++i) {
      const int k = my_col(i);
      if (cs.jw[i] >= 0) {
        const float G = g[k] * lx[0] + g[kGainCols + k] * lx[1] + g[2 * kGainCols + k] * lx[2];
        const float lap = G - cs.c[i] * cs.lprev[i];
        const float q_t = sm.stage[st][1][vl * kGainCols + k];
        const float in1 = t - cs.d[i] - 1 >= 0 ? sm.stage[st][2][vl * kGainCols + k] : 0.0f;
        const float ap_t = fmaf(cs.c[i], q_t, in1);  // the forward's all-pass output at step t
        cs.dg[i][0] = cs.dg[i][0] + lx[0] * ap_t;
        cs.dg[i][1] = cs.dg[i][1] + lx[1] * ap_t;
        cs.dg[i][2] = cs.dg[i][2] + lx[2] * ap_t;
        cs.dc[i] = cs.dc[i] + lap * q_t;
        const int ts = t - cs.d[i];
        if (ts >= 0) p.inbox[(size_t)(ts & rmask) * pitch + cs.jw[i]] = cs.c[i] * lap + cs.lprev[i];
        cs.lprev[i] = lap;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[st]);
    issue_xm(cs, sm, p, st, v0, nv, t - NS, t - NS >= t_end);
    if (threadIdx.x == 0 && t - NS >= t_end)
      if (!issue_stage(cs, sm, p, st, v0, nv, t - NS, t_lo, status)) sm.abort = 1;
  }
  return true;
}

// After a timed-out wait: let every bulk copy still in flight land (bounded) before the CTA leaves.
template <int NS>
__device__ __forceinline__ void drain_stages(Cols& cs, AdjSmem<NS>& sm, int32_t* status) {
  if (threadIdx.x == 0)
    for (int st = 0; st < NS; ++st)
      if (cs.inflight & (1u << st)) mbar_wait(&sm.full[st], (cs.full_ph >> st) & 1u, status);
}

template <int NS>
__global__ void __launch_bounds__(kAdjThreads, 1) adjoint_kernel(AdjLaunch L) {  // <= 128 registers
  extern __shared__ __align__(16) unsigned char smem_raw[];
  AdjSmem<NS>& sm = *reinterpret_cast<AdjSmem<NS>*>(smem_raw);
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
    for (int st = 0; st < NS; ++st) {
      mbar_init(&sm.full[st], 1);
      mbar_init(&sm.empty[st], kWarps);
    }
    mbar_init(&sm.meta_bar, 1);
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  Cols cs;
  cs.full_ph = cs.empty_ph = cs.empty_wait = cs.inflight = cs.meta_ph = 0;
  int cur_scn = -1, v0 = 0, nv = 0;
  if (resident && (int)blockIdx.x < ntiles) {
    tile_of(L, blockIdx.x, &cur_scn, &v0);
    load_scn(sm, L, cur_scn);
    nv = min(kTileVoxels, sm.sp.V - v0);
    if (!load_cols(cs, sm, sm.sp, v0, nv, false, L.status)) return;
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
        __syncthreads();  // recomputed rows (and the previous tile's tables) done with by every thread
        if (!resident && !load_cols(cs, sm, sm.sp, v0, nv, true, L.status)) return;
        if (!backward_block(cs, sm, sm.sp, v0, nv, ta, t_end, t_lo, L.status)) {
          drain_stages(cs, sm, L.status);
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
    if (cudaFuncSetAttribute(adjoint_kernel<kStagesSingle>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(AdjSmem<kStagesSingle>)) != cudaSuccess ||
        cudaFuncSetAttribute(adjoint_kernel<kStagesBatch>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(AdjSmem<kStagesBatch>)) != cudaSuccess)
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
  // both forms fit one CTA per SM (kAdjThreads threads of at most 128 registers)
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel<kStagesBatch>, kAdjThreads,
                                                sizeof(AdjSmem<kStagesBatch>));
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
  if (l.tiles)  // a batch's tile list
    return launch_cooperative((const void*)adjoint_kernel<kStagesBatch>, grid, kAdjThreads, args,
                              sizeof(AdjSmem<kStagesBatch>), stream);
  return launch_cooperative((const void*)adjoint_kernel<kStagesSingle>, grid, kAdjThreads, args,
                            sizeof(AdjSmem<kStagesSingle>), stream);
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
  l.ckpt_steps = d.ckpt_k;
  l.status = d.status;
  l.barrier = d.barrier;
  return launch_adjoint_tiles(l, d.adj_grid, stream);
}

}  // namespace ct
