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
//     barriers (monotone counter, ct_sync.cuh). (Waiting per tile for only the
//     tiles of its neighbourhood was measured slower: 3.58 against 2.92 ms on
//     the 20x20x20 cuboid, T = 2,000.)
//   * The all-pass state is deduplicated: ap_outputs[3v+a, 3n+b] does not
//     depend on the row component a (same input state, coefficient and zero
//     start, prediction.rs:56-79), so it is kept as [V, 26*3].
//   * Resident form (forward_ring_kernel): warp specialisation. A block of L
//     steps runs as rounds of kRound steps through a double-buffered ring of
//     all-pass outputs in shared memory. Producer warps: one thread per
//     (voxel, offset) runs the three all-pass chains of the round; its
//     3 (kRound + 1) history loads are independent. Consumer warps: one thread
//     per (voxel, step) accumulates the three rows x[t, 3v+a] over the 78
//     columns in order k = 0..77, adds the control input, stores the states
//     and the voxel's max-regularisation term. Named barriers hand the two
//     buffers back and forth.
//   * Streaming forms (forward_stream_kernel, forward_batch_kernel): every
//     thread takes both roles in turn, separated by CTA barriers: producer of
//     4-5 (voxel, offset) items, then consumer of one (step, row, voxel) state
//     (one accumulation chain over k = 0..77 per thread, three times the
//     consumer threads of the resident form). During the consumer phase each
//     thread already has the next round's history loads in flight, or in a
//     visit's last round the next tile's staging loads.
//   * Shared memory per tile: gains (absent neighbours zeroed, which adds
//     exact zeros where the reference skips), (neighbour, delay, coefficient)
//     per (voxel, offset), the chain state, and the round buffers. A CTA that
//     owns one tile stages it once per launch.
//   * History reads go through L1: within one launch a history row is read
//     only after the grid barrier's acquire, which orders its writes before the
//     read.
#include <cuda_runtime.h>

#include "ct_internal.cuh"
#include "ct_sync.cuh"

namespace ct {
namespace {

constexpr int kTileVoxels = kFwdTileVoxels;
constexpr int kFwdScnCache = 64;  // scenarios of a batched launch kept in shared memory
constexpr int kTileStates = 3 * kTileVoxels;
constexpr int kTileItems = kTileVoxels * kOffsets;  // (voxel, offset) pairs
constexpr int kRound = 2;                            // steps per round
constexpr int kProducers = 128;                      // 4 warps
constexpr int kConsumers = kRound * kTileVoxels;     // 2 warps: (step, voxel)
constexpr int kThreads = kProducers + kConsumers;
constexpr int kBarFull = 1;   // named barriers kBarFull + buffer, kBarEmpty + buffer (resident form)
constexpr int kBarEmpty = 3;
constexpr int kItemsPerProducer = (kTileItems + kProducers - 1) / kProducers;  // resident form
static_assert(kRound == 2, "the producers' fast paths step two chains");

// Streaming forms (a CTA walks several tiles, re-staging each per block of steps). All 192 threads
// take both roles in turn: producers, one thread per (voxel, offset) item (4-5 items each), then
// consumers, one thread per (step, row a, voxel) state of the round; CTA barriers separate the two.
// While the consumers work, each thread already holds the next round's history loads (or, in a
// visit's last round, the next tile's staging loads) in flight.
constexpr int kApPitch = kGainCols + 1;  // odd row pitch of the round buffer: conflict-free reads
constexpr int kLsItems = (kTileItems + kThreads - 1) / kThreads;
static_assert(kRound * 3 * kTileVoxels == kThreads, "one consumer thread per (step, row, voxel)");

struct Smem {
  float g[3][kGainCols][kTileVoxels];             // gain g[3v+a][k] at [a][k][v] (absent neighbours zero)
  float ap_out[kRound][kTileVoxels * kApPitch];   // all-pass outputs of the round's steps
  float ap_state[kTileVoxels * kGainCols];
  int32_t j[kTileItems];                          // 3 * neighbour, -1 if absent
  int32_t d[kTileItems];
  float c[kTileItems];
  float ctrl[kTileStates];
  float xs[kRound][3][kTileVoxels];               // the round's states, for the regularisation term
  float part[kMaxStepBlock];
};

__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void named_arrive(int id, int count) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// A tile's staging loads, held in registers between their issue and their store to shared
// memory, so that they can be issued before the previous tile's visit ends.
constexpr int kStageItems = (kTileItems + kThreads - 1) / kThreads;
constexpr int kStageCols = (kGainCols * kTileVoxels + kThreads - 1) / kThreads;
static_assert(kTileStates <= kThreads, "one control entry per thread");

struct StageRegs {
  int32_t nb[kStageItems], dl[kStageItems];
  float cf[kStageItems];
  float gx[kStageCols], gy[kStageCols], gz[kStageCols], ap[kStageCols];
  float ctl;
};

// Issue every global load of tile v0 of scenario p (metadata, the three gain rows, chain state,
// control column) into registers; nothing waits for them here.
__device__ __forceinline__ void stage_load(StageRegs& r, const FwdArgs& p, int v0) {
  const int nv = min(kTileVoxels, p.V - v0);
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < kStageItems; ++i) {
    const int e = tid + i * kThreads;
    const bool ok = e < kTileItems && e / kOffsets < nv;
    const int gi = v0 * kOffsets + (ok ? e : 0);
    r.nb[i] = ok ? p.nbr[gi] : -1;
    r.dl[i] = ok ? p.delays[gi] : 1;
    r.cf[i] = ok ? p.coefs[gi] : 0.0f;
  }
#pragma unroll
  for (int i = 0; i < kStageCols; ++i) {
    const int e = tid + i * kThreads;
    const int k = e / kTileVoxels, vl = e - k * kTileVoxels;
    const bool ok = e < kGainCols * kTileVoxels && vl < nv;
    const float* row = p.gains + (size_t)3 * (v0 + (ok ? vl : 0)) * kGainCols + (ok ? k : 0);
    r.gx[i] = ok ? row[0] : 0.0f;
    r.gy[i] = ok ? row[kGainCols] : 0.0f;
    r.gz[i] = ok ? row[2 * kGainCols] : 0.0f;
    r.ap[i] = (e < nv * kGainCols) ? p.ap[(size_t)v0 * kGainCols + e] : 0.0f;
  }
  r.ctl = (tid < 3 * nv) ? p.ctrl[3 * v0 + tid] : 0.0f;
}

// Store staged registers to shared memory (all threads, after every read of the previous tile's
// shared data); the gain mask needs the neighbour table and is applied after a barrier.
__device__ __forceinline__ void stage_store(Smem& sm, const StageRegs& r) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < kStageItems; ++i) {
    const int e = tid + i * kThreads;
    if (e < kTileItems) {
      sm.j[e] = r.nb[i] < 0 ? -1 : 3 * r.nb[i];
      sm.d[e] = r.dl[i];
      sm.c[e] = r.cf[i];
    }
  }
  if (tid < kTileStates) sm.ctrl[tid] = r.ctl;
#pragma unroll
  for (int i = 0; i < kStageCols; ++i) {
    const int e = tid + i * kThreads;
    if (e < kTileVoxels * kGainCols) sm.ap_state[e] = r.ap[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kStageCols; ++i) {
    const int e = tid + i * kThreads;
    if (e < kGainCols * kTileVoxels) {
      const int k = e / kTileVoxels, vl = e - k * kTileVoxels;
      const bool live = sm.j[vl * kOffsets + k / 3] >= 0;  // absent neighbours add exact zeros
      sm.g[0][k][vl] = live ? r.gx[i] : 0.0f;
      sm.g[1][k][vl] = live ? r.gy[i] : 0.0f;
      sm.g[2][k][vl] = live ? r.gz[i] : 0.0f;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void unstage_tile(Smem& sm, const FwdArgs& p, int v0) {
  const int nv = min(kTileVoxels, p.V - v0);
  float* a0 = p.ap + (size_t)v0 * kGainCols;
  for (int e = threadIdx.x; e < nv * kGainCols; e += blockDim.x) a0[e] = sm.ap_state[e];
}

// History of the thread's items for the round starting at tr0: h[i][q][b] = x[tr0 - d_i - 1 + q,
// j_i + b] (rows before t = 0 read as zero, prediction.rs:68-77). Every row read within a block of
// L <= dmin steps is older than the block, so these loads may be issued at any time in the block.
__device__ __forceinline__ void load_history(float (&h)[kLsItems][kRound + 1][3], const Smem& sm, const FwdArgs& p,
                                             int tr0, int R, int dmax) {
  if (R == kRound && tr0 - dmax - 1 >= 0) {
    // every row exists: unpredicated loads (an absent neighbour reads column 0; its values are unused)
#pragma unroll
    for (int i = 0; i < kLsItems; ++i) {
      const int e = threadIdx.x + i * kThreads;
      const int jb = e < kTileItems ? sm.j[e] : -1;
      const int d = jb >= 0 ? sm.d[e] : dmax;  // absent: an old row, values unused
      const float* row = p.X + (size_t)(tr0 - d - 1) * p.S + (jb >= 0 ? jb : 0);
#pragma unroll
      for (int q = 0; q <= kRound; ++q)
#pragma unroll
        for (int b = 0; b < 3; ++b) h[i][q][b] = row[(size_t)q * p.S + b];
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < kLsItems; ++i) {
    const int e = threadIdx.x + i * kThreads;
    const int jb = e < kTileItems ? sm.j[e] : -1;
    const int d = e < kTileItems ? sm.d[e] : 0;
#pragma unroll
    for (int q = 0; q <= kRound; ++q) {
      const int tr = tr0 - d - 1 + q;
      const bool ok = jb >= 0 && q <= R && tr >= 0;
      const float* row = p.X + (size_t)(ok ? tr : 0) * p.S + (jb >= 0 ? jb : 0);
#pragma unroll
      for (int b = 0; b < 3; ++b) h[i][q][b] = ok ? row[b] : 0.0f;
    }
  }
}

// Producer: all-pass chains of the thread's items for steps tr0 .. tr0+R-1 into the round buffer.
__device__ __forceinline__ void produce(Smem& sm, const FwdArgs& p, int v0, int nv, int tr0, int R,
                                        const float (&h)[kLsItems][kRound + 1][3]) {
  // adjoint checkpoint inside this round: step index after which the state is stored, or -1
  int ck_s = -1;
  float* ck_row = nullptr;
  if (p.ckpt) {
    const int tc = ((tr0 + p.ckpt_k) & ~(p.ckpt_k - 1)) - 1;  // first step t >= tr0 with (t+1) % K == 0
    if (tc < tr0 + R && tc + 1 < p.T) {
      ck_s = tc - tr0;
      ck_row = p.ckpt + (size_t)((tc + 1) / p.ckpt_k) * p.V * kGainCols + (size_t)v0 * kGainCols;
    }
  }
  if (R == kRound && ck_s < 0 && !(tr0 <= p.T - 2 && p.T - 2 < tr0 + kRound)) {
    // common round: no per-element checks (same arithmetic)
#pragma unroll
    for (int i = 0; i < kLsItems; ++i) {
      const int e = threadIdx.x + i * kThreads;
      if (e >= kTileItems) break;
      const int vl = e / kOffsets;
      const int n = e - vl * kOffsets;
      float* st = sm.ap_state + vl * kGainCols + 3 * n;
      float* out0 = sm.ap_out[0] + vl * kApPitch + 3 * n;
      if (sm.j[e] >= 0) {
        const float c = sm.c[e];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          float a = fmaf(c, h[i][1][b] - st[b], h[i][0][b]);
          out0[b] = a;
          a = fmaf(c, h[i][2][b] - a, h[i][1][b]);
          out0[kTileVoxels * kApPitch + b] = a;
          st[b] = a;
        }
      } else {
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          out0[b] = 0.0f;
          out0[kTileVoxels * kApPitch + b] = 0.0f;
        }
      }
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < kLsItems; ++i) {
    const int e = threadIdx.x + i * kThreads;
    if (e >= kTileItems) break;
    const int vl = e / kOffsets;
    const int n = e - vl * kOffsets;
    const int jb = sm.j[e];
    float* st = sm.ap_state + vl * kGainCols + 3 * n;
    float* out0 = sm.ap_out[0] + vl * kApPitch + 3 * n;
    if (jb >= 0) {
      const float c = sm.c[e];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        float a = st[b];
#pragma unroll
        for (int s = 0; s < kRound; ++s) {
          if (s < R) {
            a = fmaf(c, h[i][s + 1][b] - a, h[i][s][b]);
            out0[s * (kTileVoxels * kApPitch) + b] = a;
            if (tr0 + s == p.T - 2) p.ap_last[(size_t)(v0 + vl) * kGainCols + 3 * n + b] = a;
            if (s == ck_s) ck_row[vl * kGainCols + 3 * n + b] = a;
          }
        }
        st[b] = a;
      }
    } else {
#pragma unroll
      for (int s = 0; s < kRound; ++s)
        if (s < R)
#pragma unroll
          for (int b = 0; b < 3; ++b) out0[s * (kTileVoxels * kApPitch) + b] = 0.0f;
      if (vl < nv && p.T - 2 >= tr0 && p.T - 2 < tr0 + R)
#pragma unroll
        for (int b = 0; b < 3; ++b) p.ap_last[(size_t)(v0 + vl) * kGainCols + 3 * n + b] = st[b];
    }
  }
}

// Consumer: the state x[tr0 + s, 3 (v0 + vl) + a] (thread = (s, a, vl)), accumulated over the 78
// columns in the reference's order, plus the control input; stored to X and to the round's xs.
__device__ __forceinline__ void consume(Smem& sm, const FwdArgs& p, int v0, int nv, int tr0, int R) {
  const int s = threadIdx.x / (3 * kTileVoxels);
  const int a = (threadIdx.x / kTileVoxels) % 3;
  const int vl = threadIdx.x % kTileVoxels;
  if (s >= R || vl >= nv) return;
  const float* aps = sm.ap_out[s] + vl * kApPitch;
  const float* gs = &sm.g[a][0][vl];
  float x = 0.0f;
#pragma unroll 13
  for (int k = 0; k < kGainCols; ++k) x = x + gs[k * kTileVoxels] * aps[k];
  const int t = tr0 + s;
  x = x + p.u[t] * sm.ctrl[3 * vl + a];
  p.X[(size_t)t * p.S + 3 * (v0 + vl) + a] = x;
  sm.xs[s][a][vl] = x;
}

// The voxels' max-regularisation terms of the round's step s (warp s * 3 of the consumers, lane =
// voxel), reduced over the warp in lane order and added to part[r0 + s].
__device__ __forceinline__ void regularise(Smem& sm, const FwdArgs& p, int nv, int R, int r0) {
  const int s = threadIdx.x / (3 * kTileVoxels);
  const int a = (threadIdx.x / kTileVoxels) % 3;
  const int vl = threadIdx.x % kTileVoxels;
  if (a != 0 || s >= R) return;  // warp-uniform
  float f2 = 0.0f;
  if (vl < nv) {
    const float sum = fabsf(sm.xs[s][0][vl]) + fabsf(sm.xs[s][1][vl]) + fabsf(sm.xs[s][2][vl]);
    if (sum > p.threshold) {
      const float f = sum - p.threshold;
      f2 = f * f;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) f2 = f2 + __shfl_down_sync(0xffffffffu, f2, off);
  if (vl == 0) sm.part[r0 + s] = sm.part[r0 + s] + f2;
}

// One visit of a tile: L steps from t0 in rounds of kRound. `h` holds the first round's history on
// entry; with `next` set, the last round's consumer phase also issues the next tile's staging loads
// into `nx` (stored by the caller after this visit).
__device__ __forceinline__ void visit_tile(Smem& sm, const FwdArgs& p, int v0, int nv, int t0, int L, int dmax,
                                           float (&h)[kLsItems][kRound + 1][3], const FwdArgs* next, int next_v0,
                                           StageRegs& nx) {
  for (int r0 = 0; r0 < L; r0 += kRound) {
    const int R = (L - r0) < kRound ? (L - r0) : kRound;
    produce(sm, p, v0, nv, t0 + r0, R, h);
    __syncthreads();
    if (r0 + kRound < L) {
      const int Rn = (L - r0 - kRound) < kRound ? (L - r0 - kRound) : kRound;
      load_history(h, sm, p, t0 + r0 + kRound, Rn, dmax);
    } else if (next) {
      stage_load(nx, *next, next_v0);
    }
    consume(sm, p, v0, nv, t0 + r0, R);
    __syncthreads();
    regularise(sm, p, nv, R, r0);
  }
}

__global__ void __launch_bounds__(kThreads, 2) forward_stream_kernel(FwdArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);

  const int V = p.V, T = p.T;
  const int num_tiles = (V + kTileVoxels - 1) / kTileVoxels;
  const bool resident = num_tiles <= (int)gridDim.x;  // this CTA owns at most one tile
  int dmin = p.dmin[0];
  if (dmin < 1) dmin = 1;
  const int dmax = p.dmin[1] > dmin ? p.dmin[1] : dmin;
  const int Lmax = dmin < kMaxStepBlock ? dmin : kMaxStepBlock;
  float h[kLsItems][kRound + 1][3];
  StageRegs nx;

  if (resident && (int)blockIdx.x < num_tiles) {
    stage_load(nx, p, blockIdx.x * kTileVoxels);
    stage_store(sm, nx);
  }
  unsigned int barrier_number = 0;
  for (int t0 = 0; t0 < T; t0 += Lmax) {
    const int L = (T - t0) < Lmax ? (T - t0) : Lmax;
    if (threadIdx.x < kMaxStepBlock) sm.part[threadIdx.x] = 0.0f;
    // the block's first tile: staged now (resident tiles stay staged)
    if (!resident && (int)blockIdx.x < num_tiles) {
      __syncthreads();
      stage_load(nx, p, blockIdx.x * kTileVoxels);
      stage_store(sm, nx);
    } else {
      __syncthreads();
    }
    for (int tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
      const int v0 = tile * kTileVoxels;
      const int nv = min(kTileVoxels, V - v0);
      const int nt = tile + (int)gridDim.x;
      const bool more = !resident && nt < num_tiles;
      load_history(h, sm, p, t0, L < kRound ? L : kRound, dmax);
      visit_tile(sm, p, v0, nv, t0, L, dmax, h, more ? &p : nullptr, nt * kTileVoxels, nx);
      if (!resident) {
        unstage_tile(sm, p, v0);
        if (more) {
          __syncthreads();  // every thread's chain state is out before the next tile's lands
          stage_store(sm, nx);
        }
      }
    }
    __syncthreads();
    if ((int)threadIdx.x < L) p.stepsum_part[(size_t)(t0 + threadIdx.x) * gridDim.x + blockIdx.x] = sm.part[threadIdx.x];
    if (t0 + L < T) {
      if (!grid_barrier(p.barrier, barrier_number++, p.status)) return;
    }
  }
  if (resident && (int)blockIdx.x < num_tiles) {
    __syncthreads();
    unstage_tile(sm, p, blockIdx.x * kTileVoxels);
  }
}


// ---- batched form: the streaming schedule over the tiles of several scenarios
//
// Every tile names its scenario; all scenarios advance through the same
// absolute steps (a scenario whose beat is shorter idles once it is done),
// L = the smallest min(dmin, kMaxStepBlock) of any scenario. Each tile writes
// its own per-step max-regularisation partial, stepsum_part[t * part_stride +
// tile of the scenario], so the step metrics of every scenario sum the same
// partials in the same order. A visit's last round issues the staging loads
// of the CTA's next live tile (whatever its scenario).
__global__ void __launch_bounds__(kThreads, 2) forward_batch_kernel(FwdBatch B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  // the launch's first kFwdScnCache scenarios, copied into shared memory once; a tile of any other
  // scenario loads it into `over` at the start of its visit
  __shared__ FwdArgs cache[kFwdScnCache];
  __shared__ FwdArgs over;
  for (int i = threadIdx.x; i < min(B.nscn, kFwdScnCache); i += blockDim.x) cache[i] = B.scns[i];
  auto scn_of = [&](int s) -> const FwdArgs& { return s < kFwdScnCache ? cache[s] : B.scns[s]; };
  int Lmax = kMaxStepBlock;
  for (int s = 0; s < B.nscn; ++s) {
    int dmin = B.scns[s].dmin[0];
    if (dmin < 1) dmin = 1;
    if (dmin < Lmax) Lmax = dmin;
  }
  float h[kLsItems][kRound + 1][3];
  StageRegs nx;
  // the CTA's first tile at or after list index `from` whose scenario still runs at step t0
  auto next_live = [&](int from, int t0) {
    int tile = from;
    while (tile < B.ntiles && t0 >= scn_of(B.tiles[tile].x).T) tile += gridDim.x;
    return tile;
  };
  __syncthreads();
  unsigned int barrier_number = 0;
  for (int t0 = 0; t0 < B.Tmax; t0 += Lmax) {
    int tile = next_live(blockIdx.x, t0);
    __syncthreads();
    if (tile < B.ntiles) {
      const int2 tl = B.tiles[tile];
      stage_load(nx, scn_of(tl.x), tl.y);
      stage_store(sm, nx);
    }
    while (tile < B.ntiles) {
      const int2 tl = B.tiles[tile];
      if (threadIdx.x == 0 && tl.x >= kFwdScnCache) over = B.scns[tl.x];
      if (threadIdx.x < kMaxStepBlock) sm.part[threadIdx.x] = 0.0f;
      __syncthreads();
      const FwdArgs& sp = tl.x < kFwdScnCache ? cache[tl.x] : over;
      const int L = (sp.T - t0) < Lmax ? (sp.T - t0) : Lmax;
      const int v0 = tl.y;
      const int nv = min(kTileVoxels, sp.V - v0);
      const int nt = next_live(tile + (int)gridDim.x, t0);
      const bool more = nt < B.ntiles;
      const int2 ntl = more ? B.tiles[nt] : make_int2(0, 0);
      const int dmax = max(sp.dmin[1], 1);
      load_history(h, sm, sp, t0, L < kRound ? L : kRound, dmax);
      visit_tile(sm, sp, v0, nv, t0, L, dmax, h, more ? &scn_of(ntl.x) : nullptr, ntl.y, nx);
      unstage_tile(sm, sp, v0);
      __syncthreads();  // the last round's regularisation terms are in part[]
      if ((int)threadIdx.x < L)
        sp.stepsum_part[(size_t)(t0 + threadIdx.x) * sp.part_stride + v0 / kTileVoxels] = sm.part[threadIdx.x];
      __syncthreads();  // chain state and partials are out, sp is free, before the next tile lands
      if (more) stage_store(sm, nx);
      tile = nt;
    }
    if (t0 + Lmax < B.Tmax) {
      if (!grid_barrier(B.barrier, barrier_number++, B.status)) return;
    }
  }
}

// ---- resident form: one tile per CTA for the whole launch, neighbour history in a shared ring
//
// Each tile's halo (the device voxels its 26-neighbourhoods touch, at most
// kHaloMax) is listed on the host; producer thread p owns the items
// e = p + kProducers * i and keeps their halo slot, delay, coefficient and
// three chain states in registers for the whole launch. History rows live
// in a ring of kRingRows rows x halo states in shared memory: each round
// needs rows [t - dmax - 1, t + kRound - 1 - dmin], stages the rows new to
// the window with cp.async one round ahead (the first round of a block
// stages after the grid barrier, since its rows were produced in the
// previous block), and the chains read only shared memory. When the spread
// of delays does not fit the ring, the producers read the history from
// global memory instead (same arithmetic, same results).

constexpr int kHaloMax = kFwdHaloMax;
constexpr int kRingRows = 16;  // power of two: slot = row & (kRingRows - 1)
constexpr int kBarProducers = 5;

struct RingSmem {
  float4 g[kGainCols][kTileVoxels];
  float ap_out[2][kRound][kTileVoxels * kGainCols];
  float ring[kRingRows][kHaloMax * 3];
  int32_t halo[kHaloMax];  // device voxel of each halo slot
  float ctrl[kTileStates];
  float part[kMaxStepBlock];
};

struct RingArgs {
  const int32_t* halo;    // [tiles, kHaloMax], -1 padded
  const int16_t* hslot;   // [tiles, kTileItems], halo slot of the item's neighbour, -1 if absent
  const int32_t* nhalo;   // [tiles]
};

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// Producer p stages the ring columns q = p + kProducers * i (i < kStageSlots) of every history row;
// col[i] is the state index 3 * halo[q / 3] + q % 3 of column q, or -1 beyond the halo's 3 nh columns
// (computed once per launch, so a staged element costs an address add and the copy).
constexpr int kStageSlots = (kHaloMax * 3 + kProducers - 1) / kProducers;

// Producers: copy history rows [r_lo, r_hi] of the halo into the ring (rows before t = 0 are zero).
__device__ __forceinline__ void stage_rows(RingSmem& sm, const FwdArgs& p, const int (&col)[kStageSlots], int r_lo,
                                           int r_hi) {
  for (int row = r_lo; row <= r_hi; ++row) {
    float* dst = sm.ring[row & (kRingRows - 1)] + threadIdx.x;
    const float* src = p.X + (size_t)(row < 0 ? 0 : row) * p.S;
#pragma unroll
    for (int i = 0; i < kStageSlots; ++i) {
      if (col[i] < 0) continue;
      if (row < 0)
        dst[i * kProducers] = 0.0f;
      else
        cp_async4(dst + i * kProducers, src + col[i]);
    }
  }
}

// Two CTAs per SM (<= 170 registers) keep up to 296 tiles co-resident.
__global__ void __launch_bounds__(kThreads, 2) forward_ring_kernel(FwdArgs p, RingArgs ra) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RingSmem& sm = *reinterpret_cast<RingSmem*>(smem_raw);
  const int T = p.T, S = p.S;
  const int tile = blockIdx.x;
  const int v0 = tile * kTileVoxels;
  const int nv = min(kTileVoxels, p.V - v0);
  const int nh = ra.nhalo[tile];
  const bool producer = threadIdx.x < kProducers;
  int dmin = p.dmin[0], dmax = p.dmin[1];
  if (dmin < 1) dmin = 1;
  if (dmax < dmin) dmax = dmin;
  const int Lmax = dmin < kMaxStepBlock ? dmin : kMaxStepBlock;
  // rows a round reads: [tr0 - dmax - 1, tr0 + kRound - 1 - dmin]; plus kRound rows staged ahead
  const bool use_ring = (dmax - dmin + kRound + 1) + kRound <= kRingRows;
  // rows a block reads: [t0 - dmax - 1, t0 + L - 1 - dmin], all produced before the block; when they
  // fit the ring together, they are staged once at the block's start (one wait per block instead of
  // one per round)
  const bool stage_block = use_ring && (dmax - dmin + Lmax + 1) <= kRingRows;

  // ---- set-up: gains (transposed, masked), control, halo list, zeroed ring
  for (int e = threadIdx.x; e < kGainCols * kTileVoxels; e += blockDim.x) {
    const int k = e / kTileVoxels, vl = e - k * kTileVoxels;
    float4 g = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (vl < nv && p.nbr[(v0 + vl) * kOffsets + k / 3] >= 0) {
      const float* row = p.gains + (size_t)3 * (v0 + vl) * kGainCols + k;
      g.x = row[0];
      g.y = row[kGainCols];
      g.z = row[2 * kGainCols];
    }
    sm.g[k][vl] = g;
  }
  for (int e = threadIdx.x; e < kTileStates; e += blockDim.x) sm.ctrl[e] = (e < 3 * nv) ? p.ctrl[3 * v0 + e] : 0.0f;
  for (int e = threadIdx.x; e < kHaloMax; e += blockDim.x) sm.halo[e] = e < nh ? ra.halo[tile * kHaloMax + e] : 0;
  for (int e = threadIdx.x; e < kRingRows * kHaloMax * 3; e += blockDim.x) (&sm.ring[0][0])[e] = 0.0f;

  // producer item registers
  int hs[kItemsPerProducer], dd[kItemsPerProducer], jj[kItemsPerProducer];
  float cc[kItemsPerProducer], st[kItemsPerProducer][3];
#pragma unroll
  for (int i = 0; i < kItemsPerProducer; ++i) {
    const int e = threadIdx.x + i * kProducers;
    hs[i] = -1;
    dd[i] = 1;
    jj[i] = 0;
    cc[i] = 0.0f;
    st[i][0] = st[i][1] = st[i][2] = 0.0f;
    if (producer && e < kTileItems && e / kOffsets < nv) {
      const int gi = v0 * kOffsets + e;
      const int32_t nb = p.nbr[gi];
      if (nb >= 0) {
        hs[i] = ra.hslot[(size_t)tile * kTileItems + e];
        dd[i] = p.delays[gi];
        cc[i] = p.coefs[gi];
        jj[i] = 3 * nb;
      }
    }
  }
  __syncthreads();
  int stage_col[kStageSlots];
#pragma unroll
  for (int i = 0; i < kStageSlots; ++i) {
    const int q = threadIdx.x + i * kProducers;
    stage_col[i] = (producer && q < 3 * nh) ? 3 * sm.halo[q / 3] + q % 3 : -1;
  }

  int round = 0;
  unsigned int barrier_number = 0;
  int staged_top = -dmin - 1 + kRound - 1 - kRound;  // highest ring row staged so far (none)

  for (int t0 = 0; t0 < T; t0 += Lmax) {
    const int L = (T - t0) < Lmax ? (T - t0) : Lmax;
    if (threadIdx.x < kMaxStepBlock) sm.part[threadIdx.x] = 0.0f;
    __syncthreads();
    for (int r0 = 0; r0 < L; r0 += kRound, ++round) {
      const int R = (L - r0) < kRound ? (L - r0) : kRound;
      const int tr0 = t0 + r0;
      const int buf = round & 1;
      const int top = tr0 + R - 1 - dmin;  // newest history row this round reads
      if (producer) {
        if (stage_block) {
          if (r0 == 0) {
            const int top_blk = t0 + L - 1 - dmin;  // newest history row the block reads
            if (top_blk > staged_top) {
              stage_rows(sm, p, stage_col, staged_top + 1, top_blk);
              staged_top = top_blk;
            }
            cp_async_commit_wait_all();
            named_sync(kBarProducers, kProducers);  // the block's ring rows visible to all producers
          }
        } else if (use_ring) {
          if (r0 == 0 && top > staged_top) {  // first round of a block: rows produced in the previous block
            stage_rows(sm, p, stage_col, staged_top + 1, top);
            staged_top = top;
          }
          cp_async_commit_wait_all();
          named_sync(kBarProducers, kProducers);  // ring rows of this round visible to all producers
          // stage the next round's new rows (all older than t0) while this round computes
          const int r0n = r0 + kRound;
          if (r0n < L) {
            const int Rn = (L - r0n) < kRound ? (L - r0n) : kRound;
            const int topn = t0 + r0n + Rn - 1 - dmin;
            if (topn > staged_top) {
              stage_rows(sm, p, stage_col, staged_top + 1, topn);
              staged_top = topn;
            }
          }
          cp_async_commit();
        }
        if (round >= 2) named_sync(kBarEmpty + buf, kThreads);
        // adjoint checkpoint inside this round: step index s2 after which the state is stored, or -1
        int ck_s = -1;
        float* ck_row = nullptr;
        if (p.ckpt) {
          const int tc = ((tr0 + p.ckpt_k) & ~(p.ckpt_k - 1)) - 1;  // first step t >= tr0 with (t+1) % K == 0
          if (tc < tr0 + R && tc + 1 < T) {
            ck_s = tc - tr0;
            ck_row = p.ckpt + (size_t)((tc + 1) / p.ckpt_k) * p.V * kGainCols + (size_t)v0 * kGainCols;
          }
        }
        // common round: full length, every history row from the ring at t >= 0, no checkpoint and
        // no ap_last step: the chains without per-element checks (same arithmetic)
        const bool fast = use_ring && R == kRound && tr0 - dmax - 1 >= 0 && ck_s < 0 &&
                          !(tr0 <= T - 2 && T - 2 < tr0 + kRound);
        if (fast) {
#pragma unroll
          for (int i = 0; i < kItemsPerProducer; ++i) {
            const int e = threadIdx.x + i * kProducers;
            if (e >= kTileItems) break;
            const int vl = e / kOffsets;
            const int n = e - vl * kOffsets;
            float* out0 = sm.ap_out[buf][0] + vl * kGainCols + 3 * n;
            if (hs[i] >= 0) {
              const int base = tr0 - dd[i] - 1;
              const float* h0 = &sm.ring[base & (kRingRows - 1)][3 * hs[i]];
              const float* h1 = &sm.ring[(base + 1) & (kRingRows - 1)][3 * hs[i]];
              const float* h2 = &sm.ring[(base + 2) & (kRingRows - 1)][3 * hs[i]];
#pragma unroll
              for (int b = 0; b < 3; ++b) {
                const float x0 = h0[b], x1 = h1[b], x2 = h2[b];
                float a = fmaf(cc[i], x1 - st[i][b], x0);
                out0[b] = a;
                a = fmaf(cc[i], x2 - a, x1);
                out0[kTileVoxels * kGainCols + b] = a;
                st[i][b] = a;
              }
            } else {
#pragma unroll
              for (int b = 0; b < 3; ++b) {
                out0[b] = 0.0f;
                out0[kTileVoxels * kGainCols + b] = 0.0f;
              }
            }
          }
        } else {
#pragma unroll
        for (int i = 0; i < kItemsPerProducer; ++i) {
          const int e = threadIdx.x + i * kProducers;
          if (e >= kTileItems) break;
          const int vl = e / kOffsets;
          const int n = e - vl * kOffsets;
          float* out0 = sm.ap_out[buf][0] + vl * kGainCols + 3 * n;
          if (hs[i] >= 0) {
            float h[kRound + 1][3];
#pragma unroll
            for (int q = 0; q <= kRound; ++q) {
              const int row = tr0 - dd[i] - 1 + q;
              const bool ok = q <= R && row >= 0;
              if (use_ring) {
                const float* src = &sm.ring[row & (kRingRows - 1)][3 * hs[i]];
#pragma unroll
                for (int b = 0; b < 3; ++b) h[q][b] = ok ? src[b] : 0.0f;
              } else {
                const float* src = p.X + (size_t)(ok ? row : 0) * S + jj[i];
#pragma unroll
                for (int b = 0; b < 3; ++b) h[q][b] = ok ? src[b] : 0.0f;
              }
            }
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              float a = st[i][b];
#pragma unroll
              for (int s2 = 0; s2 < kRound; ++s2) {
                if (s2 < R) {
                  a = fmaf(cc[i], h[s2 + 1][b] - a, h[s2][b]);
                  out0[s2 * (kTileVoxels * kGainCols) + b] = a;
                  if (tr0 + s2 == T - 2) p.ap_last[(size_t)(v0 + vl) * kGainCols + 3 * n + b] = a;
                  if (s2 == ck_s) ck_row[vl * kGainCols + 3 * n + b] = a;
                }
              }
              st[i][b] = a;
            }
          } else {
#pragma unroll
            for (int s2 = 0; s2 < kRound; ++s2)
              if (s2 < R)
#pragma unroll
                for (int b = 0; b < 3; ++b) out0[s2 * (kTileVoxels * kGainCols) + b] = 0.0f;
          }
        }
        }
        named_arrive(kBarFull + buf, kThreads);
      } else {
        named_sync(kBarFull + buf, kThreads);
        // consumers: same arithmetic as the streaming form
        const int ct = threadIdx.x - kProducers;
        const int s2 = ct / kTileVoxels, vl = ct - s2 * kTileVoxels;
        if (s2 < R) {
          float f2 = 0.0f;
          if (vl < nv) {
            const float* aps = sm.ap_out[buf][s2] + vl * kGainCols;
            float x0 = 0.0f, x1 = 0.0f, x2 = 0.0f;
#pragma unroll
            for (int k = 0; k < kGainCols; k += 2) {
              const float2 a = *reinterpret_cast<const float2*>(aps + k);
              const float4 g0 = sm.g[k][vl];
              const float4 g1 = sm.g[k + 1][vl];
              x0 = x0 + g0.x * a.x;
              x1 = x1 + g0.y * a.x;
              x2 = x2 + g0.z * a.x;
              x0 = x0 + g1.x * a.y;
              x1 = x1 + g1.y * a.y;
              x2 = x2 + g1.z * a.y;
            }
            const int t = tr0 + s2;
            const float uc = p.u[t];
            x0 = x0 + uc * sm.ctrl[3 * vl];
            x1 = x1 + uc * sm.ctrl[3 * vl + 1];
            x2 = x2 + uc * sm.ctrl[3 * vl + 2];
            float* xo = p.X + (size_t)t * S + 3 * (v0 + vl);
            xo[0] = x0;
            xo[1] = x1;
            xo[2] = x2;
            const float sum = fabsf(x0) + fabsf(x1) + fabsf(x2);
            if (sum > p.threshold) {
              const float f = sum - p.threshold;
              f2 = f * f;
            }
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) f2 = f2 + __shfl_down_sync(0xffffffffu, f2, off);
          if (vl == 0) sm.part[r0 + s2] = sm.part[r0 + s2] + f2;
        }
        named_arrive(kBarEmpty + buf, kThreads);
      }
    }
    __syncthreads();
    if ((int)threadIdx.x < L) p.stepsum_part[(size_t)(t0 + threadIdx.x) * gridDim.x + blockIdx.x] = sm.part[threadIdx.x];
    if (t0 + L < T) {
      if (!grid_barrier(p.barrier, barrier_number++, p.status)) {
        if (producer) cp_async_commit_wait_all();
        return;
      }
    }
  }
  if (producer) {
    cp_async_commit_wait_all();
#pragma unroll
    for (int i = 0; i < kItemsPerProducer; ++i) {
      const int e = threadIdx.x + i * kProducers;
      if (e < kTileItems && e / kOffsets < nv)
#pragma unroll
        for (int b = 0; b < 3; ++b) p.ap[(size_t)v0 * kGainCols + 3 * e + b] = st[i][b];
    }
  }
}
}  // namespace

int forward_grid_size(int64_t V, int device) {
  static bool configured[128] = {};
  if (device >= 0 && device < 128 && !configured[device]) {
    cudaFuncSetAttribute(forward_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
    cudaFuncSetAttribute(forward_ring_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RingSmem));
    configured[device] = true;
  }
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, forward_stream_kernel, kThreads, sizeof(Smem));
  if (per_sm < 1) per_sm = 1;
  const int64_t tiles = (V + kTileVoxels - 1) / kTileVoxels;
  int64_t grid = (int64_t)sms * per_sm;
  if (tiles < grid) grid = tiles;
  if (grid < 1) grid = 1;
  return (int)grid;
}

int forward_batch_capacity(int device) {
  forward_grid_size(1, device);
  static bool configured[128] = {};
  if (device >= 0 && device < 128 && !configured[device]) {
    cudaFuncSetAttribute(forward_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
    configured[device] = true;
  }
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, forward_batch_kernel, kThreads, sizeof(Smem));
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

FwdArgs forward_scenario(const DeviceScenario& d, float threshold, float* ckpt, float* part, int part_stride) {
  FwdArgs a;
  a.V = (int)d.V;
  a.S = (int)d.S;
  a.T = (int)d.T;
  a.part_stride = part_stride;
  a.nbr = d.nbr;
  a.coefs = d.coefs;
  a.delays = d.delays;
  a.gains = d.gains;
  a.ctrl = d.ctrl;
  a.u = d.u;
  a.X = d.X;
  a.ap = d.ap;
  a.ap_last = d.ap_last;
  a.stepsum_part = part;
  a.ckpt = ckpt;
  a.ckpt_k = d.ckpt_k > 0 ? d.ckpt_k : kCkptSteps;
  a.dmin = d.dmin;
  a.threshold = threshold;
  a.status = d.status;
  a.barrier = d.barrier;
  return a;
}

cudaError_t launch_forward_batch(const FwdBatch& b, int grid, cudaStream_t stream) {
  // forward_batch_capacity (called when the batch is made) has set the shared-memory attribute
  cudaError_t err = cudaMemsetAsync(b.barrier, 0, sizeof(GridBarrier), stream);
  if (err != cudaSuccess) return err;
  FwdBatch l = b;
  void* args[] = {&l};
  return launch_cooperative((const void*)forward_batch_kernel, grid, kThreads, args, sizeof(Smem), stream);
}

int forward_ring_capacity(int device) {
  forward_grid_size(1, device);  // sets the shared-memory attributes
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, forward_ring_kernel, kThreads, sizeof(RingSmem));
  return sms * per_sm;
}

cudaError_t launch_forward(DeviceScenario& d, float threshold, float* ckpt, cudaStream_t stream) {
  FwdArgs a = forward_scenario(d, threshold, ckpt, d.stepsum_part, 0);
  cudaError_t err = cudaMemsetAsync(d.ap, 0, sizeof(float) * d.V * kGainCols, stream);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(d.ap_last, 0, sizeof(float) * d.V * kGainCols, stream);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(d.barrier, 0, sizeof(GridBarrier), stream);
  if (err != cudaSuccess) return err;
  if (d.fwd_ring) {
    RingArgs r;
    r.halo = d.halo;
    r.hslot = d.hslot;
    r.nhalo = d.nhalo;
    void* args[] = {&a, &r};
    return launch_cooperative((const void*)forward_ring_kernel, d.fwd_grid, kThreads, args, sizeof(RingSmem), stream);
  }
  void* args[] = {&a};
  return launch_cooperative((const void*)forward_stream_kernel, d.fwd_grid, kThreads, args, sizeof(Smem), stream);
}

}  // namespace ct

