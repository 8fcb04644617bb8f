// C ABI and host-side epoch driver.
//
// ct_run_epoch mirrors run_epoch (src/core/algorithm.rs:124-281): reset the
// derivatives, visit the beats in order, per beat reset the estimations and
// run prediction -> residuals -> derivation -> step metrics for all steps,
// then (per batch or per epoch) average delays -> batch derivatives ->
// APParameters::update -> batch metrics. The per-step work of one beat runs
// as five kernels over all steps (forward, H x, H^T r, derivation, metrics)
// instead of T x 15 small launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <tuple>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ct_internal.cuh"

using ct::DeviceScenario;
using ct::kGainCols;
using ct::kOffsets;

// A context lives until the caller has destroyed it and every scenario created
// on it is gone (reference count: one for the caller, one per scenario).
struct ct_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 0;
  int refs = 1;
};

struct PhaseEvents {
  int phase;
  cudaEvent_t start, stop;
};

struct ct_scn {
  ct_ctx* ctx = nullptr;
  ct_algorithm algo{};
  DeviceScenario d{};
  int64_t adam_step = 1;  // Derivatives.step, derivation.rs:100
  // TF32 product modes (index 0: CT_PREC_TF32X3, 1: CT_PREC_TF32): 0 unchecked, 1 accepted, -1 refused,
  // and the relative gradient difference the check measured
  int tf32_verdict[2] = {0, 0};
  double tf32_rel[2] = {0.0, 0.0};
  uint64_t rng = 0x9e3779b97f4a7c15ull;
  std::vector<void*> allocations;
  std::vector<int32_t> nbr_host;  // neighbour table in reference order, for validating delay writes
  std::vector<int32_t> nbr_dev;   // neighbour table in device order (adjoint reverse table)
  // Upper bound of the largest delay of a connected pair: exact after creation and delay writes,
  // +1 per update that rolls delays (roll_delays moves a delay by at most one). Sizes the
  // adjoint ring without reading the device.
  int64_t dmax_bound = 1;
  // Asynchronous read-back of the device's largest delay after an update (pinned word + event):
  // once it has landed, the bound becomes that value plus the updates enqueued since.
  int32_t* dmax_host = nullptr;
  cudaEvent_t dmax_event = nullptr;
  int64_t updates = 0;          // updates that may roll delays, enqueued so far
  int64_t updates_at_read = -1; // `updates` when the pending read-back was enqueued (-1: none)
  // bumped whenever the algorithm settings change (batches re-capture their epoch graph)
  uint64_t config_gen = 0;
  // Device voxel order: device voxel u holds reference voxel perm[u]; inv is the inverse.
  std::vector<int32_t> perm, inv;
  // launch accounting and optional per-phase CUDA-event timing
  int64_t launches = 0;
  bool profiling = false;
  double phase_ms[CT_PHASE_COUNT] = {};
  int64_t phase_launches[CT_PHASE_COUNT] = {};
  std::vector<PhaseEvents> pending;
  std::vector<cudaEvent_t> event_pool;
  // post-run pass (ct_calculate_plotting_arrays / ct_calculate_final), allocated on first use
  ct::PostBuffers post{};
  ct::PostPlan post_plan{};
  bool post_arrays = false;  // CT_FIELD_STATES_* / CT_FIELD_ACTIVATION_TIMES hold results
  // field transfers: device perm and a staging buffer of S * 78 words (voxel reordering on the device)
  int32_t* perm_dev = nullptr;
  uint32_t* xfer = nullptr;
  uint32_t* xfer_epoch = nullptr;  // [S*78 + 2*V*26] staging of ct_run_epoch_host (gains, coefs, delays)
  // ct_calculate_final: grid types and numbers [2, cells], threshold histogram, results (grown on demand)
  int64_t final_cells = 0;
  int32_t* final_grid = nullptr;
  unsigned long long* final_hist = nullptr;
  float* final_out = nullptr;
  // snapshots of the last ct_run_model_based call: snap_n stored slots of snap_cap allocated
  int64_t snap_n = 0, snap_cap = 0;
  float* snap_gains = nullptr;
  float* snap_coefs = nullptr;
  int32_t* snap_delays = nullptr;
  float* snap_X = nullptr;
  float* snap_Y = nullptr;
};

namespace {

thread_local std::string g_last_error;

int fail(int status, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

int cuda_fail(cudaError_t err, const char* what) {
  return fail(err == cudaErrorMemoryAllocation ? CT_ERR_OUT_OF_MEMORY : CT_ERR_CUDA, "%s: %s", what,
              cudaGetErrorString(err));
}

#define CT_CUDA(call, what)                    \
  do {                                         \
    cudaError_t err__ = (call);                \
    if (err__ != cudaSuccess) return cuda_fail(err__, what); \
  } while (0)

// Makes `device` current for the rest of the enclosing scope and restores the caller's current
// device when the scope ends, so that no entry point changes the calling thread's device.
struct DeviceScope {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceScope(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (prev != device) err = cudaSetDevice(device);
  }
  ~DeviceScope() {
    int now = -1;
    if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;
};
#define CT_DEVICE_SCOPE(device)           \
  DeviceScope device_scope__(device);     \
  CT_CUDA(device_scope__.err, "cudaSetDevice")

cudaEvent_t take_event(ct_scn* s) {
  if (!s->event_pool.empty()) {
    cudaEvent_t e = s->event_pool.back();
    s->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

// Runs one phase: counts its kernel launches and, when profiling, brackets it
// with CUDA events on the context stream (the stream every kernel uses).
template <typename F>
cudaError_t run_phase(ct_scn* s, int phase, int kernels, F&& body) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (s->profiling) {
    e0 = take_event(s);
    e1 = take_event(s);
    if (e0) cudaEventRecord(e0, s->ctx->stream);
  }
  cudaError_t err = body();
  s->launches += kernels;
  if (s->profiling && e0 && e1) {
    cudaEventRecord(e1, s->ctx->stream);
    s->pending.push_back({phase, e0, e1});
    s->phase_launches[phase] += kernels;
  }
  return err;
}

template <typename T>
int alloc(ct_scn* s, T** p, int64_t count) {
  void* ptr = nullptr;
  const size_t bytes = sizeof(T) * (size_t)(count > 0 ? count : 1);
  cudaError_t err = cudaMalloc(&ptr, bytes);
  if (err != cudaSuccess) return cuda_fail(err, "cudaMalloc");
  s->allocations.push_back(ptr);
  *p = static_cast<T*>(ptr);
  return CT_OK;
}

int upload(ct_scn* s, void* dst, const void* src, size_t bytes) {
  CT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->ctx->stream), "upload");
  return CT_OK;
}

int check_algo(const ct_algorithm* a) {
  if (!a) return fail(CT_ERR_INVALID_ARGUMENT, "algorithm is NULL");
  if (a->optimizer != CT_OPT_SGD && a->optimizer != CT_OPT_ADAM)
    return fail(CT_ERR_INVALID_ARGUMENT, "unknown optimizer %d", a->optimizer);
  if (a->ap_derivative != CT_AP_SIMPLE && a->ap_derivative != CT_AP_TEXTBOOK)
    return fail(CT_ERR_INVALID_ARGUMENT, "unknown ap_derivative %d", a->ap_derivative);
  if (a->batch_size < 0) return fail(CT_ERR_INVALID_ARGUMENT, "negative batch_size");
  return CT_OK;
}

// Shuffle of the beat indices when the caller passes no order (the reference
// shuffles with an unseeded generator, algorithm.rs:139-141).
void seeded_shuffle(ct_scn* s, std::vector<int32_t>& order) {
  for (size_t i = order.size(); i > 1; --i) {
    s->rng ^= s->rng << 13;
    s->rng ^= s->rng >> 7;
    s->rng ^= s->rng << 17;
    const size_t j = (size_t)(s->rng % i);
    std::swap(order[i - 1], order[j]);
  }
}

int64_t max_connected_delay(const std::vector<int32_t>& nbr, const int32_t* delays) {
  int64_t m = 1;
  for (size_t i = 0; i < nbr.size(); ++i)
    if (nbr[i] >= 0 && delays[i] > m) m = delays[i];
  return m;
}

void release(ct_scn* s, void* p) {
  if (!p) return;
  cudaFree(p);
  s->allocations.erase(std::remove(s->allocations.begin(), s->allocations.end(), p), s->allocations.end());
}

// After an update that may roll delays: count it and enqueue the read-back of the largest delay.
void note_delay_update(ct_scn* s, cudaStream_t st) {
  s->updates += 1;
  s->dmax_bound = std::min<int64_t>(s->dmax_bound + 1, 1000);
  if (!s->dmax_host) {
    void* p = nullptr;
    if (cudaMallocHost(&p, sizeof(int32_t)) != cudaSuccess) return;
    if (cudaEventCreateWithFlags(&s->dmax_event, cudaEventDisableTiming) != cudaSuccess) {
      cudaFreeHost(p);
      return;
    }
    s->dmax_host = static_cast<int32_t*>(p);
  }
  if (s->updates_at_read >= 0 && cudaEventQuery(s->dmax_event) != cudaSuccess) return;  // one in flight
  if (cudaMemcpyAsync(s->dmax_host, s->d.dmin + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaEventRecord(s->dmax_event, st) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  s->updates_at_read = s->updates;
}

// Tightens dmax_bound with a read-back that has landed.
void refresh_delay_bound(ct_scn* s) {
  if (s->updates_at_read < 0 || cudaEventQuery(s->dmax_event) != cudaSuccess) return;
  const int64_t bound = std::max<int64_t>(1, *s->dmax_host) + (s->updates - s->updates_at_read);
  s->dmax_bound = std::min<int64_t>(s->dmax_bound, bound);
  s->updates_at_read = -1;
}

bool valid_precision(int p) {
  return p == CT_PREC_FP32 || p == CT_PREC_TF32X3 || p == CT_PREC_TF32 || p == CT_PREC_BF16X6;
}

// Sliced BF16 operands (ct_slice.cu): buffers allocated on first use, H and H^T sliced once per
// measurement matrix. Synchronous when it slices (the temporary buffer of the transpose).
int prepare_sliced(ct_scn* s) {
  DeviceScenario& d = s->d;
  cudaStream_t st = s->ctx->stream;
  if (!d.H_sl) {
    const int64_t sp = ct::slice_pitch(d.S), kpm = ct::slice_pitch(d.M);
    const int64_t ngs = ct::slice_groups(d.S), ngm = ct::slice_groups(d.M);
    int rc = alloc(s, &d.H_sl, d.B * 3 * d.M * sp);
    if (!rc) rc = alloc(s, &d.H_sc, d.B * ngs * d.M);
    if (!rc) rc = alloc(s, &d.Ht_sl, d.B * 3 * d.S * kpm);
    if (!rc) rc = alloc(s, &d.Ht_sc, d.B * ngm * d.S);
    if (!rc) rc = alloc(s, &d.X_sl, 3 * d.T * sp);
    if (!rc) rc = alloc(s, &d.X_sc, d.T * ngs);
    if (!rc) rc = alloc(s, &d.R_sl, 3 * d.T * kpm);
    if (!rc) rc = alloc(s, &d.R_sc, d.T * ngm);
    if (rc) {
      for (void* p : {(void*)d.H_sl, (void*)d.H_sc, (void*)d.Ht_sl, (void*)d.Ht_sc, (void*)d.X_sl, (void*)d.X_sc,
                      (void*)d.R_sl, (void*)d.R_sc})
        release(s, p);
      d.H_sl = d.Ht_sl = d.X_sl = d.R_sl = nullptr;
      d.H_sc = d.Ht_sc = d.X_sc = d.R_sc = nullptr;
      return rc;
    }
    d.slice_ready = false;
  }
  if (!d.slice_ready) {
    CT_CUDA(ct::slice_prepare(d, st), "slicing the measurement matrix");
    CT_CUDA(cudaStreamSynchronize(st), "slicing the measurement matrix");
    s->launches += 3 * d.B;
    d.slice_ready = true;
  }
  return CT_OK;
}

// Adjoint-mode buffers, allocated on first use (or when the checkpoint interval k changes); the
// inbox ring grows with the delay bound.
int prepare_adjoint(ct_scn* s, int k = ct::kCkptSteps) {
  DeviceScenario& d = s->d;
  cudaStream_t st = s->ctx->stream;
  const int64_t V = d.V, plane = d.V * kGainCols;
  if (d.rev && d.ckpt_k != k) {  // re-made below with the new interval
    CT_CUDA(cudaStreamSynchronize(st), "adjoint re-layout");
    for (void* p : {(void*)d.rev, (void*)d.ckpt, (void*)d.seg_q}) release(s, p);
    d.rev = nullptr;
    d.ckpt = d.seg_q = nullptr;
  }
  if (!d.rev) {
    std::vector<int32_t> rev((size_t)(V * kOffsets), -1);
    for (int64_t v = 0; v < V; ++v)
      for (int n = 0; n < kOffsets; ++n) {
        const int32_t j = s->nbr_dev[(size_t)(v * kOffsets + n)];
        if (j < 0) continue;
        int32_t& slot = rev[(size_t)j * kOffsets + n];
        if (slot >= 0)
          return fail(CT_ERR_NOT_SUPPORTED,
                      "adjoint mode: two voxels reach the same neighbour along one offset (not a lattice)");
        slot = (int32_t)v;
      }
    const int64_t nseg = (d.T + k - 1) / k;
    const int64_t seg_steps = std::min<int64_t>(d.T, k);
    d.adj_pitch = (int)(((plane + 3) / 4) * 4);
    d.ckpt_k = k;
    int rc = alloc(s, &d.rev, V * kOffsets);
    if (!rc) rc = alloc(s, &d.ckpt, nseg * plane);
    if (!rc) rc = alloc(s, &d.seg_q, seg_steps * d.adj_pitch);
    if (!rc && !d.dCk) rc = alloc(s, &d.dCk, plane);
    if (rc) {
      for (void* p : {(void*)d.rev, (void*)d.ckpt, (void*)d.seg_q}) release(s, p);
      d.rev = nullptr;
      d.ckpt = d.seg_q = nullptr;
      return rc;
    }
    CT_CUDA(cudaMemcpyAsync(d.rev, rev.data(), sizeof(int32_t) * rev.size(), cudaMemcpyHostToDevice, st),
            "upload reverse table");
    CT_CUDA(cudaMemsetAsync(d.ckpt, 0, sizeof(float) * nseg * plane, st), "memset");
    CT_CUDA(cudaMemsetAsync(d.dCk, 0, sizeof(float) * plane, st), "memset");
    CT_CUDA(cudaStreamSynchronize(st), "adjoint set-up");
    d.adj_grid = (int)std::min<int64_t>((V + ct::kFwdTileVoxels - 1) / ct::kFwdTileVoxels,
                                        ct::adjoint_capacity(s->ctx->device));
  }
  if (!d.lam_state) {
    int rc = alloc(s, &d.lam_state, plane + 4);  // +4: the adjoint's bulk copies round sizes up to 16 bytes
    if (rc) return rc;
  }
  refresh_delay_bound(s);
  int need = 1;
  while (need < s->dmax_bound + ct::kMaxStepBlock + 2) need <<= 1;
  if (!d.inbox || d.adj_ring < need) {
    CT_CUDA(cudaStreamSynchronize(st), "adjoint inbox");
    release(s, d.inbox);
    d.inbox = nullptr;
    d.adj_ring = 0;
    int rc = alloc(s, &d.inbox, (int64_t)need * d.adj_pitch);
    if (rc) return rc;
    d.adj_ring = need;
  }
  return CT_OK;
}

int run_beat(ct_scn* s, int64_t beat, int precision, int grad_mode) {
  DeviceScenario& d = s->d;
  const ct_algorithm& a = s->algo;
  cudaStream_t st = s->ctx->stream;
  const bool adjoint = grad_mode == CT_GRAD_ADJOINT;
  CT_CUDA(run_phase(s, CT_PHASE_FORWARD, 1,
                    [&] {
                      return ct::launch_forward(d, a.maximum_regularization_threshold, adjoint ? d.ckpt : nullptr,
                                                st);
                    }),
          "forward kernel");
  if (precision == CT_PREC_FP32) {
    CT_CUDA(run_phase(s, CT_PHASE_MEASURE, 3, [&] { return ct::launch_measure(d, beat, true, st); }),
            "measurement kernel");
    CT_CUDA(run_phase(s, CT_PHASE_MAP_RESIDUALS, 1, [&] { return ct::launch_map_residuals(d, beat, st); }),
            "mapped-residual kernel");
  } else if (precision == CT_PREC_BF16X6) {
    CT_CUDA(run_phase(s, CT_PHASE_MEASURE, 4, [&] { return ct::launch_measure_sliced(d, beat, true, st); }),
            "sliced tensor-core measurement kernel");
    CT_CUDA(run_phase(s, CT_PHASE_MAP_RESIDUALS, 2, [&] { return ct::launch_map_residuals_sliced(d, beat, st); }),
            "sliced tensor-core mapped-residual kernel");
  } else {
    CT_CUDA(run_phase(s, CT_PHASE_MEASURE, 3,
                      [&] { return ct::launch_measure_umma(d, beat, true, precision, st); }),
            "tensor-core measurement kernel");
    CT_CUDA(run_phase(s, CT_PHASE_MAP_RESIDUALS, 1,
                      [&] { return ct::launch_map_residuals_umma(d, beat, precision, st); }),
            "tensor-core mapped-residual kernel");
  }
  if (adjoint && (!a.freeze_gains || !a.freeze_delays)) {
    ct::AdjointScalars as;
    as.mse_scaling = 1.0f / (float)d.M * a.mse_strength;
    as.reg_scaling = a.maximum_regularization_strength;
    as.threshold = a.maximum_regularization_threshold;
    as.diffreg = a.difference_regularization_strength;
    as.freeze_gains = a.freeze_gains;
    as.freeze_delays = a.freeze_delays;
    as.ap_derivative = a.ap_derivative;
    CT_CUDA(run_phase(s, CT_PHASE_DERIVE, 1, [&] { return ct::launch_adjoint(d, as, st); }), "adjoint kernel");
  } else if (!a.freeze_gains || !a.freeze_delays) {
    ct::DeriveScalars ds;
    ds.mse_scaling = 1.0f / (float)d.M * a.mse_strength;
    ds.reg_scaling = a.maximum_regularization_strength;
    ds.threshold = a.maximum_regularization_threshold;
    ds.diffreg = a.difference_regularization_strength;
    ds.freeze_gains = a.freeze_gains;
    ds.freeze_delays = a.freeze_delays;
    ds.ap_derivative = a.ap_derivative;
    CT_CUDA(run_phase(s, CT_PHASE_DERIVE, 1, [&] { return ct::launch_derive(d, ds, st); }), "derivation kernel");
  }
  CT_CUDA(run_phase(s, CT_PHASE_STEP_METRICS, 2,
                    [&] { return ct::launch_step_metrics(d, a.maximum_regularization_strength, st); }),
          "step metrics kernel");
  return CT_OK;
}

int derivatives_reset(ct_scn* s) {
  DeviceScenario& d = s->d;
  cudaStream_t st = s->ctx->stream;
  CT_CUDA(cudaMemsetAsync(d.dG, 0, sizeof(float) * d.S * kGainCols, st), "reset");
  CT_CUDA(cudaMemsetAsync(d.dC, 0, sizeof(float) * d.V * kOffsets, st), "reset");
  CT_CUDA(cudaMemsetAsync(d.fir, 0, sizeof(float) * d.V * kGainCols, st), "reset");
  CT_CUDA(cudaMemsetAsync(d.iir, 0, sizeof(float) * d.V * kGainCols, st), "reset");
  CT_CUDA(cudaMemsetAsync(d.mreg_sum, 0, sizeof(float), st), "reset");
  return CT_OK;
}

// calculate_average_delays -> calculate_batch_derivatives -> update -> calculate_batch
int batch_end(ct_scn* s, int64_t n_beats, int64_t* batch_index) {
  DeviceScenario& d = s->d;
  const ct_algorithm& a = s->algo;
  cudaStream_t st = s->ctx->stream;
  if (*batch_index < 0 || *batch_index >= d.NB)
    return fail(CT_ERR_BATCH_INDEX, "batch index %lld outside the %lld batch-wise metric slots",
                (long long)*batch_index, (long long)d.NB);
  const bool smooth = !a.freeze_delays && std::fabs(a.smoothness_regularization_strength) > 1.1920929e-7f;
  const int kernels = 1 + (smooth ? 1 : 0) + (a.freeze_gains ? 0 : 1) + (a.freeze_delays ? 0 : 4) + 1;
  cudaError_t err = run_phase(s, CT_PHASE_UPDATE, kernels, [&]() -> cudaError_t {
  cudaError_t e = ct::launch_average_delays(d, st);
  if (e != cudaSuccess) return e;
  if (smooth) {
    e = ct::launch_smoothness(d, a.smoothness_regularization_strength, st);
    if (e != cudaSuccess) return e;
  }
  const int64_t bs = (a.batch_size == 0) ? d.T * n_beats : d.T * a.batch_size;
  ct::UpdateScalars u;
  u.optimizer = a.optimizer;
  u.freeze_gains = a.freeze_gains;
  u.freeze_delays = a.freeze_delays;
  u.lr_over_bs = a.learning_rate / (float)bs;
  // update.rs:140-141: 1 - beta^step with f32 powf
  u.bias1 = 1.0f - powf(0.9f, (float)s->adam_step);
  u.bias2 = 1.0f - powf(0.999f, (float)s->adam_step);
  e = ct::launch_update(d, u, st);
  if (e != cudaSuccess) return e;
  if (!a.freeze_delays) {
    e = ct::launch_min_delay(d, st);
    if (e != cudaSuccess) return e;
  }
  return ct::launch_batch_metrics(d, *batch_index, st);
  });
  if (err != cudaSuccess) return cuda_fail(err, "update kernels");
  if (!a.freeze_delays) note_delay_update(s, st);
  s->adam_step += 1;
  *batch_index += 1;
  return CT_OK;
}

// ---- device voxel order --------------------------------------------------------------
//
// Kernels see the voxels in spatially compact 4x4x2 bricks, so the 26
// neighbours of a tile of consecutive device voxels are few and close, and
// their state history is reused from L1. Integer grid coordinates are
// recovered from the neighbour table (offset index n <-> (dx, dy, dz), the
// ordering of delay_index_to_offset, allpass.rs:597-611) by a breadth-first
// walk; each connected component is laid out on its own. Any permutation is
// correct (every per-state operation and its order is unchanged); the bricks
// only improve locality. Arrays cross the ABI in reference order.

const int kOffsetXYZ[kOffsets][3] = {
    {-1, -1, -1}, {-1, -1, 0}, {-1, -1, 1}, {-1, 0, -1}, {-1, 0, 0}, {-1, 0, 1}, {-1, 1, -1},
    {-1, 1, 0},   {-1, 1, 1},  {0, -1, -1}, {0, -1, 0},  {0, -1, 1}, {0, 0, -1},  {0, 0, 1},
    {0, 1, -1},   {0, 1, 0},   {0, 1, 1},   {1, -1, -1}, {1, -1, 0}, {1, -1, 1},  {1, 0, -1},
    {1, 0, 0},    {1, 0, 1},   {1, 1, -1},  {1, 1, 0},   {1, 1, 1}};

void brick_layout(const std::vector<int32_t>& nbr, int64_t V, std::vector<int32_t>& perm,
                  std::vector<int32_t>& inv) {
  std::vector<int64_t> cx((size_t)V), cy((size_t)V), cz((size_t)V), comp((size_t)V, -1);
  std::vector<int32_t> queue;
  queue.reserve((size_t)V);
  int64_t ncomp = 0;
  for (int64_t root = 0; root < V; ++root) {
    if (comp[(size_t)root] >= 0) continue;
    queue.clear();
    queue.push_back((int32_t)root);
    comp[(size_t)root] = ncomp;
    cx[(size_t)root] = cy[(size_t)root] = cz[(size_t)root] = 0;
    for (size_t qi = 0; qi < queue.size(); ++qi) {
      const int32_t u = queue[qi];
      for (int n = 0; n < kOffsets; ++n) {
        const int32_t w = nbr[(size_t)u * kOffsets + n];
        if (w < 0 || comp[(size_t)w] >= 0) continue;
        comp[(size_t)w] = ncomp;
        cx[(size_t)w] = cx[(size_t)u] + kOffsetXYZ[n][0];
        cy[(size_t)w] = cy[(size_t)u] + kOffsetXYZ[n][1];
        cz[(size_t)w] = cz[(size_t)u] + kOffsetXYZ[n][2];
        queue.push_back(w);
      }
    }
    // shift the component to non-negative coordinates
    int64_t mx = 0, my = 0, mz = 0;
    for (int32_t u : queue) {
      mx = std::min(mx, cx[(size_t)u]);
      my = std::min(my, cy[(size_t)u]);
      mz = std::min(mz, cz[(size_t)u]);
    }
    for (int32_t u : queue) {
      cx[(size_t)u] -= mx;
      cy[(size_t)u] -= my;
      cz[(size_t)u] -= mz;
    }
    ++ncomp;
  }
  perm.resize((size_t)V);
  for (int64_t v = 0; v < V; ++v) perm[(size_t)v] = (int32_t)v;
  auto key = [&](int32_t v) {
    return std::make_tuple(comp[(size_t)v], cx[(size_t)v] / 4, cy[(size_t)v] / 4, cz[(size_t)v] / 2,
                           cx[(size_t)v], cy[(size_t)v], cz[(size_t)v], v);
  };
  std::sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) { return key(a) < key(b); });
  inv.resize((size_t)V);
  for (int64_t u = 0; u < V; ++u) inv[(size_t)perm[(size_t)u]] = (int32_t)u;
}

// Row blocks of `rows_per_voxel` rows of `row_len` elements: device block u <- reference block perm[u].
template <typename T>
void gather_rows(T* dst, const T* src, const std::vector<int32_t>& perm, int64_t rows_per_voxel, int64_t row_len) {
  const size_t blk = (size_t)(rows_per_voxel * row_len);
  for (size_t u = 0; u < perm.size(); ++u) std::memcpy(dst + u * blk, src + (size_t)perm[u] * blk, sizeof(T) * blk);
}
// Inverse of gather_rows: reference block perm[u] <- device block u.
template <typename T>
void scatter_rows(T* dst, const T* src, const std::vector<int32_t>& perm, int64_t rows_per_voxel, int64_t row_len) {
  const size_t blk = (size_t)(rows_per_voxel * row_len);
  for (size_t u = 0; u < perm.size(); ++u) std::memcpy(dst + (size_t)perm[u] * blk, src + u * blk, sizeof(T) * blk);
}
// Columns of `rows` rows of S = 3V states: device state 3u+a <- reference state 3perm[u]+a.
void gather_state_columns(float* dst, const float* src, const std::vector<int32_t>& perm, int64_t rows) {
  const size_t S = 3 * perm.size();
  for (int64_t r = 0; r < rows; ++r) {
    const float* sr = src + (size_t)r * S;
    float* dr = dst + (size_t)r * S;
    for (size_t u = 0; u < perm.size(); ++u) {
      const size_t v = (size_t)perm[u];
      dr[3 * u] = sr[3 * v];
      dr[3 * u + 1] = sr[3 * v + 1];
      dr[3 * u + 2] = sr[3 * v + 2];
    }
  }
}
void scatter_state_columns(float* dst, const float* src, const std::vector<int32_t>& perm, int64_t rows) {
  const size_t S = 3 * perm.size();
  for (int64_t r = 0; r < rows; ++r) {
    const float* sr = src + (size_t)r * S;
    float* dr = dst + (size_t)r * S;
    for (size_t u = 0; u < perm.size(); ++u) {
      const size_t v = (size_t)perm[u];
      dr[3 * v] = sr[3 * u];
      dr[3 * v + 1] = sr[3 * u + 1];
      dr[3 * v + 2] = sr[3 * u + 2];
    }
  }
}

// Per forward tile (kFwdTileVoxels consecutive device voxels): the sorted device voxels its
// (voxel, offset) items read, and each item's slot in that list. False if a neighbourhood
// exceeds kFwdHaloMax (the resident forward form is then not used).
bool build_halos(const ct_scn* s, const std::vector<int32_t>& nbr_ref, int64_t tiles, std::vector<int32_t>& halo,
                 std::vector<int32_t>& nhalo, std::vector<int16_t>& hslot) {
  const int TV = ct::kFwdTileVoxels, HM = ct::kFwdHaloMax;
  const int64_t V = (int64_t)s->perm.size();
  halo.assign((size_t)(tiles * HM), -1);
  nhalo.assign((size_t)tiles, 0);
  hslot.assign((size_t)(tiles * TV * kOffsets), -1);
  std::vector<int32_t> list;
  for (int64_t t = 0; t < tiles; ++t) {
    list.clear();
    for (int vl = 0; vl < TV; ++vl) {
      const int64_t u = t * TV + vl;
      if (u >= V) break;
      for (int n = 0; n < kOffsets; ++n) {
        const int32_t w = nbr_ref[(size_t)s->perm[(size_t)u] * kOffsets + n];
        if (w >= 0) list.push_back(s->inv[(size_t)w]);
      }
    }
    std::sort(list.begin(), list.end());
    list.erase(std::unique(list.begin(), list.end()), list.end());
    if ((int)list.size() > HM) return false;
    nhalo[(size_t)t] = (int32_t)list.size();
    std::copy(list.begin(), list.end(), halo.begin() + (size_t)(t * HM));
    for (int vl = 0; vl < TV; ++vl) {
      const int64_t u = t * TV + vl;
      if (u >= V) break;
      for (int n = 0; n < kOffsets; ++n) {
        const int32_t w = nbr_ref[(size_t)s->perm[(size_t)u] * kOffsets + n];
        if (w < 0) continue;
        const int32_t dw = s->inv[(size_t)w];
        hslot[(size_t)((t * TV + vl) * kOffsets + n)] =
            (int16_t)(std::lower_bound(list.begin(), list.end(), dw) - list.begin());
      }
    }
  }
  return true;
}

int validate_and_build_nbr(const ct_scenario_desc* desc, std::vector<int32_t>& nbr) {
  const int64_t S = desc->num_states, V = S / 3;
  nbr.assign((size_t)(V * kOffsets), -1);
  const int32_t* osi = desc->output_state_indices;
  for (int64_t v = 0; v < V; ++v) {
    for (int n = 0; n < kOffsets; ++n) {
      const int32_t first = osi[(3 * v) * kGainCols + 3 * n];
      int32_t nb = -1;
      if (first >= 0) {
        if (first % 3 != 0 || first / 3 >= V)
          return fail(CT_ERR_INVALID_INDEX, "output_state_indices[%lld,%d] = %d is not a voxel's first state",
                      (long long)(3 * v), 3 * n, first);
        nb = first / 3;
      }
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          const int32_t got = osi[(3 * v + a) * kGainCols + 3 * n + b];
          const int32_t want = nb < 0 ? -1 : 3 * nb + b;
          if ((got < 0 ? -1 : got) != want)
            return fail(CT_ERR_INVALID_INDEX,
                        "output_state_indices[%lld,%d] = %d breaks the (voxel, offset, component) structure",
                        (long long)(3 * v + a), 3 * n + b, got);
        }
      nbr[(size_t)(v * kOffsets + n)] = nb;
      if (nb >= 0 && desc->delays[v * kOffsets + n] < 1)
        return fail(CT_ERR_INVALID_ARGUMENT, "delay of connected pair (%lld,%d) is %d; delays must be >= 1",
                    (long long)v, n, desc->delays[v * kOffsets + n]);
    }
  }
  return CT_OK;
}

void free_scenario(ct_scn* s) {
  for (void* p : s->allocations) cudaFree(p);
  s->allocations.clear();
  for (auto& pe : s->pending) {
    cudaEventDestroy(pe.start);
    cudaEventDestroy(pe.stop);
  }
  s->pending.clear();
  for (cudaEvent_t e : s->event_pool) cudaEventDestroy(e);
  s->event_pool.clear();
  if (s->dmax_host) cudaFreeHost(s->dmax_host);
  if (s->dmax_event) cudaEventDestroy(s->dmax_event);
  s->dmax_host = nullptr;
  s->dmax_event = nullptr;
}

int field_bytes(const ct_scn* s, int field, size_t* nbytes) {
  const DeviceScenario& d = s->d;
  const size_t f = sizeof(float);
  switch (field) {
    case CT_FIELD_GAINS:
    case CT_FIELD_AP_OUTPUTS_NOW:
    case CT_FIELD_AP_OUTPUTS_LAST:
    case CT_FIELD_GRAD_GAINS:
    case CT_FIELD_COEFS_FIR:
    case CT_FIELD_COEFS_IIR:
    case CT_FIELD_GAINS_FIRST_MOMENT:
    case CT_FIELD_GAINS_SECOND_MOMENT: *nbytes = f * d.S * kGainCols; return CT_OK;
    case CT_FIELD_COEFS:
    case CT_FIELD_GRAD_COEFS:
    case CT_FIELD_COEFS_FIRST_MOMENT:
    case CT_FIELD_COEFS_SECOND_MOMENT: *nbytes = f * d.V * kOffsets; return CT_OK;
    case CT_FIELD_DELAYS: *nbytes = sizeof(int32_t) * d.V * kOffsets; return CT_OK;
    case CT_FIELD_MEASUREMENTS_ACTUAL:
    case CT_FIELD_MEASUREMENTS: *nbytes = f * d.B * d.T * d.M; return CT_OK;
    case CT_FIELD_SYSTEM_STATES:
    case CT_FIELD_MAPPED_RESIDUALS_HISTORY: *nbytes = f * d.T * d.S; return CT_OK;
    case CT_FIELD_RESIDUALS: *nbytes = f * d.M; return CT_OK;
    case CT_FIELD_AVERAGE_DELAYS: *nbytes = f * d.V; return CT_OK;
    case CT_FIELD_MAPPED_RESIDUALS:
    case CT_FIELD_MAXIMUM_REGULARIZATION: *nbytes = f * d.S; return CT_OK;
    case CT_FIELD_MAXIMUM_REGULARIZATION_SUM: *nbytes = f; return CT_OK;
    case CT_FIELD_ADAM_STEP: *nbytes = sizeof(int64_t); return CT_OK;
    case CT_FIELD_LOSS:
    case CT_FIELD_LOSS_MSE:
    case CT_FIELD_LOSS_MAXIMUM_REGULARIZATION: *nbytes = f * d.T; return CT_OK;
    case CT_FIELD_LOSS_BATCH:
    case CT_FIELD_LOSS_MSE_BATCH:
    case CT_FIELD_LOSS_MAXIMUM_REGULARIZATION_BATCH: *nbytes = f * d.NB; return CT_OK;
    case CT_FIELD_STATES_MAGNITUDE:
    case CT_FIELD_STATES_THETA:
    case CT_FIELD_STATES_PHI: *nbytes = f * d.T * d.V; return CT_OK;
    case CT_FIELD_STATES_MAGNITUDE_MAX:
    case CT_FIELD_STATES_THETA_MAX:
    case CT_FIELD_STATES_PHI_MAX:
    case CT_FIELD_ACTIVATION_TIMES: *nbytes = f * d.V; return CT_OK;
    case CT_FIELD_SNAPSHOT_GAINS: *nbytes = f * s->snap_n * d.S * kGainCols; return CT_OK;
    case CT_FIELD_SNAPSHOT_COEFS: *nbytes = f * s->snap_n * d.V * kOffsets; return CT_OK;
    case CT_FIELD_SNAPSHOT_DELAYS: *nbytes = sizeof(int32_t) * s->snap_n * d.V * kOffsets; return CT_OK;
    case CT_FIELD_SNAPSHOT_SYSTEM_STATES: *nbytes = f * s->snap_n * d.T * d.S; return CT_OK;
    case CT_FIELD_SNAPSHOT_MEASUREMENTS: *nbytes = f * s->snap_n * d.B * d.T * d.M; return CT_OK;
    default: return fail(CT_ERR_INVALID_ARGUMENT, "unknown field %d", field);
  }
}

int copy_down(ct_scn* s, void* dst, const void* src, size_t bytes) {
  CT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->ctx->stream), "read field");
  CT_CUDA(cudaStreamSynchronize(s->ctx->stream), "read field");
  return CT_OK;
}

// [V,78] device order -> [S,78] reference order (row component replicated)
int copy_down_expanded(ct_scn* s, float* dst, const float* src) {
  const int64_t V = s->d.V;
  std::vector<float> tmp((size_t)(V * kGainCols));
  int rc = copy_down(s, tmp.data(), src, sizeof(float) * tmp.size());
  if (rc) return rc;
  for (int64_t u = 0; u < V; ++u) {
    const int64_t v = s->perm[(size_t)u];
    for (int a = 0; a < 3; ++a)
      std::memcpy(dst + (3 * v + a) * kGainCols, tmp.data() + u * kGainCols, sizeof(float) * kGainCols);
  }
  return CT_OK;
}

template <typename T>
int copy_down_rows_host(ct_scn* s, T* dst, const T* src, int64_t rows_per_voxel, int64_t row_len) {
  std::vector<T> tmp((size_t)(s->d.V * rows_per_voxel * row_len));
  int rc = copy_down(s, tmp.data(), src, sizeof(T) * tmp.size());
  if (rc) return rc;
  scatter_rows(dst, tmp.data(), s->perm, rows_per_voxel, row_len);
  return CT_OK;
}

// Staging buffer and device perm for reordering transfers on the device (allocated on first use).
int ensure_xfer(ct_scn* s) {
  if (s->xfer) return CT_OK;
  int rc = alloc(s, &s->perm_dev, s->d.V);
  if (!rc) rc = upload(s, s->perm_dev, s->perm.data(), sizeof(int32_t) * s->perm.size());
  if (!rc) rc = alloc(s, &s->xfer, s->d.S * kGainCols);
  if (rc) {
    release(s, s->perm_dev);
    release(s, s->xfer);
    s->perm_dev = nullptr;
    s->xfer = nullptr;
  }
  return rc;
}

// Per-voxel row blocks (rows_per_voxel x row_len elements) in device order -> reference order:
// scattered on the device into the staging buffer, then one copy to the host.
template <typename T>
int copy_down_rows(ct_scn* s, T* dst, const T* src, int64_t rows_per_voxel, int64_t row_len) {
  static_assert(sizeof(T) == 4, "32-bit elements");
  if (rows_per_voxel * row_len <= kGainCols * 3 && ensure_xfer(s) == CT_OK) {
    const int64_t words = rows_per_voxel * row_len;
    CT_CUDA(ct::launch_permute_blocks(src, s->xfer, s->perm_dev, s->d.V, words, false, s->ctx->stream),
            "permute kernel");
    return copy_down(s, dst, s->xfer, sizeof(T) * (size_t)(s->d.V * words));
  }
  return copy_down_rows_host(s, dst, src, rows_per_voxel, row_len);
}

// `rows` rows of S states in device order -> reference order.
int copy_down_state_columns(ct_scn* s, float* dst, const float* src, int64_t rows) {
  std::vector<float> tmp((size_t)(rows * s->d.S));
  int rc = copy_down(s, tmp.data(), src, sizeof(float) * tmp.size());
  if (rc) return rc;
  scatter_state_columns(dst, tmp.data(), s->perm, rows);
  return CT_OK;
}

}  // namespace

namespace ct {
int report_error(int status, const char* message) { return fail(status, "%s", message); }
}  // namespace ct

extern "C" {

int ct_version(void) { return CT_ABI_VERSION; }

const char* ct_status_string(int status) {
  switch (status) {
    case CT_OK: return "ok";
    case CT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CT_ERR_CUDA: return "CUDA error";
    case CT_ERR_OUT_OF_MEMORY: return "out of device memory";
    case CT_ERR_TIMEOUT: return "device-side wait timed out";
    case CT_ERR_INVALID_INDEX: return "output_state_indices lack the voxel/neighbour structure";
    case CT_ERR_NOT_SUPPORTED: return "not supported";
    case CT_ERR_BATCH_INDEX: return "batch index outside the metric arrays";
    case CT_ERR_NO_MAXIMUM: return "a voxel's magnitude is NaN at every step";
    default: return "unknown status";
  }
}

int ct_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return CT_ERR_INVALID_ARGUMENT;
  std::snprintf(buf, len, "%s", g_last_error.c_str());
  return CT_OK;
}

int ct_ctx_create(int device, void* stream, ct_ctx** out) {
  if (!out) return fail(CT_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  int count = 0;
  CT_CUDA(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
  if (device < 0 || device >= count) return fail(CT_ERR_INVALID_ARGUMENT, "device %d of %d", device, count);
  CT_DEVICE_SCOPE(device);
  ct_ctx* c = new ct_ctx;
  c->device = device;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (stream) {
    c->stream = static_cast<cudaStream_t>(stream);
  } else {
    cudaError_t err = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
      delete c;
      return cuda_fail(err, "cudaStreamCreate");
    }
    c->own_stream = true;
  }
  *out = c;
  return CT_OK;
}

namespace {
void ctx_release(ct_ctx* ctx) {
  if (--ctx->refs > 0) return;
  DeviceScope device_scope__(ctx->device);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}
}  // namespace

int ct_ctx_destroy(ct_ctx* ctx) {
  if (!ctx) return CT_OK;
  ctx_release(ctx);
  return CT_OK;
}

int ct_ctx_stream(ct_ctx* ctx, void** stream) {
  if (!ctx || !stream) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  *stream = ctx->stream;
  return CT_OK;
}

int ct_scenario_create(ct_ctx* ctx, const ct_scenario_desc* desc, const ct_algorithm* algo, ct_scn** out) {
  if (!ctx || !desc || !out) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  int rc = check_algo(algo);
  if (rc) return rc;
  const int64_t S = desc->num_states, M = desc->num_sensors, T = desc->num_steps, B = desc->num_beats;
  if (S <= 0 || S % 3 != 0) return fail(CT_ERR_INVALID_ARGUMENT, "num_states %lld must be a positive multiple of 3", (long long)S);
  if (M <= 0 || T <= 0 || B <= 0) return fail(CT_ERR_INVALID_ARGUMENT, "num_sensors, num_steps and num_beats must be positive");
  if (desc->num_batch_slots <= 0) return fail(CT_ERR_INVALID_ARGUMENT, "num_batch_slots must be positive");
  if (T * S >= (int64_t(1) << 31) || S * kGainCols >= (int64_t(1) << 31) || B * M * S >= (int64_t(1) << 40))
    return fail(CT_ERR_NOT_SUPPORTED, "num_steps x num_states must stay below 2^31 (32-bit state indexing)");
  if (!desc->gains || !desc->output_state_indices || !desc->coefs || !desc->delays || !desc->initial_delays ||
      !desc->control_matrix || !desc->control_function)
    return fail(CT_ERR_INVALID_ARGUMENT, "a required array pointer is NULL");
  std::vector<int32_t> nbr;
  rc = validate_and_build_nbr(desc, nbr);
  if (rc) return rc;
  CT_DEVICE_SCOPE(ctx->device);

  ct_scn* s = new ct_scn;
  s->ctx = ctx;
  s->algo = *algo;
  s->nbr_host = nbr;
  s->dmax_bound = max_connected_delay(nbr, desc->delays);
  brick_layout(nbr, S / 3, s->perm, s->inv);
  DeviceScenario& d = s->d;
  d.S = S;
  d.V = S / 3;
  d.M = M;
  d.T = T;
  d.B = B;
  d.NB = desc->num_batch_slots;
  // forward form: resident (one tile per CTA, halo ring) when every tile fits a co-resident CTA
  // and every tile's neighbourhood fits the ring; streaming otherwise
  const int64_t tiles = (d.V + ct::kFwdTileVoxels - 1) / ct::kFwdTileVoxels;
  std::vector<int32_t> h_halo, h_nhalo;
  std::vector<int16_t> h_hslot;
  d.fwd_ring = tiles <= ct::forward_ring_capacity(ctx->device) &&
               build_halos(s, nbr, tiles, h_halo, h_nhalo, h_hslot);
  d.fwd_grid = d.fwd_ring ? (int)tiles : ct::forward_grid_size(d.V, ctx->device);
  {
    const int64_t tiles = ((M + 63) / 64) * ((T + 63) / 64);
    int64_t ks = (2 * ctx->num_sms + tiles - 1) / tiles;
    ks = std::min<int64_t>(ks, std::max<int64_t>(1, S / 256));
    d.ksplit = (int)std::max<int64_t>(1, std::min<int64_t>(ks, 64));
  }
  d.umma = ct::umma_supported(M);
  d.spad = (S + 3) / 4 * 4;
  d.kpad = ((M + 31) / 32) * 32;
  d.ksplit_umma = d.umma ? ct::umma_ksplit(T, S, M, ctx->num_sms) : 1;
  d.ksplit_slice = d.umma ? ct::slice_ksplit(T, S, M, ctx->num_sms) : 1;
  const int64_t V = d.V, mpad = ((M + 63) / 64) * 64;
  const int64_t ldp_umma = ((M + ct::umma_yn(M) - 1) / ct::umma_yn(M)) * ct::umma_yn(M);
  const int64_t ldp_slice = ((M + 127) / 128) * 128;
  const int64_t part_floats =
      std::max<int64_t>(std::max<int64_t>((int64_t)d.ksplit * T * mpad,
                                          d.umma ? (int64_t)d.ksplit_umma * T * ldp_umma : 0),
                        d.umma ? (int64_t)d.ksplit_slice * T * ldp_slice : 0);
#define ALLOC(ptr, n)                    \
  do {                                   \
    int r__ = alloc(s, &(ptr), (n));     \
    if (r__) {                           \
      free_scenario(s);                  \
      delete s;                          \
      return r__;                        \
    }                                    \
  } while (0)
  // +4 elements: the adjoint kernel bulk-copies per-tile ranges rounded up to 16 bytes
  ALLOC(d.gains, S * kGainCols + 4);
  ALLOC(d.nbr, V * kOffsets + 4);
  ALLOC(d.coefs, V * kOffsets + 4);
  ALLOC(d.delays, V * kOffsets + 4);
  ALLOC(d.init_delays, V * kOffsets);
  ALLOC(d.H, B * M * S);
  ALLOC(d.ctrl, S);
  ALLOC(d.u, T);
  ALLOC(d.meas, B * T * M);
  ALLOC(d.X, T * S);
  ALLOC(d.Y, B * T * M);
  ALLOC(d.R, T * M);
  ALLOC(d.MR, T * S);
  ALLOC(d.ap, V * kGainCols);
  ALLOC(d.ap_last, V * kGainCols);
  ALLOC(d.avg_delays, V);
  ALLOC(d.dG, S * kGainCols);
  ALLOC(d.dC, V * kOffsets);
  ALLOC(d.fir, V * kGainCols);
  ALLOC(d.iir, V * kGainCols);
  ALLOC(d.mG1, S * kGainCols);
  ALLOC(d.mG2, S * kGainCols);
  ALLOC(d.mC1, V * kOffsets);
  ALLOC(d.mC2, V * kOffsets);
  ALLOC(d.mreg_sum, 1);
  ALLOC(d.loss, T);
  ALLOC(d.loss_mse, T);
  ALLOC(d.loss_mr, T);
  ALLOC(d.loss_b, d.NB);
  ALLOC(d.loss_mse_b, d.NB);
  ALLOC(d.loss_mr_b, d.NB);
  ALLOC(d.stepsum_part, T * d.fwd_grid);
  ALLOC(d.gemm_part, part_floats);
  if (d.umma) {
    ALLOC(d.H_hi, B * M * d.spad);
    ALLOC(d.H_lo, B * M * d.spad);
    if (d.spad != S) ALLOC(d.Xpad, T * d.spad);
    ALLOC(d.Ht_hi, B * S * d.kpad);
    ALLOC(d.Ht_lo, B * S * d.kpad);
    ALLOC(d.R_hi, T * d.kpad);
    ALLOC(d.R_lo, T * d.kpad);
  }
  ALLOC(d.dmin, 2);
  if (d.fwd_ring) {
    ALLOC(d.halo, tiles * ct::kFwdHaloMax);
    ALLOC(d.hslot, tiles * ct::kFwdTileVoxels * kOffsets);
    ALLOC(d.nhalo, tiles);
  }
  ALLOC(d.status, 1);
  ALLOC(d.barrier, 1);
#undef ALLOC
  cudaStream_t st = ctx->stream;
  int r = CT_OK;
  // model arrays in device voxel order (uploads are synchronous on the context stream below,
  // so the host staging vectors outlive their copies)
  std::vector<float> h_gains((size_t)(S * kGainCols)), h_coefs((size_t)(V * kOffsets)),
      h_init((size_t)(V * kOffsets)), h_ctrl((size_t)S), h_H(desc->measurement_matrix ? (size_t)(B * M * S) : 0);
  std::vector<int32_t> h_nbr((size_t)(V * kOffsets)), h_delays((size_t)(V * kOffsets));
  gather_rows(h_gains.data(), desc->gains, s->perm, 3, kGainCols);
  gather_rows(h_coefs.data(), desc->coefs, s->perm, 1, kOffsets);
  gather_rows(h_init.data(), desc->initial_delays, s->perm, 1, kOffsets);
  gather_rows(h_delays.data(), desc->delays, s->perm, 1, kOffsets);
  gather_state_columns(h_ctrl.data(), desc->control_matrix, s->perm, 1);
  if (desc->measurement_matrix) gather_state_columns(h_H.data(), desc->measurement_matrix, s->perm, B * M);
  for (int64_t u = 0; u < V; ++u)
    for (int n = 0; n < kOffsets; ++n) {
      const int32_t w = nbr[(size_t)s->perm[(size_t)u] * kOffsets + n];
      h_nbr[(size_t)(u * kOffsets + n)] = w < 0 ? -1 : s->inv[(size_t)w];
    }
  s->nbr_dev = h_nbr;
  r = r ? r : upload(s, d.gains, h_gains.data(), sizeof(float) * S * kGainCols);
  r = r ? r : upload(s, d.nbr, h_nbr.data(), sizeof(int32_t) * V * kOffsets);
  r = r ? r : upload(s, d.coefs, h_coefs.data(), sizeof(float) * V * kOffsets);
  r = r ? r : upload(s, d.delays, h_delays.data(), sizeof(int32_t) * V * kOffsets);
  r = r ? r : upload(s, d.init_delays, h_init.data(), sizeof(float) * V * kOffsets);
  if (desc->measurement_matrix) r = r ? r : upload(s, d.H, h_H.data(), sizeof(float) * B * M * S);
  r = r ? r : upload(s, d.ctrl, h_ctrl.data(), sizeof(float) * S);
  if (d.fwd_ring) {
    r = r ? r : upload(s, d.halo, h_halo.data(), sizeof(int32_t) * h_halo.size());
    r = r ? r : upload(s, d.hslot, h_hslot.data(), sizeof(int16_t) * h_hslot.size());
    r = r ? r : upload(s, d.nhalo, h_nhalo.data(), sizeof(int32_t) * h_nhalo.size());
  }
  r = r ? r : upload(s, d.u, desc->control_function, sizeof(float) * T);
  if (!r && desc->measurements) r = upload(s, d.meas, desc->measurements, sizeof(float) * B * T * M);
  if (!r && !desc->measurements) {
    cudaError_t e = cudaMemsetAsync(d.meas, 0, sizeof(float) * B * T * M, st);
    if (e != cudaSuccess) r = cuda_fail(e, "memset");
  }
  auto zero = [&](void* p, size_t bytes) {
    if (r) return;
    cudaError_t e = cudaMemsetAsync(p, 0, bytes, st);
    if (e != cudaSuccess) r = cuda_fail(e, "memset");
  };
  if (!desc->measurement_matrix) zero(d.H, sizeof(float) * B * M * S);  // ct_scenario_set_measurement_matrix fills it
  zero(d.X, sizeof(float) * T * S);
  zero(d.Y, sizeof(float) * B * T * M);
  zero(d.R, sizeof(float) * T * M);
  zero(d.MR, sizeof(float) * T * S);
  zero(d.ap, sizeof(float) * V * kGainCols);
  zero(d.ap_last, sizeof(float) * V * kGainCols);
  zero(d.dG, sizeof(float) * S * kGainCols);
  zero(d.dC, sizeof(float) * V * kOffsets);
  zero(d.fir, sizeof(float) * V * kGainCols);
  zero(d.iir, sizeof(float) * V * kGainCols);
  zero(d.mG1, sizeof(float) * S * kGainCols);
  zero(d.mG2, sizeof(float) * S * kGainCols);
  zero(d.mC1, sizeof(float) * V * kOffsets);
  zero(d.mC2, sizeof(float) * V * kOffsets);
  zero(d.mreg_sum, sizeof(float));
  zero(d.loss, sizeof(float) * T);
  zero(d.loss_mse, sizeof(float) * T);
  zero(d.loss_mr, sizeof(float) * T);
  zero(d.loss_b, sizeof(float) * d.NB);
  zero(d.loss_mse_b, sizeof(float) * d.NB);
  zero(d.loss_mr_b, sizeof(float) * d.NB);
  zero(d.status, sizeof(int32_t));
  zero(d.barrier, sizeof(ct::GridBarrier));
  std::vector<float> nan_v((size_t)V, std::nanf(""));
  r = r ? r : upload(s, d.avg_delays, nan_v.data(), sizeof(float) * V);
  if (!r) {
    cudaError_t e = ct::launch_min_delay(d, st);
    if (e != cudaSuccess) r = cuda_fail(e, "min delay kernel");
  }
  if (!r && d.umma) {
    cudaError_t e = ct::umma_prepare(d, st);
    if (e != cudaSuccess) r = cuda_fail(e, "tensor-core operand split");
  }
  if (!r) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_fail(e, "scenario upload");
  }
  if (r) {
    free_scenario(s);
    delete s;
    return r;
  }
  ctx->refs += 1;
  *out = s;
  return CT_OK;
}

int ct_scenario_destroy(ct_scn* scn) {
  if (!scn) return CT_OK;
  ct_ctx* ctx = scn->ctx;
  DeviceScope device_scope__(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  free_scenario(scn);
  delete scn;
  ctx_release(ctx);
  return CT_OK;
}

int ct_scenario_dims(ct_scn* scn, int64_t* S, int64_t* M, int64_t* T, int64_t* B) {
  if (!scn) return fail(CT_ERR_INVALID_ARGUMENT, "scenario is NULL");
  if (S) *S = scn->d.S;
  if (M) *M = scn->d.M;
  if (T) *T = scn->d.T;
  if (B) *B = scn->d.B;
  return CT_OK;
}

static int run_beat_plain(ct_scn* s, int64_t beat) {
  DeviceScenario& d = s->d;
  const ct_algorithm& a = s->algo;
  if (!d.plain_mreg) {
    int rc = alloc(s, &d.plain_mreg, d.S);
    if (!rc) rc = alloc(s, &d.plain_part, (d.V + 255) / 256);
    if (rc) return rc;
  }
  ct::PlainScalars ps;
  ps.mse_scaling = 1.0f / (float)d.M * a.mse_strength;
  ps.reg_scaling = a.maximum_regularization_strength;
  ps.threshold = a.maximum_regularization_threshold;
  ps.diffreg = a.difference_regularization_strength;
  ps.freeze_gains = a.freeze_gains;
  ps.freeze_delays = a.freeze_delays;
  ps.ap_derivative = a.ap_derivative;
  CT_CUDA(run_phase(s, CT_PHASE_FORWARD, (int)(d.T * ct::plain_step_launches(ps)),
                    [&] { return ct::launch_plain_beat(d, beat, ps, s->ctx->stream); }),
          "plain-form kernels");
  return CT_OK;
}

// The TF32 product modes accumulate with a bias (the tensor core's FP32 adds are not round-to-nearest)
// that the gradient, a near-cancelling sum of residual terms, does not average out when the residuals
// are a small fraction of the signal. Before a scenario's first epoch in such a mode, the first beat's
// reference-mode gradients are computed with the mode and with the sliced BF16 products (unbiased, within
// ~1e-4 of FP64); if they differ by more than the 1e-3 gradient target (norm-wise), the mode is refused for
// this scenario. The check leaves parameters, Adam state and the batch cursor untouched; it overwrites
// the estimation outputs of the last epoch (states, predicted measurements, residuals, step metrics).
constexpr double kTf32GradientBar = 1e-3;

int check_tf32_gradients(ct_scn* s, int precision) {
  const int slot = precision == CT_PREC_TF32 ? 1 : 0;
  if (s->tf32_verdict[slot] > 0) return CT_OK;
  if (s->tf32_verdict[slot] < 0)
    return fail(CT_ERR_NOT_SUPPORTED,
                "precision %d refused for this scenario: its first-beat gradients differ by %.2e (norm-wise) from "
                "the sliced BF16 products' (bar %.0e); use CT_PREC_BF16X6 or CT_PREC_FP32",
                precision, s->tf32_rel[slot], kTf32GradientBar);
  const ct_algorithm& a = s->algo;
  if (a.freeze_gains && a.freeze_delays) return CT_OK;  // no gradients to compare
  int rc = prepare_sliced(s);
  if (rc) return rc;
  DeviceScenario& d = s->d;
  const bool prof = s->profiling;
  s->profiling = false;
  std::vector<float> g[2], c[2];
  for (int pass = 0; pass < 2 && !rc; ++pass) {
    rc = derivatives_reset(s);
    if (!rc) rc = run_beat(s, 0, pass == 0 ? precision : CT_PREC_BF16X6, CT_GRAD_REFERENCE);
    if (!rc) {
      g[pass].resize((size_t)(d.S * kGainCols));
      c[pass].resize((size_t)(d.V * kOffsets));
      rc = copy_down(s, g[pass].data(), d.dG, sizeof(float) * g[pass].size());
      if (!rc) rc = copy_down(s, c[pass].data(), d.dC, sizeof(float) * c[pass].size());
    }
  }
  s->profiling = prof;
  if (!rc) rc = derivatives_reset(s);
  if (rc) return rc;
  auto rel = [](const std::vector<float>& x, const std::vector<float>& y) {
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < x.size(); ++i) {
      const double e = (double)x[i] - (double)y[i];
      num += e * e;
      den += (double)y[i] * (double)y[i];
    }
    return den > 0.0 ? std::sqrt(num / den) : std::sqrt(num);
  };
  const double eg = a.freeze_gains ? 0.0 : rel(g[0], g[1]);
  const double ec = a.freeze_delays ? 0.0 : rel(c[0], c[1]);
  const double e = std::max(eg, ec);
  s->tf32_rel[slot] = e;
  s->tf32_verdict[slot] = (e <= kTf32GradientBar) ? 1 : -1;
  return check_tf32_gradients(s, precision);
}

static int run_epoch_impl(ct_scn* scn, int64_t* batch_index, const int32_t* beat_order, int grad_mode,
                          int precision, bool plain) {
  if (!scn || !batch_index) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (grad_mode != CT_GRAD_REFERENCE && grad_mode != CT_GRAD_ADJOINT)
    return fail(CT_ERR_NOT_SUPPORTED, "gradient mode %d", grad_mode);
  if (!valid_precision(precision)) return fail(CT_ERR_NOT_SUPPORTED, "precision %d", precision);
  if (precision != CT_PREC_FP32 && !scn->d.umma)
    return fail(CT_ERR_NOT_SUPPORTED,
                "tensor-core precision needs the driver's TMA encoder and at most 65,536 sensor rows");
  CT_DEVICE_SCOPE(scn->ctx->device);
  if (precision == CT_PREC_BF16X6 && !plain) {
    int rc0 = prepare_sliced(scn);
    if (rc0) return rc0;
  }
  if ((precision == CT_PREC_TF32X3 || precision == CT_PREC_TF32) && !plain) {
    int rc0 = check_tf32_gradients(scn, precision);
    if (rc0) return rc0;
  }
  DeviceScenario& d = scn->d;
  const ct_algorithm& a = scn->algo;
  std::vector<int32_t> order((size_t)d.B);
  if (beat_order) {
    for (int64_t i = 0; i < d.B; ++i) {
      if (beat_order[i] < 0 || beat_order[i] >= d.B)
        return fail(CT_ERR_INVALID_ARGUMENT, "beat_order[%lld] = %d out of range", (long long)i, beat_order[i]);
      order[(size_t)i] = beat_order[i];
    }
  } else {
    for (int64_t i = 0; i < d.B; ++i) order[(size_t)i] = (int32_t)i;
    seeded_shuffle(scn, order);
  }
  int rc = derivatives_reset(scn);
  if (rc) return rc;
  if (grad_mode == CT_GRAD_ADJOINT && (!a.freeze_gains || !a.freeze_delays)) {
    rc = prepare_adjoint(scn, scn->d.rev ? scn->d.ckpt_k : ct::kCkptSteps);
    if (rc) return rc;
  }
  int64_t batch = 0;
  const bool batched = a.batch_size != 0;
  for (int32_t beat : order) {
    rc = plain ? run_beat_plain(scn, beat) : run_beat(scn, beat, precision, grad_mode);
    if (rc) return rc;
    if (batched) {
      batch += 1;
      if (batch == a.batch_size) {
        rc = batch_end(scn, batch, batch_index);
        if (rc) return rc;
        rc = derivatives_reset(scn);
        if (rc) return rc;
        batch = 0;
      }
    }
  }
  if (batched) return batch > 0 ? batch_end(scn, batch, batch_index) : CT_OK;
  return batch_end(scn, d.B, batch_index);
}

int ct_run_epoch(ct_scn* scn, int64_t* batch_index, const int32_t* beat_order, int grad_mode, int precision) {
  return run_epoch_impl(scn, batch_index, beat_order, grad_mode, precision, false);
}

int ct_run_epoch_plain(ct_scn* scn, int64_t* batch_index, const int32_t* beat_order) {
  return run_epoch_impl(scn, batch_index, beat_order, CT_GRAD_REFERENCE, CT_PREC_FP32, true);
}

// One epoch for a caller that keeps the model in host memory, as the reference's run_epoch
// (src/core/algorithm.rs:124-129) mutates `results.model` in place: every copy, reordering kernel
// and the epoch go onto the context stream back to back, and the call waits once at the end.
int ct_run_epoch_host(ct_scn* scn, int64_t* batch_index, const int32_t* beat_order, int grad_mode, int precision,
                      float* gains, float* coefs, int32_t* delays, const float* measurements, float* loss_batch) {
  if (!scn || !batch_index || !gains || !coefs || !delays) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  CT_DEVICE_SCOPE(scn->ctx->device);
  DeviceScenario& d = scn->d;
  cudaStream_t st = scn->ctx->stream;
  // the delays of connected pairs must be >= 1, as ct_write_field checks; their largest sizes the
  // adjoint's inbox ring
  const std::vector<int32_t>& nbr = scn->nbr_host;
  int64_t dmax = 1;
  for (size_t i = 0; i < nbr.size(); ++i) {
    if (nbr[i] < 0) continue;
    if (delays[i] < 1)
      return fail(CT_ERR_INVALID_ARGUMENT, "delay %zu of a connected pair is %d; delays must be >= 1", i, delays[i]);
    if (delays[i] > dmax) dmax = delays[i];
  }
  int rc = ensure_xfer(scn);
  if (rc) return rc;
  const int64_t ng = d.S * kGainCols, nc = d.V * kOffsets;
  if (!scn->xfer_epoch) {
    rc = alloc(scn, &scn->xfer_epoch, ng + 2 * nc);
    if (rc) return rc;
  }
  uint32_t* sg = scn->xfer_epoch;
  uint32_t* sc = sg + ng;
  uint32_t* sd = sc + nc;
  // inputs: host -> staging -> device voxel order
  CT_CUDA(cudaMemcpyAsync(sg, gains, sizeof(float) * ng, cudaMemcpyHostToDevice, st), "copy gains");
  CT_CUDA(ct::launch_permute_blocks(sg, d.gains, scn->perm_dev, d.V, 3 * kGainCols, true, st), "permute kernel");
  CT_CUDA(cudaMemcpyAsync(sc, coefs, sizeof(float) * nc, cudaMemcpyHostToDevice, st), "copy coefs");
  CT_CUDA(ct::launch_permute_blocks(sc, d.coefs, scn->perm_dev, d.V, kOffsets, true, st), "permute kernel");
  CT_CUDA(cudaMemcpyAsync(sd, delays, sizeof(int32_t) * nc, cudaMemcpyHostToDevice, st), "copy delays");
  CT_CUDA(ct::launch_permute_blocks(sd, d.delays, scn->perm_dev, d.V, kOffsets, true, st), "permute kernel");
  if (measurements)
    CT_CUDA(cudaMemcpyAsync(d.meas, measurements, sizeof(float) * d.B * d.T * d.M, cudaMemcpyHostToDevice, st),
            "copy measurements");
  CT_CUDA(ct::launch_min_delay(d, st), "min delay kernel");
  scn->launches += 4;
  scn->dmax_bound = dmax;
  scn->updates_at_read = -1;
  rc = ct_run_epoch(scn, batch_index, beat_order, grad_mode, precision);
  if (rc) {
    cudaStreamSynchronize(st);
    return rc;
  }
  // outputs: device voxel order -> staging -> host (the same arrays, updated in place)
  CT_CUDA(ct::launch_permute_blocks(d.gains, sg, scn->perm_dev, d.V, 3 * kGainCols, false, st), "permute kernel");
  CT_CUDA(cudaMemcpyAsync(gains, sg, sizeof(float) * ng, cudaMemcpyDeviceToHost, st), "copy gains");
  CT_CUDA(ct::launch_permute_blocks(d.coefs, sc, scn->perm_dev, d.V, kOffsets, false, st), "permute kernel");
  CT_CUDA(cudaMemcpyAsync(coefs, sc, sizeof(float) * nc, cudaMemcpyDeviceToHost, st), "copy coefs");
  CT_CUDA(ct::launch_permute_blocks(d.delays, sd, scn->perm_dev, d.V, kOffsets, false, st), "permute kernel");
  CT_CUDA(cudaMemcpyAsync(delays, sd, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, st), "copy delays");
  scn->launches += 3;
  if (loss_batch)
    CT_CUDA(cudaMemcpyAsync(loss_batch, d.loss_b, sizeof(float) * d.NB, cudaMemcpyDeviceToHost, st), "copy loss");
  return ct_sync(scn);
}

int ct_simulate(ct_scn* scn, float* measurements_out, float* states_out) {
  if (!scn || !measurements_out) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  CT_DEVICE_SCOPE(scn->ctx->device);
  DeviceScenario& d = scn->d;
  cudaStream_t st = scn->ctx->stream;
  for (int64_t beat = 0; beat < d.B; ++beat) {
    CT_CUDA(run_phase(scn, CT_PHASE_FORWARD, 1,
                      [&] { return ct::launch_forward(d, scn->algo.maximum_regularization_threshold, nullptr, st); }),
            "forward kernel");
    CT_CUDA(run_phase(scn, CT_PHASE_MEASURE, 2, [&] { return ct::launch_measure(d, beat, false, st); }),
            "measurement kernel");
  }
  int rc = ct_sync(scn);
  if (rc) return rc;
  rc = copy_down(scn, measurements_out, d.Y, sizeof(float) * d.B * d.T * d.M);
  if (rc) return rc;
  if (states_out) rc = copy_down_state_columns(scn, states_out, d.X, d.T);
  return rc;
}

int ct_set_algorithm(ct_scn* scn, const ct_algorithm* algo) {
  if (!scn) return fail(CT_ERR_INVALID_ARGUMENT, "scenario is NULL");
  int rc = check_algo(algo);
  if (rc) return rc;
  scn->algo = *algo;
  scn->config_gen += 1;
  return CT_OK;
}

int ct_set_freeze(ct_scn* scn, int freeze_gains, int freeze_delays) {
  if (!scn) return fail(CT_ERR_INVALID_ARGUMENT, "scenario is NULL");
  scn->algo.freeze_gains = freeze_gains != 0;
  scn->algo.freeze_delays = freeze_delays != 0;
  scn->config_gen += 1;
  return CT_OK;
}

int ct_set_learning_rate(ct_scn* scn, float learning_rate) {
  if (!scn) return fail(CT_ERR_INVALID_ARGUMENT, "scenario is NULL");
  scn->algo.learning_rate = learning_rate;
  scn->config_gen += 1;
  return CT_OK;
}

int ct_field_size(ct_scn* scn, int field, size_t* nbytes) {
  if (!scn || !nbytes) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  return field_bytes(scn, field, nbytes);
}

int ct_read_field(ct_scn* scn, int field, void* dst, size_t nbytes) {
  if (!scn || !dst) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  size_t want = 0;
  int rc = field_bytes(scn, field, &want);
  if (rc) return rc;
  if (want != nbytes) return fail(CT_ERR_INVALID_ARGUMENT, "field %d has %zu bytes, got %zu", field, want, nbytes);
  CT_DEVICE_SCOPE(scn->ctx->device);
  DeviceScenario& d = scn->d;
  float* out = static_cast<float*>(dst);
  switch (field) {
    case CT_FIELD_GAINS: return copy_down_rows(scn, out, d.gains, 3, kGainCols);
    case CT_FIELD_COEFS: return copy_down_rows(scn, out, d.coefs, 1, kOffsets);
    case CT_FIELD_DELAYS: return copy_down_rows(scn, static_cast<int32_t*>(dst), d.delays, 1, kOffsets);
    case CT_FIELD_MEASUREMENTS_ACTUAL: return copy_down(scn, dst, d.meas, nbytes);
    case CT_FIELD_SYSTEM_STATES: return copy_down_state_columns(scn, out, d.X, d.T);
    case CT_FIELD_MEASUREMENTS: return copy_down(scn, dst, d.Y, nbytes);
    case CT_FIELD_RESIDUALS: return copy_down(scn, dst, d.R + (d.T - 1) * d.M, nbytes);
    case CT_FIELD_AP_OUTPUTS_NOW: return copy_down_expanded(scn, out, d.ap);
    case CT_FIELD_AP_OUTPUTS_LAST: return copy_down_expanded(scn, out, d.ap_last);
    case CT_FIELD_AVERAGE_DELAYS: return copy_down_rows(scn, out, d.avg_delays, 1, 1);
    case CT_FIELD_GRAD_GAINS: return copy_down_rows(scn, out, d.dG, 3, kGainCols);
    case CT_FIELD_GRAD_COEFS: return copy_down_rows(scn, out, d.dC, 1, kOffsets);
    case CT_FIELD_COEFS_FIR: return copy_down_expanded(scn, out, d.fir);
    case CT_FIELD_COEFS_IIR: return copy_down_expanded(scn, out, d.iir);
    case CT_FIELD_MAPPED_RESIDUALS: return copy_down_state_columns(scn, out, d.MR + (d.T - 1) * d.S, 1);
    case CT_FIELD_MAXIMUM_REGULARIZATION: {
      // derived from the last step's states into a temporary device buffer (read-back path only)
      float* tmp = nullptr;
      CT_CUDA(cudaMallocAsync((void**)&tmp, nbytes, scn->ctx->stream), "cudaMallocAsync");
      cudaError_t e = ct::launch_last_max_reg(d, scn->algo.maximum_regularization_threshold, tmp, scn->ctx->stream);
      int r2 = e == cudaSuccess ? copy_down_state_columns(scn, out, tmp, 1) : cuda_fail(e, "max reg kernel");
      cudaFreeAsync(tmp, scn->ctx->stream);
      return r2;
    }
    case CT_FIELD_MAXIMUM_REGULARIZATION_SUM: return copy_down(scn, dst, d.mreg_sum, nbytes);
    case CT_FIELD_ADAM_STEP: std::memcpy(dst, &scn->adam_step, sizeof(int64_t)); return CT_OK;
    case CT_FIELD_GAINS_FIRST_MOMENT: return copy_down_rows(scn, out, d.mG1, 3, kGainCols);
    case CT_FIELD_GAINS_SECOND_MOMENT: return copy_down_rows(scn, out, d.mG2, 3, kGainCols);
    case CT_FIELD_COEFS_FIRST_MOMENT: return copy_down_rows(scn, out, d.mC1, 1, kOffsets);
    case CT_FIELD_COEFS_SECOND_MOMENT: return copy_down_rows(scn, out, d.mC2, 1, kOffsets);
    case CT_FIELD_MAPPED_RESIDUALS_HISTORY: return copy_down_state_columns(scn, out, d.MR, d.T);
    case CT_FIELD_LOSS: return copy_down(scn, dst, d.loss, nbytes);
    case CT_FIELD_LOSS_MSE: return copy_down(scn, dst, d.loss_mse, nbytes);
    case CT_FIELD_LOSS_MAXIMUM_REGULARIZATION: return copy_down(scn, dst, d.loss_mr, nbytes);
    case CT_FIELD_LOSS_BATCH: return copy_down(scn, dst, d.loss_b, nbytes);
    case CT_FIELD_LOSS_MSE_BATCH: return copy_down(scn, dst, d.loss_mse_b, nbytes);
    case CT_FIELD_LOSS_MAXIMUM_REGULARIZATION_BATCH: return copy_down(scn, dst, d.loss_mr_b, nbytes);
    case CT_FIELD_STATES_MAGNITUDE:
    case CT_FIELD_STATES_THETA:
    case CT_FIELD_STATES_PHI:
    case CT_FIELD_STATES_MAGNITUDE_MAX:
    case CT_FIELD_STATES_THETA_MAX:
    case CT_FIELD_STATES_PHI_MAX:
    case CT_FIELD_ACTIVATION_TIMES: {
      if (!scn->post_arrays) return fail(CT_ERR_INVALID_ARGUMENT, "field %d: call ct_calculate_plotting_arrays first", field);
      const ct::PostBuffers& b = scn->post;
      const float* src = field == CT_FIELD_STATES_MAGNITUDE     ? b.mag
                         : field == CT_FIELD_STATES_THETA       ? b.theta
                         : field == CT_FIELD_STATES_PHI         ? b.phi
                         : field == CT_FIELD_STATES_MAGNITUDE_MAX ? b.mag_max
                         : field == CT_FIELD_STATES_THETA_MAX   ? b.theta_max
                         : field == CT_FIELD_STATES_PHI_MAX     ? b.phi_max
                                                                : b.activation_ms;
      return copy_down(scn, dst, src, nbytes);  // written in reference voxel order
    }
    case CT_FIELD_SNAPSHOT_GAINS:
    case CT_FIELD_SNAPSHOT_COEFS:
    case CT_FIELD_SNAPSHOT_DELAYS:
    case CT_FIELD_SNAPSHOT_SYSTEM_STATES: {
      for (int64_t i = 0; i < scn->snap_n; ++i) {
        int r = CT_OK;
        if (field == CT_FIELD_SNAPSHOT_GAINS) {
          const int64_t n = d.S * kGainCols;
          r = copy_down_rows(scn, out + i * n, scn->snap_gains + i * n, 3, kGainCols);
        } else if (field == CT_FIELD_SNAPSHOT_COEFS) {
          const int64_t n = d.V * kOffsets;
          r = copy_down_rows(scn, out + i * n, scn->snap_coefs + i * n, 1, kOffsets);
        } else if (field == CT_FIELD_SNAPSHOT_DELAYS) {
          const int64_t n = d.V * kOffsets;
          r = copy_down_rows(scn, static_cast<int32_t*>(dst) + i * n, scn->snap_delays + i * n, 1, kOffsets);
        } else {
          const int64_t n = d.T * d.S;
          r = copy_down_state_columns(scn, out + i * n, scn->snap_X + i * n, d.T);
        }
        if (r) return r;
      }
      return CT_OK;
    }
    case CT_FIELD_SNAPSHOT_MEASUREMENTS:
      return scn->snap_n ? copy_down(scn, dst, scn->snap_Y, nbytes) : CT_OK;
    default: return fail(CT_ERR_INVALID_ARGUMENT, "unknown field %d", field);
  }
}

int ct_write_field(ct_scn* scn, int field, const void* src, size_t nbytes) {
  if (!scn || !src) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  size_t want = 0;
  int rc = field_bytes(scn, field, &want);
  if (rc) return rc;
  if (want != nbytes) return fail(CT_ERR_INVALID_ARGUMENT, "field %d has %zu bytes, got %zu", field, want, nbytes);
  CT_DEVICE_SCOPE(scn->ctx->device);
  DeviceScenario& d = scn->d;
  void* dst = nullptr;
  switch (field) {
    case CT_FIELD_GAINS: dst = d.gains; break;
    case CT_FIELD_COEFS: dst = d.coefs; break;
    case CT_FIELD_DELAYS: {
      const int32_t* del = static_cast<const int32_t*>(src);
      const std::vector<int32_t>& nbr = scn->nbr_host;
      for (size_t i = 0; i < nbr.size(); ++i)
        if (nbr[i] >= 0 && del[i] < 1)
          return fail(CT_ERR_INVALID_ARGUMENT, "delay %zu of a connected pair is %d; delays must be >= 1", i, del[i]);
      dst = d.delays;
      scn->dmax_bound = max_connected_delay(nbr, del);
      scn->updates_at_read = -1;
      break;
    }
    case CT_FIELD_MEASUREMENTS_ACTUAL: dst = d.meas; break;
    default: return fail(CT_ERR_INVALID_ARGUMENT, "field %d is read-only", field);
  }
  // reorder into device voxel order on the device (measurements are in sensor space: no reordering)
  if (field == CT_FIELD_MEASUREMENTS_ACTUAL) {
    CT_CUDA(cudaMemcpyAsync(dst, src, nbytes, cudaMemcpyHostToDevice, scn->ctx->stream), "write field");
  } else if (ensure_xfer(scn) == CT_OK) {
    const int64_t words = field == CT_FIELD_GAINS ? 3 * kGainCols : kOffsets;
    CT_CUDA(cudaMemcpyAsync(scn->xfer, src, nbytes, cudaMemcpyHostToDevice, scn->ctx->stream), "write field");
    CT_CUDA(ct::launch_permute_blocks(scn->xfer, dst, scn->perm_dev, d.V, words, true, scn->ctx->stream),
            "permute kernel");
  } else {
    std::vector<unsigned char> staged(nbytes);
    if (field == CT_FIELD_GAINS)
      gather_rows(reinterpret_cast<float*>(staged.data()), static_cast<const float*>(src), scn->perm, 3, kGainCols);
    else if (field == CT_FIELD_COEFS)
      gather_rows(reinterpret_cast<float*>(staged.data()), static_cast<const float*>(src), scn->perm, 1, kOffsets);
    else
      gather_rows(reinterpret_cast<int32_t*>(staged.data()), static_cast<const int32_t*>(src), scn->perm, 1,
                  kOffsets);
    CT_CUDA(cudaMemcpyAsync(dst, staged.data(), nbytes, cudaMemcpyHostToDevice, scn->ctx->stream), "write field");
    CT_CUDA(cudaStreamSynchronize(scn->ctx->stream), "write field");
  }
  if (field == CT_FIELD_DELAYS) CT_CUDA(ct::launch_min_delay(d, scn->ctx->stream), "min delay kernel");
  CT_CUDA(cudaStreamSynchronize(scn->ctx->stream), "write field");
  return CT_OK;
}

int ct_sync(ct_scn* scn) {
  if (!scn) return fail(CT_ERR_INVALID_ARGUMENT, "scenario is NULL");
  CT_DEVICE_SCOPE(scn->ctx->device);
  CT_CUDA(cudaStreamSynchronize(scn->ctx->stream), "cudaStreamSynchronize");
  int32_t status = 0;
  CT_CUDA(cudaMemcpy(&status, scn->d.status, sizeof(int32_t), cudaMemcpyDeviceToHost), "read status");
  if (status != 0) {
    cudaMemset(scn->d.status, 0, sizeof(int32_t));
    return fail(status, "device-side failure: %s", ct_status_string(status));
  }
  return CT_OK;
}

int ct_kernel_launches(ct_scn* scn, int64_t* launches) {
  if (!scn || !launches) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  *launches = scn->launches;
  return CT_OK;
}

int ct_set_profiling(ct_scn* scn, int enable) {
  if (!scn) return fail(CT_ERR_INVALID_ARGUMENT, "scenario is NULL");
  CT_DEVICE_SCOPE(scn->ctx->device);
  CT_CUDA(cudaStreamSynchronize(scn->ctx->stream), "cudaStreamSynchronize");
  for (auto& pe : scn->pending) {
    scn->event_pool.push_back(pe.start);
    scn->event_pool.push_back(pe.stop);
  }
  scn->pending.clear();
  scn->profiling = enable != 0;
  if (scn->profiling) {
    for (int i = 0; i < CT_PHASE_COUNT; ++i) {
      scn->phase_ms[i] = 0.0;
      scn->phase_launches[i] = 0;
    }
  }
  return CT_OK;
}

int ct_read_profile(ct_scn* scn, double* ms, int64_t* launches) {
  if (!scn || !ms || !launches) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  CT_DEVICE_SCOPE(scn->ctx->device);
  CT_CUDA(cudaStreamSynchronize(scn->ctx->stream), "cudaStreamSynchronize");
  for (auto& pe : scn->pending) {
    float t = 0.0f;
    CT_CUDA(cudaEventElapsedTime(&t, pe.start, pe.stop), "cudaEventElapsedTime");
    scn->phase_ms[pe.phase] += t;
    scn->event_pool.push_back(pe.start);
    scn->event_pool.push_back(pe.stop);
  }
  scn->pending.clear();
  for (int i = 0; i < CT_PHASE_COUNT; ++i) {
    ms[i] = scn->phase_ms[i];
    launches[i] = scn->phase_launches[i];
  }
  return CT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- batched scenarios
//
// A batch runs one epoch of every member scenario as one schedule: per beat
// index b, one cooperative forward launch over the tiles of every scenario
// that has a beat b, the measurement products of each scenario on parallel
// streams, then one cooperative adjoint launch (or the per-scenario reference
// derivations), the step metrics, and finally every scenario's update. The
// whole epoch is captured once as a CUDA graph and replayed; the values that
// change from epoch to epoch (Adam bias corrections, batch-metric slots) are
// read by the kernels from a small device array written before each replay.

// Checkpoint interval of batch members in adjoint mode: segment buffers (2K planes) plus
// checkpoints (T/K planes) are smallest near K = sqrt(T/2), 22..45 for 1,000..4,000 steps.
constexpr int kBatchCkptSteps = 64;

struct EpochDev {
  float bias[2];        // 1 - beta1^step, 1 - beta2^step (host powf, as in update.rs:140-141)
  int64_t batch_index;  // batch-wise metric slot
};

struct ct_batch {
  ct_ctx* ctx = nullptr;
  std::vector<ct_scn*> scns;
  int grad_mode = CT_GRAD_REFERENCE;
  int precision = CT_PREC_FP32;
  int nbeats_max = 0;
  int fwd_grid = 0, adj_grid = 0;
  std::vector<std::vector<int2>> beat_tiles;  // per beat index: tiles of the scenarios with that beat
  std::vector<int> beat_tmax;
  std::vector<int2*> beat_tiles_dev;
  std::vector<float*> parts;                  // per scenario [T, tiles] step partials
  std::vector<int> ntiles;
  ct::FwdArgs* fwd_dev = nullptr;
  ct::AdjScn* adj_dev = nullptr;
  EpochDev* epoch_dev = nullptr;
  std::vector<void*> allocations;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> fork_ev, join_ev;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool use_graph = true;
  std::vector<int> captured_ring;
  std::vector<uint64_t> captured_gen;
  int64_t graph_kernels = 0;
  // tuned choices (ct_batch_autotune): adjoint checkpoint interval, tile order
  int ckpt_k = kBatchCkptSteps;
  int tile_order = 0;
  int captured_k = 0;
  // optional per-phase timing (eager launches, CUDA events on the context stream)
  bool profiling = false;
  cudaEvent_t open_event = nullptr;
  std::vector<PhaseEvents> pending;
  double phase_ms[CT_PHASE_COUNT] = {};
};

namespace {

int batch_alloc(ct_batch* b, void** p, size_t bytes) {
  cudaError_t err = cudaMalloc(p, bytes > 0 ? bytes : 1);
  if (err != cudaSuccess) return cuda_fail(err, "cudaMalloc (batch)");
  b->allocations.push_back(*p);
  return CT_OK;
}

void batch_free(ct_batch* b) {
  for (auto& pe : b->pending) {
    cudaEventDestroy(pe.start);
    cudaEventDestroy(pe.stop);
  }
  b->pending.clear();
  if (b->open_event) cudaEventDestroy(b->open_event);
  b->open_event = nullptr;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  for (void* p : b->allocations) cudaFree(p);
  b->allocations.clear();
  for (cudaStream_t s : b->side) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->fork_ev) cudaEventDestroy(e);
  for (cudaEvent_t e : b->join_ev) cudaEventDestroy(e);
  b->side.clear();
  b->fork_ev.clear();
  b->join_ev.clear();
}

// Fork every side stream off the main stream / join them back (event record + wait; captured as graph edges).
cudaError_t fork_side(ct_batch* b) {
  cudaStream_t st = b->ctx->stream;
  for (size_t i = 0; i < b->side.size(); ++i) {
    cudaError_t e = cudaEventRecord(b->fork_ev[i], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->side[i], b->fork_ev[i], 0);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
cudaError_t join_side(ct_batch* b) {
  cudaStream_t st = b->ctx->stream;
  for (size_t i = 0; i < b->side.size(); ++i) {
    cudaError_t e = cudaEventRecord(b->join_ev[i], b->side[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->join_ev[i], 0);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

#define B_CUDA(expr)                         \
  do {                                       \
    cudaError_t e__ = (expr);                \
    if (e__ != cudaSuccess) return e__;      \
  } while (0)

// Profiling: closes the phase opened by the previous mark (closes_phase >= 0) and opens the next one.
// Every event belongs to exactly one (start, stop) pair.
cudaError_t batch_mark(ct_batch* b, int closes_phase) {
  if (!b->profiling) return cudaSuccess;
  cudaStream_t st = b->ctx->stream;
  cudaError_t err;
  if (b->open_event && closes_phase >= 0) {
    cudaEvent_t stop = nullptr;
    if ((err = cudaEventCreate(&stop)) != cudaSuccess) return err;
    if ((err = cudaEventRecord(stop, st)) != cudaSuccess) return err;
    b->pending.push_back({closes_phase, b->open_event, stop});
  } else if (b->open_event) {
    cudaEventDestroy(b->open_event);
  }
  b->open_event = nullptr;
  cudaEvent_t start = nullptr;
  if ((err = cudaEventCreate(&start)) != cudaSuccess) return err;
  if ((err = cudaEventRecord(start, st)) != cudaSuccess) return err;
  b->open_event = start;
  return cudaSuccess;
}

// Everything of one epoch, enqueued on the context stream and the side streams.
cudaError_t batch_enqueue_epoch(ct_batch* b) {
  cudaStream_t st = b->ctx->stream;
  const size_t n = b->scns.size();
  B_CUDA(batch_mark(b, -1));
  auto side_of = [&](size_t i) { return b->side[i % b->side.size()]; };
  const bool adjoint = b->grad_mode == CT_GRAD_ADJOINT;
  // Derivatives::reset of every scenario
  B_CUDA(fork_side(b));
  for (size_t i = 0; i < n; ++i) {
    DeviceScenario& d = b->scns[i]->d;
    cudaStream_t s = side_of(i);
    B_CUDA(cudaMemsetAsync(d.dG, 0, sizeof(float) * d.S * kGainCols, s));
    B_CUDA(cudaMemsetAsync(d.dC, 0, sizeof(float) * d.V * kOffsets, s));
    B_CUDA(cudaMemsetAsync(d.fir, 0, sizeof(float) * d.V * kGainCols, s));
    B_CUDA(cudaMemsetAsync(d.iir, 0, sizeof(float) * d.V * kGainCols, s));
    B_CUDA(cudaMemsetAsync(d.mreg_sum, 0, sizeof(float), s));
  }
  B_CUDA(join_side(b));
  for (int beat = 0; beat < b->nbeats_max; ++beat) {
    // forward of every scenario with this beat
    B_CUDA(fork_side(b));
    for (size_t i = 0; i < n; ++i) {
      DeviceScenario& d = b->scns[i]->d;
      if (beat >= d.B) continue;
      B_CUDA(cudaMemsetAsync(d.ap, 0, sizeof(float) * d.V * kGainCols, side_of(i)));
      B_CUDA(cudaMemsetAsync(d.ap_last, 0, sizeof(float) * d.V * kGainCols, side_of(i)));
      if (adjoint) {
        B_CUDA(cudaMemsetAsync(d.inbox, 0, sizeof(float) * d.adj_ring * (size_t)d.adj_pitch, side_of(i)));
        B_CUDA(cudaMemsetAsync(d.lam_state, 0, sizeof(float) * d.V * kGainCols, side_of(i)));
      }
    }
    B_CUDA(join_side(b));
    DeviceScenario& d0 = b->scns[0]->d;
    ct::FwdBatch fb;
    fb.scns = b->fwd_dev;
    fb.nscn = (int)n;
    fb.tiles = b->beat_tiles_dev[(size_t)beat];
    fb.ntiles = (int)b->beat_tiles[(size_t)beat].size();
    fb.Tmax = b->beat_tmax[(size_t)beat];
    fb.status = d0.status;
    fb.barrier = d0.barrier;
    B_CUDA(ct::launch_forward_batch(fb, std::min(b->fwd_grid, fb.ntiles), st));
    B_CUDA(batch_mark(b, CT_PHASE_FORWARD));
    // measurement products, residuals, (reference) derivations and step metrics per scenario
    B_CUDA(fork_side(b));
    for (size_t i = 0; i < n; ++i) {
      ct_scn* s = b->scns[i];
      DeviceScenario& d = s->d;
      if (beat >= d.B) continue;
      cudaStream_t ss = side_of(i);
      const ct_algorithm& a = s->algo;
      // members whose states cannot be tensor-mapped (num_states not a multiple of 4) use FP32 products
      if (b->precision == CT_PREC_FP32 || !d.umma) {
        B_CUDA(ct::launch_measure(d, beat, true, ss));
        B_CUDA(ct::launch_map_residuals(d, beat, ss));
      } else if (b->precision == CT_PREC_BF16X6) {
        B_CUDA(ct::launch_measure_sliced(d, beat, true, ss));
        B_CUDA(ct::launch_map_residuals_sliced(d, beat, ss));
      } else {
        B_CUDA(ct::launch_measure_umma(d, beat, true, b->precision, ss));
        B_CUDA(ct::launch_map_residuals_umma(d, beat, b->precision, ss));
      }
      if (!adjoint && (!a.freeze_gains || !a.freeze_delays)) {
        ct::DeriveScalars ds;
        ds.mse_scaling = 1.0f / (float)d.M * a.mse_strength;
        ds.reg_scaling = a.maximum_regularization_strength;
        ds.threshold = a.maximum_regularization_threshold;
        ds.diffreg = a.difference_regularization_strength;
        ds.freeze_gains = a.freeze_gains;
        ds.freeze_delays = a.freeze_delays;
        ds.ap_derivative = a.ap_derivative;
        B_CUDA(ct::launch_derive(d, ds, ss));
      }
      B_CUDA(ct::launch_step_metrics_parts(d, b->parts[i], b->ntiles[i], a.maximum_regularization_strength, ss));
    }
    B_CUDA(join_side(b));
    if (adjoint) {
      ct::AdjLaunch al;
      al.scns = b->adj_dev;
      al.nscn = (int)n;
      al.tiles = fb.tiles;
      al.ntiles = fb.ntiles;
      al.Tmax = fb.Tmax;
      al.ckpt_steps = b->ckpt_k;
      al.status = d0.status;
      al.barrier = d0.barrier;
      B_CUDA(batch_mark(b, CT_PHASE_MEASURE));
      B_CUDA(ct::launch_adjoint_tiles(al, std::min(b->adj_grid, fb.ntiles), st));
      B_CUDA(batch_mark(b, CT_PHASE_DERIVE));
    } else {
      B_CUDA(batch_mark(b, CT_PHASE_MEASURE));
    }
  }
  // calculate_average_delays -> batch derivatives -> update -> batch metrics, per scenario
  B_CUDA(fork_side(b));
  for (size_t i = 0; i < n; ++i) {
    ct_scn* s = b->scns[i];
    DeviceScenario& d = s->d;
    const ct_algorithm& a = s->algo;
    cudaStream_t ss = side_of(i);
    B_CUDA(ct::launch_average_delays(d, ss));
    if (!a.freeze_delays && std::fabs(a.smoothness_regularization_strength) > 1.1920929e-7f)
      B_CUDA(ct::launch_smoothness(d, a.smoothness_regularization_strength, ss));
    ct::UpdateScalars u;
    u.optimizer = a.optimizer;
    u.freeze_gains = a.freeze_gains;
    u.freeze_delays = a.freeze_delays;
    u.lr_over_bs = a.learning_rate / (float)(d.T * d.B);
    u.bias1 = u.bias2 = 1.0f;
    u.bias_dev = b->epoch_dev[i].bias;
    B_CUDA(ct::launch_update(d, u, ss));
    if (!a.freeze_delays) B_CUDA(ct::launch_min_delay(d, ss));
    B_CUDA(ct::launch_batch_metrics_dev(d, &b->epoch_dev[i].batch_index, ss));
  }
  B_CUDA(join_side(b));
  B_CUDA(batch_mark(b, CT_PHASE_UPDATE));
  return cudaSuccess;
}

// (Re)builds the per-scenario device descriptors and, if possible, the epoch graph.
int batch_prepare(ct_batch* b) {
  cudaStream_t st = b->ctx->stream;
  const size_t n = b->scns.size();
  bool stale = b->exec == nullptr && b->use_graph;
  for (size_t i = 0; i < n; ++i) {
    ct_scn* s = b->scns[i];
    if (b->grad_mode == CT_GRAD_ADJOINT) {
      const int before = s->d.adj_ring;
      int rc = prepare_adjoint(s, b->ckpt_k);
      if (rc) return rc;
      if (s->d.adj_ring != before) stale = true;
    }
    if (b->captured_ring.size() == n && b->captured_ring[i] != s->d.adj_ring) stale = true;
    if (b->captured_gen.size() == n && b->captured_gen[i] != s->config_gen) stale = true;
  }
  if (b->captured_k != b->ckpt_k) stale = true;
  if (!stale && b->captured_ring.size() == n) return CT_OK;
  // descriptors
  std::vector<ct::FwdArgs> fa(n);
  std::vector<ct::AdjScn> aa(n);
  for (size_t i = 0; i < n; ++i) {
    ct_scn* s = b->scns[i];
    const ct_algorithm& a = s->algo;
    DeviceScenario& d = s->d;
    const bool adjoint = b->grad_mode == CT_GRAD_ADJOINT && (!a.freeze_gains || !a.freeze_delays);
    fa[i] = ct::forward_scenario(d, a.maximum_regularization_threshold, adjoint ? d.ckpt : nullptr, b->parts[i],
                                 b->ntiles[i]);
    ct::AdjointScalars as;
    as.mse_scaling = 1.0f / (float)d.M * a.mse_strength;
    as.reg_scaling = a.maximum_regularization_strength;
    as.threshold = a.maximum_regularization_threshold;
    as.diffreg = a.difference_regularization_strength;
    as.freeze_gains = a.freeze_gains || !adjoint;
    as.freeze_delays = a.freeze_delays || !adjoint;
    as.ap_derivative = a.ap_derivative;
    aa[i] = b->grad_mode == CT_GRAD_ADJOINT ? ct::adjoint_scenario(d, as) : ct::AdjScn{};
  }
  CT_CUDA(cudaMemcpyAsync(b->fwd_dev, fa.data(), sizeof(ct::FwdArgs) * n, cudaMemcpyHostToDevice, st), "batch upload");
  if (b->grad_mode == CT_GRAD_ADJOINT)
    CT_CUDA(cudaMemcpyAsync(b->adj_dev, aa.data(), sizeof(ct::AdjScn) * n, cudaMemcpyHostToDevice, st),
            "batch upload");
  CT_CUDA(cudaStreamSynchronize(st), "batch upload");
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_kernels = 0;
  if (b->use_graph) {
    cudaError_t err = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      cudaError_t body = batch_enqueue_epoch(b);
      cudaGraph_t g = nullptr;
      err = cudaStreamEndCapture(st, &g);
      if (body == cudaSuccess && err == cudaSuccess && g) {
        err = cudaGraphInstantiate(&b->exec, g, 0);
        b->graph = g;
        if (err == cudaSuccess) {
          size_t count = 0;
          cudaGraphGetNodes(g, nullptr, &count);
          std::vector<cudaGraphNode_t> nodes(count);
          cudaGraphGetNodes(g, nodes.data(), &count);
          for (cudaGraphNode_t nd : nodes) {
            cudaGraphNodeType ty;
            if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++b->graph_kernels;
          }
        }
      } else if (g) {
        cudaGraphDestroy(g);
      }
      if (body != cudaSuccess || err != cudaSuccess || !b->exec) {
        // capture refused (e.g. a driver without cooperative graph nodes): run the same schedule eagerly
        cudaGetLastError();
        if (b->exec) cudaGraphExecDestroy(b->exec);
        if (b->graph) cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
        b->use_graph = false;
      }
    } else {
      cudaGetLastError();
      b->use_graph = false;
    }
  }
  b->captured_k = b->ckpt_k;
  b->captured_ring.assign(n, 0);
  b->captured_gen.assign(n, 0);
  for (size_t i = 0; i < n; ++i) {
    b->captured_ring[i] = b->scns[i]->d.adj_ring;
    b->captured_gen[i] = b->scns[i]->config_gen;
  }
  return CT_OK;
}

// Tile lists per beat index. Order 0: scenarios by decreasing beat length, each scenario's tiles
// together, so that at any step the live tiles form a prefix of the list, which the round-robin
// tile -> CTA assignment (CTA c takes tiles c, c + G, ...) spreads evenly. Order 1: the same list
// folded back and forth over the adjoint grid (chunk k of G tiles reversed when k is odd), so that
// no CTA always gets the first tile of a chunk. Order 2: scenarios by decreasing beat length, their
// tiles interleaved one at a time.
int batch_build_tiles(ct_batch* b, bool upload) {
  const size_t n = b->scns.size();
  std::vector<size_t> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return b->scns[x]->d.T > b->scns[y]->d.T; });
  b->beat_tiles.assign((size_t)b->nbeats_max, {});
  b->beat_tmax.assign((size_t)b->nbeats_max, 0);
  for (int beat = 0; beat < b->nbeats_max; ++beat) {
    std::vector<int2>& tl = b->beat_tiles[(size_t)beat];
    if (b->tile_order == 2) {
      for (int t = 0;; ++t) {
        bool any = false;
        for (size_t i : order) {
          DeviceScenario& d = b->scns[i]->d;
          if (beat >= d.B || t >= b->ntiles[i]) continue;
          tl.push_back(make_int2((int)i, t * ct::kFwdTileVoxels));
          any = true;
        }
        if (!any) break;
      }
    } else {
      for (size_t i : order) {
        DeviceScenario& d = b->scns[i]->d;
        if (beat >= d.B) continue;
        for (int t = 0; t < b->ntiles[i]; ++t) tl.push_back(make_int2((int)i, t * ct::kFwdTileVoxels));
      }
      if (b->tile_order == 1 && b->adj_grid > 0) {
        const size_t G = (size_t)b->adj_grid;
        for (size_t k = 1; k * G < tl.size(); k += 2)
          std::reverse(tl.begin() + (ptrdiff_t)(k * G), tl.begin() + (ptrdiff_t)std::min(tl.size(), (k + 1) * G));
      }
    }
    for (const int2& t : tl)
      b->beat_tmax[(size_t)beat] = std::max<int>(b->beat_tmax[(size_t)beat], (int)b->scns[(size_t)t.x]->d.T);
  }
  if (upload)
    for (int beat = 0; beat < b->nbeats_max; ++beat) {
      const auto& tl = b->beat_tiles[(size_t)beat];
      CT_CUDA(cudaMemcpy(b->beat_tiles_dev[(size_t)beat], tl.data(), sizeof(int2) * tl.size(), cudaMemcpyHostToDevice),
              "batch tiles");
    }
  return CT_OK;
}

}  // namespace

extern "C" {

int ct_batch_create(ct_ctx* ctx, ct_scn* const* scenarios, int64_t count, int grad_mode, int precision,
                    ct_batch** out) {
  if (!ctx || !scenarios || !out || count <= 0) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument or empty batch");
  *out = nullptr;
  if (grad_mode != CT_GRAD_REFERENCE && grad_mode != CT_GRAD_ADJOINT)
    return fail(CT_ERR_NOT_SUPPORTED, "gradient mode %d", grad_mode);
  if (!valid_precision(precision)) return fail(CT_ERR_NOT_SUPPORTED, "precision %d", precision);
  for (int64_t i = 0; i < count; ++i) {
    ct_scn* s = scenarios[i];
    if (!s) return fail(CT_ERR_INVALID_ARGUMENT, "scenario %lld is NULL", (long long)i);
    if (s->ctx != ctx) return fail(CT_ERR_INVALID_ARGUMENT, "scenario %lld belongs to another context", (long long)i);
    if (s->algo.batch_size != 0)
      return fail(CT_ERR_NOT_SUPPORTED, "scenario %lld: batches need batch_size 0 (one update per epoch)",
                  (long long)i);
    for (int64_t j = 0; j < i; ++j)
      if (scenarios[j] == s) return fail(CT_ERR_INVALID_ARGUMENT, "scenario %lld appears twice", (long long)i);
  }
  CT_DEVICE_SCOPE(ctx->device);
  if (precision == CT_PREC_BF16X6)  // slice every member's H before the epoch graph is captured
    for (int64_t i = 0; i < count; ++i)
      if (scenarios[i]->d.umma) {
        int rc0 = prepare_sliced(scenarios[i]);
        if (rc0) return rc0;
      }
  if (precision == CT_PREC_TF32X3 || precision == CT_PREC_TF32)  // the members' gradient check
    for (int64_t i = 0; i < count; ++i)
      if (scenarios[i]->d.umma) {
        int rc0 = check_tf32_gradients(scenarios[i], precision);
        if (rc0) return rc0;
      }
  ct_batch* b = new ct_batch;
  b->ctx = ctx;
  b->grad_mode = grad_mode;
  b->precision = precision;
  b->scns.assign(scenarios, scenarios + count);
  const size_t n = b->scns.size();
  int rc = CT_OK;
  b->ntiles.resize(n);
  for (size_t i = 0; i < n; ++i) {
    DeviceScenario& d = b->scns[i]->d;
    b->ntiles[i] = (int)((d.V + ct::kFwdTileVoxels - 1) / ct::kFwdTileVoxels);
    b->nbeats_max = std::max<int>(b->nbeats_max, (int)d.B);
  }
  b->fwd_grid = ct::forward_batch_capacity(ctx->device);
  b->adj_grid = ct::adjoint_capacity(ctx->device);
  batch_build_tiles(b, false);
  void* p = nullptr;
  rc = batch_alloc(b, &p, sizeof(ct::FwdArgs) * n);
  b->fwd_dev = static_cast<ct::FwdArgs*>(p);
  if (!rc) {
    rc = batch_alloc(b, &p, sizeof(ct::AdjScn) * n);
    b->adj_dev = static_cast<ct::AdjScn*>(p);
  }
  if (!rc) {
    rc = batch_alloc(b, &p, sizeof(EpochDev) * n);
    b->epoch_dev = static_cast<EpochDev*>(p);
  }
  for (size_t i = 0; i < n && !rc; ++i) {
    DeviceScenario& d = b->scns[i]->d;
    rc = batch_alloc(b, &p, sizeof(float) * (size_t)d.T * b->ntiles[i]);
    b->parts.push_back(static_cast<float*>(p));
  }
  for (int beat = 0; beat < b->nbeats_max && !rc; ++beat) {
    const auto& tl = b->beat_tiles[(size_t)beat];
    rc = batch_alloc(b, &p, sizeof(int2) * tl.size());
    b->beat_tiles_dev.push_back(static_cast<int2*>(p));
    if (!rc) {
      cudaError_t e = cudaMemcpy(p, tl.data(), sizeof(int2) * tl.size(), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) rc = cuda_fail(e, "batch tiles");
    }
  }
  const int nside = (int)std::min<size_t>(n, 8);
  for (int i = 0; i < nside && !rc; ++i) {
    cudaStream_t s = nullptr;
    cudaEvent_t e1 = nullptr, e2 = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&e1, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&e2, cudaEventDisableTiming);
    if (e != cudaSuccess) rc = cuda_fail(e, "batch streams");
    if (s) b->side.push_back(s);
    if (e1) b->fork_ev.push_back(e1);
    if (e2) b->join_ev.push_back(e2);
  }
  if (rc) {
    batch_free(b);
    delete b;
    return rc;
  }
  ctx->refs += 1;
  *out = b;
  return CT_OK;
}

int ct_batch_destroy(ct_batch* b) {
  if (!b) return CT_OK;
  ct_ctx* ctx = b->ctx;
  DeviceScope device_scope__(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  batch_free(b);
  delete b;
  ctx_release(ctx);
  return CT_OK;
}

int ct_batch_run_epoch(ct_batch* b, int64_t* batch_indices) {
  if (!b || !batch_indices) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  CT_DEVICE_SCOPE(b->ctx->device);
  const size_t n = b->scns.size();
  for (size_t i = 0; i < n; ++i) {
    ct_scn* s = b->scns[i];
    if (s->algo.batch_size != 0)
      return fail(CT_ERR_NOT_SUPPORTED, "scenario %zu: batches need batch_size 0 (one update per epoch)", i);
    if (batch_indices[i] < 0 || batch_indices[i] >= s->d.NB)
      return fail(CT_ERR_BATCH_INDEX, "scenario %zu: batch index %lld outside the %lld batch-wise metric slots", i,
                  (long long)batch_indices[i], (long long)s->d.NB);
  }
  int rc = batch_prepare(b);
  if (rc) return rc;
  std::vector<EpochDev> ep(n);
  for (size_t i = 0; i < n; ++i) {
    ct_scn* s = b->scns[i];
    ep[i].bias[0] = 1.0f - powf(0.9f, (float)s->adam_step);
    ep[i].bias[1] = 1.0f - powf(0.999f, (float)s->adam_step);
    ep[i].batch_index = batch_indices[i];
  }
  cudaStream_t st = b->ctx->stream;
  // pageable source: the copy is staged before the call returns, so `ep` may go out of scope
  CT_CUDA(cudaMemcpyAsync(b->epoch_dev, ep.data(), sizeof(EpochDev) * n, cudaMemcpyHostToDevice, st),
          "batch epoch scalars");
  if (b->exec && !b->profiling) {
    CT_CUDA(cudaGraphLaunch(b->exec, st), "cudaGraphLaunch");
  } else {
    CT_CUDA(batch_enqueue_epoch(b), "batch epoch");
  }
  for (size_t i = 0; i < n; ++i) {
    ct_scn* s = b->scns[i];
    s->adam_step += 1;
    batch_indices[i] += 1;
    if (!s->algo.freeze_delays) note_delay_update(s, st);
  }
  return CT_OK;
}

int ct_batch_autotune(ct_batch* b, int64_t* batch_indices, int* ckpt_k, int* tile_order, double* best_ms) {
  if (!b || !batch_indices) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  CT_DEVICE_SCOPE(b->ctx->device);
  cudaStream_t st = b->ctx->stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CT_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
  CT_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
  const bool was_profiling = b->profiling;
  b->profiling = false;
  auto trial = [&](int k, int order, double* ms) -> int {
    b->ckpt_k = k;
    b->tile_order = order;
    int rc = batch_build_tiles(b, true);
    if (rc) return rc;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->captured_ring.clear();
    rc = batch_prepare(b);  // re-layout for k, capture
    if (rc) return rc;
    CT_CUDA(cudaStreamSynchronize(st), "autotune");
    CT_CUDA(cudaEventRecord(e0, st), "cudaEventRecord");
    rc = ct_batch_run_epoch(b, batch_indices);
    if (rc) return rc;
    CT_CUDA(cudaEventRecord(e1, st), "cudaEventRecord");
    rc = ct_batch_sync(b);
    if (rc) return rc;
    float t = 0.0f;
    CT_CUDA(cudaEventElapsedTime(&t, e0, e1), "cudaEventElapsedTime");
    *ms = t;
    return CT_OK;
  };
  int best_k = b->ckpt_k, best_o = b->tile_order;
  double best = 1e300;
  int rc = CT_OK;
  const int ks[3] = {32, 64, 128};
  for (int k : ks) {
    double ms = 0.0;
    if (b->grad_mode != CT_GRAD_ADJOINT && k != kBatchCkptSteps) continue;  // the interval only matters for adjoint
    rc = trial(k, 0, &ms);
    if (rc) break;
    if (ms < best) best = ms, best_k = k, best_o = 0;
  }
  for (int o = 1; o <= 2 && !rc; ++o) {
    double ms = 0.0;
    rc = trial(best_k, o, &ms);
    if (rc) break;
    if (ms < best) best = ms, best_o = o;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->profiling = was_profiling;
  if (rc) return rc;
  b->ckpt_k = best_k;
  b->tile_order = best_o;
  rc = batch_build_tiles(b, true);
  if (rc) return rc;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->captured_ring.clear();
  if (ckpt_k) *ckpt_k = best_k;
  if (tile_order) *tile_order = best_o;
  if (best_ms) *best_ms = best;
  return CT_OK;
}

int ct_batch_sync(ct_batch* b) {
  if (!b) return fail(CT_ERR_INVALID_ARGUMENT, "batch is NULL");
  for (ct_scn* s : b->scns) {
    int rc = ct_sync(s);
    if (rc) return rc;
  }
  return CT_OK;
}

int ct_batch_set_profiling(ct_batch* b, int enable) {
  if (!b) return fail(CT_ERR_INVALID_ARGUMENT, "batch is NULL");
  b->profiling = enable != 0;
  for (double& m : b->phase_ms) m = 0.0;
  return CT_OK;
}

int ct_batch_read_profile(ct_batch* b, double* ms) {
  if (!b || !ms) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  CT_DEVICE_SCOPE(b->ctx->device);
  CT_CUDA(cudaStreamSynchronize(b->ctx->stream), "cudaStreamSynchronize");
  for (auto& pe : b->pending) {
    float t = 0.0f;
    CT_CUDA(cudaEventElapsedTime(&t, pe.start, pe.stop), "cudaEventElapsedTime");
    b->phase_ms[pe.phase] += t;
    cudaEventDestroy(pe.start);
    cudaEventDestroy(pe.stop);
  }
  b->pending.clear();
  if (b->open_event) cudaEventDestroy(b->open_event);
  b->open_event = nullptr;
  for (int i = 0; i < CT_PHASE_COUNT; ++i) ms[i] = b->phase_ms[i];
  return CT_OK;
}

int ct_batch_info(ct_batch* b, int64_t* graph_kernels, int* uses_graph, int* forward_ctas, int* adjoint_ctas) {
  if (!b) return fail(CT_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (graph_kernels) *graph_kernels = b->graph_kernels;
  if (uses_graph) *uses_graph = b->exec != nullptr ? 1 : 0;
  if (forward_ctas) *forward_ctas = b->fwd_grid;
  if (adjoint_ctas) *adjoint_ctas = b->adj_grid;
  return CT_OK;
}

}  // extern "C"

// ---- the callers either side of the epoch: the scenario loop and the post-run metrics

namespace {

static_assert(sizeof(ct_final_metrics) == sizeof(float) * (4 * CT_THRESHOLDS + 5),
              "ct_final_metrics is a plain float array on the device");

// Post-run buffers: the scan partials always, the spherical arrays when `arrays`.
int ensure_post(ct_scn* s, bool arrays) {
  DeviceScenario& d = s->d;
  ct::PostBuffers& b = s->post;
  int rc = CT_OK;
  if (!b.inv) {
    s->post_plan = ct::post_plan(d.V, d.T, s->ctx->num_sms);
    const int64_t np = (int64_t)s->post_plan.parts * d.V;
    if (!rc) rc = alloc(s, &b.inv, d.V);
    if (!rc) rc = upload(s, b.inv, s->inv.data(), sizeof(int32_t) * (size_t)d.V);
    if (!rc) rc = alloc(s, &b.maxmag, d.V);
    if (!rc) rc = alloc(s, &b.part_val, np);
    if (!rc) rc = alloc(s, &b.part_idx, np);
    if (rc) {
      release(s, b.inv);
      release(s, b.maxmag);
      release(s, b.part_val);
      release(s, b.part_idx);
      b = ct::PostBuffers{};
      return rc;
    }
  }
  if (arrays && !b.mag) {
    float** big[] = {&b.mag, &b.theta, &b.phi};
    float** small[] = {&b.mag_max, &b.theta_max, &b.phi_max, &b.activation_ms};
    for (float** p : big)
      if (!rc) rc = alloc(s, p, d.T * d.V);
    for (float** p : small)
      if (!rc) rc = alloc(s, p, d.V);
    if (rc) {
      for (float** p : big) release(s, *p), *p = nullptr;
      for (float** p : small) release(s, *p), *p = nullptr;
    }
  }
  return rc;
}

// Snapshot slots for `n` snapshots (re-allocated only when more are needed).
int ensure_snapshots(ct_scn* s, int64_t n) {
  s->snap_n = 0;
  if (n <= s->snap_cap) return CT_OK;
  DeviceScenario& d = s->d;
  release(s, s->snap_gains);
  release(s, s->snap_coefs);
  release(s, s->snap_delays);
  release(s, s->snap_X);
  release(s, s->snap_Y);
  s->snap_gains = s->snap_coefs = s->snap_X = s->snap_Y = nullptr;
  s->snap_delays = nullptr;
  s->snap_cap = 0;
  int rc = alloc(s, &s->snap_gains, n * d.S * kGainCols);
  if (!rc) rc = alloc(s, &s->snap_coefs, n * d.V * kOffsets);
  if (!rc) rc = alloc(s, &s->snap_delays, n * d.V * kOffsets);
  if (!rc) rc = alloc(s, &s->snap_X, n * d.T * d.S);
  if (!rc) rc = alloc(s, &s->snap_Y, n * d.B * d.T * d.M);
  if (!rc) s->snap_cap = n;
  return rc;
}

// Snapshots::push (results.rs:224-247): parameters after the epoch's update, states and predicted
// measurements of its last beat, stored in slot `i` (device order, converted on read).
int push_snapshot(ct_scn* s, int64_t i) {
  DeviceScenario& d = s->d;
  cudaStream_t st = s->ctx->stream;
  const size_t f = sizeof(float);
  CT_CUDA(cudaMemcpyAsync(s->snap_gains + i * d.S * kGainCols, d.gains, f * d.S * kGainCols,
                          cudaMemcpyDeviceToDevice, st), "snapshot");
  CT_CUDA(cudaMemcpyAsync(s->snap_coefs + i * d.V * kOffsets, d.coefs, f * d.V * kOffsets, cudaMemcpyDeviceToDevice, st),
          "snapshot");
  CT_CUDA(cudaMemcpyAsync(s->snap_delays + i * d.V * kOffsets, d.delays, sizeof(int32_t) * d.V * kOffsets,
                          cudaMemcpyDeviceToDevice, st), "snapshot");
  CT_CUDA(cudaMemcpyAsync(s->snap_X + i * d.T * d.S, d.X, f * d.T * d.S, cudaMemcpyDeviceToDevice, st), "snapshot");
  CT_CUDA(cudaMemcpyAsync(s->snap_Y + i * d.B * d.T * d.M, d.Y, f * d.B * d.T * d.M, cudaMemcpyDeviceToDevice, st),
          "snapshot");
  return CT_OK;
}

// Enqueues the read-back of the three batch losses at slot batch_index - 1 (the summary fields
// run_model_based copies after every epoch, scenario.rs:753-756).
int enqueue_summary_read(ct_scn* s, int64_t batch_index, float* out3) {
  DeviceScenario& d = s->d;
  if (batch_index < 1 || batch_index > d.NB)
    return fail(CT_ERR_BATCH_INDEX, "batch index %lld outside the %lld slots", (long long)batch_index, (long long)d.NB);
  cudaStream_t st = s->ctx->stream;
  const int64_t i = batch_index - 1;
  CT_CUDA(cudaMemcpyAsync(out3 + 0, d.loss_b + i, sizeof(float), cudaMemcpyDeviceToHost, st), "summary");
  CT_CUDA(cudaMemcpyAsync(out3 + 1, d.loss_mse_b + i, sizeof(float), cudaMemcpyDeviceToHost, st), "summary");
  CT_CUDA(cudaMemcpyAsync(out3 + 2, d.loss_mr_b + i, sizeof(float), cudaMemcpyDeviceToHost, st), "summary");
  return CT_OK;
}

int check_run_config(const ct_run_config* c) {
  if (c->epochs < 0) return fail(CT_ERR_INVALID_ARGUMENT, "negative epochs");
  if (c->learning_rate_reduction_interval < 0) return fail(CT_ERR_INVALID_ARGUMENT, "negative reduction interval");
  if (c->snapshots_interval < 0) return fail(CT_ERR_INVALID_ARGUMENT, "negative snapshots interval");
  return CT_OK;
}

// Learning rate of epoch `e` given the running rate of epoch e-1 (scenario.rs:737-747).
float scheduled_rate(const ct_run_config* c, int64_t e, float running, float original) {
  float lr = running;
  if (e == 0)
    lr = 0.0f;
  else if (e == 1)
    lr = original;
  if (c->learning_rate_reduction_interval != 0 && e % c->learning_rate_reduction_interval == 0)
    lr = lr * c->learning_rate_reduction_factor;
  return lr;
}

}  // namespace

extern "C" {

int ct_run_model_based(ct_scn* scn, const ct_run_config* cfg, const int32_t* beat_orders, int64_t* batch_index,
                       float* epoch_losses, ct_run_summary* summary) {
  if (!scn || !cfg || !batch_index || !summary) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  int rc = check_run_config(cfg);
  if (rc) return rc;
  CT_DEVICE_SCOPE(scn->ctx->device);
  *summary = ct_run_summary{};
  const int64_t nsnap = cfg->snapshots_interval == 0 ? 0 : cfg->epochs / cfg->snapshots_interval + 1;
  rc = ensure_snapshots(scn, nsnap);
  if (rc) return rc;
  const float original = scn->algo.learning_rate;
  float lr = original;
  float host[3] = {0.0f, 0.0f, 0.0f};
  for (int64_t e = 0; e < cfg->epochs && !rc; ++e) {
    lr = scheduled_rate(cfg, e, lr, original);
    ct_set_learning_rate(scn, lr);
    const int32_t* order = beat_orders ? beat_orders + e * scn->d.B : nullptr;
    rc = ct_run_epoch(scn, batch_index, order, cfg->grad_mode, cfg->precision);
    if (!rc) rc = enqueue_summary_read(scn, *batch_index, host);
    const bool snap = cfg->snapshots_interval != 0 && e % cfg->snapshots_interval == 0;
    if (!rc && snap) rc = push_snapshot(scn, scn->snap_n);
    if (!rc) rc = ct_sync(scn);
    if (rc) break;
    if (snap) scn->snap_n += 1;
    summary->epochs_run = e + 1;
    summary->loss = host[0];
    summary->loss_mse = host[1];
    summary->loss_maximum_regularization = host[2];
    if (epoch_losses) std::memcpy(epoch_losses + 3 * e, host, sizeof(host));
    if (!std::isnormal(host[0])) break;  // the algorithm diverged (scenario.rs:778-781)
  }
  summary->snapshots = scn->snap_n;
  ct_set_learning_rate(scn, original);
  if (rc) return rc;
  // calculate_average_delays of the final parameters (scenario.rs:783-790)
  CT_CUDA(ct::launch_average_delays(scn->d, scn->ctx->stream), "average delays kernel");
  scn->launches += 1;
  return ct_sync(scn);
}

int ct_batch_run_model_based(ct_batch* batch, const ct_run_config* cfg, int64_t* batch_indices, float* epoch_losses,
                             ct_run_summary* summaries) {
  if (!batch || !cfg || !batch_indices || !summaries) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  int rc = check_run_config(cfg);
  if (rc) return rc;
  if (cfg->snapshots_interval != 0) return fail(CT_ERR_NOT_SUPPORTED, "batched runs store no snapshots");
  if (cfg->grad_mode != batch->grad_mode || cfg->precision != batch->precision)
    return fail(CT_ERR_INVALID_ARGUMENT, "the batch was created with another gradient mode or precision");
  CT_DEVICE_SCOPE(batch->ctx->device);
  const size_t n = batch->scns.size();
  std::vector<float> original(n), lr(n), host(3 * n, 0.0f);
  for (size_t i = 0; i < n; ++i) {
    original[i] = lr[i] = batch->scns[i]->algo.learning_rate;
    summaries[i] = ct_run_summary{};
  }
  std::vector<size_t> members(n);  // batch member index of each scenario of `cur`
  for (size_t i = 0; i < n; ++i) members[i] = i;
  ct_batch* cur = batch;
  ct_batch* sub = nullptr;  // smaller batch once a member has stopped
  std::vector<int64_t> idx;
  for (int64_t e = 0; e < cfg->epochs && !rc && !members.empty(); ++e) {
    for (size_t i : members) {
      lr[i] = scheduled_rate(cfg, e, lr[i], original[i]);
      ct_set_learning_rate(batch->scns[i], lr[i]);
    }
    idx.resize(members.size());
    for (size_t k = 0; k < members.size(); ++k) idx[k] = batch_indices[members[k]];
    rc = ct_batch_run_epoch(cur, idx.data());
    for (size_t k = 0; k < members.size() && !rc; ++k) {
      batch_indices[members[k]] = idx[k];
      rc = enqueue_summary_read(batch->scns[members[k]], idx[k], host.data() + 3 * members[k]);
    }
    if (!rc) rc = ct_batch_sync(cur);
    if (rc) break;
    std::vector<size_t> still;
    for (size_t i : members) {
      const float* h = host.data() + 3 * i;
      summaries[i].epochs_run = e + 1;
      summaries[i].loss = h[0];
      summaries[i].loss_mse = h[1];
      summaries[i].loss_maximum_regularization = h[2];
      if (epoch_losses) std::memcpy(epoch_losses + (i * (size_t)cfg->epochs + (size_t)e) * 3, h, 3 * sizeof(float));
      if (std::isnormal(h[0])) still.push_back(i);
    }
    if (still.size() != members.size() && !still.empty() && e + 1 < cfg->epochs) {
      // members whose loss stopped being normal leave; the others go on as a smaller batch
      std::vector<ct_scn*> scns;
      for (size_t i : still) scns.push_back(batch->scns[i]);
      ct_batch* nb = nullptr;
      rc = ct_batch_create(batch->ctx, scns.data(), (int64_t)scns.size(), batch->grad_mode, batch->precision, &nb);
      if (!rc) {
        nb->ckpt_k = batch->ckpt_k;
        nb->tile_order = batch->tile_order;
        rc = batch_build_tiles(nb, true);
      }
      if (sub) ct_batch_destroy(sub);
      sub = nb;
      cur = nb;
    }
    members.swap(still);
  }
  if (sub) ct_batch_destroy(sub);
  for (size_t i = 0; i < n; ++i) ct_set_learning_rate(batch->scns[i], original[i]);
  if (rc) return rc;
  for (ct_scn* s : batch->scns) {
    CT_CUDA(ct::launch_average_delays(s->d, s->ctx->stream), "average delays kernel");
    s->launches += 1;
  }
  return ct_batch_sync(batch);
}

int ct_calculate_plotting_arrays(ct_scn* scn, float sample_rate_hz) {
  if (!scn) return fail(CT_ERR_INVALID_ARGUMENT, "scenario is NULL");
  CT_DEVICE_SCOPE(scn->ctx->device);
  int rc = ensure_post(scn, true);
  if (rc) return rc;
  CT_CUDA(ct::launch_spherical(scn->d, scn->post, scn->post_plan, true, sample_rate_hz, scn->ctx->stream),
          "spherical kernels");
  scn->launches += 2;
  rc = ct_sync(scn);
  if (rc == CT_OK || rc == CT_ERR_NO_MAXIMUM) scn->post_arrays = true;
  return rc;
}

int ct_calculate_final(ct_scn* scn, const int32_t* ground_truth_types, const int32_t* voxel_numbers, int64_t nx,
                       int64_t ny, int64_t nz, ct_final_metrics* out) {
  if (!scn || !ground_truth_types || !voxel_numbers || !out) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (nx <= 0 || ny <= 0 || nz <= 0) return fail(CT_ERR_INVALID_ARGUMENT, "empty grid");
  const int64_t cells = nx * ny * nz;
  const DeviceScenario& d = scn->d;
  for (int64_t g = 0; g < cells; ++g) {
    const int32_t num = voxel_numbers[g];
    if (num != -1 && (num < 0 || num >= d.S || num % 3 != 0))
      return fail(CT_ERR_INVALID_ARGUMENT, "voxel number %d of cell %lld is not a state index of this scenario",
                  num, (long long)g);
  }
  CT_DEVICE_SCOPE(scn->ctx->device);
  int rc = ensure_post(scn, false);
  if (rc) return rc;
  if (!scn->final_hist) {
    rc = alloc(scn, &scn->final_hist, 2 * (CT_THRESHOLDS + 1));
    if (!rc) rc = alloc(scn, &scn->final_out, (int64_t)(sizeof(ct_final_metrics) / sizeof(float)));
    if (rc) return rc;
  }
  if (cells > scn->final_cells) {
    release(scn, scn->final_grid);
    scn->final_grid = nullptr;
    scn->final_cells = 0;
    rc = alloc(scn, &scn->final_grid, 2 * cells);
    if (rc) return rc;
    scn->final_cells = cells;
  }
  cudaStream_t st = scn->ctx->stream;
  const size_t grid_bytes = sizeof(int32_t) * (size_t)cells;
  int32_t* types = scn->final_grid;
  int32_t* numbers = scn->final_grid + cells;
  cudaError_t e = cudaMemcpyAsync(types, ground_truth_types, grid_bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(numbers, voxel_numbers, grid_bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = ct::launch_spherical(d, scn->post, scn->post_plan, false, 1.0f, st);
  if (e == cudaSuccess)
    e = ct::launch_final_metrics(scn->post, types, numbers, cells, scn->final_hist, scn->final_out,
                                 scn->ctx->num_sms, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, scn->final_out, sizeof(ct_final_metrics), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return cuda_fail(e, "final metrics");
  scn->launches += 4;
  return ct_sync(scn);
}


// ---- model construction on the device

}  // extern "C"

namespace {

// Device buffers of one model-construction call, freed on every return path (cudaFree waits for
// the device, so nothing in flight still uses them).
struct TempBuffers {
  std::vector<void*> ptrs;
  ~TempBuffers() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  cudaError_t get(T** p, int64_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * (size_t)(count > 0 ? count : 1));
    if (e == cudaSuccess) {
      ptrs.push_back(q);
      *p = static_cast<T*>(q);
    }
    return e;
  }
};

bool is_connectable(int32_t t) { return t >= 1 && t <= 6; }  // voxels.rs:690-700

// The voxel grid of a spatial description: connectable cells must carry the voxel numbers
// 0, 3, .., S-3 once each (the reference's numbering, voxels.rs:407-424). cell_of[v] = the cell
// of voxel v.
int check_grid(const ct_spatial_desc* g, std::vector<int64_t>& cell_of) {
  if (!g->voxel_types || !g->voxel_numbers || !g->voxel_positions_mm)
    return fail(CT_ERR_INVALID_ARGUMENT, "a voxel grid array is NULL");
  if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0) return fail(CT_ERR_INVALID_ARGUMENT, "empty voxel grid");
  if (g->nx * g->ny >= (int64_t(1) << 31) || g->nx * g->ny * g->nz >= (int64_t(1) << 31) / kOffsets)
    return fail(CT_ERR_NOT_SUPPORTED, "voxel grid too large");
  const int64_t cells = g->nx * g->ny * g->nz;
  int64_t V = 0;
  for (int64_t c = 0; c < cells; ++c) V += is_connectable(g->voxel_types[c]) ? 1 : 0;
  if (V == 0) return fail(CT_ERR_INVALID_ARGUMENT, "the voxel grid has no connectable voxel");
  cell_of.assign((size_t)V, -1);
  for (int64_t c = 0; c < cells; ++c) {
    if (!is_connectable(g->voxel_types[c])) continue;
    const int32_t num = g->voxel_numbers[c];
    if (num < 0 || num % 3 != 0 || num / 3 >= V || cell_of[(size_t)(num / 3)] >= 0)
      return fail(CT_ERR_INVALID_ARGUMENT,
                  "voxel number %d of connectable cell %lld: connectable cells must number 0, 3, .., %lld once each",
                  num, (long long)c, (long long)(3 * V - 3));
    cell_of[(size_t)(num / 3)] = c;
  }
  return CT_OK;
}

int check_sensors(const ct_spatial_desc* g) {
  if (!g->sensor_positions_mm || !g->sensor_orientations || !g->sensor_array_offsets_mm)
    return fail(CT_ERR_INVALID_ARGUMENT, "a sensor array is NULL");
  if (g->num_sensors <= 0 || g->num_beats <= 0)
    return fail(CT_ERR_INVALID_ARGUMENT, "num_sensors and num_beats must be positive");
  return CT_OK;
}

// H [B, M, ldh] on the device from a voxel list (vpos[i], first column col[i]).
int fill_lead_field(ct_ctx* ctx, const ct_spatial_desc* g, const std::vector<float>& vpos,
                    const std::vector<int32_t>& col, float* H, int64_t ldh) {
  const int64_t nv = (int64_t)col.size(), M = g->num_sensors, B = g->num_beats;
  cudaStream_t st = ctx->stream;
  TempBuffers tb;
  float *dv = nullptr, *dsp = nullptr, *dso = nullptr, *doff = nullptr;
  int32_t* dc = nullptr;
  CT_CUDA(tb.get(&dv, 3 * nv), "cudaMalloc");
  CT_CUDA(tb.get(&dc, nv), "cudaMalloc");
  CT_CUDA(tb.get(&dsp, 3 * M), "cudaMalloc");
  CT_CUDA(tb.get(&dso, 3 * M), "cudaMalloc");
  CT_CUDA(tb.get(&doff, 3 * B), "cudaMalloc");
  CT_CUDA(cudaMemcpyAsync(dv, vpos.data(), sizeof(float) * vpos.size(), cudaMemcpyHostToDevice, st), "upload");
  CT_CUDA(cudaMemcpyAsync(dc, col.data(), sizeof(int32_t) * col.size(), cudaMemcpyHostToDevice, st), "upload");
  CT_CUDA(cudaMemcpyAsync(dsp, g->sensor_positions_mm, sizeof(float) * 3 * M, cudaMemcpyHostToDevice, st), "upload");
  CT_CUDA(cudaMemcpyAsync(dso, g->sensor_orientations, sizeof(float) * 3 * M, cudaMemcpyHostToDevice, st), "upload");
  CT_CUDA(cudaMemcpyAsync(doff, g->sensor_array_offsets_mm, sizeof(float) * 3 * B, cudaMemcpyHostToDevice, st),
          "upload");
  CT_CUDA(ct::launch_lead_field(dv, dc, nv, dsp, dso, doff, M, B, ct::lead_field_factor(g->voxel_size_mm), H, ldh,
                                ctx->num_sms, st),
          "lead field kernel");
  CT_CUDA(cudaStreamSynchronize(st), "lead field");
  return CT_OK;
}

}  // namespace

extern "C" {

int ct_measurement_matrix(ct_ctx* ctx, const ct_spatial_desc* desc, float* out, size_t nbytes) {
  if (!ctx || !desc || !out) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::vector<int64_t> cell_of;
  int rc = check_grid(desc, cell_of);
  if (!rc) rc = check_sensors(desc);
  if (rc) return rc;
  const int64_t V = (int64_t)cell_of.size(), S = 3 * V, M = desc->num_sensors, B = desc->num_beats;
  if (B * M * S >= (int64_t(1) << 40)) return fail(CT_ERR_NOT_SUPPORTED, "measurement matrix too large");
  const size_t want = sizeof(float) * (size_t)(B * M * S);
  if (nbytes != want) return fail(CT_ERR_INVALID_ARGUMENT, "measurement matrix has %zu bytes, got %zu", want, nbytes);
  std::vector<float> vpos((size_t)(3 * V));
  std::vector<int32_t> col((size_t)V);
  for (int64_t v = 0; v < V; ++v) {
    for (int k = 0; k < 3; ++k) vpos[(size_t)(3 * v + k)] = desc->voxel_positions_mm[3 * cell_of[(size_t)v] + k];
    col[(size_t)v] = (int32_t)(3 * v);
  }
  CT_DEVICE_SCOPE(ctx->device);
  TempBuffers tb;
  float* dH = nullptr;
  CT_CUDA(tb.get(&dH, B * M * S), "cudaMalloc");
  rc = fill_lead_field(ctx, desc, vpos, col, dH, S);
  if (rc) return rc;
  CT_CUDA(cudaMemcpyAsync(out, dH, want, cudaMemcpyDeviceToHost, ctx->stream), "download");
  CT_CUDA(cudaStreamSynchronize(ctx->stream), "download");
  return CT_OK;
}

int ct_scenario_set_measurement_matrix(ct_scn* scn, const ct_spatial_desc* desc) {
  if (!scn || !desc) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::vector<int64_t> cell_of;
  int rc = check_grid(desc, cell_of);
  if (!rc) rc = check_sensors(desc);
  if (rc) return rc;
  DeviceScenario& d = scn->d;
  if ((int64_t)cell_of.size() != d.V || desc->num_sensors != d.M || desc->num_beats != d.B)
    return fail(CT_ERR_INVALID_ARGUMENT,
                "spatial description has %lld voxels, %lld sensors, %lld beats; the scenario %lld, %lld, %lld",
                (long long)cell_of.size(), (long long)desc->num_sensors, (long long)desc->num_beats, (long long)d.V,
                (long long)d.M, (long long)d.B);
  // voxel list in device order: device voxel u is reference voxel perm[u]
  std::vector<float> vpos((size_t)(3 * d.V));
  std::vector<int32_t> col((size_t)d.V);
  for (int64_t u = 0; u < d.V; ++u) {
    const int64_t c = cell_of[(size_t)scn->perm[(size_t)u]];
    for (int k = 0; k < 3; ++k) vpos[(size_t)(3 * u + k)] = desc->voxel_positions_mm[3 * c + k];
    col[(size_t)u] = (int32_t)(3 * u);
  }
  CT_DEVICE_SCOPE(scn->ctx->device);
  CT_CUDA(cudaStreamSynchronize(scn->ctx->stream), "scenario stream");
  rc = fill_lead_field(scn->ctx, desc, vpos, col, d.H, d.S);
  if (rc) return rc;
  scn->launches += 1;
  if (d.umma) {
    CT_CUDA(ct::umma_prepare(d, scn->ctx->stream), "tensor-core operand split");
    scn->launches += 2;
  }
  d.slice_ready = false;
  if (d.H_sl) {
    rc = prepare_sliced(scn);
    if (rc) return rc;
  }
  CT_CUDA(cudaStreamSynchronize(scn->ctx->stream), "measurement matrix");
  return CT_OK;
}

int ct_delay_samples(ct_ctx* ctx, const ct_spatial_desc* desc, float* initial_delays, int32_t* delays, float* coefs,
                     int64_t count) {
  if (!ctx || !desc || !initial_delays || !delays || !coefs || !desc->propagation_velocities_m_per_s)
    return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::vector<int64_t> cell_of;
  int rc = check_grid(desc, cell_of);
  if (rc) return rc;
  const int64_t V = (int64_t)cell_of.size(), cells = desc->nx * desc->ny * desc->nz;
  if (count != V * kOffsets)
    return fail(CT_ERR_INVALID_ARGUMENT, "delay arrays have %lld elements, got %lld", (long long)(V * kOffsets),
                (long long)count);
  CT_DEVICE_SCOPE(ctx->device);
  cudaStream_t st = ctx->stream;
  TempBuffers tb;
  int32_t *dt = nullptr, *dn = nullptr, *dd = nullptr;
  float *dp = nullptr, *dvel = nullptr, *ds = nullptr, *dcoef = nullptr;
  unsigned long long* bad = nullptr;
  CT_CUDA(tb.get(&dt, cells), "cudaMalloc");
  CT_CUDA(tb.get(&dn, cells), "cudaMalloc");
  CT_CUDA(tb.get(&dp, 3 * cells), "cudaMalloc");
  CT_CUDA(tb.get(&dvel, 10), "cudaMalloc");
  CT_CUDA(tb.get(&ds, V * kOffsets), "cudaMalloc");
  CT_CUDA(tb.get(&dd, V * kOffsets), "cudaMalloc");
  CT_CUDA(tb.get(&dcoef, V * kOffsets), "cudaMalloc");
  CT_CUDA(tb.get(&bad, 1), "cudaMalloc");
  CT_CUDA(cudaMemcpyAsync(dt, desc->voxel_types, sizeof(int32_t) * cells, cudaMemcpyHostToDevice, st), "upload");
  CT_CUDA(cudaMemcpyAsync(dn, desc->voxel_numbers, sizeof(int32_t) * cells, cudaMemcpyHostToDevice, st), "upload");
  CT_CUDA(cudaMemcpyAsync(dp, desc->voxel_positions_mm, sizeof(float) * 3 * cells, cudaMemcpyHostToDevice, st),
          "upload");
  CT_CUDA(cudaMemcpyAsync(dvel, desc->propagation_velocities_m_per_s, sizeof(float) * 10, cudaMemcpyHostToDevice, st),
          "upload");
  CT_CUDA(cudaMemsetAsync(bad, 0xFF, sizeof(unsigned long long), st), "memset");
  CT_CUDA(ct::launch_delay_samples(dt, dn, dp, desc->nx, desc->ny, desc->nz, dvel, desc->sample_rate_hz, ds, dd, dcoef,
                                   bad, ctx->num_sms, st),
          "delay samples kernel");
  unsigned long long first_bad = 0;
  CT_CUDA(cudaMemcpyAsync(&first_bad, bad, sizeof(first_bad), cudaMemcpyDeviceToHost, st), "download");
  CT_CUDA(cudaMemcpyAsync(initial_delays, ds, sizeof(float) * V * kOffsets, cudaMemcpyDeviceToHost, st), "download");
  CT_CUDA(cudaMemcpyAsync(delays, dd, sizeof(int32_t) * V * kOffsets, cudaMemcpyDeviceToHost, st), "download");
  CT_CUDA(cudaMemcpyAsync(coefs, dcoef, sizeof(float) * V * kOffsets, cudaMemcpyDeviceToHost, st), "download");
  CT_CUDA(cudaStreamSynchronize(st), "delay samples");
  if (first_bad != ~0ull) {
    const long long c = (long long)(first_bad / kOffsets), n = (long long)(first_bad % kOffsets);
    const long long z = c % desc->nz, y = c / desc->nz % desc->ny, x = c / (desc->ny * desc->nz);
    return fail(CT_ERR_INVALID_ARGUMENT,
                "can not configure delays below 1 sample (or not below 2^31): voxel (%lld, %lld, %lld), offset "
                "column %lld",
                x, y, z, n);
  }
  return CT_OK;
}

int ct_connect_voxels(const ct_spatial_desc* desc, float current_factor_in_pathology, float* gains, size_t gains_bytes,
                      float* activation_time_ms) {
  if (!desc || !gains || !activation_time_ms || !desc->propagation_velocities_m_per_s)
    return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::vector<int64_t> cell_of;
  int rc = check_grid(desc, cell_of);
  if (rc) return rc;
  const int64_t S = 3 * (int64_t)cell_of.size();
  const size_t want = sizeof(float) * (size_t)(S * kGainCols);
  if (gains_bytes != want) return fail(CT_ERR_INVALID_ARGUMENT, "gains have %zu bytes, got %zu", want, gains_bytes);
  std::fill(gains, gains + S * kGainCols, 0.0f);
  ct::connect_voxels_host(desc->voxel_types, desc->voxel_numbers, desc->voxel_positions_mm, desc->nx, desc->ny,
                          desc->nz, desc->propagation_velocities_m_per_s, current_factor_in_pathology, gains,
                          activation_time_ms);
  return CT_OK;
}

int ct_output_state_indices(const ct_spatial_desc* desc, int32_t* out, size_t nbytes) {
  if (!desc || !out) return fail(CT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::vector<int64_t> cell_of;
  int rc = check_grid(desc, cell_of);
  if (rc) return rc;
  const int64_t S = 3 * (int64_t)cell_of.size();
  const size_t want = sizeof(int32_t) * (size_t)(S * kGainCols);
  if (nbytes != want) return fail(CT_ERR_INVALID_ARGUMENT, "output_state_indices have %zu bytes, got %zu", want, nbytes);
  ct::output_state_indices_host(desc->voxel_types, desc->voxel_numbers, desc->nx, desc->ny, desc->nz, cell_of, out);
  return CT_OK;
}

}  // extern "C"
