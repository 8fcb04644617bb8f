/*
 * cardiotrust_cuda.h — C ABI of the B200 estimation-epoch library.
 *
 * One scenario = one CardioTrust `Results` + `Model` + `Data` triple living in
 * GPU memory. The entry points replace the reference crate's estimation epoch
 * (paths relative to the crate root):
 *
 *   ct_run_epoch          <- run_epoch                    src/core/algorithm.rs:124-129
 *   ct_run_epoch_host     <- run_epoch, model in host memory (copies in, epoch, copies out)
 *                            EpochKernel::execute         src/core/algorithm/gpu/epoch.rs:96-117
 *   ct_scenario_create    <- Results::to_gpu              src/core/scenario/results.rs:121-133
 *                            EpochKernel::new             src/core/algorithm/gpu/epoch.rs:29-37
 *   ct_read_field         <- Results::update_from_gpu     src/core/scenario/results.rs:136-147
 *   ct_write_field        <- Results::to_gpu (per array)  src/core/scenario/results.rs:121-133
 *   ct_set_freeze         <- EpochKernel::set_freeze_*    src/core/algorithm/gpu/epoch.rs:118-125
 *   ct_set_learning_rate  <- Algorithm::learning_rate     src/core/config/algorithm.rs:35
 *                            (mutated by the caller's schedule, src/core/scenario.rs:737-747)
 *   ct_simulate           <- Simulation::run (forward)    src/core/data/simulation.rs:129-150
 *   ct_ctx_create         <- GPU::new                     src/core/algorithm/gpu.rs:31-64
 *   ct_run_model_based    <- run_model_based              src/core/scenario.rs:725-795
 *   ct_calculate_plotting_arrays <- calculate_plotting_arrays (estimations) src/core/scenario.rs:636-690
 *   ct_calculate_final    <- metrics::calculate_final     src/core/algorithm/metrics.rs:226-242
 *                            + optimal threshold summary  src/core/scenario.rs:601-617
 *   ct_measurement_matrix <- MeasurementMatrix::from_model_spatial_description
 *                                                         src/core/model/functional/measurement.rs:66-123
 *   ct_delay_samples      <- calculate_delay_samples_array src/core/model/functional/allpass/delay.rs:35-111
 *                            (+ delays/coefs of APParameters::from_model_config, allpass.rs:86-100)
 *   ct_connect_voxels     <- connect_voxels               src/core/model/functional/allpass.rs:295-494
 *   ct_output_state_indices <- init_output_state_indicies src/core/model/functional/allpass.rs:212-289
 *
 * Conventions: every function returns a status (CT_OK = 0, negative CT_ERR_*),
 * never throws and never aborts. Host arrays passed in are copied; the caller
 * keeps ownership. Handles are not thread-safe: use one scenario per host
 * thread. All arrays are C-order, f32 unless stated, i32 for indices/delays.
 * Shapes: S states, V = S/3 voxels, M sensor rows, T steps, B beats.
 */
#ifndef CARDIOTRUST_CUDA_H
#define CARDIOTRUST_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CT_ABI_VERSION 1

enum ct_status {
  CT_OK = 0,
  CT_ERR_INVALID_ARGUMENT = -1, /* null pointer, bad shape, bad enum */
  CT_ERR_CUDA = -2,             /* a CUDA runtime call failed */
  CT_ERR_OUT_OF_MEMORY = -3,    /* device allocation failed */
  CT_ERR_TIMEOUT = -4,          /* a device-side wait hit its iteration limit */
  CT_ERR_INVALID_INDEX = -5,    /* output_state_indices lack the voxel/neighbour structure */
  CT_ERR_NOT_SUPPORTED = -6,    /* mode not available for this scenario */
  CT_ERR_BATCH_INDEX = -7,      /* batch-wise metric index outside the metric arrays */
  CT_ERR_NO_MAXIMUM = -8        /* a voxel's magnitude is NaN at every step (argmax_skipnan finds none) */
};

/* Optimizer, src/core/algorithm/refinement.rs:8-12 */
enum ct_optimizer { CT_OPT_SGD = 0, CT_OPT_ADAM = 1 };
/* APDerivative, src/core/config/algorithm.rs:17-21 */
enum ct_ap_derivative { CT_AP_SIMPLE = 0, CT_AP_TEXTBOOK = 1 };
/* Gradient definition used by ct_run_epoch. */
enum ct_grad_mode {
  CT_GRAD_REFERENCE = 0, /* the reference's per-step derivation, derivation.rs:173-229 */
  /* Exact gradient of the stated loss sum_t (mse/M)/2 |r_t|^2 + reg/2 sum_v relu(|x_v|_1 - thr)^2
   * by back-propagation through time (no counterpart in the reference), plus the reference's
   * difference-regularisation term. All-pass state is checkpointed every 256 steps and the
   * segments in between are recomputed. Forward, metrics and update are those of mode 0. */
  CT_GRAD_ADJOINT = 1
};
/* Arithmetic of the two measurement products (H x and H^T r). */
enum ct_precision {
  CT_PREC_FP32 = 0,   /* FP32 CUDA-core GEMMs */
  CT_PREC_TF32X3 = 1, /* tcgen05 TF32 with a hi/lo split of both operands (hi*hi + hi*lo + lo*hi), FP32
                         accumulate. The tensor core's accumulation is biased toward zero: when residuals are a
                         small fraction of the signal, gradients drift ~1e-2 from the FP64 result. Guarded: see
                         below. */
  CT_PREC_TF32 = 2,   /* tcgen05 TF32, one pass (operands rounded to TF32). Guarded: see below. */
  CT_PREC_BF16X6 = 3  /* tcgen05 BF16 on error-free slices: every operand row is cut into groups of 512 values
                         sharing a power-of-two scale and split into three 8-bit integer slices (exact in BF16);
                         six slice products accumulate exactly in FP32 tensor memory and are folded into an FP32
                         sum, rounding to nearest, every 512 values. Unbiased like FP32 CUDA-core products. */
};
/* Guard of the TF32 modes: before a scenario's first epoch in CT_PREC_TF32X3 or CT_PREC_TF32 (ct_run_epoch,
 * ct_run_model_based, ct_batch_create), the first beat's reference-mode gradients are computed with the mode and
 * with CT_PREC_BF16X6. If they differ by more than 1e-3 (norm-wise relative, the gradient target), the call
 * returns CT_ERR_NOT_SUPPORTED with the measured difference in ct_last_error, and every later call in that mode
 * on that scenario does too. Parameters, derivatives, Adam state and the batch cursor are left untouched; the
 * last epoch's estimation outputs (states, predicted measurements, residuals, step metrics) are overwritten. */

/* The Algorithm fields the epoch reads, src/core/config/algorithm.rs:25-58. */
typedef struct ct_algorithm {
  int32_t optimizer;     /* ct_optimizer */
  int32_t ap_derivative; /* ct_ap_derivative */
  int32_t freeze_gains;
  int32_t freeze_delays;
  int64_t batch_size; /* 0 = one update per epoch */
  float learning_rate;
  float mse_strength;
  float maximum_regularization_strength;
  float maximum_regularization_threshold;
  float difference_regularization_strength;
  float smoothness_regularization_strength;
} ct_algorithm;

/* Host arrays describing one scenario (Model.functional_description + Data). */
typedef struct ct_scenario_desc {
  int64_t num_states;  /* S, multiple of 3 */
  int64_t num_sensors; /* M */
  int64_t num_steps;   /* T */
  int64_t num_beats;   /* B */
  int64_t num_batch_slots; /* length of the batch-wise metric arrays (epochs x batches) */
  const float* gains;                  /* [S,78]  APParameters.gains, allpass.rs:30 */
  const int32_t* output_state_indices; /* [S,78]  -1 = None, allpass.rs:31 / :146 */
  const float* coefs;                  /* [V,26]  allpass.rs:32 */
  const int32_t* delays;               /* [V,26]  allpass.rs:33 (usize, <= 1000 after roll_delays) */
  const float* initial_delays;         /* [V,26]  allpass.rs:34 */
  const float* measurement_matrix;     /* [B,M,S] measurement.rs:22; NULL = zero until ct_scenario_set_measurement_matrix */
  const float* control_matrix;         /* [S]     control.rs:23 */
  const float* control_function;       /* [T]     control.rs:142 */
  const float* measurements;           /* [B,T,M] data.simulation.measurements; may be NULL */
} ct_scenario_desc;

/* Arrays readable/writable with ct_read_field / ct_write_field. */
enum ct_field {
  /* model (read/write) */
  CT_FIELD_GAINS = 0,           /* [S,78] f32 */
  CT_FIELD_COEFS = 1,           /* [V,26] f32 */
  CT_FIELD_DELAYS = 2,          /* [V,26] i32 */
  CT_FIELD_MEASUREMENTS_ACTUAL = 3, /* [B,T,M] f32 */
  /* estimations (read) */
  CT_FIELD_SYSTEM_STATES = 10,  /* [T,S] f32 of the last beat run */
  CT_FIELD_MEASUREMENTS = 11,   /* [B,T,M] f32 predicted */
  CT_FIELD_RESIDUALS = 12,      /* [M] f32 last step */
  CT_FIELD_AP_OUTPUTS_NOW = 13, /* [S,78] f32 */
  CT_FIELD_AP_OUTPUTS_LAST = 14,/* [S,78] f32 */
  CT_FIELD_AVERAGE_DELAYS = 15, /* [V] f32, NaN = None */
  /* derivatives (read) */
  CT_FIELD_GRAD_GAINS = 20,     /* [S,78] f32 */
  CT_FIELD_GRAD_COEFS = 21,     /* [V,26] f32 */
  CT_FIELD_COEFS_FIR = 22,      /* [S,78] f32 */
  CT_FIELD_COEFS_IIR = 23,      /* [S,78] f32 */
  CT_FIELD_MAPPED_RESIDUALS = 24,     /* [S] f32 last step */
  CT_FIELD_MAXIMUM_REGULARIZATION = 25, /* [S] f32 last step */
  CT_FIELD_MAXIMUM_REGULARIZATION_SUM = 26, /* [1] f32 */
  CT_FIELD_ADAM_STEP = 27,      /* [1] i64, Derivatives.step */
  CT_FIELD_GAINS_FIRST_MOMENT = 28,  /* [S,78] */
  CT_FIELD_GAINS_SECOND_MOMENT = 29, /* [S,78] */
  CT_FIELD_COEFS_FIRST_MOMENT = 30,  /* [V,26] */
  CT_FIELD_COEFS_SECOND_MOMENT = 31, /* [V,26] */
  CT_FIELD_MAPPED_RESIDUALS_HISTORY = 32, /* [T,S] f32 H^T r of every step of the last beat */
  /* metrics (read) */
  CT_FIELD_LOSS = 40,           /* [T] */
  CT_FIELD_LOSS_MSE = 41,       /* [T] */
  CT_FIELD_LOSS_MAXIMUM_REGULARIZATION = 42, /* [T] */
  CT_FIELD_LOSS_BATCH = 43,     /* [num_batch_slots] */
  CT_FIELD_LOSS_MSE_BATCH = 44,
  CT_FIELD_LOSS_MAXIMUM_REGULARIZATION_BATCH = 45,
  /* post-run arrays of the last beat's states, reference voxel order (read; written by
   * ct_calculate_plotting_arrays, CT_ERR_INVALID_ARGUMENT before the first call) */
  CT_FIELD_STATES_MAGNITUDE = 50,      /* [T,V] SystemStatesSpherical.magnitude, shapes.rs:151-192 */
  CT_FIELD_STATES_THETA = 51,          /* [T,V] */
  CT_FIELD_STATES_PHI = 52,            /* [T,V] */
  CT_FIELD_STATES_MAGNITUDE_MAX = 53,  /* [V] SystemStatesSphericalMax, shapes.rs:242-277 */
  CT_FIELD_STATES_THETA_MAX = 54,      /* [V] */
  CT_FIELD_STATES_PHI_MAX = 55,        /* [V] */
  CT_FIELD_ACTIVATION_TIMES = 56,      /* [V] ActivationTimePerStateMs, shapes.rs:322-352 */
  /* snapshots of the last ct_run_model_based call (Snapshots, src/core/scenario/results.rs:179-248); N = the
   * number of snapshots that call allocated (epochs / snapshots_interval + 1, 0 without) */
  CT_FIELD_SNAPSHOT_GAINS = 60,        /* [N,S,78] */
  CT_FIELD_SNAPSHOT_COEFS = 61,        /* [N,V,26] */
  CT_FIELD_SNAPSHOT_DELAYS = 62,       /* [N,V,26] i32 */
  CT_FIELD_SNAPSHOT_SYSTEM_STATES = 63,/* [N,T,S] */
  CT_FIELD_SNAPSHOT_MEASUREMENTS = 64  /* [N,B,T,M] */
};

typedef struct ct_ctx ct_ctx;
typedef struct ct_scn ct_scn;

int ct_version(void);
const char* ct_status_string(int status);
/* Last error message of the calling thread (empty if none). */
int ct_last_error(char* buf, size_t len);

/* Context = device + stream. stream == NULL creates a private non-blocking stream;
 * otherwise the context issues all work on the given cudaStream_t. A destroyed context
 * stays alive until the last scenario created on it is destroyed. */
int ct_ctx_create(int device, void* stream, ct_ctx** out);
int ct_ctx_destroy(ct_ctx* ctx);
int ct_ctx_stream(ct_ctx* ctx, void** stream);

/* Copies the description to the device; Derivatives.step starts at 1 (derivation.rs:100). */
int ct_scenario_create(ct_ctx* ctx, const ct_scenario_desc* desc, const ct_algorithm* algo, ct_scn** out);
int ct_scenario_destroy(ct_scn* scn);
int ct_scenario_dims(ct_scn* scn, int64_t* S, int64_t* M, int64_t* T, int64_t* B);

/* One estimation epoch, enqueued on the context stream (asynchronous).
 * beat_order: B beat indices, or NULL for the library's seeded shuffle.
 * batch_index: in/out batch-wise metric cursor (algorithm.rs:126).
 * grad_mode: ct_grad_mode. CT_GRAD_ADJOINT allocates its checkpoint and segment buffers on
 * first use (about (T/256 + 256 * 2 + ring) x V x 78 floats) and needs every voxel pair to be
 * connected along at most one offset (true of the reference's lattice).
 * Device-side failures are reported by ct_sync. */
int ct_run_epoch(ct_scn* scn, int64_t* batch_index, const int32_t* beat_order, int grad_mode, int precision);

/* The plain GPU form of ct_run_epoch (CT_GRAD_REFERENCE, FP32 products): every phase of every
 * step is its own kernel launch with one thread per output, one scenario at a time - the
 * straightforward port of the reference's OpenCL epoch (src/core/algorithm/gpu/epoch.rs:96-117,
 * prediction/derivation/metrics kernels per step). Kept as the baseline the persistent and
 * batched forms are measured against. Same arguments, results (within tolerance) and error
 * behaviour as ct_run_epoch. */
int ct_run_epoch_plain(ct_scn* scn, int64_t* batch_index, const int32_t* beat_order);

/* ct_run_epoch for a caller that keeps the model in host memory, as the reference's
 * run_epoch(results, batch_index, data, config) (src/core/algorithm.rs:124-129) updates
 * `results.model` in place: gains [S,78], coefs [V,26] and delays [V,26] (reference order) are
 * copied in, the epoch runs, and the updated arrays are copied back into the same buffers;
 * measurements [B,T,M] (or NULL: keep the device copy) are copied in, loss_batch [num_batch_slots]
 * (or NULL) receives the batch-wise loss (results.metrics.loss_batch). Delays of connected pairs
 * must be >= 1 (CT_ERR_INVALID_ARGUMENT, nothing copied). All copies, the reordering kernels and the
 * epoch are enqueued on the context stream back to back and the call waits once, at the end
 * (device-side failures reported as by ct_sync). Pinned host memory gives full copy bandwidth. */
int ct_run_epoch_host(ct_scn* scn, int64_t* batch_index, const int32_t* beat_order, int grad_mode, int precision,
                      float* gains, float* coefs, int32_t* delays, const float* measurements, float* loss_batch);

/* ---- batched scenarios (no counterpart in the reference, which runs one scenario per OS
 * thread, src/core/scheduler.rs:93).
 * A batch runs one epoch of every member as one schedule: per beat index, one persistent
 * forward launch over the tiles of every member that has that beat, the members' measurement
 * products on parallel streams, one persistent adjoint launch (CT_GRAD_ADJOINT) or the members'
 * reference derivations, then every member's update. The epoch is captured once as a CUDA
 * graph and replayed (re-captured when a member's algorithm or adjoint ring changes).
 * Members need batch_size 0 (one update per epoch, the reference default) and the same
 * context; their beats run in index order. Results equal ct_run_epoch with beat_order
 * 0..B-1 within the tolerances of the measurement products. The members stay usable on
 * their own; a batch must be destroyed before its members. */
typedef struct ct_batch ct_batch;
int ct_batch_create(ct_ctx* ctx, ct_scn* const* scenarios, int64_t count, int grad_mode, int precision,
                    ct_batch** out);
int ct_batch_destroy(ct_batch* batch);
/* One epoch of every member, enqueued on the context stream (asynchronous).
 * batch_indices: in/out batch-wise metric cursor per member (as ct_run_epoch's batch_index). */
int ct_batch_run_epoch(ct_batch* batch, int64_t* batch_indices);
/* Autotuner: runs real epochs of the batch (each one trains and advances batch_indices like
 * ct_batch_run_epoch) under candidate schedules and keeps the fastest: the adjoint checkpoint
 * interval (32, 64, 128 steps; memory against recompute granularity) and the order of the tile
 * lists (by beat length; folded over the grid; interleaved across members), which sets how the
 * tiles of members of different sizes spread over the CTAs. Up to five epochs; synchronous.
 * Writes the choice and its epoch time (ms) to the non-NULL outputs. */
int ct_batch_autotune(ct_batch* batch, int64_t* batch_indices, int* ckpt_k, int* tile_order, double* best_ms);
/* Waits for the batch and reports any device-side failure of a member. */
int ct_batch_sync(ct_batch* batch);
/* Kernel nodes in the captured epoch graph, whether the graph is used (0: eager launches), and the
 * CTAs of the persistent forward and adjoint launches (all co-resident). NULL outputs are skipped. */
int ct_batch_info(ct_batch* batch, int64_t* graph_kernels, int* uses_graph, int* forward_ctas, int* adjoint_ctas);
/* Per-phase device time of batched epochs: while enabled, epochs run as eager launches (not the
 * graph) with CUDA events around each phase; ct_batch_read_profile waits for the batch and writes
 * CT_PHASE_COUNT totals in ms since enabling (FORWARD: memsets + forward launches; MEASURE: the
 * members' products, reference derivations and step metrics; DERIVE: adjoint launches; UPDATE). */
int ct_batch_set_profiling(ct_batch* batch, int enable);
int ct_batch_read_profile(ct_batch* batch, double* ms);

/* Forward of every beat with the current parameters (no noise); writes the predicted
 * measurements [B,T,M] and, if non-NULL, the states [T,S] of the last beat. Synchronous. */
int ct_simulate(ct_scn* scn, float* measurements_out, float* states_out);

int ct_set_algorithm(ct_scn* scn, const ct_algorithm* algo);
int ct_set_freeze(ct_scn* scn, int freeze_gains, int freeze_delays);
int ct_set_learning_rate(ct_scn* scn, float learning_rate);

/* Field access (synchronous). nbytes must equal the field size. */
int ct_field_size(ct_scn* scn, int field, size_t* nbytes);
int ct_read_field(ct_scn* scn, int field, void* dst, size_t nbytes);
int ct_write_field(ct_scn* scn, int field, const void* src, size_t nbytes);

/* Waits for the context stream and reports device-side failures (e.g. CT_ERR_TIMEOUT). */
int ct_sync(ct_scn* scn);

/* Phases of the epoch timed by ct_set_profiling. */
enum ct_phase {
  CT_PHASE_FORWARD = 0,        /* propagation kernel */
  CT_PHASE_MEASURE = 1,        /* H x, residuals, per-step MSE */
  CT_PHASE_MAP_RESIDUALS = 2,  /* H^T r */
  CT_PHASE_DERIVE = 3,         /* derivative sweep */
  CT_PHASE_STEP_METRICS = 4,   /* running max-regularisation sum, per-step loss */
  CT_PHASE_UPDATE = 5,         /* average delays, smoothness, optimizer, roll, batch metrics */
  CT_PHASE_COUNT = 6
};
/* Kernel launches issued by this scenario since creation (host-side counter; no CUDA
 * equivalent in the reference, which issues ~15 launches per step, gpu/epoch.rs:107-112). */
int ct_kernel_launches(ct_scn* scn, int64_t* launches);
/* Enable (1) / disable (0) CUDA-event timing of every phase; enabling clears the totals. */
int ct_set_profiling(ct_scn* scn, int enable);
/* Accumulated device milliseconds and launch counts per phase (arrays of CT_PHASE_COUNT).
 * Synchronizes the context stream. */
int ct_read_profile(ct_scn* scn, double* ms, int64_t* launches);

/* ---- the scenario loop and the post-run metrics (the callers either side of the epoch) */

/* Settings of the reference's epoch loop, run_model_based (src/core/scenario.rs:725-795), read from
 * the Algorithm config (src/core/config/algorithm.rs:25-58). The learning rate is the scenario's
 * (ct_set_learning_rate / the create-time algorithm): epoch 0 runs with learning rate 0, epoch 1
 * restores it, and every epoch whose index is a multiple of learning_rate_reduction_interval
 * (when non-zero) multiplies the running rate by learning_rate_reduction_factor. */
typedef struct ct_run_config {
  int64_t epochs;
  int64_t learning_rate_reduction_interval; /* 0 = never */
  float learning_rate_reduction_factor;
  int32_t grad_mode;                        /* ct_grad_mode of every epoch */
  int32_t precision;                        /* ct_precision of every epoch */
  int64_t snapshots_interval;               /* 0 = no snapshots */
} ct_run_config;

/* The loss part of the reference's Summary (src/core/scenario/summary.rs:25-42) after the loop. */
typedef struct ct_run_summary {
  int64_t epochs_run; /* epochs executed: fewer than requested when the loss stopped being normal */
  int64_t snapshots;  /* snapshots stored (CT_FIELD_SNAPSHOT_*) */
  float loss;         /* loss_batch[batch_index - 1] of the last epoch run */
  float loss_mse;
  float loss_maximum_regularization;
} ct_run_summary;

/* run_model_based: cfg->epochs epochs of ct_run_epoch under the learning-rate schedule above; after
 * each epoch the three batch losses of its last batch are read back (the summary the reference
 * sends per epoch), a snapshot is stored when the epoch index is a multiple of snapshots_interval,
 * and the loop stops early when the loss is not a normal number (zero, subnormal, infinite or
 * NaN: f32::is_normal). Then the average delays are recomputed from the final parameters
 * (CT_FIELD_AVERAGE_DELAYS) and the scenario's learning rate is restored. Synchronous.
 * beat_orders: [epochs, B] beat orders, or NULL for the library's seeded shuffle each epoch.
 * batch_index: in/out as for ct_run_epoch. epoch_losses: NULL or [epochs, 3] (loss, loss_mse,
 * loss_maximum_regularization per epoch run; rows of epochs not run are left untouched). */
int ct_run_model_based(ct_scn* scn, const ct_run_config* cfg, const int32_t* beat_orders, int64_t* batch_index,
                       float* epoch_losses, ct_run_summary* summary);

/* The same loop over every member of a batch (one ct_batch_run_epoch per epoch; beats in index
 * order). Each member follows its own learning rate through the schedule and stops on its own
 * non-normal loss; the remaining members continue as a smaller batch. No snapshots
 * (snapshots_interval must be 0). batch_indices: in/out per member. epoch_losses: NULL or
 * [count, epochs, 3]. summaries: [count]. Synchronous. */
int ct_batch_run_model_based(ct_batch* batch, const ct_run_config* cfg, int64_t* batch_indices, float* epoch_losses,
                             ct_run_summary* summaries);

/* calculate_plotting_arrays (src/core/scenario.rs:636-690), estimation side: from the last beat's
 * states, the spherical arrays (magnitude |x|+|y|+|z|, theta = acos(z / magnitude),
 * phi = atan2(y, x)), their values at each voxel's first maximum of the magnitude, and the
 * activation time (that step / sample_rate_hz * 1000, ms). Results in CT_FIELD_STATES_* and
 * CT_FIELD_ACTIVATION_TIMES. CT_ERR_NO_MAXIMUM when a voxel's magnitude is NaN at every step
 * (the reference's argmax_skipnan error). The differences against the simulation's arrays are the
 * same call on the ground-truth scenario followed by a subtraction. Synchronous. */
int ct_calculate_plotting_arrays(ct_scn* scn, float sample_rate_hz);

#define CT_THRESHOLDS 101
/* Metrics::*_over_threshold (src/core/algorithm/metrics.rs:20-37) and the Summary fields chosen at
 * the Dice-optimal threshold (src/core/scenario.rs:601-617). */
typedef struct ct_final_metrics {
  float dice_score_over_threshold[CT_THRESHOLDS]; /* threshold i / 100, i = 0..100 */
  float iou_over_threshold[CT_THRESHOLDS];
  float precision_over_threshold[CT_THRESHOLDS];
  float recall_over_threshold[CT_THRESHOLDS];
  float threshold; /* first threshold of the largest Dice score */
  float dice;
  float iou;
  float recall;
  float precision;
} ct_final_metrics;

/* metrics::calculate_final (src/core/algorithm/metrics.rs:226-447): a grid cell with a voxel number
 * is predicted pathological at threshold t when the largest magnitude of its voxel's last-beat
 * states over all steps (NaN steps skipped) is <= t; Dice, IoU, precision and recall against the
 * ground truth for t = 0, 0.01, ..., 1, and the summary at the Dice-optimal threshold.
 * ground_truth_types: [nx,ny,nz] VoxelType discriminants (voxels.rs:664-676, Pathological = 6) of
 * the simulation; voxel_numbers: [nx,ny,nz] state index of each cell's voxel (multiple of 3, < S)
 * or -1 (None), of the estimated model. Synchronous. */
int ct_calculate_final(ct_scn* scn, const int32_t* ground_truth_types, const int32_t* voxel_numbers, int64_t nx,
                       int64_t ny, int64_t nz, ct_final_metrics* out);

/* ---- model construction on the device (the step before the epoch) */

/* The parts of the reference's SpatialDescription (src/core/model/spatial.rs) and model config that
 * the measurement matrix and the delay arrays are built from. Arrays are C-order host arrays. */
typedef struct ct_spatial_desc {
  int64_t nx, ny, nz;                /* voxel grid, voxels.types.raw_dim() */
  const int32_t* voxel_types;        /* [nx,ny,nz] VoxelType discriminants (voxels.rs:664-676); 1..6 connectable */
  const int32_t* voxel_numbers;      /* [nx,ny,nz] state index 3v of each connectable cell's voxel, -1 = None
                                        (voxels.numbers); the connectable cells must number 0, 3, .., S-3 once each */
  const float* voxel_positions_mm;   /* [nx,ny,nz,3] voxels.positions_mm */
  float voxel_size_mm;               /* voxels.size_mm */
  float sample_rate_hz;              /* the simulation's sample rate (delay samples) */
  const float* propagation_velocities_m_per_s; /* [10] per VoxelType discriminant (config/model.rs:138-150) */
  int64_t num_sensors;               /* M sensor rows */
  int64_t num_beats;                 /* B */
  const float* sensor_positions_mm;  /* [M,3] sensors.positions_mm */
  const float* sensor_orientations;  /* [M,3] sensors.orientations_xyz */
  const float* sensor_array_offsets_mm; /* [B,3] sensors.array_offsets_mm */
} ct_spatial_desc;

/* MeasurementMatrix::from_model_spatial_description (src/core/model/functional/measurement.rs:66-123) on the
 * device: the Biot-Savart lead field H [B, M, S] (S = 3 x connectable cells) in reference state order,
 * written to the host buffer `out` of nbytes = 4 B M S. Bit-identical to the reference's f32 loop.
 * Needs only the geometry fields and num_sensors / num_beats / sensor arrays. Synchronous. */
int ct_measurement_matrix(ct_ctx* ctx, const ct_spatial_desc* desc, float* out, size_t nbytes);

/* calculate_delay_samples_array (src/core/model/functional/allpass/delay.rs:35-111) and the integer delays
 * and coefficients APParameters::from_model_config derives from it (allpass.rs:86-100), on the device:
 * initial_delays (f32), delays (i32) and coefs (f32), each [V, 26] with count = V x 26 elements. Pairs
 * whose neighbour is outside the grid or not connectable get 0 samples, delay 0 and coefficient
 * 0.9999, as in the reference. CT_ERR_INVALID_ARGUMENT naming the first (cell, offset) in the
 * reference's loop order whose delay is below one sample (the reference's error) or is not a finite
 * value below 2^31 (not representable as an i32 delay). Synchronous. */
int ct_delay_samples(ct_ctx* ctx, const ct_spatial_desc* desc, float* initial_delays, int32_t* delays, float* coefs,
                     int64_t count);

/* The measurement matrix of ct_measurement_matrix computed straight into the scenario's device copy
 * (and its tensor-core operand splits): no [B, M, S] host array and no host-to-device copy of it.
 * The grid's connectable cells, num_sensors and num_beats must match the scenario. A scenario may be
 * created with measurement_matrix = NULL (H zero) and filled by this call before its first epoch.
 * Synchronous. */
int ct_scenario_set_measurement_matrix(ct_scn* scn, const ct_spatial_desc* desc);

/* connect_voxels / try_to_connect (src/core/model/functional/allpass.rs:295-494): the activation-front
 * search that sets the gains. Starting from the Sinoatrial voxels at time 0 it visits activation times
 * in increasing order; the voxels whose time is relative_eq to the current one (C order) each activate
 * their allowed (voxels.rs:707-742), not yet activated neighbours first come, first served, at the
 * input's velocity; the input's current direction is (in - out) / |in - out|_1 and its gains
 * gain::calculate (gain.rs:9-29) times the pathology factor (or its inverse). Writes gains [S, 78]
 * (gains_bytes = 4 S 78) and activation_time_ms [nx, ny, nz] (NaN = never activated), bit-identical
 * to the reference's f32 loop. Host-only (sequential by definition: a voxel's gains depend on which
 * neighbour reached it first); needs the grid fields and the velocities. Synchronous. */
int ct_connect_voxels(const ct_spatial_desc* desc, float current_factor_in_pathology, float* gains, size_t gains_bytes,
                      float* activation_time_ms);

/* init_output_state_indicies (src/core/model/functional/allpass.rs:212-289): [S, 78] i32, row 3v + a,
 * column 3n + b = 3w + b for the voxel w at offset n of voxel v, -1 where there is none
 * (nbytes = 4 S 78). Host-only. */
int ct_output_state_indices(const ct_spatial_desc* desc, int32_t* out, size_t nbytes);

/* Allocation-free H x product for callers that must not see this library allocate device
 * memory: hosts that keep every device buffer in their own pool or arena or run under a fixed
 * memory budget, and callers that cannot accept the implicit device synchronisation of
 * cudaMalloc / cudaFree. No counterpart in the reference crate.
 *
 * predicted[t, m] = sum_s measurement_matrix[m, s] * states[t, s] for one beat, and, when
 * residuals is non-NULL, residuals = predicted - actual (all [T, M]). All pointers are device
 * pointers owned by the caller; work is enqueued on `stream` (NULL = legacy default stream), which
 * must belong to the current device (CT_ERR_INVALID_ARGUMENT otherwise).
 * Split-K partial sums go to one 8 MiB file-scope device array that every GPU loading the
 * library holds until exit; num_steps x ceil(num_sensors / 64) x 64 must not exceed 2,097,152
 * (CT_ERR_INVALID_ARGUMENT otherwise). The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress) with the device current and keeps it; make that first call before any
 * stream capture. A device reset (cudaDeviceReset) invalidates the kept address: do not call this
 * function after resetting a device it has run on. The function calls no cudaMalloc / cudaFree. All calls share the array:
 * calls that overlap on the GPU (other streams, other host threads) race on it. */
int ct_predict_measurements_noalloc(const float* states, const float* measurement_matrix, const float* actual,
                                    float* predicted, float* residuals, int64_t num_steps, int64_t num_states,
                                    int64_t num_sensors, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CARDIOTRUST_CUDA_H */
