// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/cardiotrust_cuda.h"

namespace ct {

constexpr int kOffsets = 26;   // neighbour offsets per voxel
constexpr int kGainCols = 78;  // 26 offsets x 3 neighbour components
constexpr int kMaxStepBlock = 8;  // steps advanced between grid barriers in the forward kernel
constexpr int kFwdTileVoxels = 32;  // voxels per forward tile (consecutive in device order)
constexpr int kFwdHaloMax = 160;    // largest neighbourhood of a tile the resident forward form stages
constexpr int kCkptSteps = 256;     // adjoint mode: default all-pass checkpoint interval (power of two)

// Device-side grid barrier state: a monotone arrival counter, zeroed before each launch.
struct GridBarrier {
  unsigned int count;
  unsigned int unused;
};

// Everything of one scenario that lives on the device.
struct DeviceScenario {
  int64_t S, V, M, T, B, NB;
  // model
  float* gains;          // [S,78]
  int32_t* nbr;          // [V,26] neighbour voxel, -1 = none (derived from output_state_indices)
  float* coefs;          // [V,26]
  int32_t* delays;       // [V,26]
  float* init_delays;    // [V,26]
  float* H;              // [B,M,S]
  float* ctrl;           // [S]
  float* u;              // [T]
  float* meas;           // [B,T,M] actual measurements
  // estimations
  float* X;              // [T,S] states of the beat being processed
  float* Y;              // [B,T,M] predicted measurements
  float* R;              // [T,M] residuals of the beat being processed
  float* MR;             // [T,S] mapped residuals of the beat being processed
  float* ap;             // [V,78] all-pass state (deduplicated over the row component)
  float* ap_last;        // [V,78] all-pass output of step T-2
  float* avg_delays;     // [V]
  // derivatives
  float* dG;             // [S,78]
  float* dC;             // [V,26]
  float* fir;            // [V,78]
  float* iir;            // [V,78]
  float* mG1, *mG2;      // [S,78] Adam moments
  float* mC1, *mC2;      // [V,26]
  float* mreg_sum;       // [1] running maximum-regularisation sum
  // metrics
  float* loss, *loss_mse, *loss_mr;          // [T]
  float* loss_b, *loss_mse_b, *loss_mr_b;    // [NB]
  // scratch
  float* stepsum_part;   // [T, fwd_grid] per-CTA partial max-regularisation sums
  float* gemm_part;      // [ksplit, T, Mpad] split-K partials of H x
  int fwd_grid;          // CTAs of the forward kernel
  int ksplit;            // split-K factor of the H x product (CUDA-core form)
  // tensor-core form (ct_umma.cu); null when the scenario does not support it
  bool umma;             // S % 4 == 0 and the TMA encoder is available
  int ksplit_umma;       // split-K factor of the tensor-core H x
  int64_t kpad;          // M rounded up to 32 (K extent of H^T r)
  int64_t spad;          // S rounded up to 4: row pitch of H_hi, H_lo and Xpad (16-byte TMA rows)
  float* H_hi, *H_lo;    // [B,M,spad] TF32 split of H, zero beyond S
  float* Xpad;           // [T,spad] copy of X for the H x operand when S % 4 != 0 (else null)
  float* Ht_hi, *Ht_lo;  // [B,S,kpad] TF32 split of H^T, zero padded
  float* R_hi, *R_lo;    // [T,kpad] TF32 split of the residuals
  // sliced BF16 form (ct_slice.cu), allocated on first use; sp = S and kpm = M rounded up to 64
  int ksplit_slice;          // split-K factor of the sliced H x (whole 512-element groups per split)
  bool slice_ready;          // H_sl / Ht_sl hold the slices of the current H
  __nv_bfloat16* H_sl;       // [B][3][M][sp] slices of H
  float* H_sc;               // [B][ceil(sp/512)][M] scales (group-major)
  __nv_bfloat16* Ht_sl;      // [B][3][S][kpm] slices of H^T
  float* Ht_sc;              // [B][ceil(kpm/512)][S]
  __nv_bfloat16* X_sl;       // [3][T][sp] slices of the beat's states
  float* X_sc;               // [T][ceil(sp/512)]
  __nv_bfloat16* R_sl;       // [3][T][kpm] slices of the beat's residuals
  float* R_sc;               // [T][ceil(kpm/512)]
  int32_t* dmin;         // [2] smallest and largest delay of a connected (voxel, offset) pair
  // resident forward form (one tile per CTA, halo history in a shared ring)
  bool fwd_ring;
  int32_t* halo;         // [tiles, kFwdHaloMax] device voxels of each tile's neighbourhood
  int16_t* hslot;        // [tiles, 26 * kFwdTileVoxels] halo slot of each item's neighbour, -1 if absent
  int32_t* nhalo;        // [tiles]
  // adjoint mode (ct_adjoint.cu), allocated on first use
  int32_t* rev;          // [V,26] voxel whose offset n points at this voxel, -1 if none
  int ckpt_k;            // checkpoint interval K (power of two)
  float* ckpt;           // [ceil(T/K), V, 78] all-pass state before step s * K
  float* seg_q;          // [min(T, K), pitch] in_t - ap[t-1] of one segment
  float* inbox;          // [adj_ring, V, 78] adjoint contributions addressed to (voxel, column) by step
  float* lam_state;      // [V,78] adjoint all-pass state between blocks of steps
  float* dCk;            // [V,78] per-column coefficient-gradient partials
  int adj_ring;          // inbox slots (power of two)
  int adj_pitch;         // floats per plane of seg_q and inbox: V * 78 rounded up to 4 (16-byte rows)
  int adj_grid;          // CTAs of the adjoint kernel
  // plain form (ct_plain.cu), allocated on first use
  float* plain_mreg;     // [S] maximum regularisation of the current step
  float* plain_part;     // [ceil(V / 256)] per-block sums of the step's regularisation terms
  int32_t* status;       // [1] device-side error code (0 = ok)
  GridBarrier* barrier;  // [1]
};

// Records `message` as the calling thread's last error (read by ct_last_error); returns status.
int report_error(int status, const char* message);

// ---- launchers (all enqueue on `stream`, return cudaError_t of the launch)

// One scenario as the forward kernels see it.
struct FwdArgs {
  int V, S, T;
  int part_stride;  // batched form: tiles of the scenario (stride of stepsum_part rows)
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
  float* ckpt;  // adjoint checkpoints [ceil(T / ckpt_k), V, 78] or null
  int ckpt_k;   // checkpoint interval (power of two)
  const int32_t* dmin;
  float threshold;
  int32_t* status;
  GridBarrier* barrier;
};
// One cooperative forward launch over the tiles of several scenarios (batched form).
struct FwdBatch {
  const FwdArgs* scns;  // device array
  int nscn;
  const int2* tiles;    // (scenario, first voxel)
  int ntiles;
  int Tmax;
  int32_t* status;
  GridBarrier* barrier;
};
FwdArgs forward_scenario(const DeviceScenario& d, float threshold, float* ckpt, float* part, int part_stride);
// The caller zeroes every scenario's ap and ap_last first.
cudaError_t launch_forward_batch(const FwdBatch& b, int grid, cudaStream_t stream);
int forward_batch_capacity(int device);

// Forward propagation of one beat: X[t,:] for t in [0,T). With ckpt non-null the all-pass
// state before every step s * d.ckpt_k (s >= 1) is stored in ckpt[s].
cudaError_t launch_forward(DeviceScenario& d, float threshold, float* ckpt, cudaStream_t stream);
// CTAs of the streaming form, and how many CTAs of the resident form fit on the device.
int forward_grid_size(int64_t V, int device);
int forward_ring_capacity(int device);

// y = H[beat] x for all steps; Y[beat] = y, R = y - meas[beat], loss_mse[t].
cudaError_t launch_measure(DeviceScenario& d, int64_t beat, bool with_residuals, cudaStream_t stream);
// MR[t,:] = H[beat]^T R[t,:] for all steps.
cudaError_t launch_map_residuals(DeviceScenario& d, int64_t beat, cudaStream_t stream);
// loss_mse[t] from R.
cudaError_t launch_mse(DeviceScenario& d, cudaStream_t stream);

// Tensor-core (tcgen05) forms, ct_umma.cu.
bool umma_supported(int64_t M);
int umma_yn(int64_t M);
int umma_ksplit(int64_t T, int64_t S, int64_t M, int sms);
cudaError_t umma_prepare(DeviceScenario& d, cudaStream_t stream);
cudaError_t launch_measure_umma(DeviceScenario& d, int64_t beat, bool with_residuals, int precision,
                                cudaStream_t stream);
cudaError_t launch_map_residuals_umma(DeviceScenario& d, int64_t beat, int precision, cudaStream_t stream);
// Sliced BF16 forms (ct_slice.cu): K extents rounded up to whole 64-element chunks, scale groups of
// 512 elements, the split-K factor of H x, the slicing of H and H^T (after every change of H;
// allocates and frees a temporary [S, kpm] buffer on the stream), and the two products.
int64_t slice_pitch(int64_t k);
int64_t slice_groups(int64_t k);
int slice_ksplit(int64_t T, int64_t S, int64_t M, int sms);
cudaError_t slice_prepare(DeviceScenario& d, cudaStream_t stream);
cudaError_t launch_measure_sliced(DeviceScenario& d, int64_t beat, bool with_residuals, cudaStream_t stream);
cudaError_t launch_map_residuals_sliced(DeviceScenario& d, int64_t beat, cudaStream_t stream);

struct DeriveScalars {
  float mse_scaling, reg_scaling, threshold, diffreg;
  int freeze_gains, freeze_delays, ap_derivative;
};
// Per-(voxel, offset) sweep over the steps of one beat: dG, dC, fir, iir.
cudaError_t launch_derive(DeviceScenario& d, const DeriveScalars& s, cudaStream_t stream);

struct AdjointScalars {
  float mse_scaling, reg_scaling, threshold, diffreg;
  int freeze_gains, freeze_delays, ap_derivative;
};
// One scenario as the adjoint kernel sees it (device pointers, sizes, scalars).
struct AdjScn {
  int V, S, T, ring;
  int pitch;  // floats between consecutive planes of seg_q and inbox (V * 78 rounded up to 4)
  const int32_t* nbr;
  const float* coefs;
  const int32_t* delays;
  const float* init_delays;
  const float* gains;
  const float* X;
  const float* MR;
  const float* ckpt;
  float* seg_q;
  float* inbox;
  float* lam_state;
  float* dG;
  float* dC;
  float* dCk;
  const int32_t* dmin;
  float mse_scaling, reg_scaling, threshold, diffreg;
  int freeze_gains, freeze_delays, ap_derivative;
};
// One cooperative adjoint launch over the tiles of one or more scenarios.
struct AdjLaunch {
  const AdjScn* scns;  // device array of nscn scenarios, or null: `single` is the only one
  AdjScn single;
  int nscn;
  const int2* tiles;  // (scenario, first voxel) per tile, or null: tiles of 32 voxels of scenario 0
  int ntiles;
  int Tmax;           // longest beat of the launch
  int ckpt_steps;     // checkpoint interval (power of two)
  int32_t* status;
  GridBarrier* barrier;
};
AdjScn adjoint_scenario(const DeviceScenario& d, const AdjointScalars& s);
// Back-propagation through time of one beat (needs X, MR and the forward's checkpoints): dG, dC.
cudaError_t launch_adjoint(DeviceScenario& d, const AdjointScalars& s, cudaStream_t stream);
// The same over a tile list; the caller zeroes every scenario's inbox and lam_state first.
cudaError_t launch_adjoint_tiles(const AdjLaunch& launch, int grid, cudaStream_t stream);
// How many CTAs of the adjoint kernel fit on the device at once.
int adjoint_capacity(int device);

struct PlainScalars {
  float mse_scaling, reg_scaling, threshold, diffreg;
  int freeze_gains, freeze_delays, ap_derivative;
};
// Plain form of one beat (prediction, reference derivation and step metrics), launched per step.
cudaError_t launch_plain_beat(DeviceScenario& d, int64_t beat, const PlainScalars& s, cudaStream_t stream);
int plain_step_launches(const PlainScalars& s);

// Step metrics of one beat: loss_mr[t] (running), loss[t]; advances mreg_sum.
cudaError_t launch_step_metrics(DeviceScenario& d, float reg_strength, cudaStream_t stream);
// Batch metrics into slot `index`; the _dev form reads the slot on the device (graph replay).
cudaError_t launch_batch_metrics(DeviceScenario& d, int64_t index, cudaStream_t stream);
cudaError_t launch_batch_metrics_dev(DeviceScenario& d, const int64_t* index_dev, cudaStream_t stream);
// Step metrics from `parts` per-step partial sums (the batched forward's per-tile partials).
cudaError_t launch_step_metrics_parts(DeviceScenario& d, const float* part, int parts, float reg_strength,
                                      cudaStream_t stream);

cudaError_t launch_average_delays(DeviceScenario& d, cudaStream_t stream);
cudaError_t launch_smoothness(DeviceScenario& d, float strength, cudaStream_t stream);

struct UpdateScalars {
  int optimizer, freeze_gains, freeze_delays;
  float lr_over_bs, bias1, bias2;
  const float* bias_dev = nullptr;  // if set: {bias1, bias2} read on the device (graph replay)
};
cudaError_t launch_update(DeviceScenario& d, const UpdateScalars& s, cudaStream_t stream);
cudaError_t launch_min_delay(DeviceScenario& d, cudaStream_t stream);

// Voxel blocks of `words` 32-bit words between reference and device voxel order (perm[u] = the
// reference voxel of device voxel u): gather dst[u] = src[perm[u]], else scatter dst[perm[u]] = src[u].
cudaError_t launch_permute_blocks(const void* src, void* dst, const int32_t* perm, int64_t V, int64_t words,
                                  bool gather, cudaStream_t stream);
// Model construction (ct_model.cu). The lead-field factor of measurement.rs:85-88 for a voxel size.
float lead_field_factor(float voxel_size_mm);
// H[b * M + m, col[i] + a] for every beat b, sensor row m, voxel-list entry i (position vpos[i]) and
// component a, with row pitch ldh.
cudaError_t launch_lead_field(const float* vpos, const int32_t* col, int64_t nv, const float* spos,
                              const float* sori, const float* off, int64_t M, int64_t B, float cf, float* H,
                              int64_t ldh, int num_sms, cudaStream_t stream);
// Delay samples, integer delays and coefficients [V, 26] from the voxel grid; *first_bad (preset to
// all ones) receives the first failing cell * 26 + offset column.
cudaError_t launch_delay_samples(const int32_t* types, const int32_t* numbers, const float* pos, int64_t nx,
                                 int64_t ny, int64_t nz, const float* vel, float rate, float* samples,
                                 int32_t* delays, float* coefs, unsigned long long* first_bad, int num_sms,
                                 cudaStream_t stream);
// connect_voxels (allpass.rs:295-494) on the host: gains [S,78] (zeroed by the caller) and activation
// times in ms [cells] (NaN = never activated).
void connect_voxels_host(const int32_t* types, const int32_t* numbers, const float* pos, int64_t nx, int64_t ny,
                         int64_t nz, const float* vel, float factor, float* gains, float* activation_ms);
// init_output_state_indicies (allpass.rs:212-289) on the host: [S,78], cell_of[v] = the cell of voxel v.
void output_state_indices_host(const int32_t* types, const int32_t* numbers, int64_t nx, int64_t ny, int64_t nz,
                               const std::vector<int64_t>& cell_of, int32_t* out);
// Expand the deduplicated [V,78] all-pass/fir/iir state into the reference [S,78] layout.
cudaError_t launch_expand_rows(const float* src, float* dst, int64_t V, cudaStream_t stream);
// Last-step maximum regularisation [S] from X[T-1].
cudaError_t launch_last_max_reg(DeviceScenario& d, float threshold, float* out, cudaStream_t stream);

// ---- post-run arrays and segmentation metrics (ct_post.cu)
struct PostPlan {
  int parts = 1;           // blocks of steps each voxel's scan is split into
  int steps_per_part = 1;
};
PostPlan post_plan(int64_t V, int64_t T, int sms);
// Device buffers of the post-run pass; the spherical arrays are reference voxel order.
struct PostBuffers {
  int32_t* inv = nullptr;          // [V] device voxel of each reference voxel
  float* mag = nullptr;            // [T,V] |x| + |y| + |z|
  float* theta = nullptr;          // [T,V]
  float* phi = nullptr;            // [T,V]
  float* mag_max = nullptr;        // [V] at the first maximum of the magnitude
  float* theta_max = nullptr;      // [V]
  float* phi_max = nullptr;        // [V]
  float* activation_ms = nullptr;  // [V]
  float* maxmag = nullptr;         // [V] largest magnitude, NaN when every step is NaN
  float* part_val = nullptr;       // [parts,V] per block of steps: largest magnitude
  int32_t* part_idx = nullptr;     // [parts,V] and its first step (-1: all NaN)
};
// Scan of X: maxmag always; with `write`, the spherical arrays, their maxima and the activation
// times (a voxel whose magnitude is NaN at every step sets CT_ERR_NO_MAXIMUM in d.status).
cudaError_t launch_spherical(const DeviceScenario& d, const PostBuffers& b, const PostPlan& plan, bool write,
                             float sample_rate_hz, cudaStream_t stream);
// Threshold sweep over `cells` grid cells (types, numbers in grid order) into `out`
// (the ct_final_metrics layout); hist is 2 x (CT_THRESHOLDS + 1) device counters.
cudaError_t launch_final_metrics(const PostBuffers& b, const int32_t* types, const int32_t* numbers, int64_t cells,
                                 unsigned long long* hist, float* out, int sms, cudaStream_t stream);

}  // namespace ct
