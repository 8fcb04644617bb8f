// Post-run arrays and segmentation metrics of one beat's states (the beat an
// epoch ran last): what the reference computes once after the epoch loop.
//
//   spherical arrays   SystemStatesSpherical::calculate      src/core/data/shapes.rs:171-192
//   their maximum      SystemStatesSphericalMax::calculate   src/core/data/shapes.rs:262-277
//   activation times   ActivationTimePerStateMs::calculate   src/core/data/shapes.rs:334-352
//   final metrics      metrics::calculate_final              src/core/algorithm/metrics.rs:226-242
//                      calculate_for_threshold / dice / iou / precision / recall / predict_voxeltype
//                                                            src/core/algorithm/metrics.rs:248-447
//   summary            optimal Dice threshold                src/core/scenario.rs:601-617
//
// Both passes are HBM-bound streams over X [T, S]: 12 bytes read per
// (step, voxel), plus 12 bytes written when the spherical arrays are kept.
// Work is split over (voxel, block of steps) so that a few hundred thousand
// threads keep loads in flight; each block of steps leaves its first maximum
// and the blocks are merged in step order, which gives the first maximum over
// all steps (ndarray-stats 0.6.0 `argmax_skipnan` keeps the earliest of equal
// maxima and skips NaN).
//
// Rounding: the magnitude is |x| + |y| + |z| added left to right; theta is
// acos(z / magnitude) and phi atan2(y, x) with CUDA's acosf / atan2f (the
// reference calls the host libm's: they agree to a few ulp, not bitwise);
// activation times, thresholds and the metric ratios are single IEEE
// divisions and products, as in the reference.

#include <math.h>

#include <algorithm>

#include "ct_internal.cuh"

namespace ct {
namespace {

constexpr int kPathological = 6;  // VoxelType::Pathological, src/core/model/spatial/voxels.rs:664-676
constexpr int kPostThreads = 128;

__device__ __forceinline__ float magnitude3(float x, float y, float z) {
  return __fadd_rn(__fadd_rn(fabsf(x), fabsf(y)), fabsf(z));
}

// One thread per (reference voxel v, block of steps). inv[v] is v's device voxel.
template <bool kWrite>
__global__ void __launch_bounds__(kPostThreads) spherical_part_kernel(
    const float* __restrict__ X, const int32_t* __restrict__ inv, int V, int64_t S, int T, int steps_per_block,
    float* __restrict__ mag, float* __restrict__ theta, float* __restrict__ phi, float* __restrict__ part_val,
    int32_t* __restrict__ part_idx) {
  const int v = blockIdx.x * kPostThreads + threadIdx.x;
  if (v >= V) return;
  const int c = blockIdx.y;
  const int t0 = c * steps_per_block;
  const int t1 = min(T, t0 + steps_per_block);
  const float* col = X + 3 * (int64_t)inv[v];
  float best = 0.0f;
  int bidx = -1;
#pragma unroll 4
  for (int t = t0; t < t1; ++t) {
    const float* row = col + (int64_t)t * S;
    const float x = __ldg(row), y = __ldg(row + 1), z = __ldg(row + 2);
    const float m = magnitude3(x, y, z);
    if (kWrite) {
      const int64_t o = (int64_t)t * V + v;
      mag[o] = m;
      theta[o] = acosf(__fdiv_rn(z, m));
      phi[o] = atan2f(y, x);
    }
    if (!isnan(m) && (bidx < 0 || m > best)) {
      best = m;
      bidx = t;
    }
  }
  part_val[(int64_t)c * V + v] = best;
  part_idx[(int64_t)c * V + v] = bidx;
}

// Merge of the step blocks in step order; maxmag[v] = max_skipnan (NaN when every step is NaN).
template <bool kWrite>
__global__ void __launch_bounds__(kPostThreads) spherical_max_kernel(
    const float* __restrict__ X, const int32_t* __restrict__ inv, int V, int64_t S, int nparts,
    const float* __restrict__ part_val, const int32_t* __restrict__ part_idx, float sample_rate_hz,
    float* __restrict__ maxmag, float* __restrict__ mag_max, float* __restrict__ theta_max,
    float* __restrict__ phi_max, float* __restrict__ activation_ms, int32_t* status) {
  const int v = blockIdx.x * kPostThreads + threadIdx.x;
  if (v >= V) return;
  float best = 0.0f;
  int bidx = -1;
  for (int c = 0; c < nparts; ++c) {
    const int i = part_idx[(int64_t)c * V + v];
    const float m = part_val[(int64_t)c * V + v];
    if (i >= 0 && (bidx < 0 || m > best)) {
      best = m;
      bidx = i;
    }
  }
  maxmag[v] = bidx < 0 ? __int_as_float(0x7fc00000) : best;
  if (!kWrite) return;
  if (bidx < 0) {
    // argmax_skipnan finds no maximum: the reference's calculate() returns an error
    atomicCAS(status, 0, (int32_t)CT_ERR_NO_MAXIMUM);
    mag_max[v] = theta_max[v] = phi_max[v] = activation_ms[v] = __int_as_float(0x7fc00000);
    return;
  }
  const float* row = X + (int64_t)bidx * S + 3 * (int64_t)inv[v];
  mag_max[v] = best;
  theta_max[v] = acosf(__fdiv_rn(row[2], best));
  phi_max[v] = atan2f(row[1], row[0]);
  activation_ms[v] = __fmul_rn(__fdiv_rn((float)bidx, sample_rate_hz), 1000.0f);
}

// Histogram of the first threshold at which each grid cell is predicted pathological
// (bin CT_THRESHOLDS = never), split by whether the ground truth is pathological.
// hist: [2][CT_THRESHOLDS + 1] counts (row 1 = pathological ground truth).
__global__ void __launch_bounds__(256) threshold_hist_kernel(const int32_t* __restrict__ types,
                                                             const int32_t* __restrict__ numbers, int64_t cells,
                                                             const float* __restrict__ maxmag,
                                                             unsigned long long* hist) {
  __shared__ float thr[CT_THRESHOLDS];
  __shared__ unsigned int h[2][CT_THRESHOLDS + 1];
  for (int i = threadIdx.x; i < CT_THRESHOLDS; i += blockDim.x) thr[i] = __fdiv_rn((float)i, 100.0f);
  for (int i = threadIdx.x; i < 2 * (CT_THRESHOLDS + 1); i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < cells; g += (int64_t)gridDim.x * blockDim.x) {
    const int p = types[g] == kPathological ? 1 : 0;
    const int num = numbers[g];
    int bin = CT_THRESHOLDS;
    if (num >= 0) {
      // predicted pathological at threshold i iff max <= i/100 (NaN: never), metrics.rs:435
      const float m = maxmag[num / 3];
      for (int i = 0; i < CT_THRESHOLDS; ++i)
        if (m <= thr[i]) {
          bin = i;
          break;
        }
    }
    atomicAdd(&h[p][bin], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 2 * (CT_THRESHOLDS + 1); i += blockDim.x) {
    const unsigned int n = (&h[0][0])[i];
    if (n) atomicAdd(hist + i, (unsigned long long)n);
  }
}

__device__ __forceinline__ float ratio(unsigned long long num, unsigned long long den) {
  return __fdiv_rn(__ull2float_rn(num), __ull2float_rn(den));
}

// Dice, IoU, precision and recall per threshold from the histogram, then the Dice-optimal
// summary. out: the ct_final_metrics layout (4 x CT_THRESHOLDS floats, then 5 summary floats).
__global__ void __launch_bounds__(128) final_metrics_kernel(const unsigned long long* __restrict__ hist,
                                                            float* __restrict__ out) {
  __shared__ float dice_s[CT_THRESHOLDS];
  const unsigned long long* hn = hist;
  const unsigned long long* hp = hist + CT_THRESHOLDS + 1;
  const int i = threadIdx.x;
  if (i < CT_THRESHOLDS) {
    unsigned long long tp = 0, fp = 0, gt = 0;
    for (int j = 0; j <= CT_THRESHOLDS; ++j) {
      gt += hp[j];
      if (j <= i) {
        tp += hp[j];
        fp += hn[j];
      }
    }
    const unsigned long long fn = gt - tp;
    const unsigned long long dden = 2 * tp + fp + fn;
    const float dice = dden == 0 ? 0.0f : ratio(2 * tp, dden);                 // metrics.rs:362-399
    const float iou = (tp + fp + fn) == 0 ? 0.0f : ratio(tp, tp + fp + fn);    // metrics.rs:330-354
    const float prec = (tp + fp) == 0 ? 0.0f : ratio(tp, tp + fp);             // metrics.rs:300-321
    const float rec = gt == 0 ? 1.0f : ratio(tp, gt);                          // metrics.rs:272-294
    out[i] = dice;
    out[CT_THRESHOLDS + i] = iou;
    out[2 * CT_THRESHOLDS + i] = prec;
    out[3 * CT_THRESHOLDS + i] = rec;
    dice_s[i] = dice;
  }
  __syncthreads();
  if (i == 0) {
    // argmax_skipnan: first of equal maxima, NaN skipped; unwrap_or_default() = 0 (scenario.rs:601-605)
    int best = -1;
    for (int j = 0; j < CT_THRESHOLDS; ++j) {
      const float dv = dice_s[j];
      if (!isnan(dv) && (best < 0 || dv > dice_s[best])) best = j;
    }
    if (best < 0) best = 0;
    float* s = out + 4 * CT_THRESHOLDS;
    s[0] = __fdiv_rn((float)best, 100.0f);
    s[1] = out[best];
    s[2] = out[CT_THRESHOLDS + best];
    s[3] = out[3 * CT_THRESHOLDS + best];
    s[4] = out[2 * CT_THRESHOLDS + best];
  }
}

}  // namespace

PostPlan post_plan(int64_t V, int64_t T, int sms) {
  PostPlan p;
  const int64_t vblocks = (V + kPostThreads - 1) / kPostThreads;
  const int64_t target = (int64_t)sms * 16;  // 16 blocks of 128 threads per SM: a full SM
  int64_t parts = std::max<int64_t>(1, std::min<int64_t>(T, (target + vblocks - 1) / vblocks));
  parts = std::min<int64_t>(parts, 4096);
  p.steps_per_part = (int)((T + parts - 1) / parts);
  p.parts = (int)((T + p.steps_per_part - 1) / p.steps_per_part);
  return p;
}

cudaError_t launch_spherical(const DeviceScenario& d, const PostBuffers& b, const PostPlan& plan, bool write,
                             float sample_rate_hz, cudaStream_t stream) {
  const dim3 grid((unsigned)((d.V + kPostThreads - 1) / kPostThreads), (unsigned)plan.parts);
  const unsigned vgrid = (unsigned)((d.V + kPostThreads - 1) / kPostThreads);
  if (write) {
    spherical_part_kernel<true><<<grid, kPostThreads, 0, stream>>>(d.X, b.inv, (int)d.V, d.S, (int)d.T,
                                                                    plan.steps_per_part, b.mag, b.theta, b.phi,
                                                                    b.part_val, b.part_idx);
    spherical_max_kernel<true><<<vgrid, kPostThreads, 0, stream>>>(d.X, b.inv, (int)d.V, d.S, plan.parts, b.part_val,
                                                                   b.part_idx, sample_rate_hz, b.maxmag, b.mag_max,
                                                                   b.theta_max, b.phi_max, b.activation_ms, d.status);
  } else {
    spherical_part_kernel<false><<<grid, kPostThreads, 0, stream>>>(d.X, b.inv, (int)d.V, d.S, (int)d.T,
                                                                     plan.steps_per_part, nullptr, nullptr, nullptr,
                                                                     b.part_val, b.part_idx);
    spherical_max_kernel<false><<<vgrid, kPostThreads, 0, stream>>>(d.X, b.inv, (int)d.V, d.S, plan.parts,
                                                                    b.part_val, b.part_idx, sample_rate_hz, b.maxmag,
                                                                    nullptr, nullptr, nullptr, nullptr, d.status);
  }
  return cudaGetLastError();
}

cudaError_t launch_final_metrics(const PostBuffers& b, const int32_t* types, const int32_t* numbers, int64_t cells,
                                 unsigned long long* hist, float* out, int sms, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * 2 * (CT_THRESHOLDS + 1), stream);
  if (e != cudaSuccess) return e;
  const int64_t want = (cells + 255) / 256;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 8));
  threshold_hist_kernel<<<grid, 256, 0, stream>>>(types, numbers, cells, b.maxmag, hist);
  final_metrics_kernel<<<1, 128, 0, stream>>>(hist, out);
  return cudaGetLastError();
}

}  // namespace ct
