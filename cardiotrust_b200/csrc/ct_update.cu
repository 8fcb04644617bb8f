// Per-batch work of the epoch: parameter update, delay roll, average delays,
// smoothness derivative, and the step / batch metrics.
//
// Elementwise arithmetic follows the reference exactly (-fmad=false, IEEE
// division and square root); for identical gradients the updated parameters
// are bit-identical to the CPU loop.
#include <cuda_runtime.h>

#include <climits>

#include "ct_internal.cuh"

namespace ct {
namespace {

// ---- APParameters::update, src/core/algorithm/refinement/update.rs:27-200

__global__ void sgd_kernel(float* __restrict__ p, const float* __restrict__ g, int64_t n, float lr_over_bs) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = p[i] - lr_over_bs * g[i];
}

// bias_dev, when set, holds {bias1, bias2} of this update (written by the host before a graph replay).
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, int64_t n, float lr_over_bs, float bias1, float bias2,
                            const float* __restrict__ bias_dev) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (bias_dev) {
    bias1 = bias_dev[0];
    bias2 = bias_dev[1];
  }
  const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  const float omb1 = 1.0f - beta1, omb2 = 1.0f - beta2;
  const float gi = g[i];
  const float m = m1[i] * beta1 + omb1 * gi;
  const float v = m2[i] * beta2 + omb2 * gi * gi;
  m1[i] = m;
  m2[i] = v;
  const float mc = m / bias1;
  const float vc = v / bias2;
  const float factor = mc / (sqrtf(vc) + eps);
  p[i] = p[i] - lr_over_bs * factor;
}

// roll_delays, update.rs:206-228
__global__ void roll_delays_kernel(float* __restrict__ coefs, int32_t* __restrict__ delays, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float margin = 1e-4f;
  float c = coefs[i];
  int32_t d = delays[i];
  if (c > 1.0f - margin) {
    if (d > 1) {
      c = 2.0f * margin;
      d -= 1;
    } else {
      c = 1.0f - margin;
    }
  } else if (c < margin) {
    if (d < 1000) {
      c = fmaf(2.0f, -margin, 1.0f);
      d += 1;
    } else {
      c = margin;
    }
  }
  coefs[i] = c;
  delays[i] = d;
}

// dmin[0] = smallest, dmin[1] = largest delay of a connected (voxel, offset) pair
__global__ void min_delay_kernel(const int32_t* __restrict__ nbr, const int32_t* __restrict__ delays, int64_t n,
                                 int32_t* __restrict__ dmin) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int32_t lo = INT_MAX, hi = INT_MIN;
  if (i < n && nbr[i] >= 0) lo = hi = delays[i];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    lo = min(lo, __shfl_down_sync(0xffffffffu, lo, off));
    hi = max(hi, __shfl_down_sync(0xffffffffu, hi, off));
  }
  if ((threadIdx.x & 31) == 0 && lo != INT_MAX) {
    atomicMin(dmin, lo);
    atomicMax(dmin + 1, hi);
  }
}

__global__ void set_min_max_kernel(int32_t* p) {
  p[0] = INT_MAX;
  p[1] = INT_MIN;
}

// ---- calculate_average_delays, derivation.rs:554-594
__device__ __forceinline__ int offset_l1(int n) {
  const int c = n > 12 ? n + 1 : n;
  return abs(c / 9 - 1) + abs((c / 3) % 3 - 1) + abs(c % 3 - 1);
}

__global__ void average_delays_kernel(const float* __restrict__ gains, const float* __restrict__ coefs,
                                      const int32_t* __restrict__ delays, int64_t V, float* __restrict__ out) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  float delay_sum = 0.0f, gain_sum = 0.0f;
  for (int n = 0; n < kOffsets; ++n) {
    const float c = coefs[v * kOffsets + n];
    const float delay = (float)delays[v * kOffsets + n] + (1.0f - c) / (c + 1.0f);
    const float corrected = delay / sqrtf((float)offset_l1(n));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        const float g = fabsf(gains[(3 * v + a) * kGainCols + 3 * n + b]);
        delay_sum = delay_sum + g * corrected;
        gain_sum = gain_sum + g;
      }
  }
  out[v] = (gain_sum == 0.0f) ? __int_as_float(0x7fc00000) : delay_sum / gain_sum;
}

// ---- calculate_smoothness_derivatives, derivation.rs:260-302
__global__ void smoothness_kernel(const float* __restrict__ avg, const int32_t* __restrict__ nbr, int64_t V,
                                  float strength, float* __restrict__ dC) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= V * kOffsets) return;
  const int64_t v = idx / kOffsets;
  const float own = avg[v];
  if (isnan(own)) return;
  float neighbourhood = own, divisor = 1.0f;
  for (int n = 0; n < kOffsets; ++n) {
    const int32_t nb = nbr[v * kOffsets + n];
    if (nb < 0) continue;
    const float dn = avg[nb];
    if (!isnan(dn)) {
      neighbourhood = neighbourhood + dn;
      divisor = divisor + 1.0f;
    }
  }
  neighbourhood = neighbourhood / divisor;
  dC[idx] = dC[idx] + strength * (neighbourhood - own);
}

// ---- metrics::calculate_step (metrics.rs:180-196) for all steps of a beat.
// stepsum[t] = sum over forward CTAs of their partial max-regularisation sums
// (step_sum_kernel: one warp per step, a fixed order), then a deterministic block
// scan gives the running sum.

// out[t] = sum over c of part[t * grid + c]: lane l adds the partials l, l + 32, ... in order, then a
// fixed butterfly combines the lanes, so every run and every caller gets the same sum.
__global__ void step_sum_kernel(const float* __restrict__ part, int grid, int64_t T, float* __restrict__ out) {
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= T) return;
  float s = 0.0f;
  for (int c = lane; c < grid; c += 32) s = s + part[t * grid + c];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) out[t] = s;
}

// `part` may alias `loss_mr`: each step's value is read before the same thread writes it.
__global__ void step_metrics_kernel(const float* part, int grid, int64_t T, float reg,
                                    float* __restrict__ mreg_sum, const float* __restrict__ loss_mse,
                                    float* loss_mr, float* __restrict__ loss) {
  constexpr int kT = 1024;
  __shared__ float warp_tot[kT / 32];
  __shared__ float carry_s;
  const int tid = threadIdx.x;
  if (tid == 0) carry_s = *mreg_sum;
  __syncthreads();
  for (int64_t base = 0; base < T; base += (int64_t)kT * 8) {
    // each thread: up to 8 consecutive steps
    float vals[8];
    float local = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t t = base + (int64_t)tid * 8 + q;
      float s = 0.0f;
      if (t < T)
        for (int c = 0; c < grid; ++c) s = s + part[t * grid + c];
      local = local + s;
      vals[q] = local;  // inclusive prefix within the thread
    }
    // warp inclusive scan of thread totals
    float x = local;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const float y = __shfl_up_sync(0xffffffffu, x, off);
      if ((tid & 31) >= off) x = x + y;
    }
    if ((tid & 31) == 31) warp_tot[tid / 32] = x;
    __syncthreads();
    if (tid < 32) {
      float w = warp_tot[tid];
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const float y = __shfl_up_sync(0xffffffffu, w, off);
        if (tid >= off) w = w + y;
      }
      warp_tot[tid] = w;
    }
    __syncthreads();
    const float carry = carry_s;
    float excl = __shfl_up_sync(0xffffffffu, x, 1);
    if ((tid & 31) == 0) excl = 0.0f;
    const float before = (tid >= 32) ? warp_tot[tid / 32 - 1] + excl : excl;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t t = base + (int64_t)tid * 8 + q;
      if (t < T) {
        const float running = carry + (before + vals[q]);
        loss_mr[t] = running;
        loss[t] = fmaf(reg, running, loss_mse[t]);
      }
    }
    __syncthreads();
    if (tid == kT - 1) carry_s = carry + (before + vals[7]);
    __syncthreads();
  }
  if (tid == 0) *mreg_sum = carry_s;
}

// ---- metrics::calculate_batch (metrics.rs:204-219): means with ndarray's
// eight-accumulator summation; thread q of each group runs accumulator q.
// index_dev, when set, holds the slot (offset of o0/o1/o2) of this batch, read on the device.
__global__ void batch_metrics_kernel(const float* __restrict__ a0, const float* __restrict__ a1,
                                     const float* __restrict__ a2, int64_t T, float* __restrict__ o0,
                                     float* __restrict__ o1, float* __restrict__ o2, const int64_t* index_dev,
                                     int64_t slots, int32_t* status) {
  __shared__ float p[3][8];
  if (index_dev) {
    const int64_t idx = *index_dev;
    if (idx < 0 || idx >= slots) {
      if (threadIdx.x == 0) atomicCAS(status, 0, (int32_t)CT_ERR_BATCH_INDEX);
      return;
    }
    o0 += idx;
    o1 += idx;
    o2 += idx;
  }
  const int which = threadIdx.x / 8, q = threadIdx.x % 8;
  const float* xs = which == 0 ? a0 : (which == 1 ? a1 : a2);
  const int64_t full = (T / 8) * 8;
  if (which < 3) {
    float acc = 0.0f;
    for (int64_t i = q; i < full; i += 8) acc = acc + xs[i];
    p[which][q] = acc;
  }
  __syncthreads();
  if (q == 0 && which < 3) {
    float acc = 0.0f;
    acc = acc + (p[which][0] + p[which][4]);
    acc = acc + (p[which][1] + p[which][5]);
    acc = acc + (p[which][2] + p[which][6]);
    acc = acc + (p[which][3] + p[which][7]);
    for (int64_t i = full; i < T; ++i) acc = acc + xs[i];
    float* o = which == 0 ? o0 : (which == 1 ? o1 : o2);
    *o = acc / (float)T;
  }
}

__global__ void expand_rows_kernel(const float* __restrict__ src, float* __restrict__ dst, int64_t V) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 3 * V * kGainCols) return;
  const int64_t row = idx / kGainCols, k = idx - row * kGainCols;
  dst[idx] = src[(row / 3) * kGainCols + k];
}

__global__ void last_max_reg_kernel(const float* __restrict__ x, int64_t V, float thr, float* __restrict__ out) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const float x0 = x[3 * v], x1 = x[3 * v + 1], x2 = x[3 * v + 2];
  const float sum = fabsf(x0) + fabsf(x1) + fabsf(x2);
  if (sum > thr) {
    const float f = sum - thr;
    out[3 * v] = f * copysignf(1.0f, x0);
    out[3 * v + 1] = f * copysignf(1.0f, x1);
    out[3 * v + 2] = f * copysignf(1.0f, x2);
  } else {
    out[3 * v] = 0.0f;
    out[3 * v + 1] = 0.0f;
    out[3 * v + 2] = 0.0f;
  }
}

inline unsigned blocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_update(DeviceScenario& d, const UpdateScalars& s, cudaStream_t stream) {
  const int64_t ng = d.S * kGainCols, nc = d.V * kOffsets;
  if (!s.freeze_gains) {
    if (s.optimizer == CT_OPT_SGD)
      sgd_kernel<<<blocks(ng, 256), 256, 0, stream>>>(d.gains, d.dG, ng, s.lr_over_bs);
    else
      adam_kernel<<<blocks(ng, 256), 256, 0, stream>>>(d.gains, d.dG, d.mG1, d.mG2, ng, s.lr_over_bs, s.bias1,
                                                       s.bias2, s.bias_dev);
  }
  if (!s.freeze_delays) {
    if (s.optimizer == CT_OPT_SGD)
      sgd_kernel<<<blocks(nc, 256), 256, 0, stream>>>(d.coefs, d.dC, nc, s.lr_over_bs);
    else
      adam_kernel<<<blocks(nc, 256), 256, 0, stream>>>(d.coefs, d.dC, d.mC1, d.mC2, nc, s.lr_over_bs, s.bias1,
                                                       s.bias2, s.bias_dev);
    roll_delays_kernel<<<blocks(nc, 256), 256, 0, stream>>>(d.coefs, d.delays, nc);
  }
  return cudaGetLastError();
}

cudaError_t launch_min_delay(DeviceScenario& d, cudaStream_t stream) {
  set_min_max_kernel<<<1, 1, 0, stream>>>(d.dmin);
  const int64_t n = d.V * kOffsets;
  min_delay_kernel<<<blocks(n, 256), 256, 0, stream>>>(d.nbr, d.delays, n, d.dmin);
  return cudaGetLastError();
}

cudaError_t launch_average_delays(DeviceScenario& d, cudaStream_t stream) {
  average_delays_kernel<<<blocks(d.V, 128), 128, 0, stream>>>(d.gains, d.coefs, d.delays, d.V, d.avg_delays);
  return cudaGetLastError();
}

cudaError_t launch_smoothness(DeviceScenario& d, float strength, cudaStream_t stream) {
  smoothness_kernel<<<blocks(d.V * kOffsets, 256), 256, 0, stream>>>(d.avg_delays, d.nbr, d.V, strength, d.dC);
  return cudaGetLastError();
}

// The per-step sums go to loss_mr, which the scan then overwrites with the running sum in place (each
// step's value is read and written by the same thread).
cudaError_t launch_step_metrics(DeviceScenario& d, float reg_strength, cudaStream_t stream) {
  return launch_step_metrics_parts(d, d.stepsum_part, d.fwd_grid, reg_strength, stream);
}

cudaError_t launch_batch_metrics(DeviceScenario& d, int64_t index, cudaStream_t stream) {
  batch_metrics_kernel<<<1, 32, 0, stream>>>(d.loss_mse, d.loss_mr, d.loss, d.T, d.loss_mse_b + index,
                                             d.loss_mr_b + index, d.loss_b + index, nullptr, 0, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_batch_metrics_dev(DeviceScenario& d, const int64_t* index_dev, cudaStream_t stream) {
  batch_metrics_kernel<<<1, 32, 0, stream>>>(d.loss_mse, d.loss_mr, d.loss, d.T, d.loss_mse_b, d.loss_mr_b, d.loss_b,
                                             index_dev, d.NB, d.status);
  return cudaGetLastError();
}

cudaError_t launch_step_metrics_parts(DeviceScenario& d, const float* part, int parts, float reg_strength,
                                      cudaStream_t stream) {
  const int64_t threads = d.T * 32;
  step_sum_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(part, parts, d.T, d.loss_mr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  step_metrics_kernel<<<1, 1024, 0, stream>>>(d.loss_mr, 1, d.T, reg_strength, d.mreg_sum, d.loss_mse, d.loss_mr,
                                              d.loss);
  return cudaGetLastError();
}

// Voxel blocks of `words` 32-bit words: gather dst[u] = src[perm[u]] (reference -> device order) or
// scatter dst[perm[u]] = src[u] (device -> reference order).
template <bool kGather>
__global__ void permute_blocks_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                      const int32_t* __restrict__ perm, int64_t V, int64_t words) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V * words) return;
  const int64_t u = i / words, w = i - u * words;
  const int64_t r = perm[u];
  if (kGather)
    dst[i] = src[r * words + w];
  else
    dst[r * words + w] = src[i];
}

cudaError_t launch_permute_blocks(const void* src, void* dst, const int32_t* perm, int64_t V, int64_t words,
                                  bool gather, cudaStream_t stream) {
  const int64_t n = V * words;
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (gather)
    permute_blocks_kernel<true><<<grid, 256, 0, stream>>>(static_cast<const uint32_t*>(src), static_cast<uint32_t*>(dst),
                                                          perm, V, words);
  else
    permute_blocks_kernel<false><<<grid, 256, 0, stream>>>(static_cast<const uint32_t*>(src),
                                                           static_cast<uint32_t*>(dst), perm, V, words);
  return cudaGetLastError();
}

cudaError_t launch_expand_rows(const float* src, float* dst, int64_t V, cudaStream_t stream) {
  expand_rows_kernel<<<blocks(3 * V * kGainCols, 256), 256, 0, stream>>>(src, dst, V);
  return cudaGetLastError();
}

cudaError_t launch_last_max_reg(DeviceScenario& d, float threshold, float* out, cudaStream_t stream) {
  last_max_reg_kernel<<<blocks(d.V, 128), 128, 0, stream>>>(d.X + (d.T - 1) * d.S, d.V, threshold, out);
  return cudaGetLastError();
}

}  // namespace ct
