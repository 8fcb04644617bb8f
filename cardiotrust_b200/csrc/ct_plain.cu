// Plain GPU form of one beat: the straightforward port, kept as the baseline
// the persistent and batched forms are measured against. Like the reference's
// OpenCL path (src/core/algorithm/gpu/epoch.rs:96-117: prediction,
// derivation and metrics kernels launched once per step), every phase of
// every step is its own launch with one thread per output:
//   all-pass update (v, k) -> states (i) -> H x and residuals (sensor) ->
//   H^T r (i) -> maximum regularisation (v) -> step metrics (1 block) ->
//   gain derivatives (i, k) -> fir/iir (v, k) -> coefficient derivatives (v, n).
// Arithmetic follows the reference loops (prediction.rs:40-130,
// derivation.rs:173-551, metrics.rs:180-196): the states and the H^T r
// products are in the reference's order; H x and the metric sums reduce in a
// tree, so downstream values agree within the stated tolerances.
#include <cuda_runtime.h>

#include "ct_internal.cuh"

namespace ct {
namespace {

constexpr int kBlock = 256;

int64_t nblocks(int64_t n, int per) { return (n + per - 1) / per; }

__global__ void plain_ap_kernel(const int32_t* __restrict__ nbr, const float* __restrict__ coefs,
                                const int32_t* __restrict__ delays, const float* __restrict__ X, float* __restrict__ ap,
                                float* __restrict__ ap_last, int64_t V, int64_t S, int t) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= V * kGainCols) return;
  const int64_t v = e / kGainCols;
  const int k = (int)(e - v * kGainCols), n = k / 3, b = k - 3 * n;
  const float prev = ap[e];
  ap_last[e] = prev;
  const int32_t j = nbr[v * kOffsets + n];
  if (j < 0) return;
  const int d = delays[v * kOffsets + n];
  const float in = d <= t ? X[(int64_t)(t - d) * S + 3 * j + b] : 0.0f;
  const float in1 = d < t ? X[(int64_t)(t - d - 1) * S + 3 * j + b] : 0.0f;
  ap[e] = fmaf(coefs[v * kOffsets + n], in - prev, in1);
}

__global__ void plain_states_kernel(const int32_t* __restrict__ nbr, const float* __restrict__ gains,
                                    const float* __restrict__ ap, const float* __restrict__ ctrl,
                                    const float* __restrict__ u, float* __restrict__ X, int64_t S, int t) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S) return;
  const int64_t v = i / 3;
  float x = 0.0f;
  for (int k = 0; k < kGainCols; ++k)
    if (nbr[v * kOffsets + k / 3] >= 0) x = x + gains[i * kGainCols + k] * ap[v * kGainCols + k];
  x = x + u[t] * ctrl[i];
  X[(int64_t)t * S + i] = x;
}

// One block per sensor row: y = H x, residual r = y - z.
__global__ void plain_predict_kernel(const float* __restrict__ H, const float* __restrict__ x,
                                     const float* __restrict__ z, float* __restrict__ y, float* __restrict__ r,
                                     int64_t S) {
  __shared__ float red[kBlock];
  const int64_t m = blockIdx.x;
  const float* h = H + m * S;
  float s = 0.0f;
  for (int64_t i = threadIdx.x; i < S; i += blockDim.x) s = s + h[i] * x[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    y[m] = red[0];
    r[m] = red[0] - z[m];
  }
}

// mr[i] = sum_m H[m, i] r[m], fused multiply-adds in m order in blocks of 256 rows (matrixmultiply sgemm).
__global__ void plain_mapped_kernel(const float* __restrict__ H, const float* __restrict__ r, float* __restrict__ mr,
                                    int64_t S, int64_t M) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S) return;
  float c = 0.0f;
  for (int64_t k0 = 0; k0 < M; k0 += 256) {
    const int64_t k1 = k0 + 256 < M ? k0 + 256 : M;
    float ab = 0.0f;
    for (int64_t m = k0; m < k1; ++m) ab = fmaf(H[m * S + i], r[m], ab);
    c = k0 == 0 ? ab : ab + c;
  }
  mr[i] = c;
}

__global__ void plain_maxreg_kernel(const float* __restrict__ x, float* __restrict__ mreg, float* __restrict__ part,
                                    int64_t V, float threshold) {
  __shared__ float red[kBlock];
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float f2 = 0.0f;
  if (v < V) {
    const float x0 = x[3 * v], x1 = x[3 * v + 1], x2 = x[3 * v + 2];
    const float sum = fabsf(x0) + fabsf(x1) + fabsf(x2);
    if (sum > threshold) {
      const float f = sum - threshold;
      f2 = f * f;
      mreg[3 * v] = f * copysignf(1.0f, x0);
      mreg[3 * v + 1] = f * copysignf(1.0f, x1);
      mreg[3 * v + 2] = f * copysignf(1.0f, x2);
    } else {
      mreg[3 * v] = mreg[3 * v + 1] = mreg[3 * v + 2] = 0.0f;
    }
  }
  red[threadIdx.x] = f2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// loss_mse[t] = sum r^2 / M; running maximum-regularisation sum; loss[t] = fma(reg, loss_mr, mse).
__global__ void plain_metrics_kernel(const float* __restrict__ r, int64_t M, const float* __restrict__ part, int nparts,
                                     float* __restrict__ mreg_sum, float* __restrict__ loss_mse,
                                     float* __restrict__ loss_mr, float* __restrict__ loss, float reg, int t) {
  __shared__ float red[kBlock];
  float s = 0.0f;
  for (int64_t m = threadIdx.x; m < M; m += blockDim.x) s = s + r[m] * r[m];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const float mse = red[0] / (float)M;
    float acc = *mreg_sum;
    for (int p = 0; p < nparts; ++p) acc = acc + part[p];
    *mreg_sum = acc;
    loss_mse[t] = mse;
    loss_mr[t] = acc;
    loss[t] = fmaf(reg, acc, mse);
  }
}

__global__ void plain_gains_kernel(const float* __restrict__ ap, const float* __restrict__ mr,
                                   const float* __restrict__ mreg, float* __restrict__ dG, int64_t S, float mse_scaling,
                                   float reg_scaling) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= S * kGainCols) return;
  const int64_t i = e / kGainCols;
  const int k = (int)(e - i * kGainCols);
  const float a = ap[(i / 3) * kGainCols + k];
  dG[e] = dG[e] + a * fmaf(mr[i], mse_scaling, mreg[i] * reg_scaling);
}

__global__ void plain_fir_iir_kernel(const int32_t* __restrict__ nbr, const float* __restrict__ coefs,
                                     const int32_t* __restrict__ delays, const float* __restrict__ X,
                                     const float* __restrict__ ap_last, float* __restrict__ fir,
                                     float* __restrict__ iir, int64_t V, int64_t S, int t) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= V * kGainCols) return;
  const int64_t v = e / kGainCols;
  const int k = (int)(e - v * kGainCols), n = k / 3, b = k - 3 * n;
  const int d = delays[v * kOffsets + n];
  if (t < d) return;
  const float c = coefs[v * kOffsets + n];
  const int32_t j = nbr[v * kOffsets + n];
  if (j >= 0) fir[e] = fmaf(-c, fir[e], X[(int64_t)(t - d) * S + 3 * j + b]);
  iir[e] = fmaf(-c, iir[e], ap_last[e]);
}

__device__ __forceinline__ float powi5(float x) {
  const float x2 = x * x;
  const float x4 = x2 * x2;
  return x * x4;
}

// dC[v, n] over the 9 (row, column) pairs in the reference's order (rows outer, columns inner).
__global__ void plain_coefs_kernel(const int32_t* __restrict__ nbr, const float* __restrict__ coefs,
                                   const int32_t* __restrict__ delays, const float* __restrict__ init_delays,
                                   const float* __restrict__ gains, const float* __restrict__ mr,
                                   const float* __restrict__ X, const float* __restrict__ ap_last,
                                   const float* __restrict__ fir, const float* __restrict__ iir,
                                   float* __restrict__ dC, int64_t V, int64_t S, int t, float mse_scaling, float diffreg,
                                   int textbook) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= V * kOffsets) return;
  const int64_t v = e / kOffsets;
  const int n = (int)(e - v * kOffsets);
  const int32_t j = nbr[e];
  const int d = delays[e];
  const float c = coefs[e];
  const float dd = powi5(init_delays[e] - ((float)d + (1.0f - c) / (c + 1.0f)));
  const float reg_term = diffreg * dd;
  float acc = dC[e];
  for (int a = 0; a < 3; ++a) {
    const int64_t i = 3 * v + a;
    for (int b = 0; b < 3; ++b) {
      const int k = 3 * n + b;
      const float g = gains[i * kGainCols + k];
      if (textbook) {
        const float diff = fir[v * kGainCols + k] - iir[v * kGainCols + k];
        acc = acc + fmaf(diff * g * mr[i], mse_scaling, reg_term);
      } else if (j >= 0 && t >= d) {
        const float sv = X[(int64_t)(t - d) * S + 3 * j + b];
        acc = acc + fmaf((sv - ap_last[v * kGainCols + k]) * g * mr[i], mse_scaling, reg_term);
      }
    }
  }
  dC[e] = acc;
}

}  // namespace

int plain_step_launches(const PlainScalars& s) {
  return 6 + (s.freeze_gains ? 0 : 1) + (s.freeze_delays ? 0 : (s.ap_derivative == CT_AP_TEXTBOOK ? 2 : 1));
}

cudaError_t launch_plain_beat(DeviceScenario& d, int64_t beat, const PlainScalars& s, cudaStream_t stream) {
  const int64_t V = d.V, S = d.S, M = d.M, T = d.T;
  cudaError_t err = cudaMemsetAsync(d.ap, 0, sizeof(float) * V * kGainCols, stream);
  if (err != cudaSuccess) return err;
  const float* H = d.H + beat * M * S;
  const int vblocks = (int)nblocks(V, kBlock);
  for (int t = 0; t < (int)T; ++t) {
    float* x = d.X + (int64_t)t * S;
    float* r = d.R + (int64_t)t * M;
    float* mr = d.MR + (int64_t)t * S;
    plain_ap_kernel<<<nblocks(V * kGainCols, kBlock), kBlock, 0, stream>>>(d.nbr, d.coefs, d.delays, d.X, d.ap,
                                                                            d.ap_last, V, S, t);
    plain_states_kernel<<<nblocks(S, kBlock), kBlock, 0, stream>>>(d.nbr, d.gains, d.ap, d.ctrl, d.u, d.X, S, t);
    plain_predict_kernel<<<(int)M, kBlock, 0, stream>>>(H, x, d.meas + (beat * T + t) * M,
                                                        d.Y + (beat * T + t) * M, r, S);
    plain_mapped_kernel<<<nblocks(S, kBlock), kBlock, 0, stream>>>(H, r, mr, S, M);
    plain_maxreg_kernel<<<vblocks, kBlock, 0, stream>>>(x, d.plain_mreg, d.plain_part, V, s.threshold);
    plain_metrics_kernel<<<1, kBlock, 0, stream>>>(r, M, d.plain_part, vblocks, d.mreg_sum, d.loss_mse, d.loss_mr,
                                                   d.loss, s.reg_scaling, t);
    if (!s.freeze_gains)
      plain_gains_kernel<<<nblocks(S * kGainCols, kBlock), kBlock, 0, stream>>>(d.ap, mr, d.plain_mreg, d.dG, S,
                                                                                 s.mse_scaling, s.reg_scaling);
    if (!s.freeze_delays) {
      const bool textbook = s.ap_derivative == CT_AP_TEXTBOOK;
      if (textbook)
        plain_fir_iir_kernel<<<nblocks(V * kGainCols, kBlock), kBlock, 0, stream>>>(
            d.nbr, d.coefs, d.delays, d.X, d.ap_last, d.fir, d.iir, V, S, t);
      plain_coefs_kernel<<<nblocks(V * kOffsets, kBlock), kBlock, 0, stream>>>(
          d.nbr, d.coefs, d.delays, d.init_delays, d.gains, mr, d.X, d.ap_last, d.fir, d.iir, d.dC, V, S, t,
          s.mse_scaling, s.diffreg, textbook ? 1 : 0);
    }
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

}  // namespace ct
