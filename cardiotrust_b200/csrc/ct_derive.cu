// Reference-mode derivation of one beat: the per-step accumulation of
// calculate_step_derivatives (src/core/algorithm/refinement/derivation.rs:173-229)
// run for all steps of the beat after the forward pass.
//
// The reference derivative at step t uses only quantities of steps <= t (the
// all-pass outputs of t and t-1, the states x[t] and x[t-d], the mapped
// residuals of t) and never feeds the states, so every (voxel, offset) pair
// is an independent sequential sweep over t once the states and mapped
// residuals of the beat exist. One thread owns one coefficient (v, n): the
// three all-pass / fir / iir chains (v, n, b), the nine gain derivatives
// dG[3v+a, 3n+b] and the coefficient derivative dC[v, n].
//
// Rounding follows the reference exactly (-fmad=false, fmaf where the
// reference calls mul_add, the same operand order), so for identical mapped
// residuals the gradients are bit-identical to the CPU loop:
//   gains     dG += ap * fma(mr, mse/M, maxreg * reg)                 derivation.rs:307-329
//   textbook  fir = fma(-c, fir, x[t-d]) ; iir = fma(-c, iir, ap_last) derivation.rs:418-465
//             dC += fma((fir - iir) * g * mr, mse/M, diff * delta^5)   derivation.rs:467-498
//   simple    dC += fma((x[t-d] - ap_last) * g * mr, mse/M, diff * delta^5)  derivation.rs:346-395
//   maxreg    f = |x0|+|x1|+|x2| - thr if positive, times signum(x_a)  derivation.rs:509-535
// The dC update visits (a, b) in the reference's row-major (state, column) order.
#include <cuda_runtime.h>

#include "ct_internal.cuh"

namespace ct {
namespace {

struct DeriveArgs {
  int64_t V, S, T;
  const int32_t* nbr;
  const float* coefs;
  const int32_t* delays;
  const float* init_delays;
  const float* gains;
  const float* X;
  const float* MR;
  float* dG;
  float* dC;
  float* fir;
  float* iir;
  DeriveScalars s;
};

__global__ void __launch_bounds__(128) derive_kernel(DeriveArgs p) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= p.V * kOffsets) return;
  const int64_t v = idx / kOffsets;
  const int n = (int)(idx - v * kOffsets);
  const int64_t S = p.S, T = p.T;
  const int32_t nb = p.nbr[idx];
  const bool valid = nb >= 0;
  const int64_t j0 = valid ? 3 * (int64_t)nb : 0;
  const int64_t d = p.delays[idx];
  const float c = p.coefs[idx];
  const float minus_c = -c;
  // delay_delta^5 (powi(5) = x * ((x*x)*(x*x)))
  const float delay = (float)d + (1.0f - c) / (c + 1.0f);
  const float dx = p.init_delays[idx] - delay;
  const float dx2 = dx * dx;
  const float dx4 = dx2 * dx2;
  const float dr_dd = p.s.diffreg * (dx * dx4);

  float g[3][3], dG[3][3];
  float ap[3] = {0.0f, 0.0f, 0.0f}, fir[3], iir[3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      g[a][b] = p.gains[(3 * v + a) * kGainCols + 3 * n + b];
      dG[a][b] = p.dG[(3 * v + a) * kGainCols + 3 * n + b];
    }
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    fir[b] = p.fir[v * kGainCols + 3 * n + b];
    iir[b] = p.iir[v * kGainCols + 3 * n + b];
  }
  float dC = p.dC[idx];
  const float mse_s = p.s.mse_scaling, reg_s = p.s.reg_scaling, thr = p.s.threshold;
  const bool do_gains = !p.s.freeze_gains, do_coefs = !p.s.freeze_delays;
  const bool textbook = p.s.ap_derivative != 0;

  // Step t needs x[t-d] (all-pass input, fir input), x[t-d-1] (= the input of step t-1),
  // x[t, 3v..3v+2] and mr[t, 3v..3v+2]. The loads of step t+1 are issued before the
  // arithmetic of step t (two-stage software pipeline).
  const float* xv = p.X + 3 * v;
  const float* mrv = p.MR + 3 * v;
  float in_prev[3] = {0.0f, 0.0f, 0.0f};
  float nin[3], nx[3], nmr[3];
#pragma unroll
  for (int b = 0; b < 3; ++b) nin[b] = (valid && d <= 0) ? __ldg(p.X + j0 + b) : 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    nx[a] = __ldg(xv + a);
    nmr[a] = __ldg(mrv + a);
  }
  for (int64_t t = 0; t < T; ++t) {
    float in[3], x[3], mr[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      in[q] = nin[q];
      x[q] = nx[q];
      mr[q] = nmr[q];
    }
    if (t + 1 < T) {
      const int64_t tn = t + 1;
#pragma unroll
      for (int b = 0; b < 3; ++b) nin[b] = (valid && d <= tn) ? __ldg(p.X + (tn - d) * S + j0 + b) : 0.0f;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        nx[a] = __ldg(xv + tn * S + a);
        nmr[a] = __ldg(mrv + tn * S + a);
      }
    }
    float ap_last[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      ap_last[b] = ap[b];
      // in_prev = x[t-d-1] (zero while t-d-1 < 0), prediction.rs:73-77
      if (valid) ap[b] = fmaf(c, in[b] - ap[b], in_prev[b]);
      in_prev[b] = in[b];
    }
    float mreg[3];
    const float sum = fabsf(x[0]) + fabsf(x[1]) + fabsf(x[2]);
    const bool over = sum > thr;
    const float f = sum - thr;
#pragma unroll
    for (int a = 0; a < 3; ++a) mreg[a] = over ? f * copysignf(1.0f, x[a]) : 0.0f;
    if (do_gains) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float q = fmaf(mr[a], mse_s, mreg[a] * reg_s);
#pragma unroll
        for (int b = 0; b < 3; ++b) dG[a][b] = dG[a][b] + ap[b] * q;
      }
    }
    if (do_coefs) {
      if (textbook) {
        if (t >= d) {
#pragma unroll
          for (int b = 0; b < 3; ++b) {
            if (valid) fir[b] = fmaf(minus_c, fir[b], in[b]);
            iir[b] = fmaf(minus_c, iir[b], ap_last[b]);
          }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) dC = dC + fmaf((fir[b] - iir[b]) * g[a][b] * mr[a], mse_s, dr_dd);
      } else if (valid && t >= d) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) dC = dC + fmaf((in[b] - ap_last[b]) * g[a][b] * mr[a], mse_s, dr_dd);
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) p.dG[(3 * v + a) * kGainCols + 3 * n + b] = dG[a][b];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    p.fir[v * kGainCols + 3 * n + b] = fir[b];
    p.iir[v * kGainCols + 3 * n + b] = iir[b];
  }
  p.dC[idx] = dC;
}

}  // namespace

cudaError_t launch_derive(DeviceScenario& d, const DeriveScalars& s, cudaStream_t stream) {
  DeriveArgs a;
  a.V = d.V;
  a.S = d.S;
  a.T = d.T;
  a.nbr = d.nbr;
  a.coefs = d.coefs;
  a.delays = d.delays;
  a.init_delays = d.init_delays;
  a.gains = d.gains;
  a.X = d.X;
  a.MR = d.MR;
  a.dG = d.dG;
  a.dC = d.dC;
  a.fir = d.fir;
  a.iir = d.iir;
  a.s = s;
  const int64_t n = d.V * kOffsets;
  derive_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace ct
