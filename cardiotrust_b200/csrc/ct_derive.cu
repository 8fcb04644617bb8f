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

  // Lanes b = 0, 1 of every (a, b) quantity are packed in a float2 and stepped with the packed FP32
  // instructions (fma2 / mul2 / add2 / sub2: each lane rounded to nearest like the scalar operation);
  // lane b = 2 stays scalar. The dC sum is accumulated term by term in the reference's (a, b) order.
  float2 g01[3], dG01[3];
  float g2[3], dG2[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float* gr = p.gains + (3 * v + a) * kGainCols + 3 * n;
    const float* dr = p.dG + (3 * v + a) * kGainCols + 3 * n;
    g01[a] = make_float2(gr[0], gr[1]);
    g2[a] = gr[2];
    dG01[a] = make_float2(dr[0], dr[1]);
    dG2[a] = dr[2];
  }
  const float* fr = p.fir + v * kGainCols + 3 * n;
  const float* ir = p.iir + v * kGainCols + 3 * n;
  float2 fir01 = make_float2(fr[0], fr[1]), iir01 = make_float2(ir[0], ir[1]);
  float fir2 = fr[2], iir2 = ir[2];
  float2 ap01 = make_float2(0.0f, 0.0f);
  float ap2 = 0.0f;
  float dC = p.dC[idx];
  const float mse_s = p.s.mse_scaling, reg_s = p.s.reg_scaling, thr = p.s.threshold;
  const float2 c2 = make_float2(c, c), mc2 = make_float2(minus_c, minus_c);
  const float2 mse2 = make_float2(mse_s, mse_s), reg2 = make_float2(reg_s, reg_s), drdd2 = make_float2(dr_dd, dr_dd);
  const bool do_gains = !p.s.freeze_gains, do_coefs = !p.s.freeze_delays;
  const bool textbook = p.s.ap_derivative != 0;

  // Step t needs x[t-d] (all-pass input, fir input), x[t-d-1] (= the input of step t-1),
  // x[t, 3v..3v+2] and mr[t, 3v..3v+2]. The loads of step t+1 are issued before the
  // arithmetic of step t (two-stage software pipeline).
  const float* xv = p.X + 3 * v;
  const float* mrv = p.MR + 3 * v;
  float2 inp01 = make_float2(0.0f, 0.0f);
  float inp2 = 0.0f;
  float nin[3], nx[3], nmr[3];
#pragma unroll
  for (int b = 0; b < 3; ++b) nin[b] = (valid && d <= 0) ? __ldg(p.X + j0 + b) : 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    nx[a] = __ldg(xv + a);
    nmr[a] = __ldg(mrv + a);
  }
  for (int64_t t = 0; t < T; ++t) {
    const float2 in01 = make_float2(nin[0], nin[1]);
    const float in2 = nin[2];
    const float x0 = nx[0], x1 = nx[1], x2 = nx[2];
    const float2 mr01 = make_float2(nmr[0], nmr[1]);
    const float mr2 = nmr[2];
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
    // all-pass step, prediction.rs:73-79 (in_prev = x[t-d-1], zero while t-d-1 < 0)
    const float2 apl01 = ap01;
    const float apl2 = ap2;
    if (valid) {
      ap01 = fma2(c2, sub2(in01, ap01), inp01);
      ap2 = fmaf(c, in2 - ap2, inp2);
    }
    inp01 = in01;
    inp2 = in2;
    // maximum regularisation, derivation.rs:509-535
    const float sum = fabsf(x0) + fabsf(x1) + fabsf(x2);
    const bool over = sum > thr;
    const float f = sum - thr;
    const float2 mreg01 = over ? mul2(make_float2(f, f), make_float2(copysignf(1.0f, x0), copysignf(1.0f, x1)))
                               : make_float2(0.0f, 0.0f);
    const float mreg2 = over ? f * copysignf(1.0f, x2) : 0.0f;
    if (do_gains) {
      // q[a] = fma(mr[a], mse/M, maxreg[a] * reg); dG[a][b] += ap[b] * q[a]
      const float2 q01 = fma2(mr01, mse2, mul2(mreg01, reg2));
      const float q[3] = {q01.x, q01.y, fmaf(mr2, mse_s, mreg2 * reg_s)};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        dG01[a] = add2(dG01[a], mul2(ap01, make_float2(q[a], q[a])));
        dG2[a] = dG2[a] + ap2 * q[a];
      }
    }
    if (do_coefs) {
      float2 e01;
      float e2;
      bool add = true;
      if (textbook) {
        if (t >= d) {
          if (valid) {
            fir01 = fma2(mc2, fir01, in01);
            fir2 = fmaf(minus_c, fir2, in2);
          }
          iir01 = fma2(mc2, iir01, apl01);
          iir2 = fmaf(minus_c, iir2, apl2);
        }
        e01 = sub2(fir01, iir01);
        e2 = fir2 - iir2;
      } else {
        add = valid && t >= d;
        e01 = sub2(in01, apl01);
        e2 = in2 - apl2;
      }
      if (add) {
        const float mr[3] = {mr01.x, mr01.y, mr2};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          // ((e[b] * g[a][b]) * mr[a]) then fma(., mse/M, diff * delta^5), summed in (a, b) order
          const float2 t01 = fma2(mul2(mul2(e01, g01[a]), make_float2(mr[a], mr[a])), mse2, drdd2);
          const float t2 = fmaf((e2 * g2[a]) * mr[a], mse_s, dr_dd);
          dC = dC + t01.x;
          dC = dC + t01.y;
          dC = dC + t2;
        }
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float* dr = p.dG + (3 * v + a) * kGainCols + 3 * n;
    dr[0] = dG01[a].x;
    dr[1] = dG01[a].y;
    dr[2] = dG2[a];
  }
  float* fw = p.fir + v * kGainCols + 3 * n;
  float* iw = p.iir + v * kGainCols + 3 * n;
  fw[0] = fir01.x;
  fw[1] = fir01.y;
  fw[2] = fir2;
  iw[0] = iir01.x;
  iw[1] = iir01.y;
  iw[2] = iir2;
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
