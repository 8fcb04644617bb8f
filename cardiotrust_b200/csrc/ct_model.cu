// Model construction on the device: the Biot-Savart measurement matrix and the all-pass delay
// arrays, the two O(voxels x ...) fills that build a scenario before its first epoch.
//
//   lead_field_kernel    <- MeasurementMatrix::from_model_spatial_description
//                           src/core/model/functional/measurement.rs:66-123
//   delay_samples_kernel <- calculate_delay_samples_array src/core/model/functional/allpass/delay.rs:35-111
//                           + from_samples_to_usize / from_samples_to_coef (allpass.rs:86-100, 644-660)
//
// Both are elementwise and bound by their HBM writes (12 bytes per (beat, sensor row, voxel) of H;
// 12 bytes per (voxel, offset) of the delay arrays). Every product, sum, quotient and square root
// is an explicitly rounded intrinsic in the reference's order, and `mul_add` is fmaf, so the
// results equal the reference's f32 arithmetic bit for bit.

#include "ct_internal.cuh"

namespace ct {
namespace {

__device__ __forceinline__ bool connectable(int32_t t) { return t >= 1 && t <= 6; }  // voxels.rs:690-700

// One thread per (row = beat x sensor, entry i of the voxel list), grid-stride. Entry i is the voxel
// at vpos[i] whose three states are columns col[i] .. col[i] + 2 of every row of H (pitch ldh).
__global__ void lead_field_kernel(const float* __restrict__ vpos, const int32_t* __restrict__ col, int64_t nv,
                                  const float* __restrict__ spos, const float* __restrict__ sori,
                                  const float* __restrict__ off, int64_t M, int64_t rows, float cf,
                                  float* __restrict__ H, int64_t ldh) {
  const int64_t total = rows * nv;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = idx / nv, i = idx - row * nv;
    const int64_t m = row % M, b = row / M;
    float d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
      d[k] = __fdiv_rn(__fsub_rn(__fadd_rn(spos[3 * m + k], off[3 * b + k]), vpos[3 * i + k]), 1000.0f);
    float sq = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) sq = __fadd_rn(sq, __fmul_rn(d[k], d[k]));
    const float r = __fsqrt_rn(sq);
    const float r3 = __fmul_rn(__fmul_rn(r, r), r);
    const float o0 = sori[3 * m], o1 = sori[3 * m + 1], o2 = sori[3 * m + 2];
    float* h = H + row * ldh + col[i];
    h[0] = __fdiv_rn(__fmul_rn(cf, fmaf(o2, d[1], -__fmul_rn(o1, d[2]))), r3);
    h[1] = __fdiv_rn(__fmul_rn(cf, fmaf(o0, d[2], -__fmul_rn(o2, d[0]))), r3);
    h[2] = __fdiv_rn(__fmul_rn(cf, fmaf(o1, d[0], -__fmul_rn(o0, d[1]))), r3);
  }
}

// One thread per (grid cell, offset column n). A connectable cell with voxel number 3v writes row v
// of the three [V, 26] arrays; a pair whose neighbour is outside the grid or not connectable keeps
// 0 samples (Coefs::empty). A delay below one sample (the reference's error), or one that is not a
// finite value below 2^31 (not representable as an i32 delay), records the smallest failing
// cell * 26 + n in *first_bad: the reference stops at the first failure in this order.
__global__ void delay_samples_kernel(const int32_t* __restrict__ types, const int32_t* __restrict__ numbers,
                                     const float* __restrict__ pos, int64_t nx, int64_t ny, int64_t nz,
                                     const float* __restrict__ vel, float rate, float* __restrict__ samples,
                                     int32_t* __restrict__ delays, float* __restrict__ coefs,
                                     unsigned long long* __restrict__ first_bad) {
  const int64_t total = nx * ny * nz * kOffsets;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = idx / kOffsets;
    const int n = (int)(idx - c * kOffsets);
    const int32_t t = types[c];
    if (!connectable(t)) continue;
    // delay_index_to_offset (allpass.rs:597-611)
    const int cc = n > 12 ? n + 1 : n;
    const int ox = cc / 9 - 1, oy = cc / 3 % 3 - 1, oz = cc % 3 - 1;
    const int64_t z = c % nz, y = c / nz % ny, x = c / (ny * nz);
    const int64_t X = x + ox, Y = y + oy, Z = z + oz;
    float s = 0.0f;
    if (X >= 0 && X < nx && Y >= 0 && Y < ny && Z >= 0 && Z < nz) {
      const int64_t co = (X * ny + Y) * nz + Z;
      if (connectable(types[co])) {
        // calculate_delay_s (delay.rs:14-23): |(in - out) / 1000| / velocity, then x sample rate
        float sq = 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float dk = __fdiv_rn(__fsub_rn(pos[3 * c + k], pos[3 * co + k]), 1000.0f);
          sq = __fadd_rn(sq, __fmul_rn(dk, dk));
        }
        s = __fmul_rn(__fdiv_rn(__fsqrt_rn(sq), vel[t]), rate);
        if (!(s >= 1.0f) || !(s < 2147483648.0f)) {
          atomicMin(first_bad, (unsigned long long)idx);
          s = 1.0f;  // keeps the cast below defined; the call reports the failure and no result
        }
      }
    }
    const int64_t o = (int64_t)(numbers[c] / 3) * kOffsets + n;
    samples[o] = s;
    delays[o] = (int32_t)s;  // from_samples_to_usize truncates
    // from_samples_to_coef: (1 - frac) / (1 + frac) clamped to [1e-4, 1 - 1e-4]
    const float frac = fmodf(s, 1.0f);
    const float coef = __fdiv_rn(__fsub_rn(1.0f, frac), __fadd_rn(1.0f, frac));
    coefs[o] = fminf(fmaxf(coef, 1e-4f), __fsub_rn(1.0f, 1e-4f));
  }
}

unsigned fill_grid(int64_t n, int num_sms) {
  const int64_t blocks = (n + 255) / 256;
  const int64_t cap = (int64_t)num_sms * 16;
  return (unsigned)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

}  // namespace

float lead_field_factor(float voxel_size_mm) {
  // (VACUUM_MAG_PERMEABILITY as f32 * voxel_volume_m3) / (4 * PI) * 1e12 (measurement.rs:85-88)
  const float mu0 = 1.25663706212e-6f;
  const float pi = 3.14159265358979323846f;
  const float size_m = voxel_size_mm / 1000.0f;
  const float volume = (size_m * size_m) * size_m;
  return (mu0 * volume) / (4.0f * pi) * 1e12f;
}

cudaError_t launch_lead_field(const float* vpos, const int32_t* col, int64_t nv, const float* spos,
                              const float* sori, const float* off, int64_t M, int64_t B, float cf, float* H,
                              int64_t ldh, int num_sms, cudaStream_t stream) {
  if (nv <= 0 || M <= 0 || B <= 0) return cudaSuccess;
  lead_field_kernel<<<fill_grid(B * M * nv, num_sms), 256, 0, stream>>>(vpos, col, nv, spos, sori, off, M, B * M,
                                                                        cf, H, ldh);
  return cudaGetLastError();
}

cudaError_t launch_delay_samples(const int32_t* types, const int32_t* numbers, const float* pos, int64_t nx,
                                 int64_t ny, int64_t nz, const float* vel, float rate, float* samples,
                                 int32_t* delays, float* coefs, unsigned long long* first_bad, int num_sms,
                                 cudaStream_t stream) {
  const int64_t n = nx * ny * nz * kOffsets;
  if (n <= 0) return cudaSuccess;
  delay_samples_kernel<<<fill_grid(n, num_sms), 256, 0, stream>>>(types, numbers, pos, nx, ny, nz, vel, rate,
                                                                   samples, delays, coefs, first_bad);
  return cudaGetLastError();
}

}  // namespace ct
