// Model construction: the Biot-Savart measurement matrix and the all-pass delay arrays on the device
// (the two O(voxels x ...) fills that build a scenario before its first epoch), and the
// activation-front gain search and the neighbour index table on the host.
//
//   lead_field_kernel    <- MeasurementMatrix::from_model_spatial_description
//                           src/core/model/functional/measurement.rs:66-123
//   delay_samples_kernel <- calculate_delay_samples_array src/core/model/functional/allpass/delay.rs:35-111
//                           + from_samples_to_usize / from_samples_to_coef (allpass.rs:86-100, 644-660)
//   connect_voxels_host  <- connect_voxels / try_to_connect src/core/model/functional/allpass.rs:295-494
//   output_state_indices_host <- init_output_state_indicies allpass.rs:212-289
//
// Both are elementwise and bound by their HBM writes (12 bytes per (beat, sensor row, voxel) of H;
// 12 bytes per (voxel, offset) of the delay arrays). Every product, sum, quotient and square root
// is an explicitly rounded intrinsic in the reference's order, and `mul_add` is fmaf, so the
// results equal the reference's f32 arithmetic bit for bit.

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

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

// ---- the activation-front search on the host (sequential by definition: a voxel's gains depend on
// which neighbour reached it first)

namespace ct {
namespace {

// approx::relative_eq! with epsilon = max_relative = f32::EPSILON.
bool relative_eq(float a, float b) {
  if (a == b) return true;
  if (std::isinf(a) || std::isinf(b)) return false;
  const float eps = 1.1920929e-7f;
  const float diff = std::fabs(a - b);
  return diff <= eps || diff <= std::fmax(std::fabs(a), std::fabs(b)) * eps;
}

bool host_connectable(int32_t t) { return t >= 1 && t <= 6; }

// voxels::is_connection_allowed(output, input), voxels.rs:707-742 (bit i of the mask: input type i).
bool allowed(int32_t out, int32_t in) {
  static const unsigned mask[10] = {0u,
                                    (1u << 2) | (1u << 5) | (1u << 6),
                                    (1u << 1) | (1u << 2) | (1u << 3) | (1u << 6),
                                    (1u << 2) | (1u << 4) | (1u << 6),
                                    (1u << 3) | (1u << 4) | (1u << 5) | (1u << 6),
                                    (1u << 4) | (1u << 5) | (1u << 6),
                                    0x3FFu,
                                    0u,
                                    0u,
                                    0u};
  if (out < 0 || out > 9 || in < 0 || in > 9) return false;
  return (mask[out] >> in) & 1u;
}

}  // namespace

// connect_voxels / try_to_connect (allpass.rs:295-494) with the reference's exact visiting rule:
// `current` runs through 0 and then each next larger activation time; at each, the voxels whose time
// is relative_eq to it (C order, a snapshot) try their 26 offsets (x outer, z inner), each activating
// an allowed, not yet activated input first come, first served. The activation times live in an
// ordered map, so a sweep step touches only the voxels near `current` instead of the whole grid.
// Voxel numbers must be valid for every connectable cell (checked by the caller).
void connect_voxels_host(const int32_t* types, const int32_t* numbers, const float* pos, int64_t nx, int64_t ny,
                         int64_t nz, const float* vel, float factor, float* gains, float* activation_ms) {
  const int64_t cells = nx * ny * nz;
  const float nan = std::nanf("");
  std::vector<float> t((size_t)cells, nan);
  std::vector<float> dir((size_t)(3 * cells), 0.0f);
  std::map<float, std::vector<int64_t>> by_time;
  for (int64_t c = 0; c < cells; ++c)
    if (types[c] == 1) {  // Sinoatrial
      t[(size_t)c] = 0.0f;
      dir[(size_t)(3 * c)] = 1.0f;
      by_time[0.0f].push_back(c);
    }
  const bool skip_patho = relative_eq(factor, 0.0f);
  const float inv = 1.0f / factor;
  float current = 0.0f;
  std::vector<int64_t> cand;
  for (;;) {
    // the times relative_eq to `current` lie within 2 max(eps, |current| eps) of it
    const float w = 2.0f * std::fmax(1.1920929e-7f, std::fabs(current) * 1.1920929e-7f);
    cand.clear();
    for (auto it = by_time.lower_bound(current - w); it != by_time.end() && it->first <= current + w; ++it)
      if (relative_eq(it->first, current)) cand.insert(cand.end(), it->second.begin(), it->second.end());
    std::sort(cand.begin(), cand.end());
    for (int64_t out : cand) {
      const int64_t xo = out / (ny * nz), yo = out / nz % ny, zo = out % nz;
      const int32_t type_out = types[out];
      for (int ox = -1; ox <= 1; ++ox)
        for (int oy = -1; oy <= 1; ++oy)
          for (int oz = -1; oz <= 1; ++oz) {
            if (ox == 0 && oy == 0 && oz == 0) continue;
            const int64_t xi = xo - ox, yi = yo - oy, zi = zo - oz;
            if (xi < 0 || xi >= nx || yi < 0 || yi >= ny || zi < 0 || zi >= nz) continue;
            const int64_t in = (xi * ny + yi) * nz + zi;
            const int32_t type_in = types[in];
            if (!host_connectable(type_in) || !std::isnan(t[(size_t)in])) continue;
            if (!allowed(type_out, type_in)) continue;
            if (type_in == 6 && skip_patho) continue;
            const float* pin = pos + 3 * in;
            const float* pout = pos + 3 * out;
            float d[3], sq = 0.0f, norm = 0.0f;
            for (int k = 0; k < 3; ++k) {
              d[k] = (pin[k] - pout[k]) / 1000.0f;
              sq = sq + d[k] * d[k];
              norm = norm + std::fabs(d[k]);
            }
            const float ti = t[(size_t)out] + std::sqrt(sq) / vel[type_in];  // calculate_delay_s
            t[(size_t)in] = ti;
            by_time[ti].push_back(in);
            for (int k = 0; k < 3; ++k) dir[(size_t)(3 * in + k)] = d[k] / norm;  // direction::calculate
            int k0 = (oz + 1) * 3 + (oy + 1) * 9 + (ox + 1) * 27;  // offset_to_gain_index, output dim 0
            if (k0 > 27 + 9 + 3) k0 -= 3;
            for (int i = 0; i < 3; ++i)
              for (int o = 0; o < 3; ++o) {
                const float c = dir[(size_t)(3 * out + o)];
                const float mult = relative_eq(c, 0.0f) ? 0.0f : (c > 0.0f ? 1.0f : -1.0f);
                float g = dir[(size_t)(3 * in + i)] * mult;  // gain::calculate
                if (type_in == 6 && type_out != 6) g = g * factor;
                if (type_out == 6 && type_in != 6) g = g * inv;
                gains[((int64_t)numbers[in] + i) * kGainCols + k0 + o] = g;
              }
          }
    }
    auto next = by_time.upper_bound(current);
    // no later activation time: the reference's next sweep step finds no voxel and ends the loop
    if (next == by_time.end()) break;
    current = next->first;
  }
  for (int64_t c = 0; c < cells; ++c) activation_ms[c] = t[(size_t)c] * 1000.0f;
}

// init_output_state_indicies (allpass.rs:212-289): row 3v + a, column 3n + b holds 3 w + b for the
// voxel w at offset n of voxel v (in the grid and connectable), -1 otherwise. `cell_of[v]` = the cell
// of voxel v.
void output_state_indices_host(const int32_t* types, const int32_t* numbers, int64_t nx, int64_t ny, int64_t nz,
                               const std::vector<int64_t>& cell_of, int32_t* out) {
  const int64_t V = (int64_t)cell_of.size();
  for (int64_t v = 0; v < V; ++v) {
    const int64_t c = cell_of[(size_t)v];
    const int64_t x = c / (ny * nz), y = c / nz % ny, z = c % nz;
    int n = 0;
    for (int ox = -1; ox <= 1; ++ox)
      for (int oy = -1; oy <= 1; ++oy)
        for (int oz = -1; oz <= 1; ++oz) {
          if (ox == 0 && oy == 0 && oz == 0) continue;
          const int col = n++;
          const int64_t X = x + ox, Y = y + oy, Z = z + oz;
          int32_t w = -1;
          if (X >= 0 && X < nx && Y >= 0 && Y < ny && Z >= 0 && Z < nz) {
            const int64_t co = (X * ny + Y) * nz + Z;
            if (host_connectable(types[co])) w = numbers[co];
          }
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) out[(3 * v + a) * kGainCols + 3 * col + b] = w < 0 ? -1 : w + b;
        }
  }
}

}  // namespace ct
