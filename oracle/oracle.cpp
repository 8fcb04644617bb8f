// CPU restatement of the CardioTrust estimation epoch (`run_epoch`).
//
// TEST INFRASTRUCTURE ONLY. This file is the parity checker for the CUDA
// library: it is loaded by tests/, by __graft_entry__.smoke() and by the
// CPU-baseline leg of bench.py, and by nothing else. The product path never
// links or calls it.
//
// Every function follows one function of the reference crate, cited by
// file:line relative to the crate root. The f32 instantiation keeps the
// reference's loop order and rounding: `a.mul_add(b, c)` becomes std::fma,
// every other `a * b + c` is two rounded operations (the file is compiled
// with -ffp-contract=off). The f64 instantiation is the same code in double
// precision, used for error reports.
//
// Third-party arithmetic on the path (not vendored in the reference tree):
//   * ndarray 0.16.1 `ArrayBase::dot` (matrix x vector) -> `unrolled_dot`,
//     an eight-accumulator dot product, used by predict_measurements;
//   * ndarray 0.16.1 `sum` -> `unrolled_fold`, same eight-accumulator shape,
//     used by the MSE metric and the batch means;
//   * ndarray 0.16.1 `general_mat_mul` -> matrixmultiply 0.3.10 `sgemm`,
//     whose x86-64 FMA micro-kernel accumulates each output element with
//     fused multiply-adds in k order inside blocks of KC = 256 and adds the
//     blocks to C in order; used by calculate_mapped_residuals.
// These are restated from the crates' published algorithms; their exact
// summation order is not pinned by any test in the reference tree, so the
// GPU is compared against these products with a tolerance, never bitwise.

#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int kOffsets = 26;
constexpr int kGainCols = 78;

struct Algo {
  int32_t optimizer;       // 0 = Sgd, 1 = Adam           (refinement.rs:8-12)
  int32_t ap_derivative;   // 0 = Simple, 1 = Textbook    (config/algorithm.rs:17-21)
  int32_t freeze_gains;
  int32_t freeze_delays;
  int64_t batch_size;
  float learning_rate;
  float mse_strength;
  float maximum_regularization_strength;
  float maximum_regularization_threshold;
  float difference_regularization_strength;
  float smoothness_regularization_strength;
};

// Model + Results, as raw arrays owned by the caller. Field names follow the
// reference structs (APParameters allpass.rs:29-36, Estimations
// estimation.rs:24-36, Derivatives derivation.rs:31-58, Metrics
// metrics.rs:20-37). Every float pointer has the instantiation's type T.
template <typename T>
struct Epoch {
  int64_t num_states, num_voxels, num_sensors, num_steps, num_beats, num_batch_slots;
  // model
  T* gains;                           // [S,78]
  const int32_t* output_state_indices;  // [S,78], -1 = None
  T* coefs;                           // [V,26]
  int32_t* delays;                    // [V,26]
  const T* initial_delays;            // [V,26]
  const T* measurement_matrix;        // [B,M,S]
  const T* control_matrix;            // [S]
  const T* control_function_values;   // [T]
  const T* actual_measurements;       // [B,T,M]
  // estimations
  T* ap_outputs_now;   // [S,78]
  T* ap_outputs_last;  // [S,78]
  T* system_states;    // [T,S]
  T* measurements;     // [B,T,M]
  T* residuals;        // [M]
  T* average_delays;   // [V], NaN = None
  // derivatives
  T* d_gains;          // [S,78]
  T* d_coefs;          // [V,26]
  T* coefs_iir;        // [S,78]
  T* coefs_fir;        // [S,78]
  T* mapped_residuals; // [S]
  T* maximum_regularization;  // [S]
  T* maximum_regularization_sum;  // [1]
  int64_t* step;       // [1], starts at 1
  T* gains_first_moment;   // [S,78] (Adam)
  T* gains_second_moment;  // [S,78]
  T* coefs_first_moment;   // [V,26]
  T* coefs_second_moment;  // [V,26]
  // metrics
  T* loss;       // [T]
  T* loss_mse;   // [T]
  T* loss_maximum_regularization;  // [T]
  T* loss_batch;       // [num_batch_slots]
  T* loss_mse_batch;
  T* loss_maximum_regularization_batch;
  // optional: mapped residuals per (beat, step) [B,T,S] used instead of H^T r
  const T* mapped_residuals_override;
  // optional: receives H^T r per (beat, step) [B,T,S]
  T* mapped_residuals_history;
};

// ---------------------------------------------------------------- threads

// Thread count of the parallel loops (0 = OpenMP's default). Only loops whose iterations write
// disjoint outputs, each in the reference's own order, run in parallel, so every result is
// bit-identical for any count. Process-wide, so replicas run from several host threads can ask for
// one thread each.
int g_threads = 0;
inline int oracle_threads() { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

// ---------------------------------------------------------------- ndarray / matrixmultiply

template <typename T>
T unrolled_dot(const T* xs, const T* ys, int64_t n) {
  T sum = 0, p0 = 0, p1 = 0, p2 = 0, p3 = 0, p4 = 0, p5 = 0, p6 = 0, p7 = 0;
  int64_t i = 0;
  for (; n - i >= 8; i += 8) {
    p0 = p0 + xs[i + 0] * ys[i + 0];
    p1 = p1 + xs[i + 1] * ys[i + 1];
    p2 = p2 + xs[i + 2] * ys[i + 2];
    p3 = p3 + xs[i + 3] * ys[i + 3];
    p4 = p4 + xs[i + 4] * ys[i + 4];
    p5 = p5 + xs[i + 5] * ys[i + 5];
    p6 = p6 + xs[i + 6] * ys[i + 6];
    p7 = p7 + xs[i + 7] * ys[i + 7];
  }
  sum = sum + (p0 + p4);
  sum = sum + (p1 + p5);
  sum = sum + (p2 + p6);
  sum = sum + (p3 + p7);
  for (int64_t j = 0; i < n && j < 7; ++i, ++j) sum = sum + xs[i] * ys[i];
  return sum;
}

template <typename T>
T unrolled_sum(const T* xs, int64_t n) {
  T acc = 0, p0 = 0, p1 = 0, p2 = 0, p3 = 0, p4 = 0, p5 = 0, p6 = 0, p7 = 0;
  int64_t i = 0;
  for (; n - i >= 8; i += 8) {
    p0 = p0 + xs[i + 0];
    p1 = p1 + xs[i + 1];
    p2 = p2 + xs[i + 2];
    p3 = p3 + xs[i + 3];
    p4 = p4 + xs[i + 4];
    p5 = p5 + xs[i + 5];
    p6 = p6 + xs[i + 6];
    p7 = p7 + xs[i + 7];
  }
  acc = acc + (p0 + p4);
  acc = acc + (p1 + p5);
  acc = acc + (p2 + p6);
  acc = acc + (p3 + p7);
  for (int64_t j = 0; i < n && j < 7; ++i, ++j) acc = acc + xs[i];
  return acc;
}

template <typename T>
T mean(const T* xs, int64_t n) {
  return unrolled_sum(xs, n) / static_cast<T>(n);
}

// ---------------------------------------------------------------- allpass helpers

template <typename T>
T from_coef_to_samples(T coef) {  // allpass.rs:661-665
  return (T(1) - coef) / (coef + T(1));
}

float from_samples_to_coef_f32(float samples) {  // allpass.rs:640-646
  float fractional = std::fmod(samples, 1.0f);
  float coef = (1.0f - fractional) / (1.0f + fractional);
  if (coef < 1e-4f) coef = 1e-4f;
  if (coef > 1.0f - 1e-4f) coef = 1.0f - 1e-4f;
  return coef;
}

template <typename T>
T powi5(T x) {  // f32::powi(5): x * ((x*x)*(x*x))
  T x2 = x * x;
  T x4 = x2 * x2;
  return x * x4;
}

template <typename T>
T signum(T x) {  // f32::signum: +-1 with the sign bit of x, NaN for NaN
  if (std::isnan(x)) return x;
  return std::copysign(T(1), x);
}

// ---------------------------------------------------------------- prediction

// innovate_system_states_v1, estimation/prediction.rs:40-86
template <typename T>
void innovate_system_states(Epoch<T>& e, int64_t step) {
  const int64_t S = e.num_states;
  std::memcpy(e.ap_outputs_last, e.ap_outputs_now, sizeof(T) * S * kGainCols);
  T* x_now = e.system_states + step * S;
  // every state's sum is computed by one thread in the reference's k order
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
  for (int64_t i = 0; i < S; ++i) {
    for (int k = 0; k < kGainCols; ++k) {
      const int32_t out = e.output_state_indices[i * kGainCols + k];
      if (out < 0) continue;
      const int64_t ci = (i / 3) * kOffsets + k / 3;
      const T coef = e.coefs[ci];
      const int64_t delay = e.delays[ci];
      const T input = (delay <= step) ? e.system_states[(step - delay) * S + out] : T(0);
      const T input_delayed = (delay < step) ? e.system_states[(step - delay - 1) * S + out] : T(0);
      T& ap = e.ap_outputs_now[i * kGainCols + k];
      ap = std::fma(coef, input - ap, input_delayed);
      x_now[i] += e.gains[i * kGainCols + k] * ap;
    }
  }
}

// add_control_function, prediction.rs:94-106 (ndarray scaled_add: y = y + alpha * x)
template <typename T>
void add_control_function(Epoch<T>& e, int64_t step) {
  const int64_t S = e.num_states;
  const T u = e.control_function_values[step];
  T* x_now = e.system_states + step * S;
  for (int64_t i = 0; i < S; ++i) x_now[i] = x_now[i] + u * e.control_matrix[i];
}

// predict_measurements, prediction.rs:112-130
template <typename T>
void predict_measurements(Epoch<T>& e, int64_t beat, int64_t step) {
  const int64_t S = e.num_states, M = e.num_sensors, Tn = e.num_steps;
  const T* H = e.measurement_matrix + beat * M * S;
  const T* x = e.system_states + step * S;
  T* y = e.measurements + (beat * Tn + step) * M;
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
  for (int64_t m = 0; m < M; ++m) y[m] = unrolled_dot(H + m * S, x, S) * T(1);
}

// calculate_residuals, estimation.rs:146-153
template <typename T>
void calculate_residuals(Epoch<T>& e, int64_t beat, int64_t step) {
  const int64_t M = e.num_sensors, Tn = e.num_steps;
  const T* y = e.measurements + (beat * Tn + step) * M;
  const T* z = e.actual_measurements + (beat * Tn + step) * M;
  for (int64_t m = 0; m < M; ++m) e.residuals[m] = y[m] - z[m];
}

// ---------------------------------------------------------------- derivation

// calculate_mapped_residuals, derivation.rs:538-551 (matrixmultiply sgemm, n = 1)
template <typename T>
void calculate_mapped_residuals(Epoch<T>& e, int64_t beat, int64_t step) {
  const int64_t S = e.num_states, M = e.num_sensors, Tn = e.num_steps;
  if (e.mapped_residuals_override) {
    std::memcpy(e.mapped_residuals, e.mapped_residuals_override + (beat * Tn + step) * S, sizeof(T) * S);
  } else {
    const T* H = e.measurement_matrix + beat * M * S;
    constexpr int64_t KC = 256;
    // per state s: c = sum over KC-blocks (in order) of the block's fma chain in m order. The loops
    // run m-outer over a block of states (rows of H streamed), which keeps every state's order.
    constexpr int64_t SB = 512;
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
    for (int64_t s0 = 0; s0 < S; s0 += SB) {
      const int64_t s1 = (s0 + SB < S) ? s0 + SB : S;
      T c[SB], ab[SB];
      for (int64_t k0 = 0; k0 < M; k0 += KC) {
        const int64_t k1 = (k0 + KC < M) ? k0 + KC : M;
        for (int64_t s = s0; s < s1; ++s) ab[s - s0] = 0;
        for (int64_t m = k0; m < k1; ++m) {
          const T rm = e.residuals[m];
          const T* Hm = H + m * S;
          for (int64_t s = s0; s < s1; ++s) ab[s - s0] = std::fma(Hm[s], rm, ab[s - s0]);
        }
        for (int64_t s = s0; s < s1; ++s) c[s - s0] = (k0 == 0) ? ab[s - s0] : ab[s - s0] + c[s - s0];
      }
      for (int64_t s = s0; s < s1; ++s) e.mapped_residuals[s] = M > 0 ? c[s - s0] : T(0);
    }
  }
  if (e.mapped_residuals_history)
    std::memcpy(e.mapped_residuals_history + (beat * Tn + step) * S, e.mapped_residuals, sizeof(T) * S);
}

// calculate_maximum_regularization, derivation.rs:509-535
template <typename T>
void calculate_maximum_regularization(Epoch<T>& e, int64_t step, T threshold) {
  const int64_t S = e.num_states;
  const T* x = e.system_states + step * S;
  T* mr = e.maximum_regularization;
  // the per-voxel terms in parallel, their running sum in voxel order
  std::vector<T> sq((size_t)(S / 3));
  std::vector<char> over((size_t)(S / 3));
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
  for (int64_t i = 0; i < S; i += 3) {
    const T sum = std::fabs(x[i]) + std::fabs(x[i + 1]) + std::fabs(x[i + 2]);
    if (sum > threshold) {
      const T factor = sum - threshold;
      sq[(size_t)(i / 3)] = factor * factor;
      over[(size_t)(i / 3)] = 1;
      mr[i] = factor * signum(x[i]);
      mr[i + 1] = factor * signum(x[i + 1]);
      mr[i + 2] = factor * signum(x[i + 2]);
    } else {
      over[(size_t)(i / 3)] = 0;
      mr[i] = 0;
      mr[i + 1] = 0;
      mr[i + 2] = 0;
    }
  }
  for (int64_t v = 0; v < S / 3; ++v)
    if (over[(size_t)v]) *e.maximum_regularization_sum += sq[(size_t)v];
}

// calculate_derivatives_gains, derivation.rs:307-329
template <typename T>
void calculate_derivatives_gains(Epoch<T>& e, const Algo& a) {
  const int64_t S = e.num_states;
  const T mse_scaling = T(1) / static_cast<T>(e.num_sensors) * static_cast<T>(a.mse_strength);
  const T reg_scaling = static_cast<T>(a.maximum_regularization_strength);
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
  for (int64_t i = 0; i < S; ++i) {
    const T max_reg = e.maximum_regularization[i];
    const T residual = e.mapped_residuals[i];
    for (int k = 0; k < kGainCols; ++k) {
      const T ap = e.ap_outputs_now[i * kGainCols + k];
      e.d_gains[i * kGainCols + k] += ap * std::fma(residual, mse_scaling, max_reg * reg_scaling);
    }
  }
}

template <typename T>
T delay_delta(const Epoch<T>& e, int64_t ci) {
  const T delay = static_cast<T>(e.delays[ci]) + from_coef_to_samples(e.coefs[ci]);
  return powi5(e.initial_delays[ci] - delay);
}

// calculate_derivatives_coefs_simple, derivation.rs:338-398
template <typename T>
void calculate_derivatives_coefs_simple(Epoch<T>& e, int64_t step, const Algo& a) {
  const int64_t S = e.num_states;
  const T mse_scaling = T(1) / static_cast<T>(e.num_sensors) * static_cast<T>(a.mse_strength);
  const T diff = static_cast<T>(a.difference_regularization_strength);
  // parallel over voxels: d_coefs[ci] of voxel v receives its terms from rows 3v..3v+2 only, in order
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
  for (int64_t v = 0; v < S / 3; ++v)
  for (int64_t i = 3 * v; i < 3 * v + 3; ++i) {
    for (int k = 0; k < kGainCols; ++k) {
      const int64_t ci = (i / 3) * kOffsets + k / 3;
      const T dd = delay_delta(e, ci);
      const int32_t out = e.output_state_indices[i * kGainCols + k];
      if (out < 0) continue;
      const int64_t delay = e.delays[ci];
      if (step >= delay) {
        const T ap_last = e.ap_outputs_last[i * kGainCols + k];
        const T state_val = e.system_states[(step - delay) * S + out];
        const T g = e.gains[i * kGainCols + k];
        const T mr = e.mapped_residuals[i];
        e.d_coefs[ci] += std::fma((state_val - ap_last) * g * mr, mse_scaling, diff * dd);
      }
    }
  }
}

// calculate_derivatives_coefs_textbook, derivation.rs:408-501
template <typename T>
void calculate_derivatives_coefs_textbook(Epoch<T>& e, int64_t step, const Algo& a) {
  const int64_t S = e.num_states;
  const T mse_scaling = T(1) / static_cast<T>(e.num_sensors) * static_cast<T>(a.mse_strength);
  const T diff = static_cast<T>(a.difference_regularization_strength);
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
  for (int64_t i = 0; i < S; ++i) {
    for (int k = 0; k < kGainCols; ++k) {
      const int32_t out = e.output_state_indices[i * kGainCols + k];
      if (out < 0) continue;
      const int64_t ci = (i / 3) * kOffsets + k / 3;
      const int64_t delay = e.delays[ci];
      if (step >= delay) {
        const T state_val = e.system_states[(step - delay) * S + out];
        T& fir = e.coefs_fir[i * kGainCols + k];
        fir = std::fma(-e.coefs[ci], fir, state_val);
      }
    }
  }
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
  for (int64_t i = 0; i < S; ++i) {
    for (int k = 0; k < kGainCols; ++k) {
      const int64_t ci = (i / 3) * kOffsets + k / 3;
      const int64_t delay = e.delays[ci];
      if (step >= delay) {
        T& iir = e.coefs_iir[i * kGainCols + k];
        iir = std::fma(-e.coefs[ci], iir, e.ap_outputs_last[i * kGainCols + k]);
      }
    }
  }
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
  for (int64_t v = 0; v < S / 3; ++v)
  for (int64_t i = 3 * v; i < 3 * v + 3; ++i) {
    for (int k = 0; k < kGainCols; ++k) {
      const int64_t ci = (i / 3) * kOffsets + k / 3;
      const T dd = delay_delta(e, ci);
      const T iir = e.coefs_iir[i * kGainCols + k];
      const T fir = e.coefs_fir[i * kGainCols + k];
      const T g = e.gains[i * kGainCols + k];
      const T mr = e.mapped_residuals[i];
      e.d_coefs[ci] += std::fma((fir - iir) * g * mr, mse_scaling, diff * dd);
    }
  }
}

// calculate_step_derivatives, derivation.rs:173-229
template <typename T>
void calculate_step_derivatives(Epoch<T>& e, const Algo& a, int64_t step, int64_t beat) {
  calculate_mapped_residuals(e, beat, step);
  calculate_maximum_regularization(e, step, static_cast<T>(a.maximum_regularization_threshold));
  if (!a.freeze_gains) calculate_derivatives_gains(e, a);
  if (!a.freeze_delays) {
    if (a.ap_derivative == 0)
      calculate_derivatives_coefs_simple(e, step, a);
    else
      calculate_derivatives_coefs_textbook(e, step, a);
  }
}

// calculate_average_delays, derivation.rs:554-594
template <typename T>
void calculate_average_delays(Epoch<T>& e) {
  static const int kOff[26][3] = {
      {-1, -1, -1}, {-1, -1, 0}, {-1, -1, 1}, {-1, 0, -1}, {-1, 0, 0}, {-1, 0, 1}, {-1, 1, -1},
      {-1, 1, 0},   {-1, 1, 1},  {0, -1, -1}, {0, -1, 0},  {0, -1, 1}, {0, 0, -1},  {0, 0, 1},
      {0, 1, -1},   {0, 1, 0},   {0, 1, 1},   {1, -1, -1}, {1, -1, 0}, {1, -1, 1},  {1, 0, -1},
      {1, 0, 0},    {1, 0, 1},   {1, 1, -1},  {1, 1, 0},   {1, 1, 1}};
  for (int64_t v = 0; v < e.num_voxels; ++v) {
    T delay_sum = 0, gain_sum = 0;
    for (int n = 0; n < kOffsets; ++n) {
      const int xyz = std::abs(kOff[n][0]) + std::abs(kOff[n][1]) + std::abs(kOff[n][2]);
      const int64_t ci = v * kOffsets + n;
      const T delay = static_cast<T>(e.delays[ci]) + from_coef_to_samples(e.coefs[ci]);
      const T corrected = delay / std::sqrt(static_cast<T>(xyz));
      for (int in = 0; in < 3; ++in)
        for (int out = 0; out < 3; ++out) {
          const T g = e.gains[(v * 3 + in) * kGainCols + n * 3 + out];
          delay_sum += std::fabs(g) * corrected;
          gain_sum += std::fabs(g);
        }
    }
    e.average_delays[v] = (gain_sum == T(0)) ? T(NAN) : delay_sum / gain_sum;
  }
}

// calculate_smoothness_derivatives, derivation.rs:260-302
template <typename T>
void calculate_smoothness_derivatives(Epoch<T>& e, const Algo& a) {
  for (int64_t v = 0; v < e.num_voxels; ++v) {
    for (int n_out = 0; n_out < kOffsets; ++n_out) {
      const T own = e.average_delays[v];
      if (std::isnan(own)) continue;
      T neighbourhood = own;
      T divisor = 1;
      for (int n = 0; n < kOffsets; ++n) {
        const int32_t nb = e.output_state_indices[(v * 3) * kGainCols + n * 3];
        if (nb < 0) continue;
        const T d = e.average_delays[nb / 3];
        if (!std::isnan(d)) {
          neighbourhood += d;
          divisor += 1;
        }
      }
      neighbourhood /= divisor;
      e.d_coefs[v * kOffsets + n_out] += static_cast<T>(a.smoothness_regularization_strength) * (neighbourhood - own);
    }
  }
}

// calculate_batch_derivatives, derivation.rs:241-256
template <typename T>
void calculate_batch_derivatives(Epoch<T>& e, const Algo& a) {
  if (!a.freeze_delays && std::fabs(a.smoothness_regularization_strength) > 1.1920929e-7f)
    calculate_smoothness_derivatives(e, a);
}

// Derivatives::reset, derivation.rs:114-122
template <typename T>
void derivatives_reset(Epoch<T>& e) {
  const int64_t S = e.num_states, V = e.num_voxels;
  std::fill(e.d_gains, e.d_gains + S * kGainCols, T(0));
  std::fill(e.d_coefs, e.d_coefs + V * kOffsets, T(0));
  std::fill(e.coefs_iir, e.coefs_iir + S * kGainCols, T(0));
  std::fill(e.coefs_fir, e.coefs_fir + S * kGainCols, T(0));
  std::fill(e.maximum_regularization, e.maximum_regularization + S, T(0));
  *e.maximum_regularization_sum = 0;
}

// ---------------------------------------------------------------- update

template <typename T>
struct AdamConsts {
  T beta1, one_minus_beta1, beta2, one_minus_beta2, epsilon, bias1, bias2;
};

template <typename T>
AdamConsts<T> adam_consts(int64_t step) {  // update.rs:129-141 (f32 constants, powf from libm)
  AdamConsts<T> c;
  c.beta1 = static_cast<T>(0.9f);
  c.one_minus_beta1 = T(1) - c.beta1;
  c.beta2 = static_cast<T>(0.999f);
  c.one_minus_beta2 = T(1) - c.beta2;
  c.epsilon = static_cast<T>(1e-8f);
  c.bias1 = T(1) - std::pow(c.beta1, static_cast<T>(static_cast<float>(step)));
  c.bias2 = T(1) - std::pow(c.beta2, static_cast<T>(static_cast<float>(step)));
  return c;
}

template <typename T>
void adam(T* p, const T* g, T* m, T* v, int64_t n, const AdamConsts<T>& c, T lr_over_bs) {
  for (int64_t i = 0; i < n; ++i) {  // update.rs:136-145 / 190-199
    m[i] = m[i] * c.beta1 + c.one_minus_beta1 * g[i];
    v[i] = v[i] * c.beta2 + c.one_minus_beta2 * g[i] * g[i];
    const T mc = m[i] / c.bias1;
    const T vc = v[i] / c.bias2;
    const T factor = mc / (std::sqrt(vc) + c.epsilon);
    p[i] = p[i] - lr_over_bs * factor;
  }
}

template <typename T>
void sgd(T* p, const T* g, int64_t n, T lr_over_bs) {  // update.rs:106-114 / 158-168
  for (int64_t i = 0; i < n; ++i) p[i] = p[i] - lr_over_bs * g[i];
}

// roll_delays, update.rs:206-228
template <typename T>
void roll_delays(T* coefs, int32_t* delays, int64_t n) {
  const T margin = static_cast<T>(1e-4f);
  for (int64_t i = 0; i < n; ++i) {
    T& c = coefs[i];
    int32_t& d = delays[i];
    if (c > T(1) - margin) {
      if (d > 1) {
        c = T(2) * margin;
        d -= 1;
      } else {
        c = T(1) - margin;
      }
    } else if (c < margin) {
      if (d < 1000) {
        c = std::fma(T(2), -margin, T(1));
        d += 1;
      } else {
        c = margin;
      }
    }
  }
}

// APParameters::update, update.rs:27-97
template <typename T>
void ap_update(Epoch<T>& e, const Algo& a, int64_t num_steps, int64_t num_beats) {
  const int64_t S = e.num_states, V = e.num_voxels;
  const int64_t bs = (a.batch_size == 0) ? num_steps * num_beats : num_steps * a.batch_size;
  const T lr_over_bs = static_cast<T>(a.learning_rate) / static_cast<T>(static_cast<float>(bs));
  if (!a.freeze_gains) {
    if (a.optimizer == 0)
      sgd(e.gains, e.d_gains, S * kGainCols, lr_over_bs);
    else
      adam(e.gains, e.d_gains, e.gains_first_moment, e.gains_second_moment, S * kGainCols,
           adam_consts<T>(*e.step), lr_over_bs);
  }
  if (!a.freeze_delays) {
    if (a.optimizer == 0)
      sgd(e.coefs, e.d_coefs, V * kOffsets, lr_over_bs);
    else
      adam(e.coefs, e.d_coefs, e.coefs_first_moment, e.coefs_second_moment, V * kOffsets,
           adam_consts<T>(*e.step), lr_over_bs);
    roll_delays(e.coefs, e.delays, V * kOffsets);
  }
  *e.step += 1;
}

// ---------------------------------------------------------------- metrics

// metrics::calculate_step, metrics.rs:180-196
template <typename T>
void metrics_step(Epoch<T>& e, T reg_strength, int64_t step) {
  const int64_t M = e.num_sensors;
  std::vector<T> sq(M);
  for (int64_t m = 0; m < M; ++m) sq[m] = e.residuals[m] * e.residuals[m];
  e.loss_mse[step] = unrolled_sum(sq.data(), M) / static_cast<T>(M);
  e.loss_maximum_regularization[step] = *e.maximum_regularization_sum;
  e.loss[step] = std::fma(reg_strength, e.loss_maximum_regularization[step], e.loss_mse[step]);
}

// metrics::calculate_batch, metrics.rs:204-219
template <typename T>
int metrics_batch(Epoch<T>& e, int64_t index) {
  if (index < 0 || index >= e.num_batch_slots) return -3;
  const int64_t Tn = e.num_steps;
  e.loss_mse_batch[index] = mean(e.loss_mse, Tn);
  e.loss_maximum_regularization_batch[index] = mean(e.loss_maximum_regularization, Tn);
  e.loss_batch[index] = mean(e.loss, Tn);
  return 0;
}

// ---------------------------------------------------------------- epoch

// Estimations::reset, estimation.rs:82-87
template <typename T>
void estimations_reset(Epoch<T>& e) {
  std::fill(e.system_states, e.system_states + e.num_steps * e.num_states, T(0));
  std::fill(e.ap_outputs_now, e.ap_outputs_now + e.num_states * kGainCols, T(0));
}

// calculate_system_prediction, prediction.rs:15-26
template <typename T>
void system_prediction(Epoch<T>& e, int64_t beat, int64_t step) {
  innovate_system_states(e, step);
  add_control_function(e, step);
  predict_measurements(e, beat, step);
}

template <typename T>
int batch_end(Epoch<T>& e, const Algo& a, int64_t n, int64_t* batch_index) {
  calculate_average_delays(e);
  calculate_batch_derivatives(e, a);
  ap_update(e, a, e.num_steps, n);
  int rc = metrics_batch(e, *batch_index);
  *batch_index += 1;
  return rc;
}

// run_epoch, algorithm.rs:124-281. The beat order is an input (the reference
// shuffles with an unseeded generator, algorithm.rs:139-141).
template <typename T>
int run_epoch(Epoch<T>& e, const Algo& a, const int32_t* beat_order, int64_t* batch_index) {
  derivatives_reset(e);
  const T reg = static_cast<T>(a.maximum_regularization_strength);
  int64_t batch = 0;
  const bool batched = a.batch_size != 0;
  for (int64_t bi = 0; bi < e.num_beats; ++bi) {
    const int64_t beat = beat_order ? beat_order[bi] : bi;
    if (beat < 0 || beat >= e.num_beats) return -2;
    estimations_reset(e);
    for (int64_t step = 0; step < e.num_steps; ++step) {
      system_prediction(e, beat, step);
      calculate_residuals(e, beat, step);
      calculate_step_derivatives(e, a, step, beat);
      metrics_step(e, reg, step);
    }
    if (batched) {
      batch += 1;
      if (batch == a.batch_size) {
        int rc = batch_end(e, a, batch, batch_index);
        if (rc) return rc;
        derivatives_reset(e);
        batch = 0;
      }
    }
  }
  if (batched) {
    if (batch > 0) return batch_end(e, a, batch, batch_index);
    return 0;
  }
  return batch_end(e, a, e.num_beats, batch_index);
}

// Simulation::run forward part, data/simulation.rs:129-150: every beat's
// system prediction; states of the last beat stay in system_states.
template <typename T>
void simulate(Epoch<T>& e) {
  for (int64_t beat = 0; beat < e.num_beats; ++beat) {
    estimations_reset(e);
    for (int64_t step = 0; step < e.num_steps; ++step) system_prediction(e, beat, step);
  }
}

// ---------------------------------------------------------------- adjoint (no reference counterpart)
//
// Exact gradient of the stated loss of one beat,
//   L_b = sum_t [ (mse/M) * 1/2 |r_t|^2 + reg * 1/2 * sum_v relu(|x_v|_1 - thr)^2 ],
// by back-propagation through time over the forward recursion of
// innovate_system_states (prediction.rs:40-86):
//   ap[t] = c * (in_t - ap[t-1]) + in1_t,  in_t = x[t-d, j] (t >= d), in1_t = x[t-d-1, j] (t > d)
//   x[t, i] = sum_k g[i,k] * ap[t] + u[t] * B[i].
// Its instantaneous part at each step equals the reference's per-step factor
// fma(mr, mse/M, mreg * reg) (derivation.rs:307-329); the 1/2 absorbs the 2
// of the square. The difference-regularisation term is not a function of the
// states: it is added as the reference's derivation adds it, once per (i, k)
// pair per step it visits (textbook: all 9 pairs of (v, n), every step,
// derivation.rs:484-497; simple: the 9 pairs of a connected (v, n) at steps
// t >= d, derivation.rs:366-390), i.e. count * diff * delta^5.
//
// The all-pass outputs of (v, n, b) do not depend on the gain row's output
// component a, so they are kept per voxel: ap[t][v][k], k = 3n + b. The forward
// stores the all-pass state every kAdjCkpt steps; the backward recomputes each
// segment's outputs from its checkpoint and the stored states with the forward's
// own expression (bit-identical values), so memory is O(T/K + K) planes, not O(T).
constexpr int64_t kAdjCkpt = 64;

template <typename T>
T adjoint_beat(Epoch<T>& e, const Algo& a, int64_t beat, bool want_grad) {
  const int64_t S = e.num_states, V = e.num_voxels, M = e.num_sensors, Tn = e.num_steps;
  const T mse_scaling = T(1) / static_cast<T>(M) * static_cast<T>(a.mse_strength);
  const T reg = static_cast<T>(a.maximum_regularization_strength);
  const T thr = static_cast<T>(a.maximum_regularization_threshold);
  const int64_t plane = V * kGainCols;
  const int64_t nck = (Tn + kAdjCkpt - 1) / kAdjCkpt;
  std::vector<T> ck(want_grad ? (size_t)(nck * plane) : 0);  // ck[s] = all-pass state entering step s K
  estimations_reset(e);
  T loss = 0;
  for (int64_t t = 0; t < Tn; ++t) {
    if (want_grad && t % kAdjCkpt == 0) {
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
      for (int64_t v = 0; v < V; ++v)
        std::memcpy(&ck[(size_t)((t / kAdjCkpt) * plane + v * kGainCols)], e.ap_outputs_now + 3 * v * kGainCols,
                    sizeof(T) * kGainCols);
    }
    system_prediction(e, beat, t);
    calculate_residuals(e, beat, t);
    T rr = 0;
    for (int64_t m = 0; m < M; ++m) rr += e.residuals[m] * e.residuals[m];
    T rg = 0;
    const T* x = e.system_states + t * S;
    for (int64_t v = 0; v < V; ++v) {
      const T s = std::fabs(x[3 * v]) + std::fabs(x[3 * v + 1]) + std::fabs(x[3 * v + 2]);
      if (s > thr) rg += (s - thr) * (s - thr);
    }
    loss += mse_scaling * T(0.5) * rr + reg * T(0.5) * rg;
  }
  if (!want_grad) return loss;

  const T* H = e.measurement_matrix + beat * M * S;
  std::vector<T> acc((size_t)Tn * S, T(0)), lam_x(S), lap((size_t)V * kGainCols, T(0)), r(M);
  std::vector<T> seg((size_t)((kAdjCkpt + 1) * plane));  // seg[q] = all-pass output of step s K + q - 1
  std::vector<T> lnew_all((size_t)plane);
  int64_t seg_of = -1;
  for (int64_t t = Tn - 1; t >= 0; --t) {
    const int64_t sg = t / kAdjCkpt;
    if (sg != seg_of) {  // recompute the segment's all-pass outputs from its checkpoint
      const int64_t t0 = sg * kAdjCkpt, t1 = std::min<int64_t>(Tn, t0 + kAdjCkpt);
      std::memcpy(seg.data(), &ck[(size_t)(sg * plane)], sizeof(T) * plane);
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
      for (int64_t v = 0; v < V; ++v)
        for (int k = 0; k < kGainCols; ++k) {
          const int32_t out = e.output_state_indices[(3 * v) * kGainCols + k];
          const int64_t ci = v * kOffsets + k / 3;
          T ap = seg[(size_t)(v * kGainCols + k)];
          for (int64_t tt = t0; tt < t1; ++tt) {
            if (out >= 0) {  // innovate_system_states_v1's expression (prediction.rs:68-79)
              const int64_t delay = e.delays[ci];
              const T input = (delay <= tt) ? e.system_states[(tt - delay) * S + out] : T(0);
              const T input_delayed = (delay < tt) ? e.system_states[(tt - delay - 1) * S + out] : T(0);
              ap = std::fma(e.coefs[ci], input - ap, input_delayed);
            }
            seg[(size_t)((tt - t0 + 1) * plane + v * kGainCols + k)] = ap;
          }
        }
      seg_of = sg;
    }
    const int64_t q = t - sg * kAdjCkpt;
    const T* ap_now_plane = &seg[(size_t)((q + 1) * plane)];
    const T* ap_prev_plane = &seg[(size_t)(q * plane)];
    const T* x = e.system_states + t * S;
    const T* y = e.measurements + (beat * Tn + t) * M;
    const T* z = e.actual_measurements + (beat * Tn + t) * M;
    for (int64_t m = 0; m < M; ++m) r[m] = y[m] - z[m];
    // mr_i = sum over m in order of H[m,i] r[m], computed m-outer over blocks of states
    constexpr int64_t SB = 512;
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
    for (int64_t s0 = 0; s0 < S; s0 += SB) {
      const int64_t s1 = (s0 + SB < S) ? s0 + SB : S;
      T mrb[SB];
      for (int64_t i = s0; i < s1; ++i) mrb[i - s0] = 0;
      for (int64_t m = 0; m < M; ++m) {
        const T rm = r[m];
        const T* Hm = H + m * S;
        for (int64_t i = s0; i < s1; ++i) mrb[i - s0] += Hm[i] * rm;
      }
      for (int64_t i = s0; i < s1; ++i) {
        const int64_t v = i / 3;
        const T s = std::fabs(x[3 * v]) + std::fabs(x[3 * v + 1]) + std::fabs(x[3 * v + 2]);
        const T f = s > thr ? s - thr : T(0);
        lam_x[i] = mse_scaling * mrb[i - s0] + reg * f * signum(x[i]) + acc[(size_t)t * S + i];
      }
    }
    // per (v, n, b): the voxel's own gradients and adjoint state in parallel; the contributions to
    // earlier steps' state adjoints (acc, which this step does not read) in (v, n, b) order afterwards
#pragma omp parallel for schedule(static) num_threads(oracle_threads())
    for (int64_t v = 0; v < V; ++v) {
      for (int n = 0; n < kOffsets; ++n) {
        const int32_t out0 = e.output_state_indices[(3 * v) * kGainCols + 3 * n];
        if (out0 < 0) continue;
        const int64_t ci = v * kOffsets + n;
        const T c = e.coefs[ci];
        const int64_t d = e.delays[ci];
        for (int b = 0; b < 3; ++b) {
          const int k = 3 * n + b;
          const int64_t j = out0 + b;  // state index 3 * neighbour + b
          T G = 0;
          for (int c3 = 0; c3 < 3; ++c3) G += e.gains[(3 * v + c3) * kGainCols + k] * lam_x[3 * v + c3];
          const T lnew = G - c * lap[v * kGainCols + k];
          const T ap_t = ap_now_plane[v * kGainCols + k];
          const T ap_prev = ap_prev_plane[v * kGainCols + k];
          const T in = (d <= t) ? e.system_states[(t - d) * S + j] : T(0);
          if (!a.freeze_gains)
            for (int c3 = 0; c3 < 3; ++c3) e.d_gains[(3 * v + c3) * kGainCols + k] += lam_x[3 * v + c3] * ap_t;
          if (!a.freeze_delays) e.d_coefs[ci] += lnew * (in - ap_prev);
          lnew_all[(size_t)(v * kGainCols + k)] = lnew;
          lap[v * kGainCols + k] = lnew;
        }
      }
    }
    for (int64_t v = 0; v < V; ++v) {
      for (int n = 0; n < kOffsets; ++n) {
        const int32_t out0 = e.output_state_indices[(3 * v) * kGainCols + 3 * n];
        if (out0 < 0) continue;
        const int64_t ci = v * kOffsets + n;
        const T c = e.coefs[ci];
        const int64_t d = e.delays[ci];
        for (int b = 0; b < 3; ++b) {
          const T lnew = lnew_all[(size_t)(v * kGainCols + 3 * n + b)];
          const int64_t j = out0 + b;
          if (t - d >= 0) acc[(size_t)(t - d) * S + j] += c * lnew;
          if (t - d - 1 >= 0) acc[(size_t)(t - d - 1) * S + j] += lnew;
        }
      }
    }
  }
  if (!a.freeze_delays) {
    const T diff = static_cast<T>(a.difference_regularization_strength);
    for (int64_t v = 0; v < V; ++v)
      for (int n = 0; n < kOffsets; ++n) {
        const int64_t ci = v * kOffsets + n;
        int64_t count = 9 * Tn;
        if (a.ap_derivative == 0) {
          const bool connected = e.output_state_indices[(3 * v) * kGainCols + 3 * n] >= 0;
          count = connected ? 9 * std::max<int64_t>(0, Tn - e.delays[ci]) : 0;
        }
        e.d_coefs[ci] += static_cast<T>(count) * (diff * delay_delta(e, ci));
      }
  }
  return loss;
}

// run_epoch (algorithm.rs:124-281) with the derivation replaced by the
// adjoint: the forward, residuals, maximum-regularisation sum and metrics of
// every step are the reference's; gradients come from adjoint_beat.
template <typename T>
int run_epoch_adjoint(Epoch<T>& e, const Algo& a, const int32_t* beat_order, int64_t* batch_index) {
  derivatives_reset(e);
  const T reg = static_cast<T>(a.maximum_regularization_strength);
  int64_t batch = 0;
  const bool batched = a.batch_size != 0;
  for (int64_t bi = 0; bi < e.num_beats; ++bi) {
    const int64_t beat = beat_order ? beat_order[bi] : bi;
    if (beat < 0 || beat >= e.num_beats) return -2;
    adjoint_beat(e, a, beat, true);
    // metrics of the beat's forward (system_states of this beat are in place)
    for (int64_t step = 0; step < e.num_steps; ++step) {
      predict_measurements(e, beat, step);
      calculate_residuals(e, beat, step);
      calculate_mapped_residuals(e, beat, step);
      calculate_maximum_regularization(e, step, static_cast<T>(a.maximum_regularization_threshold));
      metrics_step(e, reg, step);
    }
    if (batched) {
      batch += 1;
      if (batch == a.batch_size) {
        int rc = batch_end(e, a, batch, batch_index);
        if (rc) return rc;
        derivatives_reset(e);
        batch = 0;
      }
    }
  }
  if (batched) {
    if (batch > 0) return batch_end(e, a, batch, batch_index);
    return 0;
  }
  return batch_end(e, a, e.num_beats, batch_index);
}

// Stated loss summed over beats and its gradient (accumulated into d_gains /
// d_coefs after a reset); no update.
template <typename T>
T adjoint_gradient(Epoch<T>& e, const Algo& a, bool want_grad) {
  if (want_grad) derivatives_reset(e);
  T loss = 0;
  for (int64_t beat = 0; beat < e.num_beats; ++beat) loss += adjoint_beat(e, a, beat, want_grad);
  return loss;
}

// ---- post-run arrays and segmentation metrics (the callers after the epoch loop)

// SystemStatesSpherical::calculate (src/core/data/shapes.rs:171-192): magnitude, theta, phi [T,V].
void spherical(const float* X, int64_t T, int64_t S, float* mag, float* theta, float* phi) {
  const int64_t V = S / 3;
  for (int64_t t = 0; t < T; ++t)
    for (int64_t v = 0; v < V; ++v) {
      const float* x = X + t * S + 3 * v;
      mag[t * V + v] = std::fabs(x[0]) + std::fabs(x[1]) + std::fabs(x[2]);
    }
  for (int64_t t = 0; t < T; ++t)
    for (int64_t v = 0; v < V; ++v) theta[t * V + v] = std::acos(X[t * S + 3 * v + 2] / mag[t * V + v]);
  for (int64_t t = 0; t < T; ++t)
    for (int64_t v = 0; v < V; ++v) phi[t * V + v] = std::atan2(X[t * S + 3 * v + 1], X[t * S + 3 * v]);
}

// ndarray-stats 0.6.0 `argmax_skipnan` over column v of a [T,V] array: index of the first of the
// largest non-NaN values; -1 when every value is NaN (the crate's MinMaxError::EmptyInput).
int64_t argmax_skipnan_col(const float* a, int64_t T, int64_t V, int64_t v) {
  int64_t best = -1;
  for (int64_t t = 0; t < T; ++t) {
    const float x = a[t * V + v];
    if (std::isnan(x)) continue;
    if (best < 0 || x > a[best * V + v]) best = t;
  }
  return best;
}

// ndarray-stats 0.6.0 `max_skipnan` of a 1-d array: largest non-NaN value, NaN if there is none.
float max_skipnan(const std::vector<float>& a) {
  bool any = false;
  float m = 0.0f;
  for (float x : a) {
    if (std::isnan(x)) continue;
    if (!any || x > m) m = x;
    any = true;
  }
  return any ? m : std::nanf("");
}

constexpr int kVoxelNone = 0, kVoxelVentricle = 5, kVoxelPathological = 6;  // voxels.rs:664-676

// predict_voxeltype (metrics.rs:409-447)
void predict_voxeltype(const float* X, int64_t T, int64_t S, const int32_t* numbers, int64_t cells, float threshold,
                       int32_t* pred) {
  std::vector<float> abs((size_t)T);
  for (int64_t g = 0; g < cells; ++g) {
    pred[g] = kVoxelNone;
    const int32_t n = numbers[g];
    if (n < 0) continue;
    for (int64_t t = 0; t < T; ++t)
      abs[(size_t)t] = std::fabs(X[t * S + n]) + std::fabs(X[t * S + n + 1]) + std::fabs(X[t * S + n + 2]);
    pred[g] = max_skipnan(abs) <= threshold ? kVoxelPathological : kVoxelVentricle;
  }
}

// calculate_dice / calculate_iou / calculate_precision / calculate_recall (metrics.rs:268-399)
void segmentation_scores(const int32_t* pred, const int32_t* gt, int64_t cells, float* dice, float* iou,
                         float* precision, float* recall) {
  size_t tp = 0, fp = 0, fn = 0, gt_pos = 0, pred_pos = 0, uni = 0;
  for (int64_t g = 0; g < cells; ++g) {
    const bool p = pred[g] == kVoxelPathological, q = gt[g] == kVoxelPathological;
    tp += p && q;
    fp += p && !q;
    fn += !p && q;
    gt_pos += q;
    pred_pos += p;
    uni += p || q;
  }
  const size_t den = 2 * tp + fp + fn;
  *dice = den == 0 ? 0.0f : static_cast<float>(2 * tp) / static_cast<float>(den);
  *iou = uni == 0 ? 0.0f : static_cast<float>(tp) / static_cast<float>(uni);
  *precision = pred_pos == 0 ? 0.0f : static_cast<float>(tp) / static_cast<float>(pred_pos);
  *recall = gt_pos == 0 ? 1.0f : static_cast<float>(tp) / static_cast<float>(gt_pos);
}

// ---- model construction (the step before the epoch)

// VoxelType::is_connectable (voxels.rs:690-700): Sinoatrial..Pathological = 1..6.
bool connectable(int32_t t) { return t >= 1 && t <= 6; }

// calculate_delay_s (allpass/delay.rs:14-23): |(in - out) / 1000| / velocity, f32; the norm is
// ndarray's sum of the squared components ((0 + a) + b) + c (unrolled_fold on three elements).
float delay_s(const float* p_in, const float* p_out, float velocity) {
  float sq = 0.0f;
  for (int c = 0; c < 3; ++c) {
    const float d = (p_in[c] - p_out[c]) / 1000.0f;
    sq = sq + d * d;
  }
  return std::sqrt(sq) / velocity;
}

// approx::relative_eq! with the defaults epsilon = max_relative = f32::EPSILON.
bool relative_eq_f32(float a, float b) {
  if (a == b) return true;
  if (std::isinf(a) || std::isinf(b)) return false;
  const float eps = 1.1920929e-7f;
  const float diff = std::fabs(a - b);
  if (diff <= eps) return true;
  return diff <= std::fmax(std::fabs(a), std::fabs(b)) * eps;
}

// voxels::is_connection_allowed(output, input) (voxels.rs:707-742); discriminants voxels.rs:664-676.
bool connection_allowed(int32_t out, int32_t in) {
  switch (out) {
    case 1: return in == 2 || in == 6 || in == 5;            // Sinoatrial <- Atrium, Pathological, Ventricle
    case 2: return in == 1 || in == 2 || in == 3 || in == 6;  // Atrium <- SA, Atrium, AV, Pathological
    case 3: return in == 2 || in == 4 || in == 6;             // AV <- Atrium, HPS, Pathological
    case 4: return in == 4 || in == 3 || in == 5 || in == 6;  // HPS <- HPS, AV, Ventricle, Pathological
    case 5: return in == 5 || in == 4 || in == 6;             // Ventricle <- Ventricle, HPS, Pathological
    case 6: return true;                                      // Pathological
    default: return false;                                    // None, Vessel, Torso, Chamber
  }
}

}  // namespace

extern "C" {

// connect_voxels / try_to_connect (allpass.rs:295-494), literal: the activation-time sweep visits
// `current` = 0, then the smallest activation time above it, and so on; at each, every voxel whose
// time is relative_eq to `current` (a snapshot, C order) tries the 26 offsets (x outer, z inner) and
// activates each allowed, not yet activated input voxel (first come, first served) with
// time(out) + delay at the input's velocity, the direction (in - out) / |in - out|_1, and the gains
// gain::calculate (gain.rs:9-29) x the pathology factors. O(times x cells): small grids only.
// gains [S, 78] zeroed by the caller; activation_ms [cells] (NaN = None). Returns 0, or -1 when an
// activated cell has no voxel number.
int oracle_connect_voxels_f32(const int32_t* types, const int32_t* numbers, const float* positions_mm, int64_t nx,
                              int64_t ny, int64_t nz, const float* velocities, float current_factor_in_pathology,
                              float* gains, float* activation_ms) {
  const int64_t cells = nx * ny * nz;
  const float nan = std::nanf("");
  std::vector<float> t((size_t)cells, nan);
  std::vector<float> dir((size_t)(3 * cells), 0.0f);
  for (int64_t c = 0; c < cells; ++c)
    if (types[c] == 1) {
      t[(size_t)c] = 0.0f;
      dir[(size_t)(3 * c)] = 1.0f;
    }
  float current = 0.0f;
  bool connected = true;
  while (connected) {
    bool future = false;
    for (float v : t)
      if (!std::isnan(v) && v > current) future = true;
    if (!future) connected = false;
    std::vector<int64_t> cand;
    for (int64_t c = 0; c < cells; ++c)
      if (!std::isnan(t[(size_t)c]) && relative_eq_f32(t[(size_t)c], current)) cand.push_back(c);
    for (int64_t out : cand) {
      const int64_t xo = out / (ny * nz), yo = out / nz % ny, zo = out % nz;
      for (int ox = -1; ox <= 1; ++ox)
        for (int oy = -1; oy <= 1; ++oy)
          for (int oz = -1; oz <= 1; ++oz) {
            if (ox == 0 && oy == 0 && oz == 0) continue;
            const int64_t xi = xo - ox, yi = yo - oy, zi = zo - oz;
            if (xi < 0 || xi >= nx || yi < 0 || yi >= ny || zi < 0 || zi >= nz) continue;
            const int64_t in = (xi * ny + yi) * nz + zi;
            if (!connectable(types[in])) continue;  // is_valid_index
            if (!std::isnan(t[(size_t)in])) continue;
            if (!connection_allowed(types[out], types[in])) continue;
            if (types[in] == 6 && relative_eq_f32(current_factor_in_pathology, 0.0f)) continue;
            if (numbers[in] < 0) return -1;
            const float* pin = positions_mm + 3 * in;
            const float* pout = positions_mm + 3 * out;
            t[(size_t)in] = t[(size_t)out] + delay_s(pin, pout, velocities[types[in]]);
            // direction::calculate (direction.rs:13-22)
            float d[3], norm = 0.0f;
            for (int k = 0; k < 3; ++k) {
              d[k] = (pin[k] - pout[k]) / 1000.0f;
              norm = norm + std::fabs(d[k]);
            }
            for (int k = 0; k < 3; ++k) dir[(size_t)(3 * in + k)] = d[k] / norm;
            float g[3][3];
            for (int i = 0; i < 3; ++i)
              for (int o = 0; o < 3; ++o) {
                const float c = dir[(size_t)(3 * out + o)];
                const float mult = relative_eq_f32(c, 0.0f) ? 0.0f : (c > 0.0f ? 1.0f : (c < 0.0f ? -1.0f : c));
                g[i][o] = dir[(size_t)(3 * in + i)] * mult;
              }
            if (types[in] == 6 && types[out] != 6)
              for (auto& row : g)
                for (float& v : row) v = v * current_factor_in_pathology;
            if (types[out] == 6 && types[in] != 6) {
              const float inv = 1.0f / current_factor_in_pathology;
              for (auto& row : g)
                for (float& v : row) v = v * inv;
            }
            // assign_gain (allpass.rs:501-523) with offset_to_gain_index (allpass.rs:532-548)
            for (int i = 0; i < 3; ++i)
              for (int o = 0; o < 3; ++o) {
                int k = o + (oz + 1) * 3 + (oy + 1) * 9 + (ox + 1) * 27;
                if (k > 27 + 9 + 3) k -= 3;
                gains[((int64_t)numbers[in] + i) * kGainCols + k] = g[i][o];
              }
            connected = true;
          }
    }
    float next = nan;
    for (float v : t)
      if (!std::isnan(v) && v > current && (std::isnan(next) || v < next)) next = v;
    current = next;  // min_skipnan of the times above `current` (NaN when there are none)
  }
  for (int64_t c = 0; c < cells; ++c) activation_ms[c] = t[(size_t)c] * 1000.0f;
  return 0;
}

// MeasurementMatrix::from_model_spatial_description (measurement.rs:66-123), f32, literal loops:
// beats, then grid cells in C order (indexed_iter), connectable cells only, then sensors.
// H [B, M, S] must be zeroed by the caller (non-connectable states stay 0 in the reference too).
// Returns 0, or -1 when a connectable cell has no voxel number.
int oracle_measurement_matrix_f32(const int32_t* types, const int32_t* numbers, const float* positions_mm,
                                  int64_t nx, int64_t ny, int64_t nz, float voxel_size_mm, const float* sensor_pos,
                                  const float* sensor_ori, const float* array_offsets, int64_t M, int64_t B, int64_t S,
                                  float* H) {
  const float mu0 = 1.25663706212e-6f;  // physical_constants::VACUUM_MAG_PERMEABILITY as f32
  const float pi = 3.14159265358979323846f;  // std::f32::consts::PI
  const float size_m = voxel_size_mm / 1000.0f;
  const float volume = (size_m * size_m) * size_m;  // powi(3)
  const float cf = (mu0 * volume) / (4.0f * pi) * 1e12f;
  const int64_t cells = nx * ny * nz;
  for (int64_t b = 0; b < B; ++b)
    for (int64_t c = 0; c < cells; ++c) {
      if (!connectable(types[c])) continue;
      if (numbers[c] < 0) return -1;
      const int64_t v = numbers[c];
      const float* vp = positions_mm + 3 * c;
      for (int64_t m = 0; m < M; ++m) {
        float d[3];
        for (int k = 0; k < 3; ++k) d[k] = ((sensor_pos[3 * m + k] + array_offsets[3 * b + k]) - vp[k]) / 1000.0f;
        float sq = 0.0f;
        for (int k = 0; k < 3; ++k) sq = sq + d[k] * d[k];
        const float r = std::sqrt(sq);
        const float r3 = (r * r) * r;
        const float* o = sensor_ori + 3 * m;
        float* row = H + (b * M + m) * S;
        row[v] = cf * std::fma(o[2], d[1], -(o[1] * d[2])) / r3;
        row[v + 1] = cf * std::fma(o[0], d[2], -(o[2] * d[0])) / r3;
        row[v + 2] = cf * std::fma(o[1], d[0], -(o[0] * d[1])) / r3;
      }
    }
  return 0;
}

// calculate_delay_samples_array (allpass/delay.rs:35-111) and the integer delays and coefficients
// derived from it (APParameters::from_model_config, allpass.rs:86-100): for every connectable cell
// (C order) and offset (x outer, z inner) whose neighbour is in the grid and connectable, the delay
// in samples at the input cell's velocity (velocities indexed by VoxelType discriminant, [10]).
// samples/delays/coefs [V, 26], zeroed/filled by this function (pairs without a neighbour: 0 samples,
// delay 0, coefficient from_samples_to_coef(0)). Returns 0, or the first failing (cell * 26 + n) + 1
// negated when a delay is below one sample (the reference's error), or not a finite value below 2^31.
int64_t oracle_delay_samples_f32(const int32_t* types, const int32_t* numbers, const float* positions_mm, int64_t nx,
                                 int64_t ny, int64_t nz, const float* velocities, float sample_rate_hz, int64_t V,
                                 float* samples, int32_t* delays, float* coefs) {
  for (int64_t i = 0; i < V * kOffsets; ++i) samples[i] = 0.0f;
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        const int64_t c = (x * ny + y) * nz + z;
        if (!connectable(types[c])) continue;
        int n = 0;
        for (int ox = -1; ox <= 1; ++ox)
          for (int oy = -1; oy <= 1; ++oy)
            for (int oz = -1; oz <= 1; ++oz) {
              if (ox == 0 && oy == 0 && oz == 0) continue;
              const int col = n++;  // offset_to_delay_index (allpass.rs:578-588) in this loop order
              const int64_t X = x + ox, Y = y + oy, Z = z + oz;
              if (X < 0 || X >= nx || Y < 0 || Y >= ny || Z < 0 || Z >= nz) continue;
              const int64_t co = (X * ny + Y) * nz + Z;
              if (!connectable(types[co])) continue;
              const float s = delay_s(positions_mm + 3 * c, positions_mm + 3 * co, velocities[types[c]]) * sample_rate_hz;
              if (!(s >= 1.0f) || !(s < 2147483648.0f)) return -(c * kOffsets + col + 1);
              samples[(numbers[c] / 3) * kOffsets + col] = s;
            }
      }
  for (int64_t i = 0; i < V * kOffsets; ++i) {
    delays[i] = static_cast<int32_t>(samples[i]);  // from_samples_to_usize truncates
    coefs[i] = from_samples_to_coef_f32(samples[i]);
  }
  return 0;
}

// calculate_plotting_arrays, estimation side (scenario.rs:636-690 with shapes.rs:171-192,262-277,
// 334-352). Returns 0, or -8 when a voxel's magnitude is NaN at every step (argmax_skipnan fails;
// that voxel's maxima are left NaN).
int oracle_plotting_arrays_f32(const float* X, int64_t T, int64_t S, float sample_rate_hz, float* mag, float* theta,
                               float* phi, float* mag_max, float* theta_max, float* phi_max, float* activation_ms) {
  const int64_t V = S / 3;
  spherical(X, T, S, mag, theta, phi);
  int rc = 0;
  for (int64_t v = 0; v < V; ++v) {
    const int64_t i = argmax_skipnan_col(mag, T, V, v);
    if (i < 0) {
      rc = -8;
      mag_max[v] = theta_max[v] = phi_max[v] = activation_ms[v] = std::nanf("");
      continue;
    }
    mag_max[v] = mag[i * V + v];
    theta_max[v] = theta[i * V + v];
    phi_max[v] = phi[i * V + v];
    activation_ms[v] = static_cast<float>(i) / sample_rate_hz * 1000.0f;
  }
  return rc;
}

// metrics::calculate_final (metrics.rs:226-242) and the Dice-optimal summary (scenario.rs:601-617).
// out: dice[101], iou[101], precision[101], recall[101], threshold, dice, iou, recall, precision.
void oracle_calculate_final_f32(const float* X, int64_t T, int64_t S, const int32_t* gt, const int32_t* numbers,
                                int64_t cells, float* out) {
  std::vector<int32_t> pred((size_t)cells);
  for (int i = 0; i <= 100; ++i) {
    const float threshold = static_cast<float>(i) / 100.0f;
    predict_voxeltype(X, T, S, numbers, cells, threshold, pred.data());
    segmentation_scores(pred.data(), gt, cells, out + i, out + 101 + i, out + 202 + i, out + 303 + i);
  }
  int best = -1;
  for (int i = 0; i <= 100; ++i)
    if (!std::isnan(out[i]) && (best < 0 || out[i] > out[best])) best = i;
  if (best < 0) best = 0;  // unwrap_or_default()
  out[404] = static_cast<float>(best) / 100.0f;
  out[405] = out[best];
  out[406] = out[101 + best];
  out[407] = out[303 + best];
  out[408] = out[202 + best];
}

int oracle_abi_version() { return 1; }
// Threads of the parallel loops (every result is independent of the count).
void oracle_set_threads(int n) { g_threads = n > 0 ? n : 0; }
int oracle_max_threads() { return oracle_threads(); }

int oracle_run_epoch_adjoint_f64(Epoch<double>* e, const Algo* a, const int32_t* beat_order, int64_t* batch_index) {
  return run_epoch_adjoint(*e, *a, beat_order, batch_index);
}
int oracle_run_epoch_adjoint_f32(Epoch<float>* e, const Algo* a, const int32_t* beat_order, int64_t* batch_index) {
  return run_epoch_adjoint(*e, *a, beat_order, batch_index);
}
double oracle_adjoint_gradient_f64(Epoch<double>* e, const Algo* a, int want_grad) {
  return adjoint_gradient(*e, *a, want_grad != 0);
}

int oracle_run_epoch_f32(Epoch<float>* e, const Algo* a, const int32_t* beat_order, int64_t* batch_index) {
  return run_epoch(*e, *a, beat_order, batch_index);
}
int oracle_run_epoch_f64(Epoch<double>* e, const Algo* a, const int32_t* beat_order, int64_t* batch_index) {
  return run_epoch(*e, *a, beat_order, batch_index);
}
int oracle_simulate_f32(Epoch<float>* e) {
  simulate(*e);
  return 0;
}
int oracle_simulate_f64(Epoch<double>* e) {
  simulate(*e);
  return 0;
}

// Single-step entry points for known-answer tests.
float oracle_from_samples_to_coef(float s) { return from_samples_to_coef_f32(s); }
float oracle_from_coef_to_samples(float c) { return from_coef_to_samples(c); }
int oracle_average_delays_f32(Epoch<float>* e) {
  calculate_average_delays(*e);
  return 0;
}
void oracle_sgd_f32(float* p, const float* g, int64_t n, float lr, int64_t bs) {
  sgd(p, g, n, lr / static_cast<float>(bs));
}
void oracle_adam_f32(float* p, const float* g, float* m, float* v, int64_t n, int64_t step, float lr, int64_t bs) {
  adam(p, g, m, v, n, adam_consts<float>(step), lr / static_cast<float>(bs));
}
void oracle_roll_delays_f32(float* c, int32_t* d, int64_t n) { roll_delays(c, d, n); }
void oracle_adam_bias_f32(int64_t step, float* out2) {
  AdamConsts<float> c = adam_consts<float>(step);
  out2[0] = c.bias1;
  out2[1] = c.bias2;
}

}  // extern "C"
