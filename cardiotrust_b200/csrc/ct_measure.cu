// Measurement products of one beat over all steps:
//   y[t, m]  = sum_s H[beat, m, s] x[t, s]      predict_measurements, prediction.rs:112-130
//   r[t, m]  = y[t, m] - z[beat, t, m]          calculate_residuals, estimation.rs:146-153
//   mr[t, s] = sum_m H[beat, m, s] r[t, m]      calculate_mapped_residuals, derivation.rs:538-551
// plus the per-step MSE metric (metrics.rs:189-190).
//
// Neither product feeds the state recurrence, so each is one GEMM over the
// whole beat instead of T matrix-vector products. The k-order of these sums
// differs from the reference's (ndarray/matrixmultiply), so their results are
// compared with a tolerance. The reductions are deterministic: split-K
// partials are summed in a fixed order.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "ct_internal.cuh"

namespace ct {
namespace {

constexpr int BM = 64, BN = 64, BK = 16, kThreads = 256;

// C[m, n] (+)= sum_{k in [k0, k1)} A[m*lda + k] * B(k, n), with B(k, n) at
// B[n*ldb + k] (kBKContig) or B[k*ldb + n].
template <bool kBKContig>
__global__ void __launch_bounds__(kThreads)
    gemm_kernel(const float* __restrict__ A, int64_t lda, const float* __restrict__ Bm, int64_t ldb,
                float* __restrict__ C, int64_t ldc, int64_t c_split_stride, int64_t Mrows, int64_t Ncols, int64_t K,
                int64_t kchunk) {
  __shared__ float As[BK][BM + 4];
  __shared__ float Bs[BK][BN + 4];
  const int64_t m0 = (int64_t)blockIdx.y * BM;
  const int64_t n0 = (int64_t)blockIdx.x * BN;
  const int64_t k0 = (int64_t)blockIdx.z * kchunk;
  const int64_t k1 = (k0 + kchunk < K) ? k0 + kchunk : K;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  float acc[4][4] = {};
  for (int64_t kb = k0; kb < k1; kb += BK) {
    // A tile: BM x BK, K-contiguous rows
    for (int e = threadIdx.x; e < BM * BK; e += kThreads) {
      const int r = e / BK, c = e % BK;
      const int64_t gm = m0 + r, gk = kb + c;
      As[c][r] = (gm < Mrows && gk < k1) ? A[gm * lda + gk] : 0.0f;
    }
    if (kBKContig) {
      for (int e = threadIdx.x; e < BN * BK; e += kThreads) {
        const int r = e / BK, c = e % BK;
        const int64_t gn = n0 + r, gk = kb + c;
        Bs[c][r] = (gn < Ncols && gk < k1) ? Bm[gn * ldb + gk] : 0.0f;
      }
    } else {
      for (int e = threadIdx.x; e < BN * BK; e += kThreads) {
        const int c = e / BN, r = e % BN;
        const int64_t gn = n0 + r, gk = kb + c;
        Bs[c][r] = (gn < Ncols && gk < k1) ? Bm[gk * ldb + gn] : 0.0f;
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  float* Cz = C + (int64_t)blockIdx.z * c_split_stride;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t gm = m0 + ty * 4 + i;
    if (gm >= Mrows) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t gn = n0 + tx * 4 + j;
      if (gn < Ncols) Cz[gm * ldc + gn] = acc[i][j];
    }
  }
}

// Sum split-K partials in split order; write Y[beat], R, and optionally the residuals.
__global__ void reduce_measure_kernel(const float* __restrict__ part, int ksplit, int64_t T, int64_t M, int64_t ldp,
                                      float* __restrict__ Y, const float* __restrict__ Z, float* __restrict__ R) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= T * M) return;
  const int64_t t = idx / M, m = idx - (idx / M) * M;
  float y = 0.0f;
  for (int z = 0; z < ksplit; ++z) y = y + part[((int64_t)z * T + t) * ldp + m];
  Y[idx] = y;
  if (R) R[idx] = y - Z[idx];
}

// loss_mse[t] = sum_m r^2 / M with ndarray's eight-accumulator order (metrics.rs:189-190).
__global__ void mse_kernel(const float* __restrict__ R, int64_t T, int64_t M, float* __restrict__ loss_mse) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const float* r = R + t * M;
  float p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int64_t i = 0;
  for (; M - i >= 8; i += 8) {
#pragma unroll
    for (int q = 0; q < 8; ++q) p[q] = p[q] + r[i + q] * r[i + q];
  }
  float acc = 0.0f;
  acc = acc + (p[0] + p[4]);
  acc = acc + (p[1] + p[5]);
  acc = acc + (p[2] + p[6]);
  acc = acc + (p[3] + p[7]);
  for (; i < M; ++i) acc = acc + r[i] * r[i];
  loss_mse[t] = acc / (float)M;
}

}  // namespace

cudaError_t launch_measure(DeviceScenario& d, int64_t beat, bool with_residuals, cudaStream_t stream) {
  const int64_t T = d.T, M = d.M, S = d.S;
  const float* H = d.H + beat * M * S;
  const int64_t mpad = ((M + BN - 1) / BN) * BN;
  const int64_t kchunk = ((S + d.ksplit - 1) / d.ksplit + BK - 1) / BK * BK;
  dim3 grid((unsigned)((M + BN - 1) / BN), (unsigned)((T + BM - 1) / BM), (unsigned)d.ksplit);
  gemm_kernel<true><<<grid, kThreads, 0, stream>>>(d.X, S, H, S, d.gemm_part, mpad, T * mpad, T, M, S, kchunk);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  const int64_t n = T * M;
  reduce_measure_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
      d.gemm_part, d.ksplit, T, M, mpad, d.Y + beat * T * M, with_residuals ? d.meas + beat * T * M : nullptr,
      with_residuals ? d.R : nullptr);
  err = cudaGetLastError();
  if (err != cudaSuccess || !with_residuals) return err;
  return launch_mse(d, stream);
}

cudaError_t launch_mse(DeviceScenario& d, cudaStream_t stream) {
  mse_kernel<<<(unsigned)((d.T + 127) / 128), 128, 0, stream>>>(d.R, d.T, d.M, d.loss_mse);
  return cudaGetLastError();
}

cudaError_t launch_map_residuals(DeviceScenario& d, int64_t beat, cudaStream_t stream) {
  const int64_t T = d.T, M = d.M, S = d.S;
  const float* H = d.H + beat * M * S;
  dim3 grid((unsigned)((S + BN - 1) / BN), (unsigned)((T + BM - 1) / BM), 1);
  gemm_kernel<false><<<grid, kThreads, 0, stream>>>(d.R, M, H, S, d.MR, S, 0, T, S, M, M);
  return cudaGetLastError();
}

// ---- allocation-free variant of the H x product -------------------------------------------
//
// For callers that must not see device allocations from this library: hosts
// that place every device buffer in their own pool or arena, or run under a
// fixed device-memory budget, and callers for which the implicit device
// synchronisation of cudaMalloc / cudaFree is not acceptable. The split-K
// partial sums live in one file-scope device array instead of a per-scenario
// cudaMalloc'd buffer. Every GPU that loads the library holds this array
// (8 MiB) until the process exits.

namespace {

constexpr int64_t kStaticScratchFloats = int64_t(1) << 21;  // 2,097,152 floats = 8 MiB
__device__ __align__(256) float g_measure_scratch[kStaticScratchFloats];

constexpr int kMaxDevices = 128;
std::mutex g_scratch_mutex;
float* g_scratch_address[kMaxDevices] = {};

// Device address of g_measure_scratch on the current device. In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device with that device current, and cached.
int scratch_address(int device, float** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_address[device]) {
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_measure_scratch);
    if (err != cudaSuccess) {
      char msg[256];
      std::snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(err));
      return report_error(CT_ERR_CUDA, msg);
    }
    g_scratch_address[device] = static_cast<float*>(p);
  }
  *out = g_scratch_address[device];
  return CT_OK;
}

}  // namespace
}  // namespace ct

extern "C" int ct_predict_measurements_noalloc(const float* states, const float* measurement_matrix,
                                               const float* actual, float* predicted, float* residuals,
                                               int64_t num_steps, int64_t num_states, int64_t num_sensors,
                                               void* stream) {
  using namespace ct;
  if (!states || !measurement_matrix || !predicted)
    return report_error(CT_ERR_INVALID_ARGUMENT, "states, measurement_matrix and predicted must be device pointers");
  if (residuals && !actual) return report_error(CT_ERR_INVALID_ARGUMENT, "residuals need the actual measurements");
  const int64_t T = num_steps, S = num_states, M = num_sensors;
  if (T <= 0 || S <= 0 || M <= 0) return report_error(CT_ERR_INVALID_ARGUMENT, "num_steps, num_states and num_sensors must be positive");
  const int64_t mpad = ((M + BN - 1) / BN) * BN;
  if (T * mpad > kStaticScratchFloats) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "num_steps x ceil64(num_sensors) = %lld x %lld exceeds the static scratch of %lld floats",
                  (long long)T, (long long)mpad, (long long)kStaticScratchFloats);
    return report_error(CT_ERR_INVALID_ARGUMENT, msg);
  }
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess || device < 0 || device >= kMaxDevices)
    return report_error(CT_ERR_CUDA, "cudaGetDevice failed or device index out of range");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (st) {
    // the scratch address below is the current device's; a stream of another device would make the
    // kernels write into memory that device does not own
    int stream_device = -1;
    err = cudaStreamGetDevice(st, &stream_device);
    if (err != cudaSuccess) return report_error(CT_ERR_INVALID_ARGUMENT, "cudaStreamGetDevice failed on the stream");
    if (stream_device != device) {
      char msg[160];
      std::snprintf(msg, sizeof(msg), "the stream belongs to device %d but device %d is current", stream_device,
                    device);
      return report_error(CT_ERR_INVALID_ARGUMENT, msg);
    }
  }
  float* scratch = nullptr;
  int rc = scratch_address(device, &scratch);
  if (rc) return rc;
  int sms = 0;
  err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (err != cudaSuccess) return report_error(CT_ERR_CUDA, "cudaDeviceGetAttribute failed");
  // split-K factor: as for the scenario path, but bounded by the scratch capacity
  const int64_t tiles = ((M + BN - 1) / BN) * ((T + BM - 1) / BM);
  int64_t ks = (2 * (int64_t)sms + tiles - 1) / tiles;
  const int64_t by_k = S / 256 > 1 ? S / 256 : 1;
  const int64_t by_scratch = kStaticScratchFloats / (T * mpad);
  if (ks > by_k) ks = by_k;
  if (ks > 64) ks = 64;
  if (ks > by_scratch) ks = by_scratch;
  if (ks < 1) ks = 1;
  const int64_t kchunk = ((S + ks - 1) / ks + BK - 1) / BK * BK;
  // every (split, step, sensor) partial read below is written first, so nothing is cleared
  dim3 grid((unsigned)((M + BN - 1) / BN), (unsigned)((T + BM - 1) / BM), (unsigned)ks);
  gemm_kernel<true><<<grid, kThreads, 0, st>>>(states, S, measurement_matrix, S, scratch, mpad, T * mpad, T, M, S,
                                               kchunk);
  err = cudaGetLastError();
  if (err != cudaSuccess) return report_error(CT_ERR_CUDA, cudaGetErrorString(err));
  const int64_t n = T * M;
  reduce_measure_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(scratch, (int)ks, T, M, mpad, predicted,
                                                                    residuals ? actual : nullptr, residuals);
  err = cudaGetLastError();
  if (err != cudaSuccess) return report_error(CT_ERR_CUDA, cudaGetErrorString(err));
  return CT_OK;
}
