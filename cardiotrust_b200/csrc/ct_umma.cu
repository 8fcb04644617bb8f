// Tensor-core (tcgen05) form of the two measurement products of one beat:
//   y  = X H^T   [T, M]   predict_measurements,        prediction.rs:112-130
//   mr = R H     [T, S]   calculate_mapped_residuals,  derivation.rs:538-551
//
// Both run as TF32 MMAs (kind::tf32, FP32 accumulation in tensor memory) fed
// by TMA with 128-byte swizzled K-major tiles. Precision modes:
//   * TF32x3: every operand is split into hi = rna_tf32(v) and
//     lo = rna_tf32(v - hi) and the product accumulates hi*hi + hi*lo + lo*hi
//     (the lo*lo term, ~2^-22 relative, is dropped). Rounding lo to TF32
//     before the MMA matters: the tensor core would otherwise truncate it,
//     a biased 2^-21 error per product that accumulates over the steps of a
//     gradient when the residuals are small; rounded, the error is unbiased
//     and ~2^-22, close to FP32 products;
//   * TF32: one pass, hi*hi.
// H (and its transpose) are split once per scenario; the residuals are split
// by the reduction that produces them; the state history is split in shared
// memory by the converter warps as each tile lands (an elementwise
// operation, so the swizzled layout is irrelevant).
//
// One CTA computes a 128 x NT output tile over a range of K chunks of 32
// elements: warp 0 issues TMA loads into a ring of stages, warp 1 owns the
// tensor memory and one elected thread issues the MMAs, warps 2-5 convert
// (when the A operand is split in shared memory) and then move the
// accumulator from tensor memory to global memory. Every mbarrier wait is
// bounded (globaltimer, ~2 s); on expiry the CTA records CT_ERR_TIMEOUT,
// drains, frees its tensor memory and exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "ct_internal.cuh"
#include "ct_tcgen05.cuh"

namespace ct {
namespace {

using namespace tc;

constexpr int kBM = 128;          // output rows per tile (tensor-memory lanes)
// K chunks accumulated in tensor memory before the epilogue adds them into the promoted FP32 sum.
// The tensor core's accumulation over long chains drifts toward zero (its adds are not
// round-to-nearest). Promoting every 8 chunks cuts the relative error of H x 3x (6e-6 to 1.8e-6
// on 768 sensor rows x 141,792 states) but does not remove its bias: gradients of configs whose
// residuals are a small fraction of the signal stay ~20x above the FP32 CUDA-core products'
// error. The sliced BF16 products (ct_slice.cu) accumulate exactly and do not have this bias.
constexpr int kPromote = 8;
constexpr int kBK = 32;           // K elements per chunk (one 128-byte swizzle row of f32)
constexpr int kUmmaK = 8;         // K per tf32 MMA instruction
constexpr int kThreadsUmma = 192;  // 6 warps

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

template <int NT, int PASSES, bool SPLIT_A>
struct UmmaSmem {
  static constexpr int kStages = (NT >= 256 && PASSES == 3) ? 2 : 3;
  static constexpr int kABytes = kBM * kBK * 4;  // 16 KB
  static constexpr int kBBytes = NT * kBK * 4;
  static constexpr int kStageBytes = kABytes * (PASSES == 3 ? 2 : 1) + kBBytes * (PASSES == 3 ? 2 : 1);
  static constexpr int kBytes = kStages * kStageBytes + 1024 /* alignment */ + 256 /* barriers */;
};

// C[z][m0 + r][n0 + c] = sum over the CTA's K chunks of A[m0 + r, k] * B[n0 + c, k].
template <int NT, int PASSES, bool SPLIT_A>
__global__ void __launch_bounds__(kThreadsUmma, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_a_lo,
                     const __grid_constant__ CUtensorMap map_b, const __grid_constant__ CUtensorMap map_b_lo,
                     float* __restrict__ C, int ldc, long long c_split_stride, int rows, int cols, int kchunks,
                     int chunks_per_split, int32_t* status) {
  using L = UmmaSmem<NT, PASSES, SPLIT_A>;
  constexpr int kStages = L::kStages;
  // tensor memory: the group accumulator (columns [0, kAccCols)) and the promoted sum ([kAccCols, 2 kAccCols))
  constexpr int kAccCols = NT <= 32 ? 32 : (NT <= 64 ? 64 : (NT <= 128 ? 128 : 256));
  constexpr int kTmemCols = 2 * kAccCols;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kStages * L::kStageBytes);
  uint64_t* conv = full + kStages;
  uint64_t* empty = conv + kStages;
  uint64_t* accum = empty + kStages;  // a group of K chunks is complete in the accumulator
  uint64_t* acc_empty = accum + 1;    // the epilogue warps have promoted the group
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int n0 = blockIdx.x * NT, m0 = blockIdx.y * kBM;
  const int c_begin = blockIdx.z * chunks_per_split;
  const int c_end = min(kchunks, c_begin + chunks_per_split);
  const int nchunks = max(0, c_end - c_begin);

  auto a_hi = [&](int s) { return base + s * L::kStageBytes; };
  auto a_lo = [&](int s) { return base + s * L::kStageBytes + L::kABytes; };
  auto b_hi = [&](int s) { return base + s * L::kStageBytes + L::kABytes * (PASSES == 3 ? 2 : 1); };
  auto b_lo = [&](int s) { return b_hi(s) + L::kBBytes; };

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&conv[s], 4);  // one arrival per converter warp
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    mbar_init(acc_empty, 4);  // one arrival per epilogue warp
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const uint32_t bytes_a = L::kABytes * ((PASSES == 3 && !SPLIT_A) ? 2 : 1);
  const uint32_t bytes_b = L::kBBytes * (PASSES == 3 ? 2 : 1);

  if (warp == 0) {
    // ---- TMA producer (one elected lane)
    if (lane == 0) {
      int issued = 0;
      for (int i = 0; i < nchunks; ++i) {
        const int s = i % kStages;
        const uint32_t ph = (i / kStages) & 1;
        if (!mbar_wait(&empty[s], ph ^ 1, status, abort_flag)) break;
        mbar_expect_tx(&full[s], bytes_a + bytes_b);
        const int kx = (c_begin + i) * kBK;
        tma_load_2d(a_hi(s), &map_a, &full[s], kx, m0);
        if (PASSES == 3 && !SPLIT_A) tma_load_2d(a_lo(s), &map_a_lo, &full[s], kx, m0);
        tma_load_2d(b_hi(s), &map_b, &full[s], kx, n0);
        if (PASSES == 3) tma_load_2d(b_lo(s), &map_b_lo, &full[s], kx, n0);
        issued = i + 1;
      }
      // drain: wait until the copies of the last stages have landed before the CTA may exit
      for (int i = max(0, issued - kStages); i < issued; ++i)
        mbar_wait(&full[i % kStages], (i / kStages) & 1, status, abort_flag);
    }
  } else if (warp == 1) {
    // ---- MMA issuer (one elected lane)
    if (lane == 0) {
      const uint32_t idesc = tf32_idesc(NT);
      bool ok = true;
      for (int i = 0; i < nchunks && ok; ++i) {
        const int s = i % kStages;
        const uint32_t ph = (i / kStages) & 1;
        const int g = i / kPromote;
        const bool first = (i % kPromote) == 0;
        if (first && g > 0) {  // the accumulator is free once the previous group is promoted
          if (!mbar_wait(acc_empty, (g - 1) & 1, status, abort_flag)) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
        ok = SPLIT_A ? mbar_wait(&conv[s], ph, status, abort_flag) : mbar_wait(&full[s], ph, status, abort_flag);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t dah = sw128_desc(smem_u32(a_hi(s)));
        const uint64_t dal = sw128_desc(smem_u32(a_lo(s)));
        const uint64_t dbh = sw128_desc(smem_u32(b_hi(s)));
        const uint64_t dbl = sw128_desc(smem_u32(b_lo(s)));
#pragma unroll
        for (int kk = 0; kk < kBK / kUmmaK; ++kk) {
          const uint64_t off = (uint64_t)(kk * kUmmaK * 4) >> 4;  // K step inside the swizzle row
          const uint32_t acc = (first && kk == 0) ? 0u : 1u;
          umma_tf32(tmem, dah + off, dbh + off, idesc, acc);
          if (PASSES == 3) {
            umma_tf32(tmem, dah + off, dbl + off, idesc, 1u);
            umma_tf32(tmem, dal + off, dbh + off, idesc, 1u);
          }
        }
        umma_commit(&empty[s]);  // frees the stage once these MMAs have read it
        if ((i % kPromote) == kPromote - 1 || i == nchunks - 1) umma_commit(accum);  // group complete
      }
    }
  } else {
    // ---- converter / epilogue warps 2..5 (128 threads)
    const int ct = threadIdx.x - 64;
    const int quarter = warp % 4;  // tensor-memory lanes 32*quarter .. +31
    const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
    const int r = quarter * 32 + lane;
    const int gm = m0 + r;
    float* crow = C + (long long)blockIdx.z * c_split_stride + (long long)gm * ldc;
    const int ngroups = (nchunks + kPromote - 1) / kPromote;
    auto store16 = [&](int c0, const float* v) {
      if (gm < rows) {
        if (n0 + c0 + 16 <= cols && ((ldc & 3) == 0)) {
          float4* dst = reinterpret_cast<float4*>(crow + n0 + c0);
#pragma unroll
          for (int q = 0; q < 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (n0 + c0 + j < cols) crow[n0 + c0 + j] = v[j];
        }
      }
    };
    // Promotion of group g: promoted += accumulator (FP32 adds, round to nearest, in group order);
    // the last group goes to global memory instead.
    auto promote = [&](int g) -> bool {
      if (!mbar_wait(accum, (uint32_t)(g & 1), status, abort_flag)) return false;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const bool last = g == ngroups - 1;
#pragma unroll 1
      for (int c0 = 0; c0 < NT; c0 += 16) {
        float a[16];
        tmem_ld16(lane_base + (uint32_t)c0, a);
        if (g > 0) {
          float p[16];
          tmem_ld16(lane_base + (uint32_t)(kAccCols + c0), p);
#pragma unroll
          for (int j = 0; j < 16; ++j) a[j] = p[j] + a[j];
        }
        if (last)
          store16(c0, a);
        else
          tmem_st16(lane_base + (uint32_t)(kAccCols + c0), a);
      }
      if (!last) {
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty);
      }
      return true;
    };
    bool ok = true;
    if (SPLIT_A) {
      for (int i = 0; i < nchunks && ok; ++i) {
        const int s = i % kStages;
        const uint32_t ph = (i / kStages) & 1;
        if (!mbar_wait(&full[s], ph, status, abort_flag)) {
          ok = false;
          break;
        }
        float4* hi = reinterpret_cast<float4*>(a_hi(s));
        float4* lo = reinterpret_cast<float4*>(a_lo(s));
#pragma unroll
        for (int q = 0; q < (kBM * kBK / 4) / 128; ++q) {
          const int e = ct + q * 128;
          const float4 v = hi[e];
          float4 h, l;
          h.x = tf32_rna(v.x);
          h.y = tf32_rna(v.y);
          h.z = tf32_rna(v.z);
          h.w = tf32_rna(v.w);
          hi[e] = h;
          if (PASSES == 3) {
            l.x = tf32_rna(v.x - h.x);
            l.y = tf32_rna(v.y - h.y);
            l.z = tf32_rna(v.z - h.z);
            l.w = tf32_rna(v.w - h.w);
            lo[e] = l;
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // make the stores visible to the MMA
        __syncwarp();
        if (lane == 0) mbar_arrive(&conv[s]);
        // the group this chunk closes has no conversion left; promote it as soon as its MMAs finish
        if ((i % kPromote) == kPromote - 1 || i == nchunks - 1) ok = promote(i / kPromote);
      }
    } else {
      for (int g = 0; g < ngroups && ok; ++g) ok = promote(g);
    }
    if (ngroups == 0) {  // a split without K chunks contributes zeros to the fixed-order reduction
      float z[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) z[j] = 0.0f;
      for (int c0 = 0; c0 < NT; c0 += 16) store16(c0, z);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

// ---- operand preparation kernels

// hi/lo [rows, pitch] = split(src [rows, cols]), zero in the columns cols..pitch-1.
__global__ void split_tf32_kernel(const float* __restrict__ src, float* __restrict__ hi, float* __restrict__ lo,
                                  long long rows, int cols, int pitch) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * pitch) return;
  const long long r = i / pitch;
  const int c = (int)(i - r * pitch);
  const float v = c < cols ? src[r * cols + c] : 0.0f;
  const float h = tf32_rna(v);
  hi[i] = h;
  lo[i] = tf32_rna(v - h);
}

// dst [rows, pitch] = src [rows, cols], zero in the columns cols..pitch-1 (16-byte TMA rows).
__global__ void pad_rows_kernel(const float* __restrict__ src, float* __restrict__ dst, long long rows, int cols,
                                int pitch) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * pitch) return;
  const long long r = i / pitch;
  const int c = (int)(i - r * pitch);
  dst[i] = c < cols ? src[r * cols + c] : 0.0f;
}

// Ht[b][s][k] = split(H[b][k][s]) for k < M, zero for M <= k < kpad.
__global__ void transpose_split_kernel(const float* __restrict__ H, int M, int S, int kpad, float* __restrict__ hi,
                                       float* __restrict__ lo) {
  __shared__ float tile[32][33];
  const int b = blockIdx.z;
  const int s0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const float* Hb = H + (long long)b * M * S;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, s = s0 + threadIdx.x;
    tile[r][threadIdx.x] = (k < M && s < S) ? Hb[(long long)k * S + s] : 0.0f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int s = s0 + r, k = k0 + threadIdx.x;
    if (s < S && k < kpad) {
      const float v = tile[threadIdx.x][r];
      const float h = tf32_rna(v);
      const long long o = ((long long)b * S + s) * kpad + k;
      hi[o] = h;
      lo[o] = tf32_rna(v - h);
    }
  }
}

// Sum split-K partials in split order: Y[beat], R = Y - Z (f32), R split into hi/lo [T][kpad].
__global__ void reduce_split_kernel(const float* __restrict__ part, int ksplit, int T, int M, int ldp,
                                    float* __restrict__ Y, const float* __restrict__ Z, float* __restrict__ R,
                                    float* __restrict__ r_hi, float* __restrict__ r_lo, int kpad) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)T * kpad) return;
  const int t = (int)(idx / kpad), m = (int)(idx - (long long)t * kpad);
  float r = 0.0f;
  if (m < M) {
    float y = 0.0f;
    for (int z = 0; z < ksplit; ++z) y = y + part[((long long)z * T + t) * ldp + m];
    Y[(long long)t * M + m] = y;
    if (R) {
      r = y - Z[(long long)t * M + m];
      R[(long long)t * M + m] = r;
    }
  }
  if (r_hi) {
    const float h = tf32_rna(r);
    r_hi[idx] = h;
    r_lo[idx] = tf32_rna(r - h);
  }
}

}  // namespace

namespace tc {
EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}
}  // namespace tc

namespace {

// 2D row-major f32 matrix [rows][inner] (inner contiguous), box = 32 x box_rows, 128-byte swizzle.
bool make_map(CUtensorMap* map, const float* ptr, int64_t inner, int64_t rows, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)inner * sizeof(float)};
  cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ptr), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NT, int PASSES, bool SPLIT_A>
cudaError_t launch_gemm(const CUtensorMap& a, const CUtensorMap& a_lo, const CUtensorMap& b, const CUtensorMap& b_lo,
                        float* C, int ldc, long long split_stride, int rows, int cols, int kchunks, int ksplit,
                        int32_t* status, cudaStream_t stream) {
  using L = UmmaSmem<NT, PASSES, SPLIT_A>;
  static bool configured[128] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 128 && !configured[dev]) {
    cudaError_t e = cudaFuncSetAttribute(umma_gemm_kernel<NT, PASSES, SPLIT_A>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes);
    if (e != cudaSuccess) return e;
    configured[dev] = true;
  }
  const int per = (kchunks + ksplit - 1) / ksplit;
  dim3 grid((unsigned)((cols + NT - 1) / NT), (unsigned)((rows + kBM - 1) / kBM), (unsigned)ksplit);
  umma_gemm_kernel<NT, PASSES, SPLIT_A><<<grid, kThreadsUmma, L::kBytes, stream>>>(
      a, a_lo, b, b_lo, C, ldc, split_stride, rows, cols, kchunks, per, status);
  return cudaGetLastError();
}

}  // namespace

// ---- public launchers (ct_internal.cuh)

// Sensor rows beyond 256 take more column tiles of H x. Any state count: the K-major operands of H x
// need 16-byte rows, so H's split is stored with a pitch of S rounded up to 4 and, when S % 4 != 0,
// X is copied into a padded buffer before the product (the zero columns add exact zeros).
bool umma_supported(int64_t M) { return M <= 65536 && encode_fn() != nullptr; }

int umma_yn(int64_t M) { return M <= 128 ? 128 : 256; }

int umma_ksplit(int64_t T, int64_t S, int64_t M, int sms) {
  const int64_t tiles = ((T + kBM - 1) / kBM) * ((M + umma_yn(M) - 1) / umma_yn(M));
  const int64_t kchunks = (S + kBK - 1) / kBK;
  int64_t ks = (sms + tiles - 1) / tiles;
  if (ks > kchunks) ks = kchunks;
  if (ks > 32) ks = 32;
  return (int)(ks < 1 ? 1 : ks);
}

cudaError_t umma_prepare(DeviceScenario& d, cudaStream_t stream) {
  const long long n = (long long)d.B * d.M * d.spad;
  split_tf32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(d.H, d.H_hi, d.H_lo, (long long)d.B * d.M,
                                                                      (int)d.S, (int)d.spad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((d.S + 31) / 32), (unsigned)(d.kpad / 32), (unsigned)d.B);
  transpose_split_kernel<<<grid, dim3(32, 8), 0, stream>>>(d.H, (int)d.M, (int)d.S, (int)d.kpad, d.Ht_hi, d.Ht_lo);
  return cudaGetLastError();
}

cudaError_t launch_measure_umma(DeviceScenario& d, int64_t beat, bool with_residuals, int precision,
                                cudaStream_t stream) {
  const int T = (int)d.T, S = (int)d.spad, M = (int)d.M;
  CUtensorMap mx, mh, mhl;
  const int yn = umma_yn(M);
  const float* Hh = d.H_hi + beat * d.M * d.spad;
  const float* Hl = d.H_lo + beat * d.M * d.spad;
  const float* X = d.X;
  if (d.spad != d.S) {
    const long long n = (long long)T * d.spad;
    pad_rows_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(d.X, d.Xpad, T, (int)d.S, (int)d.spad);
    cudaError_t e0 = cudaGetLastError();
    if (e0 != cudaSuccess) return e0;
    X = d.Xpad;
  }
  if (!make_map(&mx, X, S, T, kBM) || !make_map(&mh, Hh, S, M, yn) || !make_map(&mhl, Hl, S, M, yn))
    return cudaErrorInvalidValue;
  const int kchunks = (S + kBK - 1) / kBK;
  const int ldp = ((M + yn - 1) / yn) * yn;
  cudaError_t e;
  if (precision == CT_PREC_TF32X3) {
    e = (yn == 128) ? launch_gemm<128, 3, true>(mx, mx, mh, mhl, d.gemm_part, ldp, (long long)T * ldp, T, M, kchunks,
                                                d.ksplit_umma, d.status, stream)
                    : launch_gemm<256, 3, true>(mx, mx, mh, mhl, d.gemm_part, ldp, (long long)T * ldp, T, M, kchunks,
                                                d.ksplit_umma, d.status, stream);
  } else {
    e = (yn == 128) ? launch_gemm<128, 1, true>(mx, mx, mh, mhl, d.gemm_part, ldp, (long long)T * ldp, T, M, kchunks,
                                                d.ksplit_umma, d.status, stream)
                    : launch_gemm<256, 1, true>(mx, mx, mh, mhl, d.gemm_part, ldp, (long long)T * ldp, T, M, kchunks,
                                                d.ksplit_umma, d.status, stream);
  }
  if (e != cudaSuccess) return e;
  const long long n = (long long)T * d.kpad;
  reduce_split_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
      d.gemm_part, d.ksplit_umma, T, M, ldp, d.Y + beat * d.T * d.M, with_residuals ? d.meas + beat * d.T * d.M : nullptr,
      with_residuals ? d.R : nullptr, with_residuals ? d.R_hi : nullptr, with_residuals ? d.R_lo : nullptr,
      (int)d.kpad);
  e = cudaGetLastError();
  if (e != cudaSuccess || !with_residuals) return e;
  return launch_mse(d, stream);
}

cudaError_t launch_map_residuals_umma(DeviceScenario& d, int64_t beat, int precision, cudaStream_t stream) {
  const int T = (int)d.T, S = (int)d.S;
  const int kp = (int)d.kpad;
  CUtensorMap ma, mal, mb, mbl;
  const float* Bh = d.Ht_hi + beat * d.S * d.kpad;
  const float* Bl = d.Ht_lo + beat * d.S * d.kpad;
  if (!make_map(&ma, d.R_hi, kp, T, kBM) || !make_map(&mal, d.R_lo, kp, T, kBM) || !make_map(&mb, Bh, kp, S, 256) ||
      !make_map(&mbl, Bl, kp, S, 256))
    return cudaErrorInvalidValue;
  const int kchunks = kp / kBK;
  if (precision == CT_PREC_TF32X3)
    return launch_gemm<256, 3, false>(ma, mal, mb, mbl, d.MR, S, 0, T, S, kchunks, 1, d.status, stream);
  return launch_gemm<256, 1, false>(ma, mal, mb, mbl, d.MR, S, 0, T, S, kchunks, 1, d.status, stream);
}

}  // namespace ct
