// Sliced BF16 tensor-core form (precision CT_PREC_BF16X6) of the two measurement products of one
// beat:
//   y  = X H^T   [T, M]   predict_measurements,        prediction.rs:112-130
//   mr = R H     [T, S]   calculate_mapped_residuals,  derivation.rs:538-551
//
// Why: the tensor core's FP32 accumulation is not round-to-nearest. Its adds lose low bits toward
// zero, and over K = 141,792 states that loss acts like a small gain error on H x. The gradient
// is a near-cancelling sum of residual terms, so this bias does not average out. Measured on
// 768 sensor rows x 141,792 states, the 3xTF32 form's gradients are 2e-2 away from the f64
// oracle. FP32 CUDA-core products, whose rounding is unbiased, are 1.3e-4 away.
//
// Method: error-free slicing of both operands (the splitting of Ozaki, Ogita, Oishi and Rump,
// "Error-free transformations of matrix multiplication by using fast routines of matrix
// multiplication", 2012, here with BF16 operands and FP32 tensor-memory accumulators).
// Every row of an operand is cut into groups of 512 K elements. A group whose largest magnitude
// is f 2^e (0.5 <= f < 1) gets the power-of-two scale s = 2^(e-7), and each value x becomes
//   x / s = s1 + s2 2^-8 + s3 2^-16 + err,   s1, s2, s3 integers in [-128, 128], |err| <= 2^-17,
// so x is carried to within 2^-24 of the group's largest magnitude, rounded to nearest (unbiased).
// The slices are exact in BF16. A product of two slices is an integer of magnitude <= 2^14, so
// the sum of one group's 512 products (the level-0 accumulator s1*h1) stays below 2^23 and is
// exact in FP32 whatever rounding the tensor core applies. Per group:
//   acc0 = sum s1 h1,   acc1 = sum s1 h2 + s2 h1,   acc2 = sum s1 h3 + s2 h2 + s3 h1
// (the dropped terms s2 h3, s3 h2, s3 h3 are below 2^-24 of the group's scale product, with
// random signs). Every 8 chunks the epilogue warps fold the three accumulators into one FP32 sum,
// rounding to nearest:  P += ((acc2 2^-8 + acc1) 2^-8 + acc0) * s_row * s_col.
// Only the final promotions and the fixed-order split-K reduction round, to nearest, so the
// product is unbiased like the FP32 CUDA-core GEMM. Non-finite inputs give a NaN scale, and the
// affected outputs become NaN. The tensor work is six BF16 MMAs per 16 K elements, the same
// tensor-pipe time as the three TF32 MMAs per 8 K elements of the 3xTF32 form.
//
// Operands are sliced by separate kernels into three BF16 planes plus a scale per (row, group):
// H and H^T once per measurement matrix, the states once per beat, the residuals once per beat.
// One CTA computes a 128 x NT output tile over a range of whole groups. Warp 0 issues TMA loads
// (one 3D box = the three slice planes of a tile) into a ring of stages. Warp 1 owns the tensor
// memory, and one elected thread issues the MMAs. Warps 2-5 promote the accumulators and store.
// Every mbarrier wait is bounded (ct_tcgen05.cuh).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdio>

#include "ct_internal.cuh"
#include "ct_tcgen05.cuh"

namespace ct {
namespace {

using namespace tc;

constexpr int kRows = 128;        // output rows per tile (tensor-memory lanes)
constexpr int kChunk = 64;        // K elements per chunk: one 128-byte swizzle row of BF16
constexpr int kMmaK = 16;         // K per BF16 MMA instruction
constexpr int kGroupChunks = 8;   // chunks per scale group
constexpr int kGroup = kChunk * kGroupChunks;  // 512 K elements share one scale per row
constexpr int kSlices = 3;
constexpr int kThreads = 192;     // 6 warps

// ---- operand slicing

// planes[p][r][c] (p = 0..2, plane stride `plane` elements, row pitch kp) and the scales for
// src[r][c] (row stride lds, `cols` valid columns; columns cols..kp-1 become zero): scale[r][g]
// (row-major, the A operand's layout) or scale[g][r] (group-major, the B operand's layout, so that
// one group's column scales are contiguous). One warp per (row, group of kGroup columns).
__global__ void slice_rows_kernel(const float* __restrict__ src, int64_t lds, int64_t rows, int cols,
                                  __nv_bfloat16* __restrict__ planes, int64_t plane, int kp,
                                  float* __restrict__ scale, int ng, bool group_major) {
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= rows * ng) return;
  const int64_t r = w / ng;
  const int g = (int)(w - r * ng);
  const float* row = src + r * lds;
  float v[kGroup / 32];
  float amax = 0.0f;
  bool bad = false;
#pragma unroll
  for (int j = 0; j < kGroup / 32; ++j) {
    const int c = g * kGroup + j * 32 + lane;
    v[j] = c < cols ? row[c] : 0.0f;
    const float a = fabsf(v[j]);
    bad = bad || !(a <= 3.402823466e38f);  // NaN or infinite
    amax = fmaxf(amax, a);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  bad = __any_sync(0xffffffffu, bad);
  int e = 0;
  if (!bad && amax > 0.0f) frexpf(amax, &e);  // amax = f 2^e, 0.5 <= f < 1
  if (lane == 0) scale[group_major ? (int64_t)g * rows + r : r * ng + g] = bad ? __int_as_float(0x7fc00000) : (amax > 0.0f ? ldexpf(1.0f, e - 7) : 0.0f);
  __nv_bfloat16* p0 = planes + r * kp;
  const bool live = !bad && amax > 0.0f;
#pragma unroll
  for (int j = 0; j < kGroup / 32; ++j) {
    const int c = g * kGroup + j * 32 + lane;
    if (c >= kp) break;
    float s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
    if (live) {
      const float a = ldexpf(v[j], 7 - e);  // |a| < 128, exact
      s1 = rintf(a);
      const float r1 = (a - s1) * 256.0f;   // exact: |a - s1| <= 1/2
      s2 = rintf(r1);
      const float r2 = (r1 - s2) * 256.0f;  // exact
      s3 = rintf(r2);
    }
    p0[c] = __float2bfloat16_rn(s1);
    p0[plane + c] = __float2bfloat16_rn(s2);
    p0[2 * plane + c] = __float2bfloat16_rn(s3);
  }
}

// dst[s][k] = src[k][s] for k < rows (a [rows, cols] matrix), zero for rows <= k < ldd.
__global__ void transpose_pad_kernel(const float* __restrict__ src, int rows, int cols, float* __restrict__ dst,
                                     int ldd) {
  __shared__ float tile[32][33];
  const int s0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, s = s0 + threadIdx.x;
    tile[r][threadIdx.x] = (k < rows && s < cols) ? src[(int64_t)k * cols + s] : 0.0f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int s = s0 + r, k = k0 + threadIdx.x;
    if (s < cols && k < ldd) dst[(int64_t)s * ldd + k] = tile[threadIdx.x][r];
  }
}

// Sum split-K partials in split order: Y[beat], and R = Y - Z when R is non-null.
__global__ void reduce_parts_kernel(const float* __restrict__ part, int ksplit, int64_t T, int M, int ldp,
                                    float* __restrict__ Y, const float* __restrict__ Z, float* __restrict__ R) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= T * M) return;
  const int64_t t = idx / M;
  const int m = (int)(idx - t * M);
  float y = 0.0f;
  for (int z = 0; z < ksplit; ++z) y = y + part[((int64_t)z * T + t) * ldp + m];
  Y[idx] = y;
  if (R) R[idx] = y - Z[idx];
}

// ---- the sliced GEMM

template <int NT, int STAGES>
struct SliceSmem {
  static constexpr int kA = kRows * kChunk * 2;  // one slice of an A tile: 16 KB
  static constexpr int kB = NT * kChunk * 2;     // one slice of a B tile
  static constexpr int kStage = kSlices * (kA + kB);
  static constexpr int kStages = STAGES;
  static constexpr int kBytes = kStages * kStage + 1024 /* alignment */ + 256 /* barriers */;
};

__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// C[z][m0 + r][n0 + c] = sum over the CTA's groups of the sliced product of A[m0 + r, :] and
// B[n0 + c, :]. map_a / map_b: 3D maps {K, rows, 3 slices} of BF16, box {64, 128 | NT, 3}.
// sa [rows][ng] and sb [ng][cols]: the scales. chunks_per_split is a multiple of kGroupChunks.
// STAGES: shared-memory stages of the TMA ring (2 for long K; 1 for the short K of H^T r, where two
// CTAs share an SM and one's epilogue overlaps the other's loads and MMAs).
template <int NT, int STAGES>
__global__ void __launch_bounds__(kThreads, 1)
    slice_gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                      const float* __restrict__ sa, const float* __restrict__ sb, int ng, float* __restrict__ C,
                      int ldc, long long c_split_stride, int rows, int cols, int kchunks, int chunks_per_split,
                      int32_t* status) {
  using L = SliceSmem<NT, STAGES>;
  constexpr int kStages = L::kStages;
  constexpr int kTmemCols = 4 * NT;  // acc0, acc1, acc2, promoted sum
  static_assert(kTmemCols == 256 || kTmemCols == 512, "tensor-memory allocation must be a power of two");
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kStages * L::kStage);
  uint64_t* empty = full + kStages;
  uint64_t* accum = empty + kStages;  // a group is complete in the accumulators
  uint64_t* acc_empty = accum + 1;    // the epilogue warps have promoted the group
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int n0 = blockIdx.x * NT, m0 = blockIdx.y * kRows;
  const int c_begin = blockIdx.z * chunks_per_split;
  const int c_end = min(kchunks, c_begin + chunks_per_split);
  const int nchunks = max(0, c_end - c_begin);
  const int g_begin = c_begin / kGroupChunks;

  auto a_tile = [&](int s) { return base + s * L::kStage; };
  auto b_tile = [&](int s) { return base + s * L::kStage + kSlices * L::kA; };

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
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

  if (warp == 0) {
    // ---- TMA producer (one elected lane)
    if (lane == 0) {
      const uint32_t bytes = (uint32_t)(kSlices * (L::kA + L::kB));
      int issued = 0;
      for (int i = 0; i < nchunks; ++i) {
        const int s = i % kStages;
        const uint32_t ph = (i / kStages) & 1;
        if (!mbar_wait(&empty[s], ph ^ 1, status, abort_flag)) break;
        mbar_expect_tx(&full[s], bytes);
        const int kx = (c_begin + i) * kChunk;
        tma_load_3d(a_tile(s), &map_a, &full[s], kx, m0, 0);
        tma_load_3d(b_tile(s), &map_b, &full[s], kx, n0, 0);
        issued = i + 1;
      }
      // drain: the copies of the last stages must land before the CTA may exit
      for (int i = max(0, issued - kStages); i < issued; ++i)
        mbar_wait(&full[i % kStages], (i / kStages) & 1, status, abort_flag);
    }
  } else if (warp == 1) {
    // ---- MMA issuer (one elected lane)
    if (lane == 0) {
      const uint32_t idesc = bf16_idesc(NT);
      const uint32_t t0 = tmem, t1 = tmem + NT, t2 = tmem + 2 * NT;
      for (int i = 0; i < nchunks; ++i) {
        const int s = i % kStages;
        const uint32_t ph = (i / kStages) & 1;
        const int g = i / kGroupChunks;
        const bool first = (i % kGroupChunks) == 0;
        if (first && g > 0) {  // the accumulators are free once the previous group is promoted
          if (!mbar_wait(acc_empty, (g - 1) & 1, status, abort_flag)) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
        if (!mbar_wait(&full[s], ph, status, abort_flag)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t a0 = sw128_desc(smem_u32(a_tile(s)));
        const uint64_t a1 = sw128_desc(smem_u32(a_tile(s) + L::kA));
        const uint64_t a2 = sw128_desc(smem_u32(a_tile(s) + 2 * L::kA));
        const uint64_t b0 = sw128_desc(smem_u32(b_tile(s)));
        const uint64_t b1 = sw128_desc(smem_u32(b_tile(s) + L::kB));
        const uint64_t b2 = sw128_desc(smem_u32(b_tile(s) + 2 * L::kB));
#pragma unroll
        for (int kk = 0; kk < kChunk / kMmaK; ++kk) {
          const uint64_t off = (uint64_t)(kk * kMmaK * 2) >> 4;  // K step inside the swizzle row
          const uint32_t acc = (first && kk == 0) ? 0u : 1u;
          umma_bf16(t0, a0 + off, b0 + off, idesc, acc);
          umma_bf16(t1, a0 + off, b1 + off, idesc, acc);
          umma_bf16(t1, a1 + off, b0 + off, idesc, 1u);
          umma_bf16(t2, a0 + off, b2 + off, idesc, acc);
          umma_bf16(t2, a1 + off, b1 + off, idesc, 1u);
          umma_bf16(t2, a2 + off, b0 + off, idesc, 1u);
        }
        umma_commit(&empty[s]);  // frees the stage once these MMAs have read it
        if ((i % kGroupChunks) == kGroupChunks - 1 || i == nchunks - 1) umma_commit(accum);  // group complete
      }
    }
  } else {
    // ---- epilogue warps 2..5 (128 threads): promotion of every group, store of the last
    const int quarter = warp % 4;  // tensor-memory lanes 32*quarter .. +31
    const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
    const int r = quarter * 32 + lane;
    const int gm = m0 + r;
    float* crow = C + (long long)blockIdx.z * c_split_stride + (long long)gm * ldc;
    const int ngroups = (nchunks + kGroupChunks - 1) / kGroupChunks;
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
    for (int g = 0; g < ngroups; ++g) {
      const int gg = g_begin + g;
      const float rs = gm < rows ? sa[(long long)gm * ng + gg] : 0.0f;
      const float* cs = sb + (long long)gg * cols + n0;  // this group's column scales (same for every lane)
      if (!mbar_wait(accum, (uint32_t)(g & 1), status, abort_flag)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const bool last = g == ngroups - 1;
#pragma unroll 1
      for (int c0 = 0; c0 < NT; c0 += 16) {
        uint32_t v0[16], v1[16], v2[16], vp[16];
        float csv[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) csv[j] = (n0 + c0 + j < cols) ? cs[c0 + j] : 0.0f;
        tmem_ld16_async(lane_base + (uint32_t)c0, v0);
        tmem_ld16_async(lane_base + (uint32_t)(NT + c0), v1);
        tmem_ld16_async(lane_base + (uint32_t)(2 * NT + c0), v2);
        if (g > 0) tmem_ld16_async(lane_base + (uint32_t)(3 * NT + c0), vp);
        tmem_wait_ld();
        float out[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float t = fmaf(__uint_as_float(v2[j]), 0.00390625f, __uint_as_float(v1[j]));
          const float grp = fmaf(t, 0.00390625f, __uint_as_float(v0[j]));
          const float p = g > 0 ? __uint_as_float(vp[j]) : 0.0f;
          out[j] = fmaf(grp, rs * csv[j], p);
        }
        if (last)
          store16(c0, out);
        else
          tmem_st16(lane_base + (uint32_t)(3 * NT + c0), out);
      }
      if (!last) {
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty);
      }
    }
    if (ngroups == 0) {  // a split without chunks contributes zeros to the fixed-order reduction
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

// 3D map {inner, rows, 3 slice planes} of BF16 with plane stride inner * rows, box {64, box_rows, 3},
// 128-byte swizzle; rows beyond `rows` read as zero.
bool make_slice_map(CUtensorMap* map, const __nv_bfloat16* ptr, int64_t inner, int64_t rows, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)inner, (cuuint64_t)rows, (cuuint64_t)kSlices};
  cuuint64_t strides[2] = {(cuuint64_t)inner * 2, (cuuint64_t)inner * rows * 2};
  cuuint32_t box[3] = {(cuuint32_t)kChunk, (cuuint32_t)box_rows, (cuuint32_t)kSlices};
  cuuint32_t estr[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(ptr), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Dynamic shared memory of a launch: the layout's bytes, raised so that at most kCtasPerSm CTAs share
// an SM (their tensor memory, 4 NT columns each, must fit the SM's 512 together).
template <int NT, int STAGES>
constexpr int slice_smem_bytes() {
  constexpr int kCtasPerSm = 512 / (4 * NT);
  constexpr int kFloor = (232448 / (kCtasPerSm + 1)) + 1024;
  return SliceSmem<NT, STAGES>::kBytes > kFloor ? SliceSmem<NT, STAGES>::kBytes : kFloor;
}

template <int NT, int STAGES>
cudaError_t launch_slice_gemm(const CUtensorMap& a, const CUtensorMap& b, const float* sa, const float* sb, int ng,
                              float* C, int ldc, long long split_stride, int rows, int cols, int kchunks, int per,
                              int ksplit, int32_t* status, cudaStream_t stream) {
  constexpr int kSmem = slice_smem_bytes<NT, STAGES>();
  static_assert(kSmem <= 232448, "shared memory per CTA");
  static bool configured[128] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 128 && !configured[dev]) {
    cudaError_t e =
        cudaFuncSetAttribute(slice_gemm_kernel<NT, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
    if (e != cudaSuccess) return e;
    configured[dev] = true;
  }
  dim3 grid((unsigned)((cols + NT - 1) / NT), (unsigned)((rows + kRows - 1) / kRows), (unsigned)ksplit);
  slice_gemm_kernel<NT, STAGES><<<grid, kThreads, kSmem, stream>>>(a, b, sa, sb, ng, C, ldc, split_stride, rows,
                                                                   cols, kchunks, per, status);
  return cudaGetLastError();
}

cudaError_t launch_slice_rows(const float* src, int64_t lds, int64_t rows, int cols, __nv_bfloat16* planes,
                              int64_t plane, int kp, float* scale, bool group_major, cudaStream_t stream) {
  const int ng = (kp + kGroup - 1) / kGroup;
  const int64_t warps = rows * ng;
  if (warps <= 0) return cudaSuccess;
  slice_rows_kernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, stream>>>(src, lds, rows, cols, planes, plane, kp,
                                                                              scale, ng, group_major);
  return cudaGetLastError();
}

}  // namespace

// ---- public launchers (ct_internal.cuh)

int64_t slice_pitch(int64_t k) { return (k + kChunk - 1) / kChunk * kChunk; }
int64_t slice_groups(int64_t k) { return (slice_pitch(k) + kGroup - 1) / kGroup; }

int slice_ksplit(int64_t T, int64_t S, int64_t M, int sms) {
  const int64_t tiles = ((T + kRows - 1) / kRows) * ((M + 127) / 128);
  const int64_t groups = slice_groups(S);
  int64_t ks = (sms + tiles - 1) / tiles;
  if (ks > groups) ks = groups;
  if (ks > 32) ks = 32;
  if (ks < 1) ks = 1;
  // whole groups per split, and no split without groups
  const int64_t per = (groups + ks - 1) / ks;
  return (int)((groups + per - 1) / per);
}

cudaError_t slice_prepare(DeviceScenario& d, cudaStream_t stream) {
  const int64_t sp = slice_pitch(d.S), kpm = slice_pitch(d.M);
  const int64_t ngs = slice_groups(d.S), ngm = slice_groups(d.M);
  float* tmp = nullptr;
  cudaError_t e = cudaMallocAsync(&tmp, sizeof(float) * (size_t)(d.S * kpm), stream);
  if (e != cudaSuccess) return e;
  for (int64_t b = 0; b < d.B && e == cudaSuccess; ++b) {
    const float* Hb = d.H + b * d.M * d.S;
    e = launch_slice_rows(Hb, d.S, d.M, (int)d.S, d.H_sl + b * kSlices * d.M * sp, d.M * sp, (int)sp,
                          d.H_sc + b * d.M * ngs, true, stream);
    if (e != cudaSuccess) break;
    dim3 grid((unsigned)((d.S + 31) / 32), (unsigned)(kpm / 32));
    transpose_pad_kernel<<<grid, dim3(32, 8), 0, stream>>>(Hb, (int)d.M, (int)d.S, tmp, (int)kpm);
    e = cudaGetLastError();
    if (e != cudaSuccess) break;
    e = launch_slice_rows(tmp, kpm, d.S, (int)d.M, d.Ht_sl + b * kSlices * d.S * kpm, d.S * kpm, (int)kpm,
                          d.Ht_sc + b * d.S * ngm, true, stream);
  }
  cudaError_t e2 = cudaFreeAsync(tmp, stream);
  return e != cudaSuccess ? e : e2;
}

cudaError_t launch_measure_sliced(DeviceScenario& d, int64_t beat, bool with_residuals, cudaStream_t stream) {
  const int64_t T = d.T, S = d.S, M = d.M;
  const int64_t sp = slice_pitch(S), ngs = slice_groups(S);
  cudaError_t e = launch_slice_rows(d.X, S, T, (int)S, d.X_sl, T * sp, (int)sp, d.X_sc, false, stream);
  if (e != cudaSuccess) return e;
  CUtensorMap ma, mb;
  if (!make_slice_map(&ma, d.X_sl, sp, T, kRows) ||
      !make_slice_map(&mb, d.H_sl + beat * kSlices * M * sp, sp, M, 128))
    return cudaErrorInvalidValue;
  const int kchunks = (int)(sp / kChunk);
  const int groups = (int)ngs;
  // whole groups per split; every split of the grid has at least one group, and the reduction
  // below sums exactly the splits the grid writes (ks <= d.ksplit_slice, the partial buffer's count)
  const int per_groups = (groups + d.ksplit_slice - 1) / d.ksplit_slice;
  const int ks = (groups + per_groups - 1) / per_groups;
  const int per = per_groups * kGroupChunks;
  const int ldp = (int)(((M + 127) / 128) * 128);
  e = launch_slice_gemm<128, 2>(ma, mb, d.X_sc, d.H_sc + beat * M * ngs, (int)ngs, d.gemm_part, ldp,
                             (long long)T * ldp, (int)T, (int)M, kchunks, per, ks, d.status, stream);
  if (e != cudaSuccess) return e;
  const int64_t n = T * M;
  reduce_parts_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
      d.gemm_part, ks, T, (int)M, ldp, d.Y + beat * T * M, with_residuals ? d.meas + beat * T * M : nullptr,
      with_residuals ? d.R : nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess || !with_residuals) return e;
  return launch_mse(d, stream);
}

cudaError_t launch_map_residuals_sliced(DeviceScenario& d, int64_t beat, cudaStream_t stream) {
  const int64_t T = d.T, S = d.S, M = d.M;
  const int64_t kpm = slice_pitch(M), ngm = slice_groups(M);
  cudaError_t e = launch_slice_rows(d.R, M, T, (int)M, d.R_sl, T * kpm, (int)kpm, d.R_sc, false, stream);
  if (e != cudaSuccess) return e;
  CUtensorMap ma, mb;
  if (!make_slice_map(&ma, d.R_sl, kpm, T, kRows) ||
      !make_slice_map(&mb, d.Ht_sl + beat * kSlices * S * kpm, kpm, S, 64))
    return cudaErrorInvalidValue;
  const int kchunks = (int)(kpm / kChunk);
  return launch_slice_gemm<64, 1>(ma, mb, d.R_sc, d.Ht_sc + beat * S * ngm, (int)ngm, d.MR, (int)S, 0, (int)T, (int)S,
                                kchunks, (int)(ngm * kGroupChunks), 1, d.status, stream);
}

}  // namespace ct
