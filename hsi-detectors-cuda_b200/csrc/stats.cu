// stats.cu - scene moments on the 5th-generation tensor cores.
//
// Computes, for one BSQ frame, the raw first and second moments the detector
// statistics are built from (reference: SpectralMoments, include/hsi/linalg.hpp
// :22-51, accumulated by src/detectors_cpu.cpp:77-93 on the CPU and by the
// never-called src/stats.cu:72-165 on the GPU).
//
// Arithmetic (precision measured against the FP64 oracle before writing it):
//   d = x - r, r a per-band reference near the mean (the reference's shifted
//   accumulation, include/hsi/linalg.hpp:53-90);
//   d is split into BF16 hi + lo, H = bf16(d), L = bf16(d - H), and the tensor
//   cores accumulate  G' = H H^T + L L^T + H (2L)^T  (three MMAs per K-step),
//   so that S = (G' + G'^T)/2 = H H^T + L L^T + H L^T + L H^T -- all four
//   products, because dropping L L^T biases the variances;
//   a ones-row at band B makes the same GEMM produce sum(d) and the pixel count;
//   FP32 accumulation in TMEM is limited to 1024-pixel chunks, each folded into
//   an FP64 accumulator that also lives in TMEM (the reference's FP32-block ->
//   FP64 hierarchy, tests/test_linalg.cpp:290-350);
//   partial sums of all CTAs are reduced in a fixed order (deterministic), and
//   the raw moments are rebuilt in FP64 (src/linalg.cpp:81-103).
//
// Kernel roles (one CTA per SM, 14 warps):
//   warp 0       TMA producer: 2-D tiles of 64 pixels x 128 bands
//   warp 1       TMEM allocator + single-thread MMA issuer
//   warps 2-9    converters: FP32 tile -> BF16 H, L, 2L in the UMMA
//                128-byte-swizzled K-major layout
//   warps 10-13  epilogue: TMEM chunk -> FP64 TMEM accumulator -> global
// TMEM: columns [0,128) and [128,256) double-buffer the FP32 chunk
// accumulator; [256,512) hold the FP64 accumulator (two columns per value).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tc.cuh"

namespace hsi_b200 {
namespace {

constexpr int kKB = 64;          // pixels per K-block (one TMA box)
#ifndef HSI_STATS_CHUNK_KB
#define HSI_STATS_CHUNK_KB 16
#endif
constexpr int kChunkKB = HSI_STATS_CHUNK_KB;  // K-blocks per FP32 accumulation chunk
constexpr int kRows = 128;       // band rows of the GEMM (bands + ones row)
constexpr int kInStages = 3;
constexpr int kOpStages = 2;
constexpr int kConvWarps = 8;
constexpr int kEpiWarps = 4;
constexpr int kWarpTma = 0;
constexpr int kWarpMma = 1;
constexpr int kWarpConv0 = 2;
constexpr int kWarpEpi0 = kWarpConv0 + kConvWarps;
constexpr int kThreads = (kWarpEpi0 + kEpiWarps) * 32;  // 448
constexpr int kOpTileBytes = kRows * kKB * 2;           // 16 KB (BF16)
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kFp64Col = 256;
constexpr int kMaxTensorBands = kRows - 1;  // 127: room for the ones row
constexpr int kMaxCtas = 160;

template <typename T>
constexpr int in_tile_bytes() {
  return kRows * kKB * static_cast<int>(sizeof(T));
}

struct StatsSmem {
  size_t in_off, op_off, shift_off, bar_off, slot_off, total;
};

template <typename T>
__host__ __device__ inline StatsSmem stats_smem() {
  StatsSmem s;
  size_t off = 0;
  s.in_off = off;
  off += static_cast<size_t>(kInStages) * in_tile_bytes<T>();
  s.op_off = off;  // 1024-aligned: in tiles are multiples of 1024
  off += static_cast<size_t>(kOpStages) * 3 * kOpTileBytes;
  s.shift_off = off;
  off += kRows * sizeof(float);
  s.bar_off = off;
  off += (2 * kInStages + 2 * kOpStages + 5) * sizeof(uint64_t);
  s.slot_off = off;
  off += 16;
  s.total = off + 1024;  // slack to align the dynamic base to 1024
  return s;
}

// Byte offset of element (row, k) in a 128B-swizzled K-major tile of 16-bit
// values with 64 elements per row.
__device__ __forceinline__ uint32_t sw128_offset(int row, int k) {
  const int chunk = (k * 2) >> 4;
  return static_cast<uint32_t>((row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4) + ((k * 2) & 15));
}

template <typename T>
__device__ __forceinline__ float2 load_pair(const T* p);
template <>
__device__ __forceinline__ float2 load_pair<float>(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}
template <>
__device__ __forceinline__ float2 load_pair<__half>(const __half* p) {
  return __half22float2(*reinterpret_cast<const __half2*>(p));
}

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

struct StatsArgs {
  int64_t pixels;
  int bands;
  const float* shift;  // kRows floats (0 past the bands)
  double* partials;    // [gridDim.x][kRows][kRows] (column-major per CTA)
  int* status;
};

template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
    stats_gemm_kernel(const __grid_constant__ CUtensorMap cube_map, const StatsArgs args) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const StatsSmem L = stats_smem<T>();
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar_off);
  uint64_t* in_full = bars;
  uint64_t* in_empty = in_full + kInStages;
  uint64_t* op_full = in_empty + kInStages;
  uint64_t* op_empty = op_full + kOpStages;
  uint64_t* acc_full = op_empty + kOpStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* mma_done = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.slot_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.slot_off + 8);
  float* shift = reinterpret_cast<float*>(smem + L.shift_off);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t P = args.pixels;
  const int B = args.bands;
  const int64_t nkb = div_up<int64_t>(P, kKB);
  const int64_t kb0 = nkb * blockIdx.x / gridDim.x;
  const int64_t kb1 = nkb * (blockIdx.x + 1) / gridDim.x;
  const int n = static_cast<int>(kb1 - kb0);
  const int nchunks = (n + kChunkKB - 1) / kChunkKB;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kInStages; ++s) {
      mbar_init(&in_full[s], 1);
      mbar_init(&in_empty[s], kConvWarps);
    }
    for (int s = 0; s < kOpStages; ++s) {
      mbar_init(&op_full[s], kConvWarps);
      mbar_init(&op_empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&acc_full[s], 1);
      mbar_init(&acc_empty[s], kEpiWarps);
    }
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  for (int i = threadIdx.x; i < kRows; i += blockDim.x) shift[i] = args.shift[i];
  if (warp == kWarpMma) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kWarpTma) {
    if (lane == 0) {
      prefetch_tensormap(&cube_map);
      uint32_t pending = 0, parity = 0;
      for (int i = 0; i < n; ++i) {
        const int s = i % kInStages;
        const uint32_t ph = (i / kInStages) & 1u;
        if (*abort_flag || !mbar_wait(&in_empty[s], ph ^ 1u)) {
          record_error(args.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        mbar_arrive_expect_tx(&in_full[s], in_tile_bytes<T>());
        tma_load_2d(smem + L.in_off + static_cast<size_t>(s) * in_tile_bytes<T>(), &cube_map,
                    static_cast<int>((kb0 + i) * kKB), 0, &in_full[s]);
        pending |= 1u << s;
        parity = (parity & ~(1u << s)) | (ph << s);
      }
      for (int s = 0; s < kInStages; ++s)
        if ((pending >> s) & 1u) mbar_wait(&in_full[s], (parity >> s) & 1u);
    }
  } else if (warp == kWarpMma) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(kRows, kRows);
      bool issued = false;
      for (int i = 0; i < n && !*abort_flag; ++i) {
        const int chunk = i / kChunkKB, j = i % kChunkKB;
        const int buf = chunk & 1;
        if (j == 0) {
          if (!mbar_wait(&acc_empty[buf], ((chunk >> 1) & 1u) ^ 1u)) {
            record_error(args.status, HSI_E_TIMEOUT);
            *abort_flag = 1;
            break;
          }
          tc_fence_after();
        }
        const int so = i % kOpStages;
        if (!mbar_wait(&op_full[so], (i / kOpStages) & 1u)) {
          record_error(args.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        unsigned char* op = smem + L.op_off + static_cast<size_t>(so) * 3 * kOpTileBytes;
        const uint64_t dH = smem_desc_sw128(op);
        const uint64_t dL = smem_desc_sw128(op + kOpTileBytes);
        const uint64_t dL2 = smem_desc_sw128(op + 2 * kOpTileBytes);
        const uint32_t d = tmem + static_cast<uint32_t>(buf * kRows);
#pragma unroll
        for (int k = 0; k < kKB / 16; ++k) {
          const uint64_t adv = static_cast<uint64_t>(k * 2);  // 32 bytes of K, in 16-byte units
          umma_f16(d, dH + adv, dH + adv, idesc, (j > 0 || k > 0) ? 1u : 0u);
          umma_f16(d, dL + adv, dL + adv, idesc, 1u);
          umma_f16(d, dH + adv, dL2 + adv, idesc, 1u);
        }
        umma_commit(&op_empty[so]);
        if (j == kChunkKB - 1 || i == n - 1) umma_commit(&acc_full[buf]);
        issued = true;
      }
      // TMEM is freed at the end of the kernel: make sure no MMA of this
      // thread is still running by then (bounded wait).
      if (issued) {
        umma_commit(mma_done);
        if (!mbar_wait(mma_done, 0)) record_error(args.status, HSI_E_TIMEOUT);
      }
    }
  } else if (warp < kWarpEpi0) {
    // ---------------- converters ----------------
    const int cw = warp - kWarpConv0;
    float rr[kRows / kConvWarps];
#pragma unroll
    for (int t = 0; t < kRows / kConvWarps; ++t) rr[t] = shift[cw + kConvWarps * t];
    bool aborted = false;
    for (int i = 0; i < n; ++i) {
      const int s = i % kInStages, so = i % kOpStages;
      if (!aborted && (!mbar_wait(&in_full[s], (i / kInStages) & 1u) ||
                       !mbar_wait(&op_empty[so], ((i / kOpStages) & 1u) ^ 1u))) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        aborted = true;
      }
      if (aborted) break;
      const T* in = reinterpret_cast<const T*>(smem + L.in_off + static_cast<size_t>(s) * in_tile_bytes<T>());
      unsigned char* op = smem + L.op_off + static_cast<size_t>(so) * 3 * kOpTileBytes;
      const int64_t gp = (kb0 + i) * kKB + 2 * lane;
      const bool v0 = gp < P, v1 = gp + 1 < P;
#pragma unroll
      for (int t = 0; t < kRows / kConvWarps; ++t) {
        const int b = cw + kConvWarps * t;
        float d0 = 0.0f, d1 = 0.0f;
        if (b < B) {
          const float2 x = load_pair<T>(in + b * kKB + 2 * lane);
          d0 = v0 ? x.x - rr[t] : 0.0f;
          d1 = v1 ? x.y - rr[t] : 0.0f;
        } else if (b == B) {
          d0 = v0 ? 1.0f : 0.0f;
          d1 = v1 ? 1.0f : 0.0f;
        }
        const __nv_bfloat162 hi = __floats2bfloat162_rn(d0, d1);
        const float2 hf = __bfloat1622float2(hi);
        const float r0 = d0 - hf.x, r1 = d1 - hf.y;
        const __nv_bfloat162 lo = __floats2bfloat162_rn(r0, r1);
        const __nv_bfloat162 lo2 = __floats2bfloat162_rn(2.0f * r0, 2.0f * r1);
        const uint32_t off = sw128_offset(b, 2 * lane);
        *reinterpret_cast<uint32_t*>(op + off) = bf2_bits(hi);
        *reinterpret_cast<uint32_t*>(op + kOpTileBytes + off) = bf2_bits(lo);
        *reinterpret_cast<uint32_t*>(op + 2 * kOpTileBytes + off) = bf2_bits(lo2);
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&in_empty[s]);
        mbar_arrive(&op_full[so]);
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int row = q * 32 + lane;
    const uint32_t trow = tmem + (static_cast<uint32_t>(q * 32) << 16);
    uint32_t z[32];
#pragma unroll
    for (int c = 0; c < 32; ++c) z[c] = 0u;
#pragma unroll
    for (int c = 0; c < 8; ++c) tmem_st32(trow + kFp64Col + 32 * c, z);
    tmem_wait_st();
    bool aborted = false;
    for (int chunk = 0; chunk < nchunks; ++chunk) {
      const int buf = chunk & 1;
      if (!mbar_wait(&acc_full[buf], (chunk >> 1) & 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        aborted = true;
        break;
      }
      tc_fence_after();
#pragma unroll 1
      for (int cb = 0; cb < kRows / 32; ++cb) {
        uint32_t g[32], f0[32], f1[32];
        tmem_ld32(trow + buf * kRows + 32 * cb, g);
        tmem_ld32(trow + kFp64Col + 64 * cb, f0);
        tmem_ld32(trow + kFp64Col + 64 * cb + 32, f1);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          double a = __hiloint2double(static_cast<int>(f0[2 * j + 1]), static_cast<int>(f0[2 * j]));
          a += static_cast<double>(__uint_as_float(g[j]));
          f0[2 * j] = static_cast<uint32_t>(__double2loint(a));
          f0[2 * j + 1] = static_cast<uint32_t>(__double2hiint(a));
          double b = __hiloint2double(static_cast<int>(f1[2 * j + 1]), static_cast<int>(f1[2 * j]));
          b += static_cast<double>(__uint_as_float(g[16 + j]));
          f1[2 * j] = static_cast<uint32_t>(__double2loint(b));
          f1[2 * j + 1] = static_cast<uint32_t>(__double2hiint(b));
        }
        tmem_st32(trow + kFp64Col + 64 * cb, f0);
        tmem_st32(trow + kFp64Col + 64 * cb + 32, f1);
      }
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[buf]);
    }
    if (!aborted && !*abort_flag) {
      // Column-major per CTA: partial[c][col][row], so a warp's stores of one
      // column are 32 consecutive doubles.
      double* out = args.partials + static_cast<size_t>(blockIdx.x) * kRows * kRows;
#pragma unroll 1
      for (int cb = 0; cb < kRows / 32; ++cb) {
        uint32_t f0[32], f1[32];
        tmem_ld32(trow + kFp64Col + 64 * cb, f0);
        tmem_ld32(trow + kFp64Col + 64 * cb + 32, f1);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          out[static_cast<size_t>(32 * cb + j) * kRows + row] =
              __hiloint2double(static_cast<int>(f0[2 * j + 1]), static_cast<int>(f0[2 * j]));
          out[static_cast<size_t>(32 * cb + 16 + j) * kRows + row] =
              __hiloint2double(static_cast<int>(f1[2 * j + 1]), static_cast<int>(f1[2 * j]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kWarpMma) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// Shift reference: per-band mean over a regular subsample (every 16th run of
// 64 pixels), good enough to keep the shifted sums free of cancellation.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) shift_kernel(const T* __restrict__ cube, int64_t pixels, int64_t stride,
                                                    int bands, const float* __restrict__ given, float* shift) {
  const int b = blockIdx.x;
  if (b >= bands) {
    if (threadIdx.x == 0) shift[b] = 0.0f;
    return;
  }
  if (given) {
    if (threadIdx.x == 0) shift[b] = given[b];
    return;
  }
  __shared__ double s_sum[256];
  __shared__ double s_cnt[256];
  const T* plane = cube + static_cast<int64_t>(b) * stride;
  const int64_t runs = div_up<int64_t>(pixels, 64);
  const int64_t step = runs > 4096 ? 16 : 1;
  double sum = 0.0, cnt = 0.0;
  for (int64_t run = threadIdx.x / 64; run * step < runs; run += blockDim.x / 64) {
    const int64_t p = run * step * 64 + (threadIdx.x & 63);
    if (p < pixels) {
      sum += static_cast<double>(static_cast<float>(plane[p]));
      cnt += 1.0;
    }
  }
  s_sum[threadIdx.x] = sum;
  s_cnt[threadIdx.x] = cnt;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + w];
      s_cnt[threadIdx.x] += s_cnt[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) shift[b] = s_cnt[0] > 0.0 ? static_cast<float>(s_sum[0] / s_cnt[0]) : 0.0f;
}

// Sum the CTAs' partial matrices in a fixed order: block = 32 entries, each of
// 8 warps sums a slice of CTAs, then the slices are added in warp order.
__global__ void __launch_bounds__(256) stats_reduce_kernel(const double* __restrict__ partials, int ctas,
                                                          double* __restrict__ fsum) {
  __shared__ double s[8][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x * 32 + lane;  // entry index in [0, 128*128)
  double acc = 0.0;
  const int c0 = ctas * warp / 8, c1 = ctas * (warp + 1) / 8;
  for (int c = c0; c < c1; ++c) acc += partials[static_cast<size_t>(c) * kRows * kRows + e];
  s[warp][lane] = acc;
  __syncthreads();
  if (warp == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += s[w][lane];
    fsum[e] = t;
  }
}

// S = (F + F^T)/2 -> shifted sums (S1, S2, N) -> raw moments in FP64
// (moments_from_shifted, src/linalg.cpp:81-103).  fsum is column-major:
// fsum[col * 128 + row] = F[row][col].  Output: sum[B], outer[B*B] (full,
// symmetric), count.
__global__ void __launch_bounds__(256) stats_finalize_kernel(const double* __restrict__ fsum,
                                                            const float* __restrict__ shift, int bands,
                                                            double* __restrict__ moments) {
  __shared__ double s1[kRows];
  __shared__ double r[kRows];
  const int B = bands;
  auto F = [&](int row, int col) { return fsum[static_cast<size_t>(col) * kRows + row]; };
  const double N = F(B, B);
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    s1[i] = 0.5 * (F(i, B) + F(B, i));
    r[i] = static_cast<double>(shift[i]);
  }
  __syncthreads();
  double* sum = moments;
  double* outer = moments + B;
  for (int i = threadIdx.x; i < B; i += blockDim.x) sum[i] = s1[i] + N * r[i];
  // lower triangle, mirrored, so the matrix is exactly symmetric
  for (int e = threadIdx.x; e < B * B; e += blockDim.x) {
    const int i = e / B, j = e % B;
    if (j > i) continue;
    const double s2 = 0.5 * (F(i, j) + F(j, i));
    const double v = s2 + r[i] * s1[j] + s1[i] * r[j] + N * r[i] * r[j];
    outer[e] = v;
    outer[j * B + i] = v;
  }
  if (threadIdx.x == 0) moments[B + B * B] = N;
}

// ---------------------------------------------------------------------------
// Plain FP32 SIMT moments: the comparator path, and the path for B >= 128.
// Each block owns a 64-band x 64-band tile of the lower triangle over a slice
// of pixels, 4x4 register blocks per thread, FP32 sums over 1024-pixel chunks
// flushed into FP64 registers, written to per-block partials, then reduced in
// a fixed order.  The shift (and ones row) work as in the tensor path.
// ---------------------------------------------------------------------------
constexpr int kSimtTile = 64;
constexpr int kSimtPx = 32;

template <typename T>
__global__ void __launch_bounds__(256) stats_simt_kernel(const T* __restrict__ cube, int64_t pixels, int64_t stride,
                                                        int bands, const float* __restrict__ shift,
                                                        double* __restrict__ partials, int slices) {
  // blockIdx.x: pixel slice; blockIdx.y: lower-triangle tile pair
  const int tiles = (bands + 1 + kSimtTile - 1) / kSimtTile;  // rows incl. the ones row
  int ti = 0, pair = blockIdx.y;
  while (pair > ti) {
    pair -= ti + 1;
    ++ti;
  }
  const int tj = pair;
  __shared__ float si[kSimtPx][kSimtTile + 4];
  __shared__ float sj[kSimtPx][kSimtTile + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4];
  double dacc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      acc[a][c] = 0.0f;
      dacc[a][c] = 0.0;
    }
  const int64_t per = div_up<int64_t>(pixels, slices);
  const int64_t p0 = per * blockIdx.x, p1 = min(pixels, p0 + per);
  int since_flush = 0;
  for (int64_t base = p0; base < p1; base += kSimtPx) {
    for (int e = threadIdx.x; e < kSimtPx * kSimtTile; e += blockDim.x) {
      const int px = e % kSimtPx, rb = e / kSimtPx;
      const int64_t p = base + px;
      const bool valid = p < p1;
      const int bi = ti * kSimtTile + rb, bj = tj * kSimtTile + rb;
      float vi = 0.0f, vj = 0.0f;
      if (valid) {
        if (bi < bands) vi = static_cast<float>(cube[static_cast<int64_t>(bi) * stride + p]) - shift[bi];
        else if (bi == bands) vi = 1.0f;
        if (bj < bands) vj = static_cast<float>(cube[static_cast<int64_t>(bj) * stride + p]) - shift[bj];
        else if (bj == bands) vj = 1.0f;
      }
      si[px][rb] = vi;
      sj[px][rb] = vj;
    }
    __syncthreads();
#pragma unroll 8
    for (int px = 0; px < kSimtPx; ++px) {
      const float4 a = *reinterpret_cast<const float4*>(&si[px][ty * 4]);
      const float4 b = *reinterpret_cast<const float4*>(&sj[px][tx * 4]);
      const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
    }
    __syncthreads();
    since_flush += kSimtPx;
    if (since_flush >= 1024) {
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          dacc[r][c] += acc[r][c];
          acc[r][c] = 0.0f;
        }
      since_flush = 0;
    }
  }
  // partial layout: [slice][col][row] over the padded (tiles*64)^2 square
  const int n = tiles * kSimtTile;
  double* out = partials + static_cast<size_t>(blockIdx.x) * n * n;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int row = ti * kSimtTile + ty * 4 + r, col = tj * kSimtTile + tx * 4 + c;
      const double v = dacc[r][c] + acc[r][c];
      // F[row][col] for the lower-triangle tile; mirrored so that
      // (F + F^T)/2 yields the full symmetric sum.
      if (ti == tj) {
        out[static_cast<size_t>(col) * n + row] = v;
      } else {
        out[static_cast<size_t>(col) * n + row] = v;
        out[static_cast<size_t>(row) * n + col] = v;
      }
    }
}

__global__ void __launch_bounds__(256) simt_reduce_kernel(const double* __restrict__ partials, int slices, int n,
                                                         double* __restrict__ fsum) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * n) return;
  double t = 0.0;
  for (int c = 0; c < slices; ++c) t += partials[static_cast<size_t>(c) * n * n + e];
  fsum[e] = t;
}

__global__ void __launch_bounds__(256) simt_finalize_kernel(const double* __restrict__ fsum, int n,
                                                           const float* __restrict__ shift, int bands,
                                                           double* __restrict__ moments) {
  __shared__ double s1[HSI_MAX_BANDS];
  __shared__ double r[HSI_MAX_BANDS];
  const int B = bands;
  auto F = [&](int row, int col) { return fsum[static_cast<size_t>(col) * n + row]; };
  const double N = F(B, B);
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    s1[i] = F(i, B);
    r[i] = static_cast<double>(shift[i]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < B; i += blockDim.x) moments[i] = s1[i] + N * r[i];
  for (int e = threadIdx.x; e < B * B; e += blockDim.x) {
    const int i = e / B, j = e % B;
    if (j > i) continue;
    const double v = F(i, j) + r[i] * s1[j] + s1[i] * r[j] + N * r[i] * r[j];
    moments[B + e] = v;
    moments[B + j * B + i] = v;
  }
  if (threadIdx.x == 0) moments[B + B * B] = N;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

int num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

constexpr int kSimtSlices = 96;

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

struct StatsWorkspace {
  float* shift;
  double* partials;
  double* fsum;
};

size_t ws_bytes(int bands) {
  const size_t shift = align256(HSI_MAX_BANDS * sizeof(float));
  if (bands <= kMaxTensorBands) {
    return shift + align256(static_cast<size_t>(kMaxCtas) * kRows * kRows * sizeof(double)) +
           align256(kRows * kRows * sizeof(double));
  }
  const int n = ((bands + 1 + kSimtTile - 1) / kSimtTile) * kSimtTile;
  return shift + align256(static_cast<size_t>(kSimtSlices) * n * n * sizeof(double)) +
         align256(static_cast<size_t>(n) * n * sizeof(double));
}

size_t simt_ws_bytes(int bands) {
  const int n = ((bands + 1 + kSimtTile - 1) / kSimtTile) * kSimtTile;
  return align256(HSI_MAX_BANDS * sizeof(float)) + align256(static_cast<size_t>(kSimtSlices) * n * n * sizeof(double)) +
         align256(static_cast<size_t>(n) * n * sizeof(double));
}

StatsWorkspace carve(void* base, size_t partial_bytes) {
  unsigned char* p = static_cast<unsigned char*>(base);
  StatsWorkspace w;
  w.shift = reinterpret_cast<float*>(p);
  p += align256(HSI_MAX_BANDS * sizeof(float));
  w.partials = reinterpret_cast<double*>(p);
  p += align256(partial_bytes);
  w.fsum = reinterpret_cast<double*>(p);
  return w;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

template <typename T>
int launch_tensor_stats(const void* cube, int64_t P, int B, int64_t stride, double* moments, const float* reference,
                        void* workspace, cudaStream_t s, int* status) {
  CUtensorMap map;
  const int rc = encode_cube_map(&map, cube, sizeof(T) == 4 ? HSI_F32 : HSI_F16, P, B, stride, kKB, kRows);
  if (rc != HSI_OK) return rc;
  const StatsWorkspace w = carve(workspace, static_cast<size_t>(kMaxCtas) * kRows * kRows * sizeof(double));
  shift_kernel<T><<<kRows, 256, 0, s>>>(static_cast<const T*>(cube), P, stride, B, reference, w.shift);
  const int64_t nkb = div_up<int64_t>(P, kKB);
  int grid = num_sms();
  if (grid > kMaxCtas) grid = kMaxCtas;
  if (nkb < grid) grid = static_cast<int>(nkb);
  const StatsSmem L = stats_smem<T>();
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(stats_gemm_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(L.total));
    if (e != cudaSuccess) return static_cast<int>(e);
    configured = true;
  }
  StatsArgs a;
  a.pixels = P;
  a.bands = B;
  a.shift = w.shift;
  a.partials = w.partials;
  a.status = status;
  stats_gemm_kernel<T><<<grid, kThreads, L.total, s>>>(map, a);
  stats_reduce_kernel<<<kRows * kRows / 32, 256, 0, s>>>(w.partials, grid, w.fsum);
  stats_finalize_kernel<<<1, 256, 0, s>>>(w.fsum, w.shift, B, moments);
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int launch_simt_stats(const void* cube, int64_t P, int B, int64_t stride, double* moments, const float* reference,
                      void* workspace, cudaStream_t s) {
  const int tiles = (B + 1 + kSimtTile - 1) / kSimtTile;
  const int n = tiles * kSimtTile;
  const StatsWorkspace w = carve(workspace, static_cast<size_t>(kSimtSlices) * n * n * sizeof(double));
  shift_kernel<T><<<HSI_MAX_BANDS, 256, 0, s>>>(static_cast<const T*>(cube), P, stride, B, reference, w.shift);
  const dim3 grid(kSimtSlices, tiles * (tiles + 1) / 2);
  stats_simt_kernel<T><<<grid, 256, 0, s>>>(static_cast<const T*>(cube), P, stride, B, w.shift, w.partials,
                                           kSimtSlices);
  simt_reduce_kernel<<<(n * n + 255) / 256, 256, 0, s>>>(w.partials, kSimtSlices, n, w.fsum);
  simt_finalize_kernel<<<1, 256, 0, s>>>(w.fsum, n, w.shift, B, moments);
  return static_cast<int>(cudaGetLastError());
}

int check_common(const void* cube, int height, int width, int bands, int dtype, int64_t stride, double* moments) {
  if (!cube || !moments || height <= 0 || width <= 0 || bands <= 0 || bands > HSI_MAX_BANDS) return HSI_E_INVALID;
  if (dtype != HSI_F32 && dtype != HSI_F16) return HSI_E_INVALID;
  const int64_t P = static_cast<int64_t>(height) * width;
  if (stride < P || (stride & 7) != 0) return HSI_E_INVALID;
  if ((reinterpret_cast<uintptr_t>(cube) & 15u) != 0) return HSI_E_INVALID;
  return HSI_OK;
}

}  // namespace

int encode_cube_map(CUtensorMap* map, const void* cube, int dtype, int64_t pixels, int bands, int64_t stride,
                    int box_pixels, int box_bands) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return HSI_E_NO_DEVICE;
  const size_t esize = dtype == HSI_F32 ? 4 : 2;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(pixels), static_cast<cuuint64_t>(bands)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(stride) * esize};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_pixels), static_cast<cuuint32_t>(box_bands)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, dtype == HSI_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                        const_cast<void*>(cube), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HSI_OK : HSI_E_INVALID;
}

}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API size_t hsi_stats_workspace_bytes(int height, int width, int bands) {
  if (height <= 0 || width <= 0 || bands <= 0 || bands > HSI_MAX_BANDS) return 0;
  const size_t a = ws_bytes(bands), b = simt_ws_bytes(bands);
  return a > b ? a : b;
}

extern "C" HSI_API int hsi_scene_moments(const void* d_cube, int height, int width, int bands, int dtype,
                                         int64_t plane_stride, double* d_moments, const float* d_reference,
                                         void* d_workspace, size_t workspace_bytes, hsi_stream_t stream) {
  const int rc = check_common(d_cube, height, width, bands, dtype, plane_stride, d_moments);
  if (rc != HSI_OK) return rc;
  if (!d_workspace || workspace_bytes < hsi_stats_workspace_bytes(height, width, bands)) return HSI_E_WORKSPACE;
  const int64_t P = static_cast<int64_t>(height) * width;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (bands <= kMaxTensorBands) {
    return dtype == HSI_F32 ? launch_tensor_stats<float>(d_cube, P, bands, plane_stride, d_moments, d_reference,
                                                         d_workspace, s, nullptr)
                            : launch_tensor_stats<__half>(d_cube, P, bands, plane_stride, d_moments, d_reference,
                                                          d_workspace, s, nullptr);
  }
  return dtype == HSI_F32
             ? launch_simt_stats<float>(d_cube, P, bands, plane_stride, d_moments, d_reference, d_workspace, s)
             : launch_simt_stats<__half>(d_cube, P, bands, plane_stride, d_moments, d_reference, d_workspace, s);
}

extern "C" HSI_API int hsi_scene_moments_simt(const void* d_cube, int height, int width, int bands, int dtype,
                                              int64_t plane_stride, double* d_moments, const float* d_reference,
                                              void* d_workspace, size_t workspace_bytes, hsi_stream_t stream) {
  const int rc = check_common(d_cube, height, width, bands, dtype, plane_stride, d_moments);
  if (rc != HSI_OK) return rc;
  if (!d_workspace || workspace_bytes < hsi_stats_workspace_bytes(height, width, bands)) return HSI_E_WORKSPACE;
  const int64_t P = static_cast<int64_t>(height) * width;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return dtype == HSI_F32
             ? launch_simt_stats<float>(d_cube, P, bands, plane_stride, d_moments, d_reference, d_workspace, s)
             : launch_simt_stats<__half>(d_cube, P, bands, plane_stride, d_moments, d_reference, d_workspace, s);
}
