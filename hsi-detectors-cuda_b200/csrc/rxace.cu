// rxace.cu - RX and ACE scoring (whitening pass).
//
// Per pixel, with y = x - mu and the FP64-built statistics (factor.cu):
//   z = W y (W = L^-1, lower triangular);  RX = |z|^2
//   zu_t = z . u_t = y . v_t with v_t = W^T u_t (precomputed per frame)
//   ACE_t = zu_t^2 / (|u_t|^2 RX), skipped (0) when |u_t|^2 <= 0 or RX <= 0;
//   best = max with strict '>' so the lowest t wins ties, clamp to [0, 1],
//   0 and target -1 when no target is valid
// (reference rx_cpu / ace_best_cpu, src/detectors_cpu.cpp:95-156, which
// whiten in double with float statistics).
//
// Both paths treat the scoring as one GEMM  Zaug = Waug . Y  with
// Waug = [W ; V^T] ((B + T) x B): the first B rows give z, the last T rows the
// ACE numerators, and an epilogue per pixel reduces them to RX / ACE.
//
// This file holds the preparation kernel and the plain FP32 CUDA-core path
// (register-blocked 128 x 128 tiles, 8 x 8 outputs per thread, warps skip the
// all-zero upper-triangle K-chunks of W): the comparator for the tensor-core
// path in whiten.cu.
#include "common.cuh"
#include "launch_state.h"

namespace hsi_b200 {
namespace {

constexpr int kRowsTile = 128;  // output rows (bands + targets) per row tile
constexpr int kPxTile = 128;    // pixels per block tile
constexpr int kKChunk = 16;
constexpr int kThreads = 256;

// Prepared operands in the workspace (FP32 path):
//   waug[(B+T) padded to 128*R][Bk]   row-major, Bk = B rounded up to 16
//   mean_hi[B], mean_lo[B]            mu = hi + lo (double-float)
//   uu[T]
struct SimtOperands {
  float* waug;
  float* mean_hi;
  float* mean_lo;
  float* uu;
  int rows;   // padded row count (multiple of 128)
  int kpad;   // padded K (multiple of 16)
};

__host__ __device__ inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// One block per output row of Waug: rows < B copy W, rows B+t compute
// v_t = W^T u_t in FP64; the rest are zero.
__global__ void __launch_bounds__(256) prep_simt_kernel(const double* __restrict__ stats, int B, int T,
                                                       SimtOperands op) {
  const int n = blockIdx.x;
  const double* mean = stats;
  const double* W = stats + B;
  const double* tw = W + static_cast<size_t>(B) * B;
  const double* tn = tw + static_cast<size_t>(T) * B;
  float* row = op.waug + static_cast<size_t>(n) * op.kpad;
  for (int k = threadIdx.x; k < op.kpad; k += blockDim.x) {
    double v = 0.0;
    if (k < B) {
      if (n < B) {
        v = W[static_cast<size_t>(n) * B + k];
      } else if (n < B + T) {
        const double* u = tw + static_cast<size_t>(n - B) * B;
        for (int i = k; i < B; ++i) v += W[static_cast<size_t>(i) * B + k] * u[i];
      }
    }
    row[k] = static_cast<float>(v);
  }
  if (n == 0) {
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
      const float hi = static_cast<float>(mean[b]);
      op.mean_hi[b] = hi;
      op.mean_lo[b] = static_cast<float>(mean[b] - static_cast<double>(hi));
    }
    for (int t = threadIdx.x; t < T; t += blockDim.x) op.uu[t] = static_cast<float>(tn[t]);
  }
}

template <typename T>
__device__ __forceinline__ float to_f(T v);
template <>
__device__ __forceinline__ float to_f<float>(float v) {
  return v;
}
template <>
__device__ __forceinline__ float to_f<__half>(__half v) {
  return __half2float(v);
}

struct ScoreOut {
  float* rx;            // nullable
  float* ace_best;      // nullable
  int32_t* ace_target;  // nullable
  float* ace_maps;      // nullable, T maps at map_stride
  int64_t map_stride;
};

// Epilogue shared by both paths: RX and ACE for one pixel from its z-norm and
// ACE numerators.  Follows src/detectors_cpu.cpp:127-156.
__device__ __forceinline__ void write_pixel(const ScoreOut& o, int64_t p, float rx, const float* zu,
                                            const float* uu, int T) {
  if (o.rx) o.rx[p] = rx;
  float best = -1.0f;
  int32_t best_t = -1;
  for (int t = 0; t < T; ++t) {
    float a = 0.0f;
    if (uu[t] > 0.0f && rx > 0.0f) {
      a = (zu[t] * zu[t]) / (uu[t] * rx);
      if (a > best) {
        best = a;
        best_t = t;
      }
    }
    if (o.ace_maps) o.ace_maps[static_cast<int64_t>(t) * o.map_stride + p] = a;
  }
  if (o.ace_best) o.ace_best[p] = best < 0.0f ? 0.0f : fminf(best, 1.0f);
  if (o.ace_target) o.ace_target[p] = best_t;
}

struct SimtSmem {
  float w[2][kKChunk][kRowsTile];  // W chunk, k-major
  float y[2][kKChunk][kPxTile];    // Y chunk
  float rx[16][kPxTile];
  float zu[HSI_MAX_FILTERS_PER_PASS][kPxTile];
  float uu[HSI_MAX_FILTERS_PER_PASS];
};

template <typename T>
__global__ void __launch_bounds__(kThreads, 2) rxace_simt_kernel(const T* __restrict__ cube, int64_t pixels,
                                                             int64_t stride, int B, int Tn, SimtOperands op,
                                                             ScoreOut out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SimtSmem& sm = *reinterpret_cast<SimtSmem*>(smem_raw);
  const int tx = threadIdx.x & 15;  // pixel group: pixels tx*4 .. +3 and 64 + tx*4 .. +3
  const int ty = threadIdx.x >> 4;  // row group: rows ty*8 .. ty*8 + 7
  const int64_t p0 = static_cast<int64_t>(blockIdx.x) * kPxTile;
  const int kchunks = op.kpad / kKChunk;
  if (threadIdx.x < Tn) sm.uu[threadIdx.x] = op.uu[threadIdx.x];

  float rx_part[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) rx_part[j] = 0.0f;

  for (int rt = 0; rt < op.rows / kRowsTile; ++rt) {
    const int r0 = rt * kRowsTile;
    float2 acc[8][4];  // row i, pixels (2 j2, 2 j2 + 1) of this thread's 8: packed FMAs
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j2 = 0; j2 < 4; ++j2) acc[i][j2] = make_float2(0.0f, 0.0f);
    // A warp owns rows r0 + 16w .. r0 + 16w + 15; W is zero above the
    // diagonal, so K-chunks past its last row contribute nothing unless the
    // warp also holds target rows (dense).
    const int warp_rows_hi = r0 + (threadIdx.x >> 5) * 16 + 15;
    const bool warp_dense = warp_rows_hi >= B;

    // The cube elements of chunk kc + 1 are loaded into registers before chunk
    // kc's FMAs and stored to the other buffer after them, so their latency
    // overlaps the math.  W (a few hundred KB, resident in L2) is copied then.
    constexpr int kPer = kKChunk * kPxTile / kThreads;  // 8 cube elements per thread
    float yreg[kPer];
    auto fetch = [&](int kc) {
      const int k0 = kc * kKChunk;
#pragma unroll
      for (int m = 0; m < kPer; ++m) {
        const int e = threadIdx.x + kThreads * m;
        const int b = k0 + e / kPxTile;
        const int64_t p = p0 + e % kPxTile;
        float y = 0.0f;
        if (b < B && p < pixels)
          y = (to_f<T>(cube[static_cast<int64_t>(b) * stride + p]) - op.mean_hi[b]) - op.mean_lo[b];
        yreg[m] = y;
      }
    };
    auto commit = [&](int kc, int buf) {
      const int k0 = kc * kKChunk;
      for (int e = threadIdx.x; e < kKChunk * kRowsTile; e += kThreads)
        sm.w[buf][e % kKChunk][e / kKChunk] = op.waug[static_cast<size_t>(r0 + e / kKChunk) * op.kpad + k0 + e % kKChunk];
#pragma unroll
      for (int m = 0; m < kPer; ++m) {
        const int e = threadIdx.x + kThreads * m;
        sm.y[buf][e / kPxTile][e % kPxTile] = yreg[m];
      }
    };
    fetch(0);
    commit(0, 0);
    __syncthreads();
    for (int kc = 0; kc < kchunks; ++kc) {
      const int buf = kc & 1;
      if (kc + 1 < kchunks) fetch(kc + 1);
      const bool skip = !warp_dense && kc * kKChunk > warp_rows_hi;
      if (!skip) {
#pragma unroll
        for (int k = 0; k < kKChunk; ++k) {
          const float4 wa = *reinterpret_cast<const float4*>(&sm.w[buf][k][ty * 8]);
          const float4 wb = *reinterpret_cast<const float4*>(&sm.w[buf][k][ty * 8 + 4]);
          const float4 ya = *reinterpret_cast<const float4*>(&sm.y[buf][k][tx * 4]);
          const float4 yb = *reinterpret_cast<const float4*>(&sm.y[buf][k][64 + tx * 4]);
          const float wv[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
          const float2 yv[4] = {make_float2(ya.x, ya.y), make_float2(ya.z, ya.w), make_float2(yb.x, yb.y),
                                make_float2(yb.z, yb.w)};
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float2 wi = make_float2(wv[i], wv[i]);
#pragma unroll
            for (int j2 = 0; j2 < 4; ++j2) acc[i][j2] = ffma2(wi, yv[j2], acc[i][j2]);
          }
        }
      }
      // buffer buf ^ 1 was last read in iteration kc - 1, before its closing barrier
      if (kc + 1 < kchunks) commit(kc + 1, buf ^ 1);
      __syncthreads();
    }
    // fold: rows < B -> RX partials; rows B..B+T-1 -> ACE numerators
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int row = r0 + ty * 8 + i;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int px = j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4;
        const float z = (j & 1) ? acc[i][j >> 1].y : acc[i][j >> 1].x;
        if (row < B) {
          rx_part[j] = fmaf(z, z, rx_part[j]);
        } else if (row < B + Tn) {
          sm.zu[row - B][px] = z;
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) sm.rx[ty][j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4] = rx_part[j];
  __syncthreads();
  if (threadIdx.x < kPxTile) {
    const int px = threadIdx.x;
    const int64_t p = p0 + px;
    if (p < pixels) {
      float rx = 0.0f;
#pragma unroll
      for (int g = 0; g < 16; ++g) rx += sm.rx[g][px];
      float zu[HSI_MAX_FILTERS_PER_PASS];
      for (int t = 0; t < Tn; ++t) zu[t] = sm.zu[t][px];
      write_pixel(out, p, rx, zu, sm.uu, Tn);
    }
  }
}

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

SimtOperands carve_simt(void* ws, int B, int T) {
  SimtOperands op;
  op.rows = round_up(B + T, kRowsTile);
  op.kpad = round_up(B, kKChunk);
  unsigned char* p = static_cast<unsigned char*>(ws);
  op.waug = reinterpret_cast<float*>(p);
  p += align256(sizeof(float) * static_cast<size_t>(op.rows) * op.kpad);
  op.mean_hi = reinterpret_cast<float*>(p);
  p += align256(sizeof(float) * HSI_MAX_BANDS);
  op.mean_lo = reinterpret_cast<float*>(p);
  p += align256(sizeof(float) * HSI_MAX_BANDS);
  op.uu = reinterpret_cast<float*>(p);
  return op;
}

size_t simt_bytes(int B, int T) {
  return align256(sizeof(float) * static_cast<size_t>(round_up(B + T, kRowsTile)) * round_up(B, kKChunk)) +
         3 * align256(sizeof(float) * HSI_MAX_BANDS);
}

}  // namespace

// Shared with whiten.cu.
int rxace_check(const void* cube, int height, int width, int bands, int dtype, int64_t stride, const double* stats,
                int T) {
  if (!cube || !stats || height <= 0 || width <= 0 || bands <= 0 || bands > HSI_MAX_BANDS) return HSI_E_INVALID;
  if (T < 0 || T > HSI_MAX_FILTERS_PER_PASS) return HSI_E_INVALID;
  if (dtype != HSI_F32 && dtype != HSI_F16) return HSI_E_INVALID;
  const int64_t P = static_cast<int64_t>(height) * width;
  if (stride < P || (stride & 7) != 0) return HSI_E_INVALID;
  return HSI_OK;
}

}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API size_t hsi_rx_ace_simt_workspace_bytes(int bands, int num_targets) {
  if (bands <= 0 || bands > HSI_MAX_BANDS || num_targets < 0) return 0;
  return simt_bytes(bands, num_targets);
}

extern "C" HSI_API int hsi_rx_ace_simt(const void* d_cube, int height, int width, int bands, int dtype,
                                       int64_t plane_stride, const double* d_stats64, int num_targets,
                                       float* d_rx, float* d_ace_best, int32_t* d_ace_target, float* d_ace_maps,
                                       int64_t map_stride, void* d_workspace, size_t workspace_bytes,
                                       hsi_stream_t stream) {
  const int rc = rxace_check(d_cube, height, width, bands, dtype, plane_stride, d_stats64, num_targets);
  if (rc != HSI_OK) return rc;
  const int64_t P = static_cast<int64_t>(height) * width;
  if (d_ace_maps && map_stride < P) return HSI_E_INVALID;
  if (!d_workspace || workspace_bytes < simt_bytes(bands, num_targets)) return HSI_E_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const SimtOperands op = carve_simt(d_workspace, bands, num_targets);
  prep_simt_kernel<<<op.rows, 256, 0, s>>>(d_stats64, bands, num_targets, op);
  ScoreOut o{d_rx, d_ace_best, d_ace_target, d_ace_maps, map_stride};
  const unsigned blocks = static_cast<unsigned>(div_up<int64_t>(P, kPxTile));
  const int smem = static_cast<int>(sizeof(SimtSmem));
  if (dtype == HSI_F32) {
    const cudaError_t e = raise_smem_limit(rxace_simt_kernel<float>, smem);
    if (e != cudaSuccess) return static_cast<int>(e);
    rxace_simt_kernel<float><<<blocks, kThreads, smem, s>>>(static_cast<const float*>(d_cube), P, plane_stride,
                                                            bands, num_targets, op, o);
  } else {
    const cudaError_t e = raise_smem_limit(rxace_simt_kernel<__half>, smem);
    if (e != cudaSuccess) return static_cast<int>(e);
    rxace_simt_kernel<__half><<<blocks, kThreads, smem, s>>>(static_cast<const __half*>(d_cube), P, plane_stride,
                                                             bands, num_targets, op, o);
  }
  return static_cast<int>(cudaGetLastError());
}
