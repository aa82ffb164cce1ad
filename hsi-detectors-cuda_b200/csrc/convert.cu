// convert.cu - data-format kernels around the scoring path.
//
//   narrow_kernel     fp32 -> fp16, round to nearest even
//                     (reference launch_narrow_to_half, src/sam.cu:311-316,476-482)
//   transpose_kernel  BIP (pixel-major) -> BSQ planes at the caller's plane
//                     stride, through a shared-memory tile so that both the
//                     reads and the writes are coalesced
//                     (reference launch_transpose_bip_to_bsq, src/sam.cu:281-309)
//   demosaic_kernel   snapshot-mosaic frame -> BSQ cube: band b of pixel
//                     (x, y) is raw sample (y*p + oy, x*p + ox) with
//                     (oy, ox) = divmod(order[b], p)
//                     (reference demosaic, src/hot_loader.cpp:144-182)
//   shifted_kernel    raw FP64 moments -> sums about a reference spectrum,
//                     added into the caller's accumulators (the contract of
//                     reference launch_accumulate_moments, src/stats.cu:169-248)
#include <cuda_fp16.h>

#include "common.cuh"

namespace hsi_b200 {
namespace {

constexpr int kMaxOrder = 256;

__global__ void __launch_bounds__(256) narrow_kernel(const float* __restrict__ src, __half* __restrict__ dst,
                                                     int64_t count) {
  const int64_t n4 = count / 4;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n4; i += step) {
    const float4 v = reinterpret_cast<const float4*>(src)[i];
    const __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
    uint2 out;
    out.x = *reinterpret_cast<const uint32_t*>(&a);
    out.y = *reinterpret_cast<const uint32_t*>(&b);
    reinterpret_cast<uint2*>(dst)[i] = out;
  }
  for (int64_t i = n4 * 4 + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count; i += step)
    dst[i] = __float2half_rn(src[i]);
}

// 32 pixels x 32 bands per tile; block 32 x 8.
__global__ void __launch_bounds__(256) transpose_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                                        int64_t pixels, int bands, int64_t stride) {
  __shared__ float tile[32][33];
  const int64_t p0 = static_cast<int64_t>(blockIdx.x) * 32;
  const int b0 = blockIdx.y * 32;
  // read: consecutive threads walk bands of one pixel (contiguous in BIP)
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t p = p0 + i;
    const int b = b0 + threadIdx.x;
    if (p < pixels && b < bands) tile[i][threadIdx.x] = src[p * bands + b];
  }
  __syncthreads();
  // write: consecutive threads walk pixels of one band (contiguous in BSQ)
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int b = b0 + i;
    const int64_t p = p0 + threadIdx.x;
    if (p < pixels && b < bands) dst[static_cast<int64_t>(b) * stride + p] = tile[threadIdx.x][i];
  }
}

struct DemosaicParams {
  int order[kMaxOrder];
};

template <typename T>
__global__ void __launch_bounds__(256) demosaic_kernel(const float* __restrict__ raw, int raw_width, int period,
                                                       int width, int height, T* __restrict__ cube,
                                                       int64_t stride, const __grid_constant__ DemosaicParams prm) {
  const int b = blockIdx.z;
  const int y = blockIdx.y;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= width || y >= height) return;
  const int pos = prm.order[b];
  const int oy = pos / period, ox = pos - oy * period;
  const float v = raw[static_cast<int64_t>(y * period + oy) * raw_width + static_cast<int64_t>(x) * period + ox];
  const int64_t o = static_cast<int64_t>(b) * stride + static_cast<int64_t>(y) * width + x;
  if constexpr (sizeof(T) == 4) {
    cube[o] = v;
  } else {
    cube[o] = __float2half_rn(v);
  }
}

// S1 = M1 - N r;  S2 = M2 - r M1^T - M1 r^T + N r r^T (lower triangle, row-major);
// both added to the accumulators.  One thread per (row, col <= row) entry.
__global__ void __launch_bounds__(256) shifted_kernel(const double* __restrict__ m, const float* __restrict__ ref,
                                                      int bands, double* __restrict__ s1, double* __restrict__ s2) {
  const int B = bands;
  const double* sum = m;
  const double* outer = m + B;
  const double n = m[B + static_cast<int64_t>(B) * B];
  const int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  const int64_t tri = static_cast<int64_t>(B) * (B + 1) / 2;
  if (e < B) {
    const double r = ref ? static_cast<double>(ref[e]) : 0.0;
    s1[e] += sum[e] - n * r;
  }
  if (e >= tri) return;
  // row i, column j <= i, from the packed lower-triangle index
  int i = static_cast<int>((sqrt(8.0 * static_cast<double>(e) + 1.0) - 1.0) * 0.5);
  while (static_cast<int64_t>(i) * (i + 1) / 2 > e) --i;
  while (static_cast<int64_t>(i + 1) * (i + 2) / 2 <= e) ++i;
  const int j = static_cast<int>(e - static_cast<int64_t>(i) * (i + 1) / 2);
  const double ri = ref ? static_cast<double>(ref[i]) : 0.0;
  const double rj = ref ? static_cast<double>(ref[j]) : 0.0;
  const double v = outer[static_cast<int64_t>(i) * B + j] - ri * sum[j] - sum[i] * rj + n * ri * rj;
  s2[static_cast<int64_t>(i) * B + j] += v;
}

int grid_for(int64_t work, int threads) {
  const int64_t g = (work + threads - 1) / threads;
  return static_cast<int>(g < 148 * 32 ? (g > 0 ? g : 1) : 148 * 32);
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API int hsi_narrow_to_half(const float* d_src, void* d_dst, int64_t count, hsi_stream_t stream) {
  if (count < 0 || (count > 0 && (!d_src || !d_dst))) return HSI_E_INVALID;
  if (count == 0) return HSI_OK;
  if ((reinterpret_cast<uintptr_t>(d_src) & 15u) != 0 || (reinterpret_cast<uintptr_t>(d_dst) & 7u) != 0)
    return HSI_E_INVALID;
  narrow_kernel<<<grid_for(count / 4 + 1, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      d_src, static_cast<__half*>(d_dst), count);
  return static_cast<int>(cudaGetLastError());
}

extern "C" HSI_API int hsi_transpose_bip_to_bsq(const float* d_src, float* d_dst, int height, int width, int bands,
                                                int64_t plane_stride, hsi_stream_t stream) {
  if (!d_src || !d_dst || height <= 0 || width <= 0 || bands <= 0) return HSI_E_INVALID;
  const int64_t P = static_cast<int64_t>(height) * width;
  if (plane_stride < P) return HSI_E_INVALID;
  const int64_t gx = (P + 31) / 32;
  if (gx > 0x7fffffff) return HSI_E_CAPACITY;
  const dim3 grid(static_cast<unsigned>(gx), static_cast<unsigned>((bands + 31) / 32));
  transpose_kernel<<<grid, dim3(32, 8), 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_src, d_dst, P, bands,
                                                                                     plane_stride);
  return static_cast<int>(cudaGetLastError());
}

extern "C" HSI_API int hsi_demosaic(const float* d_raw, int raw_height, int raw_width, int period, int bands,
                                    const int32_t* band_order, void* d_cube, int dtype, int64_t plane_stride,
                                    hsi_stream_t stream) {
  if (!d_raw || !d_cube || period <= 0 || bands <= 0 || bands > period * period || bands > kMaxOrder)
    return HSI_E_INVALID;
  if (dtype != HSI_F32 && dtype != HSI_F16) return HSI_E_INVALID;
  const int width = raw_width / period, height = raw_height / period;
  if (width <= 0 || height <= 0) return HSI_E_INVALID;
  if (plane_stride < static_cast<int64_t>(width) * height) return HSI_E_INVALID;
  DemosaicParams prm{};
  for (int b = 0; b < bands; ++b) {
    const int pos = band_order ? band_order[b] : b;
    if (pos < 0 || pos >= period * period) return HSI_E_INVALID;
    prm.order[b] = pos;
  }
  const dim3 grid(static_cast<unsigned>((width + 255) / 256), static_cast<unsigned>(height),
                  static_cast<unsigned>(bands));
  if (grid.y > 65535) return HSI_E_CAPACITY;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (dtype == HSI_F32)
    demosaic_kernel<float><<<grid, 256, 0, s>>>(d_raw, raw_width, period, width, height,
                                                static_cast<float*>(d_cube), plane_stride, prm);
  else
    demosaic_kernel<__half><<<grid, 256, 0, s>>>(d_raw, raw_width, period, width, height,
                                                 static_cast<__half*>(d_cube), plane_stride, prm);
  return static_cast<int>(cudaGetLastError());
}

extern "C" HSI_API int hsi_accumulate_shifted_moments(const double* d_moments, const float* d_reference, int bands,
                                                      double* d_sum, double* d_sum_outer, hsi_stream_t stream) {
  if (!d_moments || !d_sum || !d_sum_outer || bands <= 0 || bands > HSI_MAX_BANDS) return HSI_E_INVALID;
  const int64_t tri = static_cast<int64_t>(bands) * (bands + 1) / 2;
  shifted_kernel<<<static_cast<unsigned>((tri + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      d_moments, d_reference, bands, d_sum, d_sum_outer);
  return static_cast<int>(cudaGetLastError());
}
