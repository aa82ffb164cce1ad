// factor.cu - detector statistics in FP64 on the device.
//
// From a frame's raw moments (sum, outer, count) and its target library,
// build everything the RX / ACE / CEM scorers index (reference
// build_statistics, src/detector.cpp:47-152, with the FP64 routines of
// src/linalg.cpp:105-162):
//   mean mu = M1/N
//   S = M2/N - mu mu^T + loading I = L L^T     (Cholesky, fails if not PD)
//   W = L^-1                                   (lower, strict upper zero)
//   u_t = W (d_t - mu),  |u_t|^2               (ACE target half)
//   R = M2/N + loading I = C C^T,  x_t = R^-1 d_t,  w_t = x_t / (d_t . x_t)
//                                              (CEM; 0 if d_t . x_t <= 0)
// All arithmetic is FP64, because the factorisation of a nearly rank-6
// covariance needs it.  One CTA per frame; frames of a batch factor in
// parallel.  Matrices live in shared memory as packed lower triangles when
// they fit (B <= 128) and in the caller's workspace otherwise.
#include "common.cuh"

namespace hsi_b200 {
namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kSmemMaxBands = 128;

__host__ __device__ inline size_t tri(int n) { return static_cast<size_t>(n) * (n + 1) / 2; }
__device__ __forceinline__ size_t pk(int i, int j) { return static_cast<size_t>(i) * (i + 1) / 2 + j; }  // j <= i

struct FactorArgs {
  int bands, targets;
  double loading;
  const double* moments;  // per frame: sum[B], outer[B*B], count
  int64_t moments_stride;
  const float* library;   // per frame: T x B, or one shared library (stride 0)
  int64_t library_stride;
  double* stats64;        // nullable, packed layout, stride = statistics_elements
  float* stats32;         // nullable, same layout narrowed to float
  float* cem32;           // nullable, T x B per frame (contiguous frames)
  int* status;            // nullable, per frame
  double* scratch;        // global scratch: per frame 2 * tri(B) doubles (B > kSmemMaxBands)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// In-place right-looking Cholesky of a packed lower triangle.  Returns false
// (to every thread) if a pivot is not positive or is NaN (src/linalg.cpp:105-122).
__device__ bool cholesky_packed(double* a, int n, int* s_flag) {
  for (int k = 0; k < n; ++k) {
    if (threadIdx.x == 0) {
      const double d = a[pk(k, k)];
      if (!(d > 0.0)) *s_flag = 1;
      else a[pk(k, k)] = sqrt(d);
    }
    __syncthreads();
    if (*s_flag) return false;
    const double piv = a[pk(k, k)];
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) a[pk(i, k)] /= piv;
    __syncthreads();
    // trailing update of rows i > k, columns k < j <= i
    const int m = n - k - 1;
    const size_t work = tri(m);
    for (size_t e = threadIdx.x; e < work; e += blockDim.x) {
      // decode e -> (ii, jj) with jj <= ii < m
      int ii = static_cast<int>((sqrt(8.0 * static_cast<double>(e) + 1.0) - 1.0) * 0.5);
      while (tri(ii + 1) <= e) ++ii;
      while (tri(ii) > e) --ii;
      const int jj = static_cast<int>(e - tri(ii));
      const int i = k + 1 + ii, j = k + 1 + jj;
      a[pk(i, j)] -= a[pk(i, k)] * a[pk(j, k)];
    }
    __syncthreads();
  }
  return true;
}

__global__ void __launch_bounds__(kThreads) factor_kernel(const FactorArgs args) {
  extern __shared__ double smem[];
  __shared__ int s_flag;
  const int f = blockIdx.x;
  const int B = args.bands, T = args.targets;
  const double* mom = args.moments + f * args.moments_stride;
  const float* lib = args.library ? args.library + f * args.library_stride : nullptr;
  const size_t per = static_cast<size_t>(B) + static_cast<size_t>(B) * B + 2 * static_cast<size_t>(T) * B + T;
  double* out64 = args.stats64 ? args.stats64 + f * per : nullptr;
  float* out32 = args.stats32 ? args.stats32 + f * per : nullptr;
  float* cem32 = args.cem32 ? args.cem32 + static_cast<size_t>(f) * T * B : nullptr;
  const bool in_smem = B <= kSmemMaxBands;
  // smem: mean[B], T x B target work vectors, one solve vector per warp,
  // then the packed matrices (in the workspace when B is large)
  double* mean = smem;
  double* vec = mean + B;
  double* xs = vec + static_cast<size_t>(T) * B;
  double* A = in_smem ? xs + static_cast<size_t>(kWarps) * B : args.scratch + static_cast<size_t>(f) * 2 * tri(B);
  double* W = A + tri(B);  // packed L^-1 (lower)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) s_flag = 0;

  const double N = mom[B + B * B];
  if (!(N > 0.0)) {
    if (threadIdx.x == 0 && args.status) args.status[f] = HSI_E_EMPTY;
    return;
  }
  const double* sum = mom;
  const double* outer = mom + B;
  for (int i = threadIdx.x; i < B; i += blockDim.x) mean[i] = sum[i] / N;
  __syncthreads();
  // covariance, loaded (src/linalg.cpp:56-79: correlation then subtract mu mu^T)
  for (size_t e = threadIdx.x; e < tri(B); e += blockDim.x) {
    int i = static_cast<int>((sqrt(8.0 * static_cast<double>(e) + 1.0) - 1.0) * 0.5);
    while (tri(i + 1) <= e) ++i;
    while (tri(i) > e) --i;
    const int j = static_cast<int>(e - tri(i));
    double v = outer[static_cast<size_t>(i) * B + j] / N - mean[i] * mean[j];
    if (i == j) v += args.loading;
    A[e] = v;
  }
  __syncthreads();
  if (!cholesky_packed(A, B, &s_flag)) {
    if (threadIdx.x == 0 && args.status) args.status[f] = HSI_E_NOT_POSITIVE_DEFINITE;
    return;
  }
  // W = L^-1, one column per thread (forward substitution down the column;
  // src/linalg.cpp:150-162)
  for (int k = threadIdx.x; k < B; k += blockDim.x) {
    W[pk(k, k)] = 1.0 / A[pk(k, k)];
    for (int i = k + 1; i < B; ++i) {
      double s = 0.0;
      for (int j = k; j < i; ++j) s -= A[pk(i, j)] * W[pk(j, k)];
      W[pk(i, k)] = s / A[pk(i, i)];
    }
  }
  __syncthreads();
  // outputs: mean, whitener (row-major, upper zero)
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    if (out64) out64[i] = mean[i];
    if (out32) out32[i] = static_cast<float>(mean[i]);
  }
  for (size_t e = threadIdx.x; e < static_cast<size_t>(B) * B; e += blockDim.x) {
    const int i = static_cast<int>(e / B), j = static_cast<int>(e % B);
    const double v = j <= i ? W[pk(i, j)] : 0.0;
    if (out64) out64[B + e] = v;
    if (out32) out32[B + e] = static_cast<float>(v);
  }
  if (T == 0) {
    if (threadIdx.x == 0 && args.status) args.status[f] = HSI_OK;
    return;
  }
  const size_t off_tw = static_cast<size_t>(B) + static_cast<size_t>(B) * B;
  const size_t off_tn = off_tw + static_cast<size_t>(T) * B;
  const size_t off_cw = off_tn + T;
  // ACE: u_t = W (d_t - mu), |u_t|^2 -- one warp per target row block
  for (size_t e = threadIdx.x; e < static_cast<size_t>(T) * B; e += blockDim.x)
    vec[e] = static_cast<double>(lib[e]) - mean[e % B];
  __syncthreads();
  for (int t = warp; t < T; t += kWarps) {
    const double* c = vec + static_cast<size_t>(t) * B;
    double norm2 = 0.0;
    for (int i = 0; i < B; ++i) {
      double s = 0.0;
      for (int j = lane; j <= i; j += 32) s += W[pk(i, j)] * c[j];
      s = warp_sum(s);
      norm2 += s * s;
      if (lane == 0) {
        if (out64) out64[off_tw + static_cast<size_t>(t) * B + i] = s;
        if (out32) out32[off_tw + static_cast<size_t>(t) * B + i] = static_cast<float>(s);
      }
    }
    if (lane == 0) {
      if (out64) out64[off_tn + t] = norm2;
      if (out32) out32[off_tn + t] = static_cast<float>(norm2);
    }
  }
  __syncthreads();
  // CEM: correlation R = M2/N + loading I, factor into A (reused)
  if (threadIdx.x == 0) s_flag = 0;
  for (size_t e = threadIdx.x; e < tri(B); e += blockDim.x) {
    int i = static_cast<int>((sqrt(8.0 * static_cast<double>(e) + 1.0) - 1.0) * 0.5);
    while (tri(i + 1) <= e) ++i;
    while (tri(i) > e) --i;
    const int j = static_cast<int>(e - tri(i));
    double v = outer[static_cast<size_t>(i) * B + j] / N;
    if (i == j) v += args.loading;
    A[e] = v;
  }
  __syncthreads();
  if (!cholesky_packed(A, B, &s_flag)) {
    if (threadIdx.x == 0 && args.status) args.status[f] = HSI_E_CORRELATION_NOT_PD;
    return;
  }
  // x_t = R^-1 d_t by forward then back substitution, one warp per target
  // (src/linalg.cpp:124-137); the raw target replaces the centred one in vec.
  for (size_t e = threadIdx.x; e < static_cast<size_t>(T) * B; e += blockDim.x) vec[e] = static_cast<double>(lib[e]);
  __syncthreads();
  for (int t = warp; t < T; t += kWarps) {
    double* x = xs + static_cast<size_t>(warp) * B;
    const double* d = vec + static_cast<size_t>(t) * B;
    for (int i = 0; i < B; ++i) {
      double s = 0.0;
      for (int k = lane; k < i; k += 32) s += A[pk(i, k)] * x[k];
      s = warp_sum(s);
      if (lane == 0) x[i] = (d[i] - s) / A[pk(i, i)];
      __syncwarp();
    }
    for (int i = B - 1; i >= 0; --i) {
      double s = 0.0;
      for (int k = i + 1 + lane; k < B; k += 32) s += A[pk(k, i)] * x[k];
      s = warp_sum(s);
      if (lane == 0) x[i] = (x[i] - s) / A[pk(i, i)];
      __syncwarp();
    }
    double g = 0.0;
    for (int i = lane; i < B; i += 32) g += d[i] * x[i];
    g = warp_sum(g);
    for (int i = lane; i < B; i += 32) {
      const double w = g > 0.0 ? x[i] / g : 0.0;
      if (out64) out64[off_cw + static_cast<size_t>(t) * B + i] = w;
      if (out32) out32[off_cw + static_cast<size_t>(t) * B + i] = static_cast<float>(w);
      if (cem32) cem32[static_cast<size_t>(t) * B + i] = static_cast<float>(w);
    }
  }
  if (threadIdx.x == 0 && args.status) args.status[f] = HSI_OK;
}

size_t smem_bytes(int B, int T) {
  const size_t vectors = static_cast<size_t>(B) + static_cast<size_t>(T) * B + static_cast<size_t>(kWarps) * B;
  if (B <= kSmemMaxBands) return sizeof(double) * (vectors + 2 * tri(B));
  return sizeof(double) * vectors;
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API size_t hsi_statistics_elements(int bands, int num_targets) {
  if (bands <= 0 || num_targets < 0) return 0;
  return static_cast<size_t>(bands) + static_cast<size_t>(bands) * bands + 2 * static_cast<size_t>(num_targets) * bands +
         num_targets;
}

extern "C" HSI_API size_t hsi_factor_workspace_bytes(int num_frames, int bands) {
  if (num_frames <= 0 || bands <= 0) return 0;
  if (bands <= kSmemMaxBands) return 0;
  return sizeof(double) * 2 * tri(bands) * static_cast<size_t>(num_frames);
}

extern "C" HSI_API int hsi_build_statistics(int num_frames, int bands, int num_targets, double loading,
                                            const double* d_moments, const float* d_library,
                                            int64_t library_stride, double* d_stats64, float* d_stats32,
                                            float* d_cem_weights, int* d_status, void* d_workspace,
                                            size_t workspace_bytes, hsi_stream_t stream) {
  if (num_frames <= 0 || bands <= 0 || bands > HSI_MAX_BANDS || num_targets < 0 || num_targets > 64 || !d_moments)
    return HSI_E_INVALID;
  if (num_targets > 0 && !d_library) return HSI_E_INVALID;
  if (!(loading >= 0.0)) return HSI_E_INVALID;
  const size_t need = hsi_factor_workspace_bytes(num_frames, bands);
  if (need > 0 && (!d_workspace || workspace_bytes < need)) return HSI_E_WORKSPACE;
  FactorArgs a;
  a.bands = bands;
  a.targets = num_targets;
  a.loading = loading;
  a.moments = d_moments;
  a.moments_stride = static_cast<int64_t>(bands) + static_cast<int64_t>(bands) * bands + 1;
  a.library = d_library;
  a.library_stride = library_stride;
  a.stats64 = d_stats64;
  a.stats32 = d_stats32;
  a.cem32 = d_cem_weights;
  a.status = d_status;
  a.scratch = static_cast<double*>(d_workspace);
  const size_t smem = smem_bytes(bands, num_targets);
  if (smem > 227 * 1024) return HSI_E_CAPACITY;
  cudaError_t e = cudaFuncSetAttribute(factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return static_cast<int>(e);
  factor_kernel<<<num_frames, kThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  return static_cast<int>(cudaGetLastError());
}
