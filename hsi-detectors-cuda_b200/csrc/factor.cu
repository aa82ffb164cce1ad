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
// they fit (B <= 128) and in the caller's workspace otherwise.  The solves use
// the explicit triangular inverses (blocked, parallel) rather than sequential
// substitution, so a single frame factors in ~0.1 ms instead of being bound by
// ~10^4 dependent FP64 steps.
#include "common.cuh"

namespace hsi_b200 {
namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kSmemMaxBands = 128;
constexpr int kChunk = 16;  // targets per pass through the per-target buffers
constexpr int kBlk = 16;    // row block of the triangular inverse

__host__ __device__ inline size_t tri(int n) { return static_cast<size_t>(n) * (n + 1) / 2; }
__device__ __forceinline__ size_t row_off(int i) { return static_cast<size_t>(i) * (i + 1) / 2; }

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

// Fill the packed lower triangle with M2/N (- mean mean^T) + loading I.
__device__ void fill_matrix(double* A, const double* outer, const double* mean, double N, double loading, int n,
                            bool centred) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = warp; i < n; i += kWarps) {
    double* ri = A + row_off(i);
    for (int j = lane; j <= i; j += 32) {
      double v = outer[static_cast<size_t>(i) * n + j] / N;
      if (centred) v -= mean[i] * mean[j];
      if (i == j) v += loading;
      ri[j] = v;
    }
  }
  __syncthreads();
}

// In-place right-looking Cholesky of a packed lower triangle, one barrier per
// elimination step: step k subtracts a_ik a_jk / a_kk from the trailing
// triangle with the column left unscaled, and all columns are scaled by
// 1/sqrt(pivot) at the end.  Returns false -- the same on every thread, which
// all read the same pivot -- if a pivot is not positive or is NaN
// (src/linalg.cpp:105-122).  `dv`: n doubles of scratch.
__device__ bool cholesky_packed(double* a, int n, double* dv) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = 0; k < n; ++k) {
    const double d = a[row_off(k) + k];
    if (!(d > 0.0)) return false;
    const double inv = 1.0 / d;
    for (int i = k + 1 + warp; i < n; i += kWarps) {
      double* ri = a + row_off(i);
      const double f = ri[k] * inv;
      for (int j = k + 1 + lane; j <= i; j += 32) ri[j] -= f * a[row_off(j) + k];
    }
    __syncthreads();
  }
  for (int k = threadIdx.x; k < n; k += blockDim.x) dv[k] = sqrt(a[row_off(k) + k]);
  __syncthreads();
  for (int i = warp; i < n; i += kWarps) {
    double* ri = a + row_off(i);
    for (int j = lane; j <= i; j += 32) ri[j] = j == i ? dv[i] : ri[j] / dv[j];
  }
  __syncthreads();
  return true;
}

// Winv = L^-1 (both packed lower) by blocked forward substitution on L X = I
// (src/linalg.cpp:150-162 solves the same system column by column).  Per row
// block [r0, r1): first every (row, column) takes the part of its sum over the
// finished rows j < r0 in parallel, then each thread finishes one column down
// the block's rows.
__device__ void triangular_inverse(const double* L, double* Winv, int n) {
  for (int r0 = 0; r0 < n; r0 += kBlk) {
    const int r1 = min(r0 + kBlk, n);
    const int work = (r1 - r0) * r1;
    for (int e = threadIdx.x; e < work; e += blockDim.x) {
      const int i = r0 + e / r1, c = e % r1;
      if (c > i) continue;
      double s = c == i ? 1.0 : 0.0;
      if (c < r0) {
        const double* li = L + row_off(i);
        for (int j = c; j < r0; ++j) s -= li[j] * Winv[row_off(j) + c];
      }
      Winv[row_off(i) + c] = s;
    }
    __syncthreads();
    for (int c = threadIdx.x; c < r1; c += blockDim.x) {
      const int j0 = max(r0, c);
      for (int i = j0; i < r1; ++i) {
        const double* li = L + row_off(i);
        double s = Winv[row_off(i) + c];
        for (int j = j0; j < i; ++j) s -= li[j] * Winv[row_off(j) + c];
        Winv[row_off(i) + c] = s / li[i];
      }
    }
    __syncthreads();
  }
}

// out[t][i] = sum_{j <= i} M[i][j] v[t][j] (M packed lower), t < nt.
__device__ void lower_matvec(const double* M, const double* v, double* out, int n, int nt) {
  for (int e = threadIdx.x; e < nt * n; e += blockDim.x) {
    const int t = e / n, i = e % n;
    const double* mi = M + row_off(i);
    const double* vt = v + static_cast<size_t>(t) * n;
    double s = 0.0;
    for (int j = 0; j <= i; ++j) s += mi[j] * vt[j];
    out[e] = s;
  }
  __syncthreads();
}

// out[t][i] = sum_{k >= i} M[k][i] v[t][k] (M^T, M packed lower), t < nt.
__device__ void upper_matvec(const double* M, const double* v, double* out, int n, int nt) {
  for (int e = threadIdx.x; e < nt * n; e += blockDim.x) {
    const int t = e / n, i = e % n;
    const double* vt = v + static_cast<size_t>(t) * n;
    double s = 0.0;
    for (int k = i; k < n; ++k) s += M[row_off(k) + i] * vt[k];
    out[e] = s;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads) factor_kernel(const FactorArgs args) {
  extern __shared__ double smem[];
  const int f = blockIdx.x;
  const int B = args.bands, T = args.targets;
  const double* mom = args.moments + f * args.moments_stride;
  const float* lib = args.library ? args.library + f * args.library_stride : nullptr;
  const size_t per = static_cast<size_t>(B) + static_cast<size_t>(B) * B + 2 * static_cast<size_t>(T) * B + T;
  double* out64 = args.stats64 ? args.stats64 + f * per : nullptr;
  float* out32 = args.stats32 ? args.stats32 + f * per : nullptr;
  float* cem32 = args.cem32 ? args.cem32 + static_cast<size_t>(f) * T * B : nullptr;
  const bool in_smem = B <= kSmemMaxBands;
  // smem: mean[B], pivots[B], two chunk buffers of kChunk x B, then the
  // packed matrices (in the workspace when B is large)
  double* mean = smem;
  double* dv = mean + B;
  double* vec = dv + B;
  double* buf = vec + static_cast<size_t>(kChunk) * B;
  double* A = in_smem ? buf + static_cast<size_t>(kChunk) * B : args.scratch + static_cast<size_t>(f) * 2 * tri(B);
  double* W = A + tri(B);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  const double N = mom[B + B * B];
  if (!(N > 0.0)) {
    if (threadIdx.x == 0 && args.status) args.status[f] = HSI_E_EMPTY;
    return;
  }
  const double* sum = mom;
  const double* outer = mom + B;
  for (int i = threadIdx.x; i < B; i += blockDim.x) mean[i] = sum[i] / N;
  __syncthreads();
  // covariance, loaded (src/linalg.cpp:56-79), its Cholesky factor and inverse
  fill_matrix(A, outer, mean, N, args.loading, B, true);
  if (!cholesky_packed(A, B, dv)) {
    if (threadIdx.x == 0 && args.status) args.status[f] = HSI_E_NOT_POSITIVE_DEFINITE;
    return;
  }
  triangular_inverse(A, W, B);
  // outputs: mean, whitener (row-major, upper zero)
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    if (out64) out64[i] = mean[i];
    if (out32) out32[i] = static_cast<float>(mean[i]);
  }
  for (size_t e = threadIdx.x; e < static_cast<size_t>(B) * B; e += blockDim.x) {
    const int i = static_cast<int>(e / B), j = static_cast<int>(e % B);
    const double v = j <= i ? W[row_off(i) + j] : 0.0;
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
  // ACE: u_t = W (d_t - mu) and |u_t|^2, kChunk targets at a time
  for (int t0 = 0; t0 < T; t0 += kChunk) {
    const int nt = min(kChunk, T - t0);
    for (int e = threadIdx.x; e < nt * B; e += blockDim.x)
      vec[e] = static_cast<double>(lib[static_cast<size_t>(t0) * B + e]) - mean[e % B];
    __syncthreads();
    lower_matvec(W, vec, buf, B, nt);
    for (int e = threadIdx.x; e < nt * B; e += blockDim.x) {
      if (out64) out64[off_tw + static_cast<size_t>(t0) * B + e] = buf[e];
      if (out32) out32[off_tw + static_cast<size_t>(t0) * B + e] = static_cast<float>(buf[e]);
    }
    for (int t = warp; t < nt; t += kWarps) {
      double s = 0.0;
      for (int i = lane; i < B; i += 32) s += buf[t * B + i] * buf[t * B + i];
      s = warp_sum(s);
      if (lane == 0) {
        if (out64) out64[off_tn + t0 + t] = s;
        if (out32) out32[off_tn + t0 + t] = static_cast<float>(s);
      }
    }
    __syncthreads();
  }
  // CEM: R = M2/N + loading I = C C^T; y_t = C^-1 d_t, x_t = C^-T y_t = R^-1 d_t,
  // d_t . x_t = |y_t|^2; w_t = x_t / |y_t|^2, 0 if that gain is not positive
  // (src/detector.cpp:128-148)
  fill_matrix(A, outer, mean, N, args.loading, B, false);
  if (!cholesky_packed(A, B, dv)) {
    if (threadIdx.x == 0 && args.status) args.status[f] = HSI_E_CORRELATION_NOT_PD;
    return;
  }
  triangular_inverse(A, W, B);
  for (int t0 = 0; t0 < T; t0 += kChunk) {
    const int nt = min(kChunk, T - t0);
    for (int e = threadIdx.x; e < nt * B; e += blockDim.x)
      vec[e] = static_cast<double>(lib[static_cast<size_t>(t0) * B + e]);
    __syncthreads();
    lower_matvec(W, vec, buf, B, nt);   // y
    upper_matvec(W, buf, vec, B, nt);   // x (d is no longer needed)
    for (int t = warp; t < nt; t += kWarps) {
      double g = 0.0;
      for (int i = lane; i < B; i += 32) g += buf[t * B + i] * buf[t * B + i];
      g = warp_sum(g);
      for (int i = lane; i < B; i += 32) {
        const double w = g > 0.0 ? vec[t * B + i] / g : 0.0;
        const size_t o = static_cast<size_t>(t0 + t) * B + i;
        if (out64) out64[off_cw + o] = w;
        if (out32) out32[off_cw + o] = static_cast<float>(w);
        if (cem32) cem32[o] = static_cast<float>(w);
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && args.status) args.status[f] = HSI_OK;
}

size_t smem_bytes(int B, int /*T*/) {
  const size_t vectors = 2 * static_cast<size_t>(B) + 2 * static_cast<size_t>(kChunk) * B;
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
