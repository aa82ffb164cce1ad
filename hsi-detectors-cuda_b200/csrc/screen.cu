// screen.cu - the learned screen: a per-pixel MLP B -> 64 -> 32 -> 1 that
// proposes candidate pixels for the plain ACE detector to re-score.
//
// No counterpart in the reference.  Trained on the device on the plain
// detector's own ACE decisions over synthetic frames, by the kernels here:
//   normaliser   per band: mean and a power-of-two scale s_b ~ 1/sigma_b
//                (power of two, so that it folds exactly into fp16 weights);
//   batch        training samples: positives drawn from the detector's
//                compacted positive list, the rest uniform over the frame;
//   gather       features (x_b - mean_b) s_b rounded to bfloat16, band-major
//                [Bp][n], and the 0/1 labels from the score map;
//   forward      one thread per sample (bfloat16 weights, FP32 accumulation,
//                h1 rounded to bfloat16 as inference does), storing the
//                activations and back-propagated deltas;
//   gradients    dW = delta^T act as small deterministic SIMT GEMMs;
//   adam         FP32 master weights; the forward reads them rounded.
// Inference (screen_tc_kernel, below) runs layers 1 and 2 on the tensor
// cores straight from the fp16 cube.
//
// Parameter layout (FP32), Bp = bands rounded up to 64:
//   W1[64][Bp] | b1[64] | W2[32][64] | b2[32] | w3[32] | b3
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "synth.h"
#include "launch_state.h"
#include "tc.cuh"

namespace hsi_b200 {
namespace {

constexpr int kH1 = 64, kH2 = 32;

__host__ __device__ inline int padded_bands(int B) { return (B + 63) / 64 * 64; }
__host__ __device__ inline int64_t param_count(int B) {
  return static_cast<int64_t>(kH1) * padded_bands(B) + kH1 + kH2 * kH1 + kH2 + kH2 + 1;
}

struct ParamView {
  float *W1, *b1, *W2, *b2, *w3, *b3;
};
__host__ __device__ inline ParamView view(float* p, int B) {
  ParamView v;
  v.W1 = p;
  v.b1 = v.W1 + static_cast<int64_t>(kH1) * padded_bands(B);
  v.W2 = v.b1 + kH1;
  v.b2 = v.W2 + kH2 * kH1;
  v.w3 = v.b2 + kH2;
  v.b3 = v.w3 + kH2;
  return v;
}

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// ---- initialisation: He-uniform from a counter hash, padding columns zero ----
__global__ void init_kernel(float* __restrict__ p, int B, uint64_t seed) {
  const int Bp = padded_bands(B);
  const int64_t n = param_count(B);
  const ParamView v = view(p, B);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double u = static_cast<double>(hsi_mix64(seed ^ (0x9E3779B97F4A7C15ull * (i + 1))) >> 11) * 0x1.0p-53;
    float val = 0.0f;
    float* q = p + i;
    if (q < v.b1) {
      const int b = static_cast<int>(i % Bp);
      if (b < B) val = static_cast<float>((2.0 * u - 1.0) * sqrt(6.0 / B));
    } else if (q >= v.W2 && q < v.b2) {
      val = static_cast<float>((2.0 * u - 1.0) * sqrt(6.0 / kH1));
    } else if (q >= v.w3 && q < v.b3) {
      val = static_cast<float>((2.0 * u - 1.0) * sqrt(6.0 / kH2));
    }
    p[i] = val;  // biases start at zero
  }
}

// ---- normaliser: mean and power-of-two scale from raw FP64 moments ----------
__global__ void normaliser_kernel(const double* __restrict__ m, int B, float* __restrict__ norm) {
  const int Bp = padded_bands(B);
  const double N = m[B + static_cast<int64_t>(B) * B];
  for (int b = threadIdx.x; b < Bp; b += blockDim.x) {
    float mu = 0.0f, s = 0.0f;
    if (b < B && N > 0.0) {
      const double mean = m[b] / N;
      const double var = m[B + static_cast<int64_t>(b) * B + b] / N - mean * mean;
      mu = static_cast<float>(mean);
      // s = 2^round(-log2 sigma): exact in fp16 weights; 1 for a constant band;
      // clamped so that |bfloat16 weight| * s stays inside the fp16 range
      s = var > 0.0 ? static_cast<float>(exp2(rint(-0.5 * log2(var)))) : 1.0f;
      s = fminf(fmaxf(s, 0x1.0p-14f), 0x1.0p12f);
    }
    norm[b] = mu;
    norm[Bp + b] = s;
  }
}

// ---- training batch: n_pos draws from the positive list, the rest uniform ----
__global__ void batch_kernel(const hsi_detection* __restrict__ pos, const uint32_t* __restrict__ pos_count,
                             int pos_capacity, int width, int64_t pixels, const float* __restrict__ score,
                             float threshold, uint64_t seed, int n_pos, int n, int32_t* __restrict__ index,
                             float* __restrict__ labels) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t np = min(*pos_count, static_cast<uint32_t>(pos_capacity));
  const uint64_t h = hsi_mix64(seed * 0x100000001B3ull + static_cast<uint64_t>(s));
  int64_t p;
  if (s < n_pos && np > 0) {
    const hsi_detection d = pos[h % np];
    p = static_cast<int64_t>(d.y) * width + d.x;
  } else {
    p = static_cast<int64_t>(h % static_cast<uint64_t>(pixels));
  }
  index[s] = static_cast<int32_t>(p);
  labels[s] = score[p] >= threshold ? 1.0f : 0.0f;
}

// ---- gather: features [Bp][n], (x - mean) s rounded to bfloat16 --------------
template <typename T>
__global__ void gather_kernel(const T* __restrict__ cube, int64_t stride, int B, const float* __restrict__ norm,
                              const int32_t* __restrict__ index, int n, float* __restrict__ features) {
  const int Bp = padded_bands(B);
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (s >= n) return;
  float v = 0.0f;
  if (b < B) {
    float x;
    if constexpr (sizeof(T) == 4) {
      x = cube[static_cast<int64_t>(b) * stride + index[s]];
    } else {
      x = __half2float(cube[static_cast<int64_t>(b) * stride + index[s]]);
    }
    v = bf16r((x - norm[b]) * norm[Bp + b]);
  }
  features[static_cast<int64_t>(b) * n + s] = v;
}

// ---- forward + deltas, one thread per sample --------------------------------
// Activations and deltas, sample-minor: H1[64][n], H2[32][n], D1[64][n],
// D2[32][n], D3[n]; per-block partial losses.
struct Acts {
  float *H1, *H2, *D1, *D2, *D3, *loss_part;
};

constexpr int kFwdThreads = 128;

__global__ void __launch_bounds__(kFwdThreads) forward_kernel(const float* __restrict__ params, int B,
                                                             const float* __restrict__ X,
                                                             const float* __restrict__ labels, int n,
                                                             float pos_weight, Acts a) {
  extern __shared__ float sw[];
  const int Bp = padded_bands(B);
  const ParamView v = view(const_cast<float*>(params), B);
  // W1 transposed to [b][64] and W2 to [j][32], both rounded to bfloat16
  float* w1t = sw;
  float* w2t = w1t + static_cast<int64_t>(Bp) * kH1;
  float* w3r = w2t + kH1 * kH2;
  __shared__ float s_loss[kFwdThreads / 32];
  for (int e = threadIdx.x; e < Bp * kH1; e += blockDim.x) {
    const int j = e / Bp, b = e % Bp;
    w1t[b * kH1 + j] = bf16r(v.W1[e]);
  }
  for (int e = threadIdx.x; e < kH2 * kH1; e += blockDim.x) {
    const int k = e / kH1, j = e % kH1;
    w2t[j * kH2 + k] = bf16r(v.W2[e]);
  }
  for (int k = threadIdx.x; k < kH2; k += blockDim.x) w3r[k] = bf16r(v.w3[k]);
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  float loss = 0.0f;
  if (s < n) {
    float z1[kH1];
#pragma unroll
    for (int j = 0; j < kH1; ++j) z1[j] = v.b1[j];
    for (int b = 0; b < B; ++b) {
      const float x = X[static_cast<int64_t>(b) * n + s];
      const float4* w = reinterpret_cast<const float4*>(w1t + b * kH1);
#pragma unroll
      for (int q = 0; q < kH1 / 4; ++q) {
        const float4 c = w[q];
        z1[4 * q] = fmaf(c.x, x, z1[4 * q]);
        z1[4 * q + 1] = fmaf(c.y, x, z1[4 * q + 1]);
        z1[4 * q + 2] = fmaf(c.z, x, z1[4 * q + 2]);
        z1[4 * q + 3] = fmaf(c.w, x, z1[4 * q + 3]);
      }
    }
#pragma unroll
    for (int j = 0; j < kH1; ++j) a.H1[static_cast<int64_t>(j) * n + s] = bf16r(fmaxf(z1[j], 0.0f));
    // layer 2 re-reads h1 (this thread's own writes) instead of keeping z1 live
    float z2[kH2];
#pragma unroll
    for (int k = 0; k < kH2; ++k) z2[k] = v.b2[k];
#pragma unroll 1
    for (int j = 0; j < kH1; ++j) {
      const float h = a.H1[static_cast<int64_t>(j) * n + s];
      const float4* w = reinterpret_cast<const float4*>(w2t + j * kH2);
#pragma unroll
      for (int q = 0; q < kH2 / 4; ++q) {
        const float4 c = w[q];
        z2[4 * q] = fmaf(c.x, h, z2[4 * q]);
        z2[4 * q + 1] = fmaf(c.y, h, z2[4 * q + 1]);
        z2[4 * q + 2] = fmaf(c.z, h, z2[4 * q + 2]);
        z2[4 * q + 3] = fmaf(c.w, h, z2[4 * q + 3]);
      }
    }
    float z3 = v.b3[0];
#pragma unroll
    for (int k = 0; k < kH2; ++k) {
      const float h2 = fmaxf(z2[k], 0.0f);
      a.H2[static_cast<int64_t>(k) * n + s] = h2;
      z3 = fmaf(w3r[k], h2, z3);
    }
    const float y = labels[s], w = y > 0.5f ? pos_weight : 1.0f;
    const float sp = z3 > 0.0f ? z3 + log1pf(expf(-z3)) : log1pf(expf(z3));
    loss = w * (sp - y * z3);
    const float d3 = w * (1.0f / (1.0f + expf(-z3)) - y) / static_cast<float>(n);
    a.D3[s] = d3;
    float d2[kH2];
#pragma unroll
    for (int k = 0; k < kH2; ++k) {
      d2[k] = z2[k] > 0.0f ? d3 * w3r[k] : 0.0f;
      a.D2[static_cast<int64_t>(k) * n + s] = d2[k];
    }
    // delta1_j = [z1_j > 0] sum_k delta2_k W2_kj  (h1_j > 0 exactly when z1_j > 0)
#pragma unroll 1
    for (int j = 0; j < kH1; ++j) {
      const float4* w2 = reinterpret_cast<const float4*>(w2t + j * kH2);
      float acc = 0.0f;
#pragma unroll
      for (int q = 0; q < kH2 / 4; ++q) {
        const float4 c = w2[q];
        acc = fmaf(d2[4 * q], c.x, acc);
        acc = fmaf(d2[4 * q + 1], c.y, acc);
        acc = fmaf(d2[4 * q + 2], c.z, acc);
        acc = fmaf(d2[4 * q + 3], c.w, acc);
      }
      const float h = a.H1[static_cast<int64_t>(j) * n + s];
      a.D1[static_cast<int64_t>(j) * n + s] = h > 0.0f ? acc : 0.0f;
    }
  }
  // block partial of the loss (fixed order: deterministic)
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if ((threadIdx.x & 31) == 0) s_loss[threadIdx.x >> 5] = loss;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < kFwdThreads / 32; ++w) t += s_loss[w];
    a.loss_part[blockIdx.x] = t;
  }
}

// C[M][N] = A[M][K] B[N][K]^T (both K-contiguous, K = samples); 32 x 32 output
// tiles, 256 threads, 4 outputs each; fixed summation order.
__global__ void __launch_bounds__(256) rowdot_kernel(const float* __restrict__ A, const float* __restrict__ Bm, int M,
                                                     int N, int K, float* __restrict__ C, int ldc) {
  __shared__ float sa[32][33];
  __shared__ float sb[32][33];
  const int m0 = blockIdx.y * 32, n0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // ty 0..7: rows ty, ty+8, ty+16, ty+24
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int k0 = 0; k0 < K; k0 += 32) {
    for (int r = ty; r < 32; r += 8) {
      const int k = k0 + tx;
      sa[r][tx] = (m0 + r < M && k < K) ? A[static_cast<int64_t>(m0 + r) * K + k] : 0.0f;
      sb[r][tx] = (n0 + r < N && k < K) ? Bm[static_cast<int64_t>(n0 + r) * K + k] : 0.0f;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      const float bv = sb[tx][k];
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = fmaf(sa[ty + 8 * i][k], bv, acc[i]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 8 * i, nn = n0 + tx;
    if (m < M && nn < N) C[static_cast<int64_t>(m) * ldc + nn] = acc[i];
  }
}

// out[r] = sum_k A[r][k], one block per row.
__global__ void __launch_bounds__(256) rowsum_kernel(const float* __restrict__ A, int K, float* __restrict__ out) {
  __shared__ float s[8];
  const float* a = A + static_cast<int64_t>(blockIdx.x) * K;
  float t = 0.0f;
  for (int k = threadIdx.x; k < K; k += blockDim.x) t += a[k];
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    float r = 0.0f;
    for (int w = 0; w < 8; ++w) r += s[w];
    out[blockIdx.x] = r;
  }
}

__global__ void loss_kernel(const float* __restrict__ part, int nparts, int n, float* __restrict__ loss) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float t = 0.0f;
    for (int i = 0; i < nparts; ++i) t += part[i];
    *loss = t / static_cast<float>(n);
  }
}

__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

struct TrainWs {
  Acts acts;
  size_t bytes;
};

TrainWs carve_train(void* ws, int n) {
  TrainWs t;
  float* f = static_cast<float*>(ws);
  const int64_t nn = n;
  t.acts.H1 = f;
  t.acts.H2 = t.acts.H1 + kH1 * nn;
  t.acts.D1 = t.acts.H2 + kH2 * nn;
  t.acts.D2 = t.acts.D1 + kH1 * nn;
  t.acts.D3 = t.acts.D2 + kH2 * nn;
  t.acts.loss_part = t.acts.D3 + nn;
  const int64_t parts = (nn + kFwdThreads - 1) / kFwdThreads;
  t.bytes = sizeof(float) * static_cast<size_t>((2 * kH1 + 2 * kH2 + 1) * nn + parts) + 256;
  return t;
}

// ---- inference on the tensor cores -------------------------------------------
//
// Per 128-pixel tile:  layer 1 on the tensor cores straight from the fp16
// cube: two 64-pixel x Bp-band TMA boxes with the 128-byte swizzle are an
// MN-major A operand; B = W1' = bf16(W1) diag(s) in fp16 (exact: s is a
// power of two), b1' = b1 - W1' mean.  Layer 2: h1 = relu(.) rounded to
// bfloat16 into a K-major shared tile, times bf16(W2).  Layer 3 (32 -> 1) on
// the CUDA cores.  Output: one FP32 logit per pixel.
// Warps: 0 TMA, 1 MMA issuer (+ TMEM), 2-5 epilogue (one per TMEM lane
// quarter).  TMEM: layer-1 accumulators double-buffered at columns 0 / 64,
// layer 2 at 128.
constexpr int kScrTile = 128, kScrBox = 64;
constexpr int kScrThreads = 6 * 32;
constexpr uint32_t kScrTmemCols = 256;

struct ScreenOps {
  unsigned char w1[4][kH1 * 128];  // up to 4 K-blocks of 64 bands: 64 rows x 128 B, fp16, swizzled K-major
  unsigned char w2[kH2 * 128];     // 32 rows x 64 hidden bf16, swizzled K-major
  float b1[kH1];
  float b2[kH2];
  float w3[kH2];
  float b3;
};

__device__ __forceinline__ uint32_t sw128(int row, int byte) {
  return static_cast<uint32_t>((row >> 3) * 1024 + (row & 7) * 128 + ((((byte >> 4) ^ (row & 7))) << 4) + (byte & 15));
}

// One block: fold the normaliser into layer 1, round and lay out the weights.
__global__ void __launch_bounds__(256) pack_kernel(const float* __restrict__ params, int B,
                                                  const float* __restrict__ norm, ScreenOps* __restrict__ ops) {
  const int Bp = padded_bands(B);
  const ParamView v = view(const_cast<float*>(params), B);
  for (int e = threadIdx.x; e < kH1 * Bp; e += blockDim.x) {
    const int j = e / Bp, b = e % Bp;
    const float w = b < B ? bf16r(v.W1[e]) * norm[Bp + b] : 0.0f;
    const __half h = __float2half_rn(w);
    *reinterpret_cast<__half*>(&ops->w1[b >> 6][sw128(j, (b & 63) * 2)]) = h;
  }
  for (int e = threadIdx.x; e < kH2 * kH1; e += blockDim.x) {
    const int k = e / kH1, j = e % kH1;
    *reinterpret_cast<__nv_bfloat16*>(&ops->w2[sw128(k, j * 2)]) = __float2bfloat16_rn(v.W2[e]);
  }
  __syncthreads();
  // b1' = b1 - sum_b W1'_jb mean_b in FP64, from the fp16 weights actually used
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = warp; j < kH1; j += blockDim.x / 32) {
    double acc = 0.0;
    for (int b = lane; b < B; b += 32)
      acc += static_cast<double>(__half2float(*reinterpret_cast<const __half*>(&ops->w1[b >> 6][sw128(j, (b & 63) * 2)]))) *
             static_cast<double>(norm[b]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) ops->b1[j] = static_cast<float>(static_cast<double>(v.b1[j]) - acc);
  }
  for (int k = threadIdx.x; k < kH2; k += blockDim.x) {
    ops->b2[k] = v.b2[k];
    ops->w3[k] = bf16r(v.w3[k]);
  }
  if (threadIdx.x == 0) ops->b3 = v.b3[0];
}

struct ScreenArgs {
  int64_t pixels;
  int bands_padded;
  const ScreenOps* ops;
  float* logits;
  int* status;
};

__global__ void __launch_bounds__(kScrThreads, 1)
    screen_tc_kernel(const __grid_constant__ CUtensorMap cube_map, const ScreenArgs args) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int Bp = args.bands_padded;
  const int kb_count = Bp / 64;
  const uint32_t box_bytes = static_cast<uint32_t>(Bp) * 128;  // Bp bands x 64 px x 2 B
  const uint32_t stage_bytes = 2 * box_bytes;
  const int kIn = (128 * 1024) / stage_bytes < 4 ? (128 * 1024) / stage_bytes : 4;  // 2 or 4 stages
  unsigned char* in = smem;                                   // kIn stages
  unsigned char* w1 = in + kIn * stage_bytes;                  // kb_count x 8 KB
  unsigned char* w2 = w1 + kb_count * kH1 * 128;               // 4 KB
  unsigned char* h1 = w2 + kH2 * 128;                          // 2 x 16 KB (1024-aligned)
  float* cst = reinterpret_cast<float*>(h1 + 2 * kScrTile * 128);  // b1, b2, w3, b3
  uint64_t* bars = reinterpret_cast<uint64_t*>(cst + kH1 + 2 * kH2 + 4);
  uint64_t* in_full = bars;
  uint64_t* in_empty = bars + 4;
  uint64_t* acc1_full = bars + 8;
  uint64_t* acc1_empty = bars + 10;
  uint64_t* h1_full = bars + 12;
  uint64_t* h1_empty = bars + 14;
  uint64_t* acc2_full = bars + 16;
  uint64_t* acc2_empty = bars + 17;
  uint64_t* w_full = bars + 18;
  uint64_t* mma_done = bars + 19;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 20);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 21);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t P = args.pixels;
  const int64_t ntiles = div_up<int64_t>(P, kScrTile);
  const int n = ntiles > blockIdx.x ? static_cast<int>((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kIn; ++s) {
      mbar_init(&in_full[s], 1);
      mbar_init(&in_empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc1_full[b], 1);
      mbar_init(&acc1_empty[b], 4);
      mbar_init(&h1_full[b], 4);
      mbar_init(&h1_empty[b], 1);
    }
    mbar_init(acc2_full, 1);
    mbar_init(acc2_empty, 4);
    mbar_init(w_full, 1);
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  for (int i = threadIdx.x; i < kH1 + 2 * kH2 + 1; i += blockDim.x) cst[i] = args.ops->b1[i];
  if (warp == 1) tmem_alloc(tmem_slot, kScrTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      prefetch_tensormap(&cube_map);
      mbar_arrive_expect_tx(w_full, kb_count * kH1 * 128 + kH2 * 128);
      for (int kb = 0; kb < kb_count; ++kb) bulk_g2s(w1 + kb * kH1 * 128, args.ops->w1[kb], kH1 * 128, w_full);
      bulk_g2s(w2, args.ops->w2, kH2 * 128, w_full);
      uint32_t pending = 0, parity = 0;
      for (int i = 0; i < n; ++i) {
        const int s = i % kIn;
        const uint32_t ph = (i / kIn) & 1u;
        if (*abort_flag || !mbar_wait(&in_empty[s], ph ^ 1u)) {
          record_error(args.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        const int64_t tile = blockIdx.x + static_cast<int64_t>(i) * gridDim.x;
        mbar_arrive_expect_tx(&in_full[s], stage_bytes);
        for (int h = 0; h < 2; ++h)
          tma_load_2d(in + s * stage_bytes + h * box_bytes, &cube_map, static_cast<int>(tile * kScrTile + h * kScrBox),
                      0, &in_full[s]);
        pending |= 1u << s;
        parity = (parity & ~(1u << s)) | (ph << s);
      }
      for (int s = 0; s < kIn; ++s)
        if ((pending >> s) & 1u) mbar_wait(&in_full[s], (parity >> s) & 1u);
      mbar_wait(w_full, 0);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t id1 = idesc_f16_amn(kScrTile, kH1);
      const uint32_t id2 = idesc_bf16_f32(kScrTile, kH2);
      bool issued = false;
      if (n > 0 && !mbar_wait(w_full, 0)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
      }
      const uint64_t dw2 = smem_desc_sw128(w2);
      // layer 2 of tile j
      auto layer2 = [&](int j) -> bool {
        const int pb = j & 1;
        if (!mbar_wait(&h1_full[pb], (j >> 1) & 1u) || !mbar_wait(acc2_empty, (j & 1u) ^ 1u)) return false;
        tc_fence_after();
        const uint64_t dh = smem_desc_sw128(h1 + pb * kScrTile * 128);
#pragma unroll
        for (int ks = 0; ks < kH1 / 16; ++ks) umma_f16(tmem + 128, dh + 2 * ks, dw2 + 2 * ks, id2, ks > 0 ? 1u : 0u);
        umma_commit(&h1_empty[pb]);
        umma_commit(acc2_full);
        return true;
      };
      for (int i = 0; i < n && !*abort_flag; ++i) {
        const int s = i % kIn, pb = i & 1;
        if (!mbar_wait(&in_full[s], (i / kIn) & 1u) || !mbar_wait(&acc1_empty[pb], ((i >> 1) & 1u) ^ 1u)) {
          record_error(args.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        unsigned char* a = in + s * stage_bytes;
        for (int ks = 0; ks < Bp / 16; ++ks) {
          const uint64_t da = smem_desc_mn_sw128(a + ks * 2048, box_bytes);
          const uint64_t db = smem_desc_sw128(w1 + (ks >> 2) * kH1 * 128) + 2 * (ks & 3);
          umma_f16(tmem + pb * kH1, da, db, id1, ks > 0 ? 1u : 0u);
        }
        umma_commit(&in_empty[s]);
        umma_commit(&acc1_full[pb]);
        issued = true;
        if (i > 0 && !layer2(i - 1)) {
          record_error(args.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
      }
      if (n > 0 && !*abort_flag && !layer2(n - 1)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
      }
      if (issued) {
        umma_commit(mma_done);
        if (!mbar_wait(mma_done, 0)) record_error(args.status, HSI_E_TIMEOUT);
      }
    }
  } else {
    // epilogue: warp -> TMEM lane quarter q, thread -> pixel q*32 + lane
    const int q = warp & 3;
    const int px = q * 32 + lane;
    const uint32_t trow = tmem + (static_cast<uint32_t>(q * 32) << 16);
    const float* b1 = cst;
    const float* b2 = cst + kH1;
    const float* w3 = b2 + kH2;
    const float b3 = w3[kH2];
    for (int i = 0; i < n; ++i) {
      const int pb = i & 1;
      if (!mbar_wait(&acc1_full[pb], (i >> 1) & 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      uint32_t r0[32], r1[32];
      tmem_ld32(trow + pb * kH1, r0);
      tmem_ld32(trow + pb * kH1 + 32, r1);
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc1_empty[pb]);
      // h1 = relu(acc + b1') as bfloat16, one 128-byte row per pixel
      uint32_t packed[32];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float a0 = fmaxf(__uint_as_float(r0[2 * j]) + b1[2 * j], 0.0f);
        const float a1 = fmaxf(__uint_as_float(r0[2 * j + 1]) + b1[2 * j + 1], 0.0f);
        const __nv_bfloat162 v2 = __floats2bfloat162_rn(a0, a1);
        packed[j] = *reinterpret_cast<const uint32_t*>(&v2);
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float a0 = fmaxf(__uint_as_float(r1[2 * j]) + b1[32 + 2 * j], 0.0f);
        const float a1 = fmaxf(__uint_as_float(r1[2 * j + 1]) + b1[32 + 2 * j + 1], 0.0f);
        const __nv_bfloat162 v2 = __floats2bfloat162_rn(a0, a1);
        packed[16 + j] = *reinterpret_cast<const uint32_t*>(&v2);
      }
      if (!mbar_wait(&h1_empty[pb], ((i >> 1) & 1u) ^ 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      unsigned char* ht = h1 + pb * kScrTile * 128;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        *reinterpret_cast<uint4*>(ht + sw128(px, c * 16)) =
            make_uint4(packed[4 * c], packed[4 * c + 1], packed[4 * c + 2], packed[4 * c + 3]);
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&h1_full[pb]);
      if (!mbar_wait(acc2_full, i & 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      uint32_t r2[32];
      tmem_ld32(trow + 128, r2);
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc2_empty);
      float z = b3;
#pragma unroll
      for (int k = 0; k < kH2; ++k) z = fmaf(w3[k], fmaxf(__uint_as_float(r2[k]) + b2[k], 0.0f), z);
      const int64_t p = (blockIdx.x + static_cast<int64_t>(i) * gridDim.x) * kScrTile + px;
      if (p < P) args.logits[p] = z;
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, kScrTmemCols);
  }
}

size_t screen_smem_bytes(int Bp) {
  const size_t stage = 2 * static_cast<size_t>(Bp) * 128;
  const size_t k_in = (128 * 1024) / stage < 4 ? (128 * 1024) / stage : 4;
  return k_in * stage + static_cast<size_t>(Bp / 64) * kH1 * 128 + kH2 * 128 + 2 * kScrTile * 128 +
         sizeof(float) * (kH1 + 2 * kH2 + 4) + 22 * sizeof(uint64_t) + 1024;
}

// ---- gather candidate pixels into a compact BSQ cube --------------------------
template <typename T>
__global__ void pick_kernel(const T* __restrict__ cube, int64_t stride, int B, int width,
                            const hsi_detection* __restrict__ cand, const uint32_t* __restrict__ count, int capacity,
                            T* __restrict__ out, int64_t out_stride) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (i >= capacity || b >= B) return;
  const uint32_t nc = min(*count, static_cast<uint32_t>(capacity));
  T v;
  if (static_cast<uint32_t>(i) < nc) {
    const int64_t p = static_cast<int64_t>(cand[i].y) * width + cand[i].x;
    v = cube[static_cast<int64_t>(b) * stride + p];
  } else {
    v = cube[static_cast<int64_t>(b) * stride];  // padding: a real pixel, its scores are ignored
  }
  out[static_cast<int64_t>(b) * out_stride + i] = v;
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API int64_t hsi_screen_param_count(int bands) {
  if (bands <= 0 || bands > HSI_MAX_BANDS) return 0;
  return param_count(bands);
}

extern "C" HSI_API int hsi_screen_init(float* d_params, int bands, uint64_t seed, hsi_stream_t stream) {
  if (!d_params || bands <= 0 || bands > HSI_MAX_BANDS) return HSI_E_INVALID;
  init_kernel<<<64, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_params, bands, seed);
  return static_cast<int>(cudaGetLastError());
}

extern "C" HSI_API int hsi_screen_normaliser(const double* d_moments, int bands, float* d_norm, hsi_stream_t stream) {
  if (!d_moments || !d_norm || bands <= 0 || bands > HSI_MAX_BANDS) return HSI_E_INVALID;
  normaliser_kernel<<<1, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_moments, bands, d_norm);
  return static_cast<int>(cudaGetLastError());
}

extern "C" HSI_API int hsi_screen_batch(const hsi_detection* d_positives, const uint32_t* d_positive_count,
                                        int positive_capacity, int height, int width, const float* d_score,
                                        float threshold, uint64_t seed, int num_positive_draws, int n,
                                        int32_t* d_index, float* d_labels, hsi_stream_t stream) {
  if (!d_positives || !d_positive_count || positive_capacity <= 0 || height <= 0 || width <= 0 || !d_score ||
      n <= 0 || num_positive_draws < 0 || !d_index || !d_labels)
    return HSI_E_INVALID;
  const int64_t P = static_cast<int64_t>(height) * width;
  if (P > 0x7fffffff) return HSI_E_CAPACITY;
  batch_kernel<<<(n + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      d_positives, d_positive_count, positive_capacity, width, P, d_score, threshold, seed, num_positive_draws, n,
      d_index, d_labels);
  return static_cast<int>(cudaGetLastError());
}

extern "C" HSI_API int hsi_screen_gather(const void* d_cube, int dtype, int64_t plane_stride, int bands,
                                         const float* d_norm, const int32_t* d_index, int n, float* d_features,
                                         hsi_stream_t stream) {
  if (!d_cube || !d_norm || !d_index || !d_features || n <= 0 || bands <= 0 || bands > HSI_MAX_BANDS)
    return HSI_E_INVALID;
  const dim3 grid((n + 255) / 256, padded_bands(bands));
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (dtype == HSI_F32)
    gather_kernel<float><<<grid, 256, 0, s>>>(static_cast<const float*>(d_cube), plane_stride, bands, d_norm,
                                              d_index, n, d_features);
  else if (dtype == HSI_F16)
    gather_kernel<__half><<<grid, 256, 0, s>>>(static_cast<const __half*>(d_cube), plane_stride, bands, d_norm,
                                               d_index, n, d_features);
  else
    return HSI_E_INVALID;
  return static_cast<int>(cudaGetLastError());
}

extern "C" HSI_API size_t hsi_screen_train_workspace_bytes(int bands, int n) {
  if (bands <= 0 || n <= 0) return 0;
  return carve_train(nullptr, n).bytes;
}

extern "C" HSI_API int hsi_screen_gradients(const float* d_params, int bands, const float* d_features,
                                            const float* d_labels, int n, float pos_weight, float* d_grads,
                                            float* d_loss, void* d_workspace, size_t workspace_bytes,
                                            hsi_stream_t stream) {
  if (!d_params || !d_features || !d_labels || !d_grads || n <= 0 || bands <= 0 || bands > HSI_MAX_BANDS)
    return HSI_E_INVALID;
  const TrainWs t = carve_train(d_workspace, n);
  if (!d_workspace || workspace_bytes < t.bytes) return HSI_E_WORKSPACE;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int Bp = padded_bands(bands);
  const size_t smem = sizeof(float) * (static_cast<size_t>(Bp) * kH1 + kH1 * kH2 + kH2);
  // the largest band count's layout, set once per device
  const cudaError_t configured =
      raise_smem_limit(forward_kernel, static_cast<int>(sizeof(float) * (256 * kH1 + kH1 * kH2 + kH2)));
  if (configured != cudaSuccess) return static_cast<int>(configured);
  const int blocks = (n + kFwdThreads - 1) / kFwdThreads;
  forward_kernel<<<blocks, kFwdThreads, smem, s>>>(d_params, bands, d_features, d_labels, n, pos_weight, t.acts);
  const ParamView g = view(d_grads, bands);
  // dW1 = D1 X^T [64][Bp], dW2 = D2 H1^T [32][64], dw3 = D3 H2^T [1][32]
  rowdot_kernel<<<dim3((Bp + 31) / 32, 2), 256, 0, s>>>(t.acts.D1, d_features, kH1, Bp, n, g.W1, Bp);
  rowdot_kernel<<<dim3(2, 1), 256, 0, s>>>(t.acts.D2, t.acts.H1, kH2, kH1, n, g.W2, kH1);
  rowdot_kernel<<<dim3(1, 1), 256, 0, s>>>(t.acts.D3, t.acts.H2, 1, kH2, n, g.w3, kH2);
  rowsum_kernel<<<kH1, 256, 0, s>>>(t.acts.D1, n, g.b1);
  rowsum_kernel<<<kH2, 256, 0, s>>>(t.acts.D2, n, g.b2);
  rowsum_kernel<<<1, 256, 0, s>>>(t.acts.D3, n, g.b3);
  if (d_loss) loss_kernel<<<1, 32, 0, s>>>(t.acts.loss_part, blocks, n, d_loss);
  return static_cast<int>(cudaGetLastError());
}

extern "C" HSI_API int hsi_screen_adam(float* d_params, float* d_adam_state, const float* d_grads, int bands,
                                       float lr, int step, hsi_stream_t stream) {
  if (!d_params || !d_adam_state || !d_grads || bands <= 0 || bands > HSI_MAX_BANDS || step < 1) return HSI_E_INVALID;
  const int64_t n = param_count(bands);
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, static_cast<float>(step)), c2 = 1.0f - powf(b2, static_cast<float>(step));
  adam_kernel<<<64, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_params, d_adam_state, d_adam_state + n,
                                                                      d_grads, n, lr, b1, b2, 1e-8f, c1, c2);
  return static_cast<int>(cudaGetLastError());
}

extern "C" HSI_API size_t hsi_screen_infer_workspace_bytes(int bands) {
  if (bands <= 0 || bands > HSI_MAX_BANDS) return 0;
  return (sizeof(ScreenOps) + 255) & ~static_cast<size_t>(255);
}

namespace hsi_b200 {
namespace {

// Screen inference on at most max_ctas CTAs (0: one per SM).  The kernel's
// static tile schedule covers every tile for any grid size.
int screen_infer(const void* d_cube, int height, int width, int bands, int dtype, int64_t plane_stride,
                 const float* d_norm, const float* d_params, float* d_logits, void* d_workspace,
                 size_t workspace_bytes, int max_ctas, hsi_stream_t stream) {
  if (max_ctas < 0) return HSI_E_INVALID;
  if (!d_cube || !d_norm || !d_params || !d_logits || height <= 0 || width <= 0 || bands <= 0 ||
      bands > HSI_MAX_BANDS)
    return HSI_E_INVALID;
  if (dtype != HSI_F16) return HSI_E_INVALID;  // the first layer reads fp16 cubes as its MMA operand
  const int64_t P = static_cast<int64_t>(height) * width;
  if (plane_stride < P || (plane_stride & 7) != 0) return HSI_E_INVALID;  // 16-byte TMA strides
  if ((reinterpret_cast<uintptr_t>(d_cube) & 15u) != 0) return HSI_E_INVALID;
  if (!d_workspace || workspace_bytes < hsi_screen_infer_workspace_bytes(bands)) return HSI_E_WORKSPACE;
  if ((reinterpret_cast<uintptr_t>(d_workspace) & 255u) != 0) return HSI_E_INVALID;
  const int Bp = padded_bands(bands);
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  ScreenOps* ops = static_cast<ScreenOps*>(d_workspace);
  pack_kernel<<<1, 256, 0, s>>>(d_params, bands, d_norm, ops);
  CUtensorMap map;
  if (encode_cube_map_sw128(&map, d_cube, HSI_F16, P, bands, plane_stride, kScrBox, Bp) != 0) return HSI_E_INVALID;
  const size_t smem = screen_smem_bytes(Bp);
  const cudaError_t e = raise_smem_limit(screen_tc_kernel, static_cast<int>(smem));
  if (e != cudaSuccess) return static_cast<int>(e);
  const int sms = device_sm_count();
  const int cap = max_ctas > 0 && max_ctas < sms ? max_ctas : sms;
  const int64_t ntiles = (P + kScrTile - 1) / kScrTile;
  const int grid = static_cast<int>(ntiles < cap ? ntiles : cap);
  ScreenArgs a{P, Bp, ops, d_logits, nullptr};
  screen_tc_kernel<<<grid, kScrThreads, smem, s>>>(map, a);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace
}  // namespace hsi_b200

extern "C" HSI_API int hsi_screen_infer(const void* d_cube, int height, int width, int bands, int dtype,
                                        int64_t plane_stride, const float* d_norm, const float* d_params,
                                        float* d_logits, void* d_workspace, size_t workspace_bytes,
                                        hsi_stream_t stream) {
  return screen_infer(d_cube, height, width, bands, dtype, plane_stride, d_norm, d_params, d_logits, d_workspace,
                      workspace_bytes, 0, stream);
}

extern "C" HSI_API int hsi_screen_infer_ctas(const void* d_cube, int height, int width, int bands, int dtype,
                                             int64_t plane_stride, const float* d_norm, const float* d_params,
                                             float* d_logits, void* d_workspace, size_t workspace_bytes,
                                             int max_ctas, hsi_stream_t stream) {
  return screen_infer(d_cube, height, width, bands, dtype, plane_stride, d_norm, d_params, d_logits, d_workspace,
                      workspace_bytes, max_ctas, stream);
}

extern "C" HSI_API int hsi_gather_candidates(const void* d_cube, int dtype, int64_t plane_stride, int bands,
                                             int width, const hsi_detection* d_candidates,
                                             const uint32_t* d_count, int capacity, void* d_out,
                                             int64_t out_stride, hsi_stream_t stream) {
  if (!d_cube || !d_candidates || !d_count || !d_out || capacity <= 0 || bands <= 0 || bands > HSI_MAX_BANDS ||
      width <= 0 || out_stride < capacity)
    return HSI_E_INVALID;
  const dim3 grid((capacity + 255) / 256, bands);
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (dtype == HSI_F32)
    pick_kernel<float><<<grid, 256, 0, s>>>(static_cast<const float*>(d_cube), plane_stride, bands, width,
                                            d_candidates, d_count, capacity, static_cast<float*>(d_out), out_stride);
  else if (dtype == HSI_F16)
    pick_kernel<__half><<<grid, 256, 0, s>>>(static_cast<const __half*>(d_cube), plane_stride, bands, width,
                                             d_candidates, d_count, capacity, static_cast<__half*>(d_out),
                                             out_stride);
  else
    return HSI_E_INVALID;
  return static_cast<int>(cudaGetLastError());
}
