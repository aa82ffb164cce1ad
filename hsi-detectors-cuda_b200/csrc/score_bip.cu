// score_bip.cu - SAM scoring of a BIP (pixel-interleaved) cube in one pass.
//
// The reference scores BIP directly with a kernel of its own (src/sam.cu:
// 80-125, SamVariant::BipDirect) next to a standalone BIP -> BSQ transpose
// (src/sam.cu:281-309).  Here the transpose is fused into the scoring pass:
// the cube crosses HBM once, and no BSQ scratch copy exists.
//
// Each warp takes tiles of 32 pixels.  A tile's 32 * B floats are contiguous
// in BIP, so the warp reads them with coalesced 16-byte loads and scatters
// them into a per-warp shared-memory buffer laid out band-major with a row
// stride of 33 floats (bank-conflict free both ways).  Then lane p scores
// pixel p: its squared norm and its dot product with every target, in band
// order with one fmaf per band -- the same operations in the same order as
// the BSQ scorer (score.cu), so the angles, best angles and best targets are
// bit-identical to scoring the transposed cube.  All targets are scored from
// shared memory in one pass over HBM (groups of 16 accumulators).
#include "common.cuh"
#include "launch_state.h"
#include "sam_math.cuh"

namespace hsi_b200 {
namespace {

constexpr int kWarps = 4;              // warps per block
constexpr int kPx = 32;                // pixels per warp tile
constexpr int kStride = kPx + 1;       // floats between band rows of the tile buffer
constexpr int kGroup = 16;             // targets per accumulator group
constexpr int kMaxTargets = 64;

struct BipArgs {
  const float* cube;
  int64_t pixels;
  int bands, targets;
  const float* lib;    // target-major targets x bands
  const float* norms;  // targets
  float* maps;         // nullable: target-major at map_stride
  int64_t map_stride;
  float* best;         // nullable
  int32_t* best_t;     // nullable
};

__host__ __device__ inline size_t bip_smem_bytes(int bands, int targets) {
  return sizeof(float) * (static_cast<size_t>(bands) * targets + kMaxTargets +
                          static_cast<size_t>(kWarps) * bands * kStride);
}

__global__ void __launch_bounds__(kWarps * 32) sam_bip_kernel(const BipArgs a) {
  extern __shared__ float sm[];
  const int B = a.bands, T = a.targets;
  float* tg = sm;                 // [b][t]
  float* scale = tg + B * T;      // [t] = 1 / |r_t| (0 for a zero target)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* buf = scale + kMaxTargets + static_cast<size_t>(warp) * B * kStride;
  for (int i = threadIdx.x; i < B * T; i += blockDim.x) {
    const int b = i / T, t = i % T;
    tg[i] = a.lib[static_cast<int64_t>(t) * B + b];
  }
  for (int t = threadIdx.x; t < T; t += blockDim.x) scale[t] = a.norms[t] > 0.0f ? 1.0f / a.norms[t] : 0.0f;
  __syncthreads();

  const int64_t ntiles = div_up<int64_t>(a.pixels, kPx);
  // 128 floats (32 lanes x one float4) advance a lane by this many pixels and bands
  const int step_p = 128 / B, step_b = 128 % B;
  for (int64_t tile = static_cast<int64_t>(blockIdx.x) * kWarps + warp; tile < ntiles;
       tile += static_cast<int64_t>(gridDim.x) * kWarps) {
    const int64_t p0 = tile * kPx;
    const int npx = static_cast<int>(a.pixels - p0 < kPx ? a.pixels - p0 : kPx);
    const float* src = a.cube + p0 * B;
    const int n = npx * B;
    // ---- load and transpose: element e = p B + b goes to buf[b * kStride + p]
    if (npx == kPx && B >= 4 && (reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
      const float4* s4 = reinterpret_cast<const float4*>(src);
      int e = 4 * lane;
      int p = e / B, b = e - p * B;
#pragma unroll 4
      for (int i = lane; i < n / 4; i += 32) {
        const float4 v = __ldg(s4 + i);
        const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          int bb = b + k, pp = p;
          if (bb >= B) {
            bb -= B;
            ++pp;
          }
          buf[bb * kStride + pp] = vv[k];
        }
        b += step_b;
        p += step_p;
        if (b >= B) {
          b -= B;
          ++p;
        }
      }
    } else {
      for (int e = lane; e < n; e += 32) {
        const int p = e / B, b = e - p * B;
        buf[b * kStride + p] = __ldg(src + e);
      }
    }
    __syncwarp();
    // ---- score: lane = pixel
    if (lane < npx) {
      const int64_t px = p0 + lane;
      float nrm = 0.0f;
      for (int b = 0; b < B; ++b) {
        const float x = buf[b * kStride + lane];
        nrm = fmaf(x, x, nrm);
      }
      const float rn = nrm > 0.0f ? rsqrtf(nrm) : 0.0f;
      float best = -2.0f;
      int32_t best_t = -1;
      for (int t0 = 0; t0 < T; t0 += kGroup) {
        const int nt = T - t0 < kGroup ? T - t0 : kGroup;
        float acc[kGroup];
#pragma unroll
        for (int k = 0; k < kGroup; ++k) acc[k] = 0.0f;
        for (int b = 0; b < B; ++b) {
          const float x = buf[b * kStride + lane];
          const float* tr = tg + b * T + t0;
#pragma unroll
          for (int k = 0; k < kGroup; ++k)
            if (k < nt) acc[k] = fmaf(x, tr[k], acc[k]);
        }
#pragma unroll
        for (int k = 0; k < kGroup; k += 2) {
          if (k >= nt) break;
          const float c0 = acc[k] * rn * scale[t0 + k];
          const float c1 = k + 1 < nt ? acc[k + 1] * rn * scale[t0 + k + 1] : -2.0f;
          if (c0 > best) {
            best = c0;
            best_t = t0 + k;
          }
          if (k + 1 < nt && c1 > best) {
            best = c1;
            best_t = t0 + k + 1;
          }
          if (a.maps) {
            const float2 ang = angle_of_cos2(make_float2(c0, c1));
            a.maps[static_cast<int64_t>(t0 + k) * a.map_stride + px] = ang.x;
            if (k + 1 < nt) a.maps[static_cast<int64_t>(t0 + k + 1) * a.map_stride + px] = ang.y;
          }
        }
      }
      if (a.best) a.best[px] = angle_of_cos(best);
      if (a.best_t) a.best_t[px] = best_t;
    }
    __syncwarp();
  }
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API int hsi_sam_bip(const float* d_cube, int height, int width, int bands, const float* d_targets,
                                   const float* d_target_norms, int num_targets, float* d_maps, int64_t map_stride,
                                   float* d_best, int32_t* d_best_target, hsi_stream_t stream) {
  const int64_t P = static_cast<int64_t>(height) * width;
  if (!d_cube || height <= 0 || width <= 0 || bands <= 0 || bands > HSI_MAX_BANDS || !d_targets ||
      !d_target_norms || num_targets <= 0 || num_targets > kMaxTargets)
    return HSI_E_INVALID;
  if (!d_maps && !d_best && !d_best_target) return HSI_E_INVALID;
  if (d_maps && map_stride < P) return HSI_E_INVALID;
  if ((reinterpret_cast<uintptr_t>(d_cube) & 3u) != 0) return HSI_E_INVALID;
  BipArgs a{d_cube, P, bands, num_targets, d_targets, d_target_norms, d_maps, map_stride, d_best, d_best_target};
  const size_t smem = bip_smem_bytes(bands, num_targets);
  if (smem > 227 * 1024) return HSI_E_CAPACITY;
  const cudaError_t e = raise_smem_limit(sam_bip_kernel, static_cast<int>(smem));
  if (e != cudaSuccess) return static_cast<int>(e);
  const int per_sm = device_residency(sam_bip_kernel, kWarps * 32, smem);
  const int64_t ntiles = div_up<int64_t>(P, kPx);
  const int64_t blocks_needed = div_up<int64_t>(ntiles, kWarps);
  const int64_t wave = static_cast<int64_t>(device_sm_count()) * (per_sm > 0 ? per_sm : 1);
  const int grid = static_cast<int>(blocks_needed < wave ? blocks_needed : wave);
  sam_bip_kernel<<<grid, kWarps * 32, smem, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  return static_cast<int>(cudaGetLastError());
}
