// score_bip.cu - SAM scoring of a BIP (pixel-interleaved) cube in one pass.
//
// The reference scores BIP directly with a kernel of its own (src/sam.cu:
// 80-125, SamVariant::BipDirect) next to a standalone BIP -> BSQ transpose
// (src/sam.cu:281-309).  Here the transpose is fused into the scoring pass:
// the cube crosses HBM once, and no BSQ scratch copy exists.
//
// Each warp takes tiles of 32 pixels on its own, as a two-step software
// pipeline.  A tile's 32 * B floats are contiguous in BIP: the warp copies
// them into a raw shared-memory buffer with 16-byte cp.async copies, then
// transposes them into a band-major buffer in which pixel p of band b sits in
// column p ^ (b / 4) mod 32 (both the transposing stores and the per-band
// reads are free of bank conflicts), then starts the next tile's copies into
// the raw buffer and scores this tile from the band-major one meanwhile.
// Lane p scores pixel p: its squared norm and its dot product with every
// target, in band order with one fmaf per band and target -- the same
// operations in the same order as the BSQ scorer (score.cu), so the angles,
// best angles and best targets are bit-identical to scoring the transposed
// cube.  All targets are scored from shared memory in one pass over HBM
// (groups of 16, two targets per packed FMA).
#include "common.cuh"
#include "launch_state.h"
#include "sam_math.cuh"

namespace hsi_b200 {
namespace {

constexpr int kWarps = 1;              // warps per block: each warp runs its own pipeline
constexpr int kPx = 32;                // pixels per warp tile
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

// floats of one warp's tile buffer: 32 pixels x bands, rounded up to 4
__host__ __device__ inline int tile_floats(int bands) { return (kPx * bands + 3) & ~3; }

// floats of the target bank, rounded up to 4 so that the tile buffers after
// it start on 16 bytes
__host__ __device__ inline int bank_floats(int bands, int targets) { return (bands * targets + 3) & ~3; }

__host__ __device__ inline size_t bip_smem_bytes(int bands, int targets) {
  return sizeof(float) * (static_cast<size_t>(bank_floats(bands, targets)) + kMaxTargets +
                          static_cast<size_t>(kWarps) * 2 * tile_floats(bands));
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Column of pixel p in band row b of the band-major buffer.
__device__ __forceinline__ int tcol(int b, int p) { return p ^ ((b >> 2) & 31); }

// Start copying the tile at p0 (npx pixels) into raw: 16-byte cp.async copies
// when the tile's start is 16-byte aligned, plain loads for the rest; the
// buffer is zero-filled to a multiple of four floats.
__device__ __forceinline__ void load_tile(float* raw, const float* src, int n, int lane, bool aligned) {
  const int n4 = aligned ? n / 4 : 0;
  for (int i = lane; i < n4; i += 32) cp_async16(raw + 4 * i, src + 4 * i);
  cp_async_commit();
  for (int e = 4 * n4 + lane; e < ((n + 3) & ~3); e += 32) raw[e] = e < n ? __ldg(src + e) : 0.0f;
}

__global__ void __launch_bounds__(kWarps * 32) sam_bip_kernel(const BipArgs a) {
  extern __shared__ __align__(16) float sm[];
  const int B = a.bands, T = a.targets;
  float* tg = sm;                              // [b][t]
  float* scale = tg + bank_floats(B, T);       // [t] = 1 / |r_t| (0 for a zero target)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tf = tile_floats(B);
  float* raw = scale + kMaxTargets + static_cast<size_t>(warp) * 2 * tf;  // [p][b] as copied, 16-byte aligned
  float* tb = raw + tf;                                                     // [b][tcol(b, p)]
  for (int i = threadIdx.x; i < B * T; i += blockDim.x) {
    const int b = i / T, t = i % T;
    tg[i] = a.lib[static_cast<int64_t>(t) * B + b];
  }
  for (int t = threadIdx.x; t < T; t += blockDim.x) scale[t] = a.norms[t] > 0.0f ? 1.0f / a.norms[t] : 0.0f;
  __syncthreads();

  const int64_t ntiles = div_up<int64_t>(a.pixels, kPx);
  const int64_t step = static_cast<int64_t>(gridDim.x) * kWarps;
  const bool base_aligned = (reinterpret_cast<uintptr_t>(a.cube) & 15u) == 0;
  // a float4 of the raw tile advances a lane's (pixel, band) by 128 floats per round
  const int step_p = 128 / B, step_b = 128 % B;
  int64_t tile = static_cast<int64_t>(blockIdx.x) * kWarps + warp;
  if (tile < ntiles) {
    const int64_t p0 = tile * kPx;
    const int npx = static_cast<int>(a.pixels - p0 < kPx ? a.pixels - p0 : kPx);
    load_tile(raw, a.cube + p0 * B, npx * B, lane, base_aligned);
  }
  for (; tile < ntiles; tile += step) {
    const int64_t p0 = tile * kPx;
    const int npx = static_cast<int>(a.pixels - p0 < kPx ? a.pixels - p0 : kPx);
    const int n = npx * B;
    cp_async_wait_all();
    __syncwarp();
    // ---- transpose raw [p][b] -> tb [b][tcol(b, p)], one float4 of raw per lane and round
    {
      int e = 4 * lane;
      int p = e / B, b = e - p * B;
      for (int i = lane; 4 * i < n; i += 32) {
        const float4 v = *reinterpret_cast<const float4*>(raw + 4 * i);
        const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          int bb = b + k, pp = p;
          while (bb >= B) {
            bb -= B;
            ++pp;
          }
          if (pp < npx) tb[bb * kPx + tcol(bb, pp)] = vv[k];
        }
        b += step_b;
        p += step_p;
        while (b >= B) {
          b -= B;
          ++p;
        }
      }
    }
    __syncwarp();
    // ---- the next tile's copies run while this one is scored
    const int64_t next = tile + step;
    if (next < ntiles) {
      const int64_t q0 = next * kPx;
      const int nq = static_cast<int>(a.pixels - q0 < kPx ? a.pixels - q0 : kPx);
      load_tile(raw, a.cube + q0 * B, nq * B, lane, base_aligned);
    }
    // ---- score: lane = pixel
    if (lane < npx) {
      const int64_t px = p0 + lane;
      float nrm = 0.0f;
      for (int b = 0; b < B; ++b) {
        const float x = tb[b * kPx + tcol(b, lane)];
        nrm = fmaf(x, x, nrm);
      }
      const float rn = nrm > 0.0f ? rsqrtf(nrm) : 0.0f;
      float best = -2.0f;
      int32_t best_t = -1;
      for (int t0 = 0; t0 < T; t0 += kGroup) {
        const int nt = T - t0 < kGroup ? T - t0 : kGroup;
        float2 acc[kGroup / 2];
#pragma unroll
        for (int k = 0; k < kGroup / 2; ++k) acc[k] = make_float2(0.0f, 0.0f);
        if (nt == kGroup && (T & 1) == 0) {
          for (int b = 0; b < B; ++b) {
            const float x = tb[b * kPx + tcol(b, lane)];
            const float2 d = make_float2(x, x);
            const float2* tr = reinterpret_cast<const float2*>(tg + b * T + t0);
#pragma unroll
            for (int k = 0; k < kGroup / 2; ++k) acc[k] = ffma2(d, tr[k], acc[k]);
          }
        } else {
          for (int b = 0; b < B; ++b) {
            const float x = tb[b * kPx + tcol(b, lane)];
            const float* tr = tg + b * T + t0;
#pragma unroll
            for (int k = 0; k < kGroup; ++k)
              if (k < nt) {
                if (k & 1)
                  acc[k / 2].y = fmaf(x, tr[k], acc[k / 2].y);
                else
                  acc[k / 2].x = fmaf(x, tr[k], acc[k / 2].x);
              }
          }
        }
#pragma unroll
        for (int k = 0; k < kGroup; k += 2) {
          if (k >= nt) break;
          const float c0 = acc[k / 2].x * rn * scale[t0 + k];
          const float c1 = k + 1 < nt ? acc[k / 2].y * rn * scale[t0 + k + 1] : -2.0f;
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
  cp_async_wait_all();  // never leave copies in flight into shared memory
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
