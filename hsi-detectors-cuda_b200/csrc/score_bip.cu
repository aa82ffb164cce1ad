// score_bip.cu - SAM scoring of a BIP (pixel-interleaved) cube in one pass.
//
// The reference scores BIP directly with a kernel of its own (src/sam.cu:
// 80-125, SamVariant::BipDirect) next to a standalone BIP -> BSQ transpose
// (src/sam.cu:281-309).  Here the transpose is fused into the scoring pass:
// the cube crosses HBM once, and no BSQ scratch copy exists.
//
// Each warp takes tiles of 32 pixels on its own, as a two-step software
// pipeline: while it scores one tile from shared memory, 16-byte cp.async
// copies bring the next.  A tile's 32 * B floats are contiguous in BIP and are
// scored where they land, with no transpose: lane p reads its own pixel's row,
// p * S floats into the tile, V bands at a time.  The row stride S and the read
// width V make those reads free of bank conflicts -- V = 1 for an odd band
// count (an odd stride spreads 32 lanes over 32 banks), V = 2 for B = 2 mod 4,
// V = 4 for B = 0 mod 4 -- and S = B except for B = 0 mod 8, where the copies
// re-stride each pixel's row to S = B + 4 (S / 4 odd).
// Lane p scores pixel p: its squared norm and its dot product with every
// target, in band order with one fmaf per band and target -- the same
// operations in the same order as the BSQ scorer (score.cu), so the angles,
// best angles and best targets are bit-identical to scoring the transposed
// cube.  All targets are scored from shared memory in one pass over HBM
// (groups of 8 or 16, two targets per packed FMA, the bank zero-padded to the
// group).  A block holds as many warps as shared memory allows, up to 8, and
// one copy of the target bank.
#include "common.cuh"
#include "launch_state.h"
#include "sam_math.cuh"

namespace hsi_b200 {
namespace {

constexpr int kPx = 32;          // pixels per warp tile
constexpr int kMaxWarps = 8;     // warps per block
constexpr int kMaxTargets = 64;
constexpr size_t kSmemCap = 227 * 1024;

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
  bool aligned;        // cube base on 16 bytes: cp.async copies
};

// Row stride (floats) of a pixel in a shared tile and the width of a lane's reads.
__host__ __device__ inline int row_stride(int bands) { return (bands & 7) == 0 ? bands + 4 : bands; }
__host__ __device__ inline int read_width(int bands) { return (bands & 3) == 0 ? 4 : (bands & 1) == 0 ? 2 : 1; }
// floats of one tile buffer, rounded up to 4 so that every buffer starts on 16 bytes
__host__ __device__ inline int tile_floats(int bands) { return (kPx * row_stride(bands) + 3) & ~3; }
__host__ __device__ inline int group_of(int targets) { return targets <= 8 ? 8 : 16; }
__host__ __device__ inline int padded_targets(int targets) {
  const int g = group_of(targets);
  return (targets + g - 1) / g * g;
}
// bytes of the bank [b][padded targets], the target scales and `warps` double-buffered tiles
__host__ __device__ inline size_t bip_fixed_bytes(int bands, int targets) {
  return sizeof(float) * (static_cast<size_t>(bands) * padded_targets(targets) + kMaxTargets);
}
__host__ __device__ inline size_t bip_warp_bytes(int bands) { return sizeof(float) * 2 * tile_floats(bands); }

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Start copying npx pixels' rows (B floats each, contiguous at src) into dst
// at row stride S: 16-byte cp.async copies when the cube is 16-byte aligned
// (every tile start then is: 32 * B floats apart), plain loads otherwise and
// for the tail of a ragged last tile.
__device__ __forceinline__ void load_tile(float* dst, const float* src, int npx, int B, int S, int lane,
                                          bool aligned) {
  const int n = npx * B;
  if (S == B) {
    const int n4 = aligned ? n / 4 : 0;
    for (int i = lane; i < n4; i += 32) cp_async16(dst + 4 * i, src + 4 * i);
    cp_async_commit();
    for (int e = 4 * n4 + lane; e < n; e += 32) dst[e] = __ldg(src + e);
  } else if (aligned) {  // B = 0 mod 8: whole 16-byte chunks, re-strided per pixel
    const int q = B / 4;
    for (int i = lane; i < npx * q; i += 32) {
      const int p = i / q;
      cp_async16(dst + p * S + 4 * (i - p * q), src + 4 * i);
    }
    cp_async_commit();
  } else {
    for (int e = lane; e < n; e += 32) {
      const int p = e / B;
      dst[p * S + (e - p * B)] = __ldg(src + e);
    }
  }
}

// acc[k] += x * bank[b][t0 + 2k, t0 + 2k + 1] over the pixel's bands in
// order (and nrm += x * x with kNorm); xr is the lane's row, tgc = bank + t0.
template <int G, int V, bool kNorm>
__device__ __forceinline__ void band_loop(const float* xr, const float* tgc, int TP, int B, float2 (&acc)[G / 2],
                                          float& nrm) {
#pragma unroll 2
  for (int b = 0; b < B; b += V) {
    float x[V];
    if constexpr (V == 4) {
      const float4 v = *reinterpret_cast<const float4*>(xr + b);
      x[0] = v.x, x[1] = v.y, x[2] = v.z, x[3] = v.w;
    } else if constexpr (V == 2) {
      const float2 v = *reinterpret_cast<const float2*>(xr + b);
      x[0] = v.x, x[1] = v.y;
    } else {
      x[0] = xr[b];
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if constexpr (kNorm) nrm = fmaf(x[v], x[v], nrm);
      const float2 d = make_float2(x[v], x[v]);
      const float4* tr = reinterpret_cast<const float4*>(tgc + (b + v) * TP);
#pragma unroll
      for (int k = 0; k < G / 4; ++k) {
        const float4 w = tr[k];
        acc[2 * k] = ffma2(d, make_float2(w.x, w.y), acc[2 * k]);
        acc[2 * k + 1] = ffma2(d, make_float2(w.z, w.w), acc[2 * k + 1]);
      }
    }
  }
}

template <int G, int V>
__global__ void __launch_bounds__(kMaxWarps * 32) sam_bip_kernel(const BipArgs a) {
  extern __shared__ __align__(16) float sm[];
  const int B = a.bands, T = a.targets, TP = (T + G - 1) / G * G, S = row_stride(B);
  float* tg = sm;                  // [b][TP], zero beyond T
  float* scale = tg + B * TP;      // [t] = 1 / |r_t| (0 for a zero target)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  const int tf = tile_floats(B);
  float* buf = scale + kMaxTargets + static_cast<size_t>(warp) * 2 * tf;  // two tiles [p][S]
  for (int i = threadIdx.x; i < B * TP; i += blockDim.x) {
    const int b = i / TP, t = i - b * TP;
    tg[i] = t < T ? a.lib[static_cast<int64_t>(t) * B + b] : 0.0f;
  }
  for (int t = threadIdx.x; t < T; t += blockDim.x) scale[t] = a.norms[t] > 0.0f ? 1.0f / a.norms[t] : 0.0f;
  __syncthreads();

  const int64_t ntiles = div_up<int64_t>(a.pixels, kPx);
  const int64_t step = static_cast<int64_t>(gridDim.x) * warps;
  int64_t tile = static_cast<int64_t>(blockIdx.x) * warps + warp;
  auto npx_of = [&](int64_t t) {
    const int64_t left = a.pixels - t * kPx;
    return static_cast<int>(left < kPx ? left : kPx);
  };
  if (tile < ntiles) load_tile(buf, a.cube + tile * kPx * B, npx_of(tile), B, S, lane, a.aligned);
  for (int it = 0; tile < ntiles; tile += step, ++it) {
    const float* cur = buf + (it & 1) * tf;
    const int npx = npx_of(tile);
    cp_async_wait_all();
    __syncwarp();
    // the next tile's copies run while this one is scored
    const int64_t next = tile + step;
    if (next < ntiles) load_tile(buf + ((it + 1) & 1) * tf, a.cube + next * kPx * B, npx_of(next), B, S, lane,
                                 a.aligned);
    if (lane < npx) {
      const int64_t px = tile * kPx + lane;
      const float* xr = cur + lane * S;
      float nrm = 0.0f, rn = 0.0f, best = -2.0f;
      int32_t best_t = -1;
      for (int t0 = 0; t0 < T; t0 += G) {
        const int nt = T - t0 < G ? T - t0 : G;
        float2 acc[G / 2];
#pragma unroll
        for (int k = 0; k < G / 2; ++k) acc[k] = make_float2(0.0f, 0.0f);
        if (t0 == 0) {
          band_loop<G, V, true>(xr, tg, TP, B, acc, nrm);
          rn = nrm > 0.0f ? rsqrtf(nrm) : 0.0f;
        } else {
          band_loop<G, V, false>(xr, tg + t0, TP, B, acc, nrm);
        }
#pragma unroll
        for (int k = 0; k < G; k += 2) {
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
    __syncwarp();  // every lane is done with cur before the next round's copies refill it
  }
  cp_async_wait_all();  // never leave copies in flight into shared memory
}

template <int G, int V>
int launch_bip(const BipArgs& a, cudaStream_t stream) {
  const size_t fixed = bip_fixed_bytes(a.bands, a.targets), per_warp = bip_warp_bytes(a.bands);
  if (fixed + per_warp > kSmemCap) return HSI_E_CAPACITY;
  const int64_t ntiles = div_up<int64_t>(a.pixels, kPx);
  int warps = static_cast<int>((kSmemCap - fixed) / per_warp);
  if (warps > kMaxWarps) warps = kMaxWarps;
  if (warps > ntiles) warps = static_cast<int>(ntiles);
  const size_t smem = fixed + static_cast<size_t>(warps) * per_warp;
  const cudaError_t e = raise_smem_limit(sam_bip_kernel<G, V>, static_cast<int>(smem));
  if (e != cudaSuccess) return static_cast<int>(e);
  const int per_sm = device_residency(sam_bip_kernel<G, V>, warps * 32, smem);
  const int64_t blocks_needed = div_up<int64_t>(ntiles, warps);
  const int64_t wave = static_cast<int64_t>(device_sm_count()) * (per_sm > 0 ? per_sm : 1);
  const int grid = static_cast<int>(blocks_needed < wave ? blocks_needed : wave);
  sam_bip_kernel<G, V><<<grid, warps * 32, smem, stream>>>(a);
  return static_cast<int>(cudaGetLastError());
}

template <int G>
int launch_bip_v(const BipArgs& a, cudaStream_t stream) {
  switch (read_width(a.bands)) {
    case 4: return launch_bip<G, 4>(a, stream);
    case 2: return launch_bip<G, 2>(a, stream);
    default: return launch_bip<G, 1>(a, stream);
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
  const bool aligned = (reinterpret_cast<uintptr_t>(d_cube) & 15u) == 0;
  BipArgs a{d_cube, P, bands, num_targets, d_targets, d_target_norms, d_maps, map_stride, d_best, d_best_target,
            aligned};
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return group_of(num_targets) == 8 ? launch_bip_v<8>(a, s) : launch_bip_v<16>(a, s);
}
