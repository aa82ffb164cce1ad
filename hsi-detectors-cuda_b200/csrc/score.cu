// score.cu - SAM / CEM filter-bank scoring: one streaming pass over a BSQ cube.
//
// Design (sm_100a):
//  * Persistent CTAs walk a static schedule of 512-pixel tiles over every
//    frame of the launch (one frame, or a batch described by a device table).
//  * One producer warp streams each tile's band planes into a ring of shared
//    memory stages with 1-D bulk copies on the TMA engine (16 FP32 or 8 FP16
//    bands x 512 px per stage), completing on mbarriers.  Nothing but the copy engine touches
//    the cube in HBM, and every HBM byte is read exactly once.
//  * Up to two consumer warpgroups read each stage from shared memory: one
//    scores the SAM library, one the CEM filters, 4 pixels per thread, with
//    the bank of the current frame held band-major in shared memory so each
//    band step is one 128-bit broadcast load per 4 filters.
//  * The epilogue turns dot products into angles (SAM) or responses (CEM),
//    writes per-target maps with 128-bit stores, and reduces the best target.
//
// Semantics follow the reference scorer: src/sam.cu:126-202 (opt kernel: rank
// on cosine, one acos, strict '>' so the lowest target wins ties, zero-norm
// pixel -> pi/2, multi-pass carry of the best cosine) and the CPU CEM
// reduction src/detectors_cpu.cpp:158-187.
#include <cuda_fp16.h>


#include "launch_state.h"
#include "sam_math.cuh"
#include "tc.cuh"

namespace hsi_b200 {
namespace {

constexpr int kGroupThreads = 128;  // one consumer warpgroup
constexpr int kPPT = 4;             // pixels per consumer thread
constexpr int kTile = kGroupThreads * kPPT;
// Both banks in one consumer group: two warpgroups, two pixels per thread
// (twice the warps of one warpgroup at four pixels, for the same tile).
constexpr int kFusedThreads = 256;
constexpr int kFusedPPT = kTile / kFusedThreads;
constexpr int kMaxTableFrames = 256;
constexpr int kFiltersPerPass = HSI_MAX_FILTERS_PER_PASS;
constexpr int kMaxInline = 64;  // frames whose descriptors travel inside one launch

template <typename T>
struct CubeTraits;
// Stage ring: with two consumer warpgroups two CTAs fit per SM, and ~190 KB
// of each SM's reads stay in flight.  With both banks in one warpgroup three
// CTAs fit (the warps hide the packed FMAs' latency better), with 64 KB of
// stages each for FP32.  FP32 stages hold 16 band planes of a tile: measured
// on 16 resident 1024^2 x 113 frames, 16 bands x 2 stages scored a frame in
// 114.6 us, 8 x 4 in 119.8, 8 x 5 (two CTAs) in 126.6, 12 x 3 in 121.7 and
// 16 x 3 in 120.4 -- fewer, larger stages halve the barrier round trips per
// band.
template <>
struct CubeTraits<float> {
  static constexpr int kStageBands = 16;  // band planes of a tile per stage
  static constexpr int kStages = 3;
  static constexpr int kStagesFused = 2;
};
template <>
struct CubeTraits<__half> {
  static constexpr int kStageBands = 8;
  static constexpr int kStages = 10;
  static constexpr int kStagesFused = 7;
};

struct ScoreParams {
  const hsi_frame* table;  // device descriptor table, or null for inline frames
  hsi_frame inline_frames[kMaxInline];
  int num_frames;
  int pass;     // filters [16*pass, 16*pass + 16) of each kind
  int dtype;    // element type every frame of the launch must have
  int max_sam;  // bounds every frame of the launch must respect
  int max_cem;
  int* status;  // nullable device error word
};

__device__ __forceinline__ const hsi_frame& frame_at(const ScoreParams& p, int f) {
  return p.table ? p.table[f] : p.inline_frames[f];
}

// Filters of one kind that this pass scores for a frame.
__device__ __forceinline__ int pass_count(int total, int pass) {
  const int n = total - pass * kFiltersPerPass;
  return n < 0 ? 0 : (n > kFiltersPerPass ? kFiltersPerPass : n);
}

template <typename T>
__device__ __forceinline__ void load4(const T* p, float v[4]);
template <>
__device__ __forceinline__ void load4<float>(const float* p, float v[4]) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  v[3] = a.w;
}
template <>
__device__ __forceinline__ void load4<__half>(const __half* p, float v[4]) {
  const uint2 raw = *reinterpret_cast<const uint2*>(p);
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}

template <typename T>
__device__ __forceinline__ float2 load2(const T* p);
template <>
__device__ __forceinline__ float2 load2<float>(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}
template <>
__device__ __forceinline__ float2 load2<__half>(const __half* p) {
  return __half22float2(*reinterpret_cast<const __half2*>(p));
}

__device__ __forceinline__ void named_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Frame of a tile: the last f with prefix[f] <= tile (frames without tiles
// are passed over).  A CTA walks its tiles in increasing order, so the search
// starts at the frame of its previous tile and only moves forward.
__device__ __forceinline__ int next_frame(const int* prefix, int n, int tile, int f) {
  while (f + 1 < n && prefix[f + 1] <= tile) ++f;
  return f;
}

struct SmemLayout {
  size_t stage_bytes, filt_off, scale_off, bar_off, prefix_off, total;
};

template <typename T>
__host__ __device__ inline SmemLayout smem_layout(int groups, int max_bands, int slots, int stages) {
  SmemLayout l;
  l.stage_bytes = static_cast<size_t>(CubeTraits<T>::kStageBands) * kTile * sizeof(T);
  size_t off = l.stage_bytes * stages;
  l.filt_off = off;
  off += static_cast<size_t>(groups) * max_bands * slots * sizeof(float);
  l.scale_off = off;
  off += static_cast<size_t>(groups) * kFiltersPerPass * sizeof(float);
  off = (off + 15) & ~static_cast<size_t>(15);
  l.bar_off = off;
  off += 2 * static_cast<size_t>(stages) * sizeof(uint64_t);
  l.prefix_off = off;
  off += (kMaxTableFrames + 1) * sizeof(int) + 16;
  l.total = off;
  return l;
}

// Accumulate one stage (nb bands) of this thread's 4 pixels against KG
// filters.  Pixels are held as pairs (p0,p1), (p2,p3); the filter bank is
// stored duplicated, (f,f), so a 128-bit shared load yields two filters ready
// for the packed FMA.
template <typename T, int KG, bool kNorm>
__device__ __forceinline__ void consume_stage(const T* stage, const float* filt2, int nb, int tid,
                                              float2 (&acc)[KG][2], float2 (&nrm)[2]) {
  const T* src = stage + tid * kPPT;
  auto band = [&](int i) {
    float v[kPPT];
    load4<T>(src + i * kTile, v);
    const float2 v01 = make_float2(v[0], v[1]), v23 = make_float2(v[2], v[3]);
    if constexpr (kNorm) {
      nrm[0] = ffma2(v01, v01, nrm[0]);
      nrm[1] = ffma2(v23, v23, nrm[1]);
    }
    const float* fr = filt2 + i * KG * 2;
    if constexpr (KG >= 2) {
#pragma unroll
      for (int k = 0; k < KG; k += 2) {
        const float4 f = ld_shared_f4(fr + 2 * k);  // (f_k, f_k, f_k+1, f_k+1)
        const float2 fa = make_float2(f.x, f.y), fb = make_float2(f.z, f.w);
        acc[k][0] = ffma2(v01, fa, acc[k][0]);
        acc[k][1] = ffma2(v23, fa, acc[k][1]);
        acc[k + 1][0] = ffma2(v01, fb, acc[k + 1][0]);
        acc[k + 1][1] = ffma2(v23, fb, acc[k + 1][1]);
      }
    } else {
      const float2 fa = *reinterpret_cast<const float2*>(fr);
      acc[0][0] = ffma2(v01, fa, acc[0][0]);
      acc[0][1] = ffma2(v23, fa, acc[0][1]);
    }
  };
  if (nb == CubeTraits<T>::kStageBands) {
#pragma unroll
    for (int i = 0; i < CubeTraits<T>::kStageBands; ++i) band(i);
  } else {
    for (int i = 0; i < nb; ++i) band(i);
  }
}

// A thread's PPT consecutive outputs: one vector store when all are valid and
// `vec` (the address is PPT * 4-byte aligned), else element by element.
template <int PPT>
__device__ __forceinline__ void storev(float* dst, const float (&v)[PPT], int valid, bool vec) {
  if (vec && valid == PPT) {
    if constexpr (PPT == 4)
      *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
    else
      *reinterpret_cast<float2*>(dst) = make_float2(v[0], v[1]);
  } else {
#pragma unroll
    for (int j = 0; j < PPT; ++j)
      if (j < valid) dst[j] = v[j];
  }
}

template <int PPT>
__device__ __forceinline__ void storevi(int32_t* dst, const int32_t (&v)[PPT], int valid, bool vec) {
  if (vec && valid == PPT) {
    if constexpr (PPT == 4)
      *reinterpret_cast<int4*>(dst) = make_int4(v[0], v[1], v[2], v[3]);
    else
      *reinterpret_cast<int2*>(dst) = make_int2(v[0], v[1]);
  } else {
#pragma unroll
    for (int j = 0; j < PPT; ++j)
      if (j < valid) dst[j] = v[j];
  }
}

// Address aligned for a PPT-float vector store.
template <int PPT>
__device__ __forceinline__ bool aligned_v(const void* p) {
  return (reinterpret_cast<uintptr_t>(p) & (PPT * 4 - 1)) == 0;
}

// SAM epilogue for one thread's PPT pixels starting at frame pixel p.
template <int KG, int PPT>
__device__ void sam_epilogue(const hsi_frame& F, int pass, int n_f, int64_t p, int valid,
                             const float (&acc)[KG][PPT], const float (&nrm)[PPT], const float* scale) {
  {
    const bool first = pass == 0;
    const bool last = pass_count(F.num_sam, pass + 1) == 0;
    const int t0 = pass * kFiltersPerPass;
    float rn[PPT], best[PPT];
    int32_t best_t[PPT];
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      rn[j] = nrm[j] > 0.0f ? rsqrtf(nrm[j]) : 0.0f;
      best[j] = -2.0f;
      best_t[j] = -1;
    }
    if (!first) {
#pragma unroll
      for (int j = 0; j < PPT; ++j) {
        if (j >= valid) continue;
        if (F.sam_best) best[j] = F.sam_best[p + j];
        if (F.sam_best_target) best_t[j] = F.sam_best_target[p + j];
      }
    }
    const bool vec_maps = F.sam_maps && aligned_v<PPT>(F.sam_maps) && (F.map_stride % PPT) == 0;
#pragma unroll
    for (int k = 0; k < KG; ++k) {
      if (k < n_f) {
        float c[PPT];
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
          c[j] = acc[k][j] * rn[j] * scale[k];
          if (c[j] > best[j]) {
            best[j] = c[j];
            best_t[j] = t0 + k;
          }
        }
        if (F.sam_maps) {
          float a[PPT];
#pragma unroll
          for (int j = 0; j < PPT; j += 2) {
            const float2 v = angle_of_cos2(make_float2(c[j], c[j + 1]));
            a[j] = v.x;
            a[j + 1] = v.y;
          }
          storev<PPT>(F.sam_maps + static_cast<int64_t>(t0 + k) * F.map_stride + p, a, valid, vec_maps);
        }
      }
    }
    if (F.sam_best) {
      float out[PPT];
#pragma unroll
      for (int j = 0; j < PPT; ++j) out[j] = last ? angle_of_cos(best[j]) : best[j];
      storev<PPT>(F.sam_best + p, out, valid, aligned_v<PPT>(F.sam_best));
    }
    if (F.sam_best_target) storevi<PPT>(F.sam_best_target + p, best_t, valid, aligned_v<PPT>(F.sam_best_target));
  }
}

template <int KG, int PPT>
__device__ void cem_epilogue(const hsi_frame& F, int pass, int n_f, int64_t p, int valid,
                             const float (&acc)[KG][PPT]) {
  {
    const bool first = pass == 0;
    const int t0 = pass * kFiltersPerPass;
    float best[PPT];
    int32_t best_t[PPT];
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      best[j] = -INFINITY;
      best_t[j] = -1;
    }
    if (!first) {
#pragma unroll
      for (int j = 0; j < PPT; ++j) {
        if (j >= valid) continue;
        if (F.cem_best) best[j] = F.cem_best[p + j];
        if (F.cem_best_target) best_t[j] = F.cem_best_target[p + j];
      }
    }
    const bool vec_maps = F.cem_maps && aligned_v<PPT>(F.cem_maps) && (F.map_stride % PPT) == 0;
#pragma unroll
    for (int k = 0; k < KG; ++k) {
      if (k < n_f) {
        float r[PPT];
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
          r[j] = acc[k][j];
          if (r[j] > best[j]) {
            best[j] = r[j];
            best_t[j] = t0 + k;
          }
        }
        if (F.cem_maps)
          storev<PPT>(F.cem_maps + static_cast<int64_t>(t0 + k) * F.map_stride + p, r, valid, vec_maps);
      }
    }
    if (F.cem_best) storev<PPT>(F.cem_best + p, best, valid, aligned_v<PPT>(F.cem_best));
    if (F.cem_best_target) storevi<PPT>(F.cem_best_target + p, best_t, valid, aligned_v<PPT>(F.cem_best_target));
  }
}

// One consumer warpgroup: walks the same tile schedule as the producer,
// reloading the filter bank whenever the frame changes.
template <typename T, int KG, bool kSam, int kStages>
__device__ __forceinline__ void consumer_loop(const ScoreParams& prm, const int* prefix, int total_tiles,
                                              unsigned char* smem, size_t stage_bytes, uint64_t* full,
                                              uint64_t* empty, volatile int* abort_flag, float* filt,
                                              float* scale, int group, int tid, int lane) {
  const int nframes = prm.num_frames;
  int cur_frame = -1;
  int n_f = 0;
  uint32_t it = 0;
  bool aborted = false;
  int fcur = 0;  // tiles only move forward, and so does their frame
  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    const int f = fcur = next_frame(prefix, nframes, tile, fcur);
    const hsi_frame& F = frame_at(prm, f);
    const int B = F.bands;
    if (f != cur_frame) {
      named_sync(1 + group, kGroupThreads);
      n_f = pass_count(kSam ? F.num_sam : F.num_cem, prm.pass);
      const float* src = kSam ? F.sam_targets : F.cem_weights;
      const int t0 = prm.pass * kFiltersPerPass;
      for (int i = tid; i < B * KG; i += kGroupThreads) {
        const int b = i / KG, k = i % KG;
        const float v = k < n_f ? src[static_cast<int64_t>(t0 + k) * B + b] : 0.0f;
        filt[2 * i] = v;
        filt[2 * i + 1] = v;
      }
      if (kSam && tid < kFiltersPerPass) {
        const float nrm = tid < n_f ? F.sam_norms[t0 + tid] : 0.0f;
        scale[tid] = nrm > 0.0f ? 1.0f / nrm : 0.0f;
      }
      named_sync(1 + group, kGroupThreads);
      cur_frame = f;
    }
    const int64_t P = static_cast<int64_t>(F.height) * F.width;
    const int64_t p0 = static_cast<int64_t>(tile - prefix[f]) * kTile;
    const bool active = n_f > 0;

    float2 acc[KG][2];
    float2 nrm[2] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
#pragma unroll
    for (int k = 0; k < KG; ++k) acc[k][0] = acc[k][1] = make_float2(0.0f, 0.0f);

    for (int b0 = 0; b0 < B; b0 += CubeTraits<T>::kStageBands) {
      const int nb = B - b0 < CubeTraits<T>::kStageBands ? B - b0 : CubeTraits<T>::kStageBands;
      const int slot = static_cast<int>(it % kStages);
      const uint32_t round = it / kStages;
      if (!aborted && !mbar_wait(&full[slot], round & 1u)) {
        record_error(prm.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        aborted = true;
      }
      if (active && !aborted) {
        const T* stage = reinterpret_cast<const T*>(smem + slot * stage_bytes);
        consume_stage<T, KG, kSam>(stage, filt + 2 * b0 * KG, nb, tid, acc, nrm);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[slot]);
      ++it;
    }
    if (active && !aborted) {
      const int64_t p = p0 + tid * kPPT;
      const int64_t rem = P - p;
      const int valid = rem <= 0 ? 0 : (rem >= kPPT ? kPPT : static_cast<int>(rem));
      if (valid > 0) {
        float a[KG][kPPT];
#pragma unroll
        for (int k = 0; k < KG; ++k) {
          a[k][0] = acc[k][0].x;
          a[k][1] = acc[k][0].y;
          a[k][2] = acc[k][1].x;
          a[k][3] = acc[k][1].y;
        }
        if constexpr (kSam) {
          const float n[kPPT] = {nrm[0].x, nrm[0].y, nrm[1].x, nrm[1].y};
          sam_epilogue<KG, kPPT>(F, prm.pass, n_f, p, valid, a, n, scale);
        } else {
          cem_epilogue<KG, kPPT>(F, prm.pass, n_f, p, valid, a);
        }
      }
    }
  }
}

// Fused consumer: two warpgroups score the SAM and the CEM bank (either may be
// empty) together, so each pixel leaves shared memory once for all KS + KC
// filters.  The bank is
// stored band-major without duplication, [b][KS SAM | KC CEM]; accumulators
// are filter pairs per pixel, (acc_k, acc_k+1) += (x, x) * (f_k, f_k+1), the
// pixel duplicated in a register pair for the packed FMA.  Two pixels per
// thread keep the accumulators at 2 * (KS + KC) registers, so 256 consumer
// threads fit per CTA at three CTAs per SM (twice the warps of one warpgroup
// at four pixels per thread, to hide the shared-memory and FMA latencies).
template <typename T, int K, bool kNorm>
__device__ __forceinline__ void consume_stage_fused(const T* stage, const float* filt, int nb, int tid,
                                                    float2 (&acc)[K / 2][kFusedPPT], float2& nrm) {
  static_assert(kFusedPPT == 2, "two pixels per fused consumer thread");
  static_assert(K % 4 == 0, "filters in groups of four");
  const T* src = stage + tid * kFusedPPT;
  auto band = [&](int i) {
    const float2 v = load2<T>(src + i * kTile);
    if constexpr (kNorm) nrm = ffma2(v, v, nrm);
    const float2 d0 = make_float2(v.x, v.x), d1 = make_float2(v.y, v.y);
    const float* fr = filt + i * K;
#pragma unroll
    for (int k = 0; k < K; k += 4) {
      const float4 f = ld_shared_f4(fr + k);  // (f_k, f_k+1, f_k+2, f_k+3)
      const float2 fa = make_float2(f.x, f.y), fb = make_float2(f.z, f.w);
      acc[k / 2][0] = ffma2(d0, fa, acc[k / 2][0]);
      acc[k / 2][1] = ffma2(d1, fa, acc[k / 2][1]);
      acc[k / 2 + 1][0] = ffma2(d0, fb, acc[k / 2 + 1][0]);
      acc[k / 2 + 1][1] = ffma2(d1, fb, acc[k / 2 + 1][1]);
    }
  };
  if (nb == CubeTraits<T>::kStageBands) {
#pragma unroll
    for (int i = 0; i < CubeTraits<T>::kStageBands; ++i) band(i);
  } else {
    for (int i = 0; i < nb; ++i) band(i);
  }
}

template <typename T, int KS, int KC, int kStages>
__device__ __forceinline__ void consumer_loop_fused(const ScoreParams& prm, const int* prefix, int total_tiles,
                                                    unsigned char* smem, size_t stage_bytes, uint64_t* full,
                                                    uint64_t* empty, volatile int* abort_flag, float* filt,
                                                    float* scale, int tid, int lane) {
  constexpr int K = KS + KC;
  constexpr int PPT = kFusedPPT;
  const int nframes = prm.num_frames;
  int cur_frame = -1;
  int n_s = 0, n_c = 0;
  uint32_t it = 0;
  bool aborted = false;
  int fcur = 0;  // tiles only move forward, and so does their frame
  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    const int f = fcur = next_frame(prefix, nframes, tile, fcur);
    const hsi_frame& F = frame_at(prm, f);
    const int B = F.bands;
    if (f != cur_frame) {
      named_sync(1, kFusedThreads);
      n_s = pass_count(F.num_sam, prm.pass);
      n_c = pass_count(F.num_cem, prm.pass);
      const int t0 = prm.pass * kFiltersPerPass;
      for (int i = tid; i < B * K; i += kFusedThreads) {
        const int b = i / K, k = i % K;
        float v = 0.0f;
        if (k < KS) {
          if (k < n_s) v = F.sam_targets[static_cast<int64_t>(t0 + k) * B + b];
        } else if (k - KS < n_c) {
          v = F.cem_weights[static_cast<int64_t>(t0 + k - KS) * B + b];
        }
        filt[i] = v;
      }
      if (tid < kFiltersPerPass) {
        const float nrm = tid < n_s ? F.sam_norms[t0 + tid] : 0.0f;
        scale[tid] = nrm > 0.0f ? 1.0f / nrm : 0.0f;
      }
      named_sync(1, kFusedThreads);
      cur_frame = f;
    }
    const int64_t P = static_cast<int64_t>(F.height) * F.width;
    const int64_t p0 = static_cast<int64_t>(tile - prefix[f]) * kTile;
    const bool active = n_s > 0 || n_c > 0;

    float2 acc[K / 2][PPT];
    float2 nrm = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int k = 0; k < K / 2; ++k)
#pragma unroll
      for (int j = 0; j < PPT; ++j) acc[k][j] = make_float2(0.0f, 0.0f);

    for (int b0 = 0; b0 < B; b0 += CubeTraits<T>::kStageBands) {
      const int nb = B - b0 < CubeTraits<T>::kStageBands ? B - b0 : CubeTraits<T>::kStageBands;
      const int slot = static_cast<int>(it % kStages);
      const uint32_t round = it / kStages;
      if (!aborted && !mbar_wait(&full[slot], round & 1u)) {
        record_error(prm.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        aborted = true;
      }
      if (active && !aborted) {
        const T* stage = reinterpret_cast<const T*>(smem + slot * stage_bytes);
        consume_stage_fused<T, K, (KS > 0)>(stage, filt + b0 * K, nb, tid, acc, nrm);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[slot]);
      ++it;
    }
    if (active && !aborted) {
      const int64_t p = p0 + tid * PPT;
      const int64_t rem = P - p;
      const int valid = rem <= 0 ? 0 : (rem >= PPT ? PPT : static_cast<int>(rem));
      if (valid > 0) {
        if constexpr (KS > 0) {
          if (n_s > 0) {
            float a[KS][PPT];
#pragma unroll
            for (int k = 0; k < KS; ++k)
#pragma unroll
              for (int j = 0; j < PPT; ++j) a[k][j] = (k & 1) ? acc[k / 2][j].y : acc[k / 2][j].x;
            const float n[PPT] = {nrm.x, nrm.y};
            sam_epilogue<KS, PPT>(F, prm.pass, n_s, p, valid, a, n, scale);
          }
        }
        if constexpr (KC > 0) {
          if (n_c > 0) {
            float a[KC][PPT];
#pragma unroll
            for (int k = 0; k < KC; ++k)
#pragma unroll
              for (int j = 0; j < PPT; ++j)
                a[k][j] = ((KS + k) & 1) ? acc[(KS + k) / 2][j].y : acc[(KS + k) / 2][j].x;
            cem_epilogue<KC, PPT>(F, prm.pass, n_c, p, valid, a);
          }
        }
      }
    }
  }
}

// One bank layout for both kinds: 0, 4, 8 or 16 filters of each kind, at most
// 16 in all (two pixels per thread keep the accumulators at 2 (KS + KC)
// registers).  Other counts (a single filter, or more than 16 in all) take one
// warpgroup per kind.
template <int KS, int KC>
constexpr bool fused_banks() {
  constexpr bool ks = KS == 0 || KS == 4 || KS == 8 || KS == 16;
  constexpr bool kc = KC == 0 || KC == 4 || KC == 8 || KC == 16;
  return ks && kc && KS + KC > 0 && KS + KC <= 16;
}

// Kernel: KS SAM filters and KC CEM filters per pass (0 = that warpgroup is
// absent; both in one consumer group of kFusedThreads when fused_banks).
// Block = consumer threads + 32; the last warp produces.
template <int KS, int KC>
constexpr int score_groups() {
  return fused_banks<KS, KC>() ? 1 : (KS > 0) + (KC > 0);
}
template <int KS, int KC>
constexpr int consumer_threads() {
  return fused_banks<KS, KC>() ? kFusedThreads : score_groups<KS, KC>() * kGroupThreads;
}
// Filter slots per band per group in shared memory (duplicated pairs in the
// two-group layout, plain in the fused one).
template <int KS, int KC>
constexpr int score_slots() {
  return fused_banks<KS, KC>() ? KS + KC : 2 * (KS > KC ? KS : KC);
}

template <typename T, int KS, int KC>
constexpr int score_stages() {
  return fused_banks<KS, KC>() ? CubeTraits<T>::kStagesFused : CubeTraits<T>::kStages;
}

template <typename T, int KS, int KC>
__global__ void __launch_bounds__(consumer_threads<KS, KC>() + 32, fused_banks<KS, KC>() ? 3 : 1)
    score_kernel(const __grid_constant__ ScoreParams prm, int max_bands) {
  constexpr int kGroups = score_groups<KS, KC>();
  constexpr int kStages = score_stages<T, KS, KC>();
  constexpr int kSlots = score_slots<KS, KC>();
  extern __shared__ __align__(128) unsigned char smem[];
  const SmemLayout L = smem_layout<T>(kGroups, max_bands, kSlots, kStages);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bar_off);
  uint64_t* empty = full + kStages;
  int* prefix = reinterpret_cast<int*>(smem + L.prefix_off);
  volatile int* abort_flag = prefix + kMaxTableFrames + 1;

  const int nframes = prm.num_frames;
  // Per-frame tile counts (frames without filters in this pass get none).
  for (int f = threadIdx.x; f < nframes; f += blockDim.x) {
    const hsi_frame& F = frame_at(prm, f);
    const int64_t P = static_cast<int64_t>(F.height) * F.width;
    // A frame outside the launch's bounds would overflow the shared-memory
    // filter bank: it is skipped and the error recorded.
    const bool ok = F.bands > 0 && F.bands <= max_bands && F.num_sam >= 0 && F.num_sam <= prm.max_sam &&
                    F.num_cem >= 0 && F.num_cem <= prm.max_cem && F.dtype == prm.dtype && P > 0 &&
                    F.plane_stride >= P && (F.plane_stride & 7) == 0;
    if (!ok && blockIdx.x == 0) record_error(prm.status, HSI_E_INVALID);
    const bool any = ok && (pass_count(F.num_sam, prm.pass) > 0 || pass_count(F.num_cem, prm.pass) > 0);
    prefix[f + 1] = any ? static_cast<int>(div_up<int64_t>(P, kTile)) : 0;
  }
  if (threadIdx.x == 0) {
    prefix[0] = 0;
    *abort_flag = 0;
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], consumer_threads<KS, KC>() / 32);
    }
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int f = 0; f < nframes; ++f) prefix[f + 1] += prefix[f];
  }
  __syncthreads();
  const int total_tiles = prefix[nframes];

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (warp == consumer_threads<KS, KC>() / 32) {
    // ---------------- producer warp ----------------
    if (lane == 0) {
      uint32_t it = 0;
      bool aborted = false;
      uint32_t pending = 0;         // bit s: slot s has copies issued
      uint32_t pending_parity = 0;  // bit s: phase parity of that issue
      int fcur = 0;  // tiles only move forward, and so does their frame
      for (int tile = blockIdx.x; tile < total_tiles && !aborted; tile += gridDim.x) {
        const int f = fcur = next_frame(prefix, nframes, tile, fcur);
        const hsi_frame& F = frame_at(prm, f);
        const int64_t P = static_cast<int64_t>(F.height) * F.width;
        const int64_t p0 = static_cast<int64_t>(tile - prefix[f]) * kTile;
        const int npx = static_cast<int>(P - p0 < kTile ? P - p0 : kTile);
        const uint32_t bytes = static_cast<uint32_t>(((npx + 7) & ~7) * sizeof(T));
        const T* cube = static_cast<const T*>(F.cube);
        for (int b0 = 0; b0 < F.bands; b0 += CubeTraits<T>::kStageBands) {
          const int nb = F.bands - b0 < CubeTraits<T>::kStageBands ? F.bands - b0 : CubeTraits<T>::kStageBands;
          const int slot = static_cast<int>(it % kStages);
          const uint32_t round = it / kStages;
          if (*abort_flag || !mbar_wait(&empty[slot], (round & 1u) ^ 1u)) {
            record_error(prm.status, HSI_E_TIMEOUT);
            *abort_flag = 1;
            aborted = true;
            break;
          }
          T* dst = reinterpret_cast<T*>(smem + slot * L.stage_bytes);
          mbar_arrive_expect_tx(&full[slot], bytes * nb);
          for (int i = 0; i < nb; ++i)
            bulk_g2s(dst + i * kTile, cube + static_cast<int64_t>(b0 + i) * F.plane_stride + p0, bytes,
                     &full[slot]);
          pending |= 1u << slot;
          pending_parity = (pending_parity & ~(1u << slot)) | ((round & 1u) << slot);
          ++it;
        }
      }
      // Never leave the CTA with copies in flight into its shared memory.
      for (int s = 0; s < kStages; ++s)
        if ((pending >> s) & 1u) mbar_wait(&full[s], (pending_parity >> s) & 1u);
    }
    return;
  }

  // ---------------- consumer warpgroups ----------------
  if constexpr (fused_banks<KS, KC>()) {
    float* filt = reinterpret_cast<float*>(smem + L.filt_off);
    float* scale = reinterpret_cast<float*>(smem + L.scale_off);
    consumer_loop_fused<T, KS, KC, kStages>(prm, prefix, total_tiles, smem, L.stage_bytes, full, empty, abort_flag,
                                            filt, scale, threadIdx.x, lane);
    return;
  }
  const int group = warp / (kGroupThreads / 32);  // 0: SAM if KS > 0, else CEM; 1: CEM
  const int tid = threadIdx.x - group * kGroupThreads;
  float* filt = reinterpret_cast<float*>(smem + L.filt_off) + static_cast<size_t>(group) * max_bands * kSlots;
  float* scale = reinterpret_cast<float*>(smem + L.scale_off) + group * kFiltersPerPass;
  if constexpr (KS > 0) {
    if (group == 0) {
      consumer_loop<T, KS, true, kStages>(prm, prefix, total_tiles, smem, L.stage_bytes, full, empty,
                                          abort_flag, filt, scale, group, tid, lane);
      return;
    }
  }
  if constexpr (KC > 0) {
    consumer_loop<T, KC, false, kStages>(prm, prefix, total_tiles, smem, L.stage_bytes, full, empty,
                                         abort_flag, filt, scale, group, tid, lane);
  }
}

// ---------------------------------------------------------------------------
// Tensor-core scorer for FP16 cubes of at most 128 bands (kind::f16 MMAs).
//
// An FP16 cube value is an exact f16 MMA operand, and a TMA box of 64 pixels x
// Bp bands loaded with the 128-byte swizzle is already the MN-major operand
// layout, so the cube goes from HBM to the tensor cores with no conversion
// pass.  Each filter f (a SAM target or CEM weight vector, FP32) is scaled by
// a power of two 2^s (its largest |weight| to [0.5, 1)) and split into an f16
// head fh = rn(f 2^s) and remainder fl = rn(f 2^s - fh), 22 significant bits
// together.  B stacks the heads over the remainders (N2 = 2 N rows), so one
// MMA per 16 bands gives x.fh and x.fl in separate TMEM columns, and
// x.f = (x.fh + x.fl) 2^-s in the epilogue.  Products are exact, sums FP32.
//
// Per 128-pixel tile, one CTA per SM:
//   warp 0       producer: two TMA boxes (64 px x Bp bands, 128-byte swizzle)
//   warp 1       TMEM allocator + MMA issuer: Bp / 16 MMAs (M 128, N N2, K 16)
//                into one of four accumulators
//   warps 2-5    readers: the pixels' squared norms (SAM) from each stage, and
//                the filter bank (heads, remainders, multipliers) at frame changes
//   warps 6-21   epilogue, two teams of eight warps taking alternate tiles (four
//                SAM, four CEM warps each; one pixel per thread): the angle /
//                response / best-target rules of the FP32 scorer.  Two teams
//                put two epilogue warps of a kind on each SM sub-partition, so
//                the per-pixel arccosines and stores of one hide the latency of
//                the other's.
// ---------------------------------------------------------------------------
constexpr int kHTile = 128;
constexpr int kHStages = 6;
constexpr int kHMaxBands = 128;
constexpr int kHAcc = 8;  // TMEM accumulators (and norm buffers) in flight
constexpr int kHThreads = 22 * 32;

struct HSmem {
  size_t stage_bytes, in_off, filt_off, norm_off, scale_off, bar_off, slot_off, total;
};

// bp: bands rounded up to 16; n2: rows of B (heads and remainders).
__host__ __device__ inline HSmem h_smem(int bp, int n2) {
  HSmem s;
  s.stage_bytes = static_cast<size_t>(2) * bp * 128;  // two 64-pixel boxes
  size_t off = 0;
  s.in_off = off;  // 1024-aligned stages (bp * 128 is a multiple of 2048)
  off += kHStages * s.stage_bytes;
  s.filt_off = off;  // K-major, 64 bands per 128-byte row: (bp / 64 rounded up) chunks of n2 rows
  off += static_cast<size_t>((bp + 63) / 64) * n2 * 128;
  s.norm_off = off;  // [kHAcc buffers][4 reader warps][128 px]
  off += kHAcc * 4 * kHTile * sizeof(float);
  s.scale_off = off;  // [2 epochs][32 filters]
  off += 2 * 32 * sizeof(float);
  s.bar_off = off;
  off += (2 * kHStages + 4 * kHAcc + 2 + 2 * 2 + 1) * sizeof(uint64_t);
  s.slot_off = off;
  off += 16;
  s.total = off + 1024;
  return s;
}

// Launch parameters: descriptors and tensor maps of up to 64 FP16 frames.
struct HParams {
  CUtensorMap maps[kMaxInline];
  hsi_frame frames[kMaxInline];
  int num_frames;
  int pass;
  int max_sam, max_cem;
  int bp;       // bands of every frame rounded up to 16, at most 128
  int* status;  // nullable device error word
};

// KS SAM and KC CEM filters per pass (each 0, 8 or 16); N = KS + KC rounded
// up to 16, N2 = 2 N.
template <int KS, int KC>
__global__ void __launch_bounds__(kHThreads, 1) score_h_kernel(const __grid_constant__ HParams prm) {
  constexpr int N = (KS + KC + 15) / 16 * 16;
  constexpr int N2 = 2 * N;
  constexpr uint32_t kCols = kHAcc * N2;  // 256 or 512 TMEM columns
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int bp = prm.bp;
  const HSmem L = h_smem(bp, N2);
  uint64_t* in_full = reinterpret_cast<uint64_t*>(smem + L.bar_off);
  uint64_t* in_empty = in_full + kHStages;
  uint64_t* acc_full = in_empty + kHStages;
  uint64_t* acc_empty = acc_full + kHAcc;
  uint64_t* norm_full = acc_empty + kHAcc;
  uint64_t* norm_empty = norm_full + kHAcc;
  uint64_t* filt_full = norm_empty + kHAcc;  // readers -> MMA: the bank of the new frame is in place
  uint64_t* filt_free = filt_full + 1;    // MMA -> readers: every MMA on the old bank has completed
  uint64_t* sc_full = filt_free + 1;      // readers -> epilogue: scales of epoch e & 1
  uint64_t* sc_empty = sc_full + 2;       // epilogue -> readers
  uint64_t* mma_done = sc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.slot_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.slot_off + 8);
  __shared__ int prefix[kMaxInline + 1];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nframes = prm.num_frames;
  for (int f = threadIdx.x; f < nframes; f += blockDim.x) {
    const hsi_frame& F = prm.frames[f];
    const int64_t P = static_cast<int64_t>(F.height) * F.width;
    const bool ok = F.bands > 0 && F.bands <= bp && F.num_sam >= 0 && F.num_sam <= prm.max_sam && F.num_cem >= 0 &&
                    F.num_cem <= prm.max_cem && F.dtype == HSI_F16 && P > 0 && F.plane_stride >= P &&
                    (F.plane_stride & 7) == 0;
    if (!ok && blockIdx.x == 0) record_error(prm.status, HSI_E_INVALID);
    const bool any = ok && (pass_count(F.num_sam, prm.pass) > 0 || pass_count(F.num_cem, prm.pass) > 0);
    prefix[f + 1] = any ? static_cast<int>(div_up<int64_t>(P, kHTile)) : 0;
  }
  if (threadIdx.x == 0) {
    prefix[0] = 0;
    *abort_flag = 0;
    for (int s = 0; s < kHStages; ++s) {
      mbar_init(&in_full[s], 1);
      mbar_init(&in_empty[s], 1 + 4);  // the MMA commit and the four reader warps
    }
    for (int s = 0; s < kHAcc; ++s) {
      mbar_init(&acc_full[s], 1);
      mbar_init(&acc_empty[s], 8);   // the eight warps of the team that takes the tile
      mbar_init(&norm_full[s], 4);
      mbar_init(&norm_empty[s], 4);  // that team's SAM warps
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&sc_full[s], 4);
      mbar_init(&sc_empty[s], 16);  // every epilogue warp
    }
    mbar_init(filt_full, 4);
    mbar_init(filt_free, 1);
    mbar_init(mma_done, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(tmem_slot, kCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0)
    for (int f = 0; f < nframes; ++f) prefix[f + 1] += prefix[f];
  __syncthreads();
  const int total_tiles = prefix[nframes];
  const uint32_t tmem = *tmem_slot;
  const uint32_t box_bytes = static_cast<uint32_t>(bp) * 128;

  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      uint32_t it = 0, pending = 0, parity = 0;
      int fcur = 0;  // tiles only move forward, and so does their frame
      for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x, ++it) {
        const int f = fcur = next_frame(prefix, nframes, tile, fcur);
        const int x0 = (tile - prefix[f]) * kHTile;
        const int s = it % kHStages;
        const uint32_t ph = (it / kHStages) & 1u;
        if (*abort_flag || !mbar_wait(&in_empty[s], ph ^ 1u)) {
          record_error(prm.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        unsigned char* dst = smem + L.in_off + static_cast<size_t>(s) * L.stage_bytes;
        mbar_arrive_expect_tx(&in_full[s], 2 * box_bytes);
        tma_load_2d(dst, &prm.maps[f], x0, 0, &in_full[s]);
        tma_load_2d(dst + box_bytes, &prm.maps[f], x0 + 64, 0, &in_full[s]);
        pending |= 1u << s;
        parity = (parity & ~(1u << s)) | (ph << s);
      }
      // never leave copies in flight into this CTA's shared memory
      for (int s = 0; s < kHStages; ++s)
        if ((pending >> s) & 1u) mbar_wait(&in_full[s], (parity >> s) & 1u);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = idesc_f16_amn(kHTile, N2);
      const unsigned char* filt = smem + L.filt_off;
      uint32_t it = 0, epoch = 0;
      int cur = -1;
      bool ok = true, issued = false;
      int fcur = 0;  // tiles only move forward, and so does their frame
      for (int tile = blockIdx.x; tile < total_tiles && ok; tile += gridDim.x, ++it) {
        const int f = fcur = next_frame(prefix, nframes, tile, fcur);
        if (f != cur) {
          // hand the bank back once every MMA on it has completed, then wait
          // for the new one
          if (cur >= 0) umma_commit(filt_free);
          if (*abort_flag || !mbar_wait(filt_full, epoch & 1u)) {
            record_error(prm.status, HSI_E_TIMEOUT);
            *abort_flag = 1;
            break;
          }
          tc_fence_after();
          cur = f;
          ++epoch;
        }
        const int s = it % kHStages, buf = it % kHAcc;
        if (!mbar_wait(&in_full[s], (it / kHStages) & 1u) || !mbar_wait(&acc_empty[buf], ((it / kHAcc) & 1u) ^ 1u)) {
          record_error(prm.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const unsigned char* a = smem + L.in_off + static_cast<size_t>(s) * L.stage_bytes;
        const int ksteps = div_up(prm.frames[f].bands, 16);
        for (int ks = 0; ks < ksteps; ++ks) {
          const uint64_t da = smem_desc_mn_sw128(a + ks * 2048, box_bytes);
          const uint64_t db = smem_desc_sw128(filt + (ks >> 2) * N2 * 128) + 2 * (ks & 3);
          umma_f16(tmem + buf * N2, da, db, idesc, ks > 0 ? 1u : 0u);
        }
        umma_commit(&in_empty[s]);
        umma_commit(&acc_full[buf]);
        issued = true;
      }
      if (issued) {
        umma_commit(mma_done);
        if (!mbar_wait(mma_done, 0)) record_error(prm.status, HSI_E_TIMEOUT);
      }
    }
  } else if (warp < 6) {
    // ---------------- readers: squared norms and the filter bank ----------------
    const int rt = threadIdx.x - 64;        // 0..127
    const int ch = rt & 15, bg = rt >> 4;   // pixels 8 ch .. 8 ch + 7; bands bg, bg + 8, ...
    const int rw = warp - 2;                // reader warp 0..3
    uint32_t it = 0, epoch = 0;
    int cur = -1;
    bool ok = true;
    int fcur = 0;  // tiles only move forward, and so does their frame
    for (int tile = blockIdx.x; tile < total_tiles && ok; tile += gridDim.x, ++it) {
      const int f = fcur = next_frame(prefix, nframes, tile, fcur);
      const hsi_frame& F = prm.frames[f];
      if (f != cur) {
        // filter n: heads in row n, remainders in row N + n; 128 / N threads per
        // filter, each over every (128 / N)-th band.  The new frame's values are
        // fetched before waiting for the MMAs on the old bank to complete.
        const int tpf = 128 / N, n = rt / tpf, j0 = rt % tpf;
        const int n_s = pass_count(F.num_sam, prm.pass), n_c = pass_count(F.num_cem, prm.pass);
        const int t0 = prm.pass * kFiltersPerPass;
        const float* src = nullptr;
        if (n < KS) {
          if (n < n_s) src = F.sam_targets + static_cast<int64_t>(t0 + n) * F.bands;
        } else if (n - KS < KC && n - KS < n_c) {
          src = F.cem_weights + static_cast<int64_t>(t0 + n - KS) * F.bands;
        }
        float v[N];  // bands j0 + i tpf, i < N, cover 0..127
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const int b = j0 + i * tpf;
          v[i] = (src && b < F.bands) ? src[b] : 0.0f;
        }
        const float nr = (n < KS && n < n_s) ? F.sam_norms[t0 + n] : 0.0f;
        float mx = 0.0f;
#pragma unroll
        for (int i = 0; i < N; ++i) mx = fmaxf(mx, fabsf(v[i]));
        for (int o = tpf / 2; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        int e2 = 0;
        if (mx > 0.0f) frexpf(mx, &e2);  // mx in [2^(e2-1), 2^e2)
        const float up = ldexpf(1.0f, -e2);
        if (epoch > 0 && !mbar_wait(filt_free, (epoch - 1) & 1u)) {
          ok = false;
          break;
        }
        if (!mbar_wait(&sc_empty[epoch & 1u], ((epoch >> 1) & 1u) ^ 1u)) {
          ok = false;
          break;
        }
        unsigned char* filt = smem + L.filt_off;
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const int b = j0 + i * tpf;
          if (b >= bp) break;
          const float w = v[i] * up;
          const __half h = __float2half_rn(w);
          const __half l = __float2half_rn(w - __half2float(h));
          const int k2 = (b & 63) * 2;
          const uint32_t row_h = static_cast<uint32_t>(n), row_l = static_cast<uint32_t>(N + n);
          const uint32_t base = static_cast<uint32_t>((b >> 6) * N2 * 128);
          const uint32_t oh = base + (row_h >> 3) * 1024 + (row_h & 7) * 128 + ((((k2 >> 4) ^ (row_h & 7))) << 4) + (k2 & 15);
          const uint32_t ol = base + (row_l >> 3) * 1024 + (row_l & 7) * 128 + ((((k2 >> 4) ^ (row_l & 7))) << 4) + (k2 & 15);
          *reinterpret_cast<__half*>(filt + oh) = h;
          *reinterpret_cast<__half*>(filt + ol) = l;
        }
        // multiplier of column pair n: x.f = (x.fh + x.fl) 2^e2, and SAM folds in 1 / |r_t|
        float mult = ldexpf(1.0f, e2);
        if (n < KS) mult = nr > 0.0f ? mult / nr : 0.0f;
        float* sc = reinterpret_cast<float*>(smem + L.scale_off) + (epoch & 1u) * 32;
        if (j0 == 0) sc[n] = mult;
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(filt_full);
          mbar_arrive(&sc_full[epoch & 1u]);
        }
        cur = f;
        ++epoch;
      }
      // squared norms of the tile's pixels
      const int s = it % kHStages, nb = it % kHAcc;
      if (!mbar_wait(&in_full[s], (it / kHStages) & 1u) || !mbar_wait(&norm_empty[nb], ((it / kHAcc) & 1u) ^ 1u)) {
        ok = false;
        break;
      }
      const unsigned char* st = smem + L.in_off + static_cast<size_t>(s) * L.stage_bytes;
      const int box = ch >> 3, c = ch & 7;  // 64-pixel box, 16-byte chunk (8 px) of its 128-byte rows
      float2 acc[4] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f),
                       make_float2(0.0f, 0.0f)};
      // rows from the frame's band count up to bp are the box's zero fill, so
      // every thread runs bp / 16 iterations of two bands (b, b + 8), loads first
      const unsigned char* col = st + box * box_bytes + ((c ^ (bg & 7)) << 4) + bg * 128;
#pragma unroll 4
      for (int b = 0; b < bp; b += 16) {
        // (b + bg) & 7 == bg & 7: the swizzled chunk is the same in every row this thread reads
        const uint4 r0 = *reinterpret_cast<const uint4*>(col + b * 128);
        const uint4 r1 = *reinterpret_cast<const uint4*>(col + b * 128 + 1024);
        const __half2* h0 = reinterpret_cast<const __half2*>(&r0);
        const __half2* h1 = reinterpret_cast<const __half2*>(&r1);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float2 v0 = __half22float2(h0[q]);
          const float2 v1 = __half22float2(h1[q]);
          acc[q] = ffma2(v0, v0, acc[q]);
          acc[q] = ffma2(v1, v1, acc[q]);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&in_empty[s]);
      // two band groups per warp (lanes 16 apart), then one partial per reader warp
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        acc[q].x += __shfl_xor_sync(0xffffffffu, acc[q].x, 16);
        acc[q].y += __shfl_xor_sync(0xffffffffu, acc[q].y, 16);
      }
      float* out = reinterpret_cast<float*>(smem + L.norm_off) + (nb * 4 + rw) * kHTile + 8 * ch;
      if (lane < 16) {
        *reinterpret_cast<float4*>(out) = make_float4(acc[0].x, acc[0].y, acc[1].x, acc[1].y);
        *reinterpret_cast<float4*>(out + 4) = make_float4(acc[2].x, acc[2].y, acc[3].x, acc[3].y);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&norm_full[nb]);
    }
    if (!ok) {
      record_error(prm.status, HSI_E_TIMEOUT);
      *abort_flag = 1;
    }
  } else {
    // ---------------- epilogue ----------------
    const int team = (warp - 6) >> 3;            // takes the tiles with it % 2 == team
    const bool cem = ((warp - 6) & 7) >= 4;
    const int quarter = warp & 3;  // TMEM lane quarter of this warp
    const int m = quarter * 32 + lane;
    const uint32_t tq = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
    uint32_t it = 0, epoch = 0;
    int cur = -1;
    float scale[16];  // multipliers of this warp's filters (SAM or CEM) for the current frame
    int fcur = 0;  // tiles only move forward, and so does their frame
    for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x, ++it) {
      const int f = fcur = next_frame(prefix, nframes, tile, fcur);
      const hsi_frame& F = prm.frames[f];
      if (f != cur) {
        if (*abort_flag || !mbar_wait(&sc_full[epoch & 1u], (epoch >> 1) & 1u)) {
          record_error(prm.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        const float* sc = reinterpret_cast<const float*>(smem + L.scale_off) + (epoch & 1u) * 32 + (cem ? KS : 0);
#pragma unroll
        for (int k = 0; k < 16; ++k) scale[k] = sc[k];
        __syncwarp();
        if (lane == 0) mbar_arrive(&sc_empty[epoch & 1u]);
        cur = f;
        ++epoch;
      }
      if (static_cast<int>(it & 1u) != team) continue;
      const int buf = it % kHAcc;
      if (*abort_flag || !mbar_wait(&acc_full[buf], (it / kHAcc) & 1u) ||
          (!cem && !mbar_wait(&norm_full[buf], (it / kHAcc) & 1u))) {
        record_error(prm.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const int64_t P = static_cast<int64_t>(F.height) * F.width;
      const int64_t p = static_cast<int64_t>(tile - prefix[f]) * kHTile + m;
      const bool in_frame = p < P;
      const uint32_t d0 = tq + buf * N2;
      const int t0 = prm.pass * kFiltersPerPass;
      // filters c .. c+7 of this kind: (head + remainder columns) x multiplier
      auto dots8 = [&](int c, float (&dot)[8]) {
        uint32_t h[8], l[8];
        const int col = (cem ? KS : 0) + c;
        tmem_ld8(d0 + col, h);
        tmem_ld8(d0 + N + col, l);
        tmem_wait_ld();
#pragma unroll
        for (int k = 0; k < 8; ++k) dot[k] = (__uint_as_float(h[k]) + __uint_as_float(l[k])) * scale[c + k];
      };
      if (!cem) {
        if constexpr (KS > 0) {
          const int n_s = pass_count(F.num_sam, prm.pass);
          const float* nrm_in = reinterpret_cast<const float*>(smem + L.norm_off) + buf * 4 * kHTile + m;
          const float nrm = (nrm_in[0] + nrm_in[kHTile]) + (nrm_in[2 * kHTile] + nrm_in[3 * kHTile]);
          __syncwarp();
          if (lane == 0) mbar_arrive(&norm_empty[buf]);
          if (n_s > 0) {
            const float rn = nrm > 0.0f ? rsqrtf(nrm) : 0.0f;
            const bool last = pass_count(F.num_sam, prm.pass + 1) == 0;
            float best = -2.0f;
            int32_t best_t = -1;
            if (prm.pass != 0 && in_frame) {
              if (F.sam_best) best = F.sam_best[p];
              if (F.sam_best_target) best_t = F.sam_best_target[p];
            }
            float cs[KS];
#pragma unroll
            for (int c = 0; c < KS; c += 8) {
              float dot[8];
              dots8(c, dot);
#pragma unroll
              for (int k = 0; k < 8; ++k) cs[c + k] = dot[k] * rn;
            }
#pragma unroll
            for (int k = 0; k < KS; ++k)
              if (k < n_s && cs[k] > best) {
                best = cs[k];
                best_t = t0 + k;
              }
            if (F.sam_maps && in_frame) {
              float* const maps = F.sam_maps + static_cast<int64_t>(t0) * F.map_stride + p;
              float ang[KS];
#pragma unroll
              for (int k = 0; k < KS; ++k) ang[k] = angle_of_cos(cs[k]);
#pragma unroll
              for (int k = 0; k < KS; ++k)
                if (k < n_s) maps[k * F.map_stride] = ang[k];
            }
            if (in_frame) {
              if (F.sam_best) F.sam_best[p] = last ? angle_of_cos(best) : best;
              if (F.sam_best_target) F.sam_best_target[p] = best_t;
            }
          }
        } else {
          __syncwarp();
          if (lane == 0) mbar_arrive(&norm_empty[buf]);
        }
      } else {
        if constexpr (KC > 0) {
          const int n_c = pass_count(F.num_cem, prm.pass);
          if (n_c > 0) {
            float best = -INFINITY;
            int32_t best_t = -1;
            if (prm.pass != 0 && in_frame) {
              if (F.cem_best) best = F.cem_best[p];
              if (F.cem_best_target) best_t = F.cem_best_target[p];
            }
            float r[KC];
#pragma unroll
            for (int c = 0; c < KC; c += 8) {
              float dot[8];
              dots8(c, dot);
#pragma unroll
              for (int k = 0; k < 8; ++k) r[c + k] = dot[k];
            }
#pragma unroll
            for (int k = 0; k < KC; ++k)
              if (k < n_c && r[k] > best) {
                best = r[k];
                best_t = t0 + k;
              }
            if (F.cem_maps && in_frame) {
              float* const maps = F.cem_maps + static_cast<int64_t>(t0) * F.map_stride + p;
#pragma unroll
              for (int k = 0; k < KC; ++k)
                if (k < n_c) maps[k * F.map_stride] = r[k];
            }
            if (in_frame) {
              if (F.cem_best) F.cem_best[p] = best;
              if (F.cem_best_target) F.cem_best_target[p] = best_t;
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[buf]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kCols);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

int sm_count() { return device_sm_count(); }

constexpr int kSupported[] = {0, 1, 4, 8, 16};

int round_filters(int n) {
  for (int v : kSupported)
    if (n <= v) return v;
  return 16;
}

template <typename T, int KS, int KC>
int launch_instance(const ScoreParams& p, int max_bands, int ctas_per_sm, cudaStream_t stream) {
  constexpr int kGroups = score_groups<KS, KC>();
  const SmemLayout L = smem_layout<T>(kGroups, max_bands, score_slots<KS, KC>(), score_stages<T, KS, KC>());
  const int threads = consumer_threads<KS, KC>() + 32;
  auto kernel = score_kernel<T, KS, KC>;
  // The layout follows the band count of the call.  The device's limit for
  // this kernel only ever rises, so a concurrent call with fewer bands cannot
  // lower it below this launch's layout; residency is per layout and device.
  const cudaError_t e = raise_smem_limit(kernel, static_cast<int>(L.total));
  if (e != cudaSuccess) return static_cast<int>(e);
  const int resident = device_residency(kernel, threads, L.total);
  const int per_sm = resident < 1 ? 1 : resident;
  // ctas_per_sm: 0 = as many as fit; otherwise that many (capped at what fits)
  const int per = ctas_per_sm > 0 && ctas_per_sm < per_sm ? ctas_per_sm : per_sm;
  const int grid = sm_count() * per;
  kernel<<<grid, threads, L.total, stream>>>(p, max_bands);
  return static_cast<int>(cudaGetLastError());
}

template <typename T, int KS>
int dispatch_kc(int kc, const ScoreParams& p, int max_bands, int cps, cudaStream_t s) {
  switch (kc) {
    case 0: if constexpr (KS > 0) return launch_instance<T, KS, 0>(p, max_bands, cps, s); else return HSI_E_INVALID;
    case 1: return launch_instance<T, KS, 1>(p, max_bands, cps, s);
    case 4: return launch_instance<T, KS, 4>(p, max_bands, cps, s);
    case 8: return launch_instance<T, KS, 8>(p, max_bands, cps, s);
    default: return launch_instance<T, KS, 16>(p, max_bands, cps, s);
  }
}

template <typename T>
int dispatch(int ks, int kc, const ScoreParams& p, int max_bands, int cps, cudaStream_t s) {
  switch (ks) {
    case 0: return dispatch_kc<T, 0>(kc, p, max_bands, cps, s);
    case 1: return dispatch_kc<T, 1>(kc, p, max_bands, cps, s);
    case 4: return dispatch_kc<T, 4>(kc, p, max_bands, cps, s);
    case 8: return dispatch_kc<T, 8>(kc, p, max_bands, cps, s);
    default: return dispatch_kc<T, 16>(kc, p, max_bands, cps, s);
  }
}

int validate_frame(const hsi_frame& f) {
  const int64_t P = static_cast<int64_t>(f.height) * f.width;
  if (!f.cube || f.height <= 0 || f.width <= 0 || f.bands <= 0 || f.bands > HSI_MAX_BANDS) return HSI_E_INVALID;
  if (f.dtype != HSI_F32 && f.dtype != HSI_F16) return HSI_E_INVALID;
  if (f.plane_stride < P || (f.plane_stride & 7) != 0) return HSI_E_INVALID;
  if ((reinterpret_cast<uintptr_t>(f.cube) & 15u) != 0) return HSI_E_INVALID;
  if (f.num_sam < 0 || f.num_cem < 0 || (f.num_sam == 0 && f.num_cem == 0)) return HSI_E_INVALID;
  if (f.num_sam > 0 && (!f.sam_targets || !f.sam_norms)) return HSI_E_INVALID;
  if (f.num_cem > 0 && !f.cem_weights) return HSI_E_INVALID;
  if ((f.sam_maps || f.cem_maps) && f.map_stride < P) return HSI_E_INVALID;
  // Several passes carry the best cosine / response through the best map.
  if (f.num_sam > kFiltersPerPass && f.sam_best_target && !f.sam_best) return HSI_E_INVALID;
  if (f.num_cem > kFiltersPerPass && f.cem_best_target && !f.cem_best) return HSI_E_INVALID;
  return HSI_OK;
}

int pass_count_host(int total, int pass) {
  const int n = total - pass * kFiltersPerPass;
  return n < 0 ? 0 : (n > kFiltersPerPass ? kFiltersPerPass : n);
}

// One launch per pass over the cube; each pass scores up to 16 filters of each kind.
int run_passes(ScoreParams& p, int dtype, int max_bands, int max_sam, int max_cem, int cps, cudaStream_t s) {
  p.dtype = dtype;
  p.max_sam = max_sam;
  p.max_cem = max_cem;
  const int most = max_sam > max_cem ? max_sam : max_cem;
  const int passes = static_cast<int>(div_up(most, kFiltersPerPass));
  for (int pass = 0; pass < passes; ++pass) {
    p.pass = pass;
    const int ks = round_filters(pass_count_host(max_sam, pass));
    const int kc = round_filters(pass_count_host(max_cem, pass));
    const int rc = dtype == HSI_F32 ? dispatch<float>(ks, kc, p, max_bands, cps, s)
                                    : dispatch<__half>(ks, kc, p, max_bands, cps, s);
    if (rc != HSI_OK) return rc;
  }
  return HSI_OK;
}

template <int KS, int KC>
int launch_h(const HParams& p, cudaStream_t stream) {
  constexpr int N2 = 2 * ((KS + KC + 15) / 16 * 16);
  auto kernel = score_h_kernel<KS, KC>;
  const HSmem L = h_smem(p.bp, N2);
  // the largest layout, set once per device
  const cudaError_t configured = raise_smem_limit(kernel, static_cast<int>(h_smem(kHMaxBands, N2).total));
  if (configured != cudaSuccess) return static_cast<int>(configured);
  kernel<<<sm_count(), kHThreads, L.total, stream>>>(p);
  return static_cast<int>(cudaGetLastError());
}

// Tensor-core filter counts per kind: 0, 8 or 16.
int round_h(int n) { return n == 0 ? 0 : (n <= 8 ? 8 : 16); }

int dispatch_h(int ks, int kc, const HParams& p, cudaStream_t s) {
  switch (ks * 100 + kc) {
    case 8: return launch_h<0, 8>(p, s);
    case 16: return launch_h<0, 16>(p, s);
    case 800: return launch_h<8, 0>(p, s);
    case 808: return launch_h<8, 8>(p, s);
    case 816: return launch_h<8, 16>(p, s);
    case 1600: return launch_h<16, 0>(p, s);
    case 1608: return launch_h<16, 8>(p, s);
    case 1616: return launch_h<16, 16>(p, s);
    default: return HSI_E_INVALID;
  }
}

// TMA pixel coordinates are 32-bit: larger frames stay on the FMA scorer.
bool tensor_core_frame(const hsi_frame& f) {
  const int64_t P = static_cast<int64_t>(f.height) * f.width;
  return f.dtype == HSI_F16 && f.bands <= kHMaxBands && P <= (int64_t(1) << 31) - 256;
}

// Tensor-core scorer over up to 64 validated FP16 frames: a 2-D tensor map
// (128-byte swizzle, boxes of 64 pixels x all bands) per cube, one launch per
// pass.
int score_h_group(const hsi_frame* const* frames, int n, int* status, cudaStream_t s) {
  static thread_local HParams p;  // 16 KB: kept off the stack, one per host thread; the launch copies it
  p = HParams{};
  p.num_frames = n;
  p.status = status;
  int max_bands = 0;
  for (int i = 0; i < n; ++i) {
    max_bands = frames[i]->bands > max_bands ? frames[i]->bands : max_bands;
    p.max_sam = frames[i]->num_sam > p.max_sam ? frames[i]->num_sam : p.max_sam;
    p.max_cem = frames[i]->num_cem > p.max_cem ? frames[i]->num_cem : p.max_cem;
  }
  p.bp = (max_bands + 15) / 16 * 16;
  for (int i = 0; i < n; ++i) {
    const hsi_frame& f = *frames[i];
    p.frames[i] = f;
    const int64_t P = static_cast<int64_t>(f.height) * f.width;
    const int rc = encode_cube_map_sw128(&p.maps[i], f.cube, HSI_F16, P, f.bands, f.plane_stride, 64, p.bp);
    if (rc != HSI_OK) return rc;
  }
  const int most = p.max_sam > p.max_cem ? p.max_sam : p.max_cem;
  const int passes = static_cast<int>(div_up(most, kFiltersPerPass));
  for (int pass = 0; pass < passes; ++pass) {
    p.pass = pass;
    const int rc = dispatch_h(round_h(pass_count_host(p.max_sam, pass)), round_h(pass_count_host(p.max_cem, pass)),
                              p, s);
    if (rc != HSI_OK) return rc;
  }
  return HSI_OK;
}

// FP32-FMA scorer over up to 64 validated frames of one element type.
int score_fma_group(const hsi_frame* const* frames, int n, int* status, cudaStream_t s) {
  static thread_local ScoreParams p;  // 8 KB: kept off the stack, one per host thread; the launch copies it
  p = ScoreParams{};
  p.table = nullptr;
  p.num_frames = n;
  p.status = status;
  int max_bands = 0, max_sam = 0, max_cem = 0;
  for (int i = 0; i < n; ++i) {
    p.inline_frames[i] = *frames[i];
    max_bands = frames[i]->bands > max_bands ? frames[i]->bands : max_bands;
    max_sam = frames[i]->num_sam > max_sam ? frames[i]->num_sam : max_sam;
    max_cem = frames[i]->num_cem > max_cem ? frames[i]->num_cem : max_cem;
  }
  return run_passes(p, frames[0]->dtype, max_bands, max_sam, max_cem, 0, s);
}

// Frames whose descriptors are on the host: FP16 cubes of at most 128 bands
// go to the tensor-core scorer, the rest to the FP32-FMA scorer, 64 frames
// per launch.
int score_host_frames(const hsi_frame* frames, int n, int* status, cudaStream_t s) {
  if (!frames || n <= 0) return HSI_E_INVALID;
  for (int i = 0; i < n; ++i) {
    const int rc = validate_frame(frames[i]);
    if (rc != HSI_OK) return rc;
  }
  const hsi_frame* group[3][kMaxInline];  // tensor-core fp16, FMA fp32, FMA fp16
  int count[3] = {0, 0, 0};
  auto flush = [&](int g) -> int {
    if (count[g] == 0) return HSI_OK;
    const int rc = g == 0 ? score_h_group(group[0], count[0], status, s) : score_fma_group(group[g], count[g], status, s);
    count[g] = 0;
    return rc;
  };
  for (int i = 0; i < n; ++i) {
    const int g = tensor_core_frame(frames[i]) ? 0 : (frames[i].dtype == HSI_F32 ? 1 : 2);
    group[g][count[g]++] = &frames[i];
    if (count[g] == kMaxInline) {
      const int rc = flush(g);
      if (rc != HSI_OK) return rc;
    }
  }
  for (int g = 0; g < 3; ++g) {
    const int rc = flush(g);
    if (rc != HSI_OK) return rc;
  }
  return HSI_OK;
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API int hsi_score_frames_batch(const hsi_frame* frames, int num_frames, int* d_status,
                                              hsi_stream_t stream) {
  return score_host_frames(frames, num_frames, d_status, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" HSI_API int hsi_score_frames(const hsi_frame* frames, int num_frames, hsi_stream_t stream) {
  if (!frames || num_frames <= 0 || num_frames > HSI_MAX_INLINE_FRAMES) return HSI_E_INVALID;
  // one element type per call, as before
  for (int i = 1; i < num_frames; ++i)
    if (frames[i].dtype != frames[0].dtype) return HSI_E_INVALID;
  return score_host_frames(frames, num_frames, nullptr, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" HSI_API int hsi_score_frames_device_grid(const hsi_frame* d_frames, int num_frames, int dtype,
                                                    int max_bands, int max_sam, int max_cem, int* d_status,
                                                    int ctas_per_sm, hsi_stream_t stream) {
  if (!d_frames || num_frames <= 0 || num_frames > kMaxTableFrames || ctas_per_sm < 0) return HSI_E_INVALID;
  if (max_bands <= 0 || max_bands > HSI_MAX_BANDS || max_sam < 0 || max_cem < 0 || max_sam + max_cem == 0)
    return HSI_E_INVALID;
  if (dtype != HSI_F32 && dtype != HSI_F16) return HSI_E_INVALID;
  ScoreParams p{};
  p.table = d_frames;
  p.num_frames = num_frames;
  p.status = d_status;
  return run_passes(p, dtype, max_bands, max_sam, max_cem, ctas_per_sm, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" HSI_API int hsi_score_frames_device(const hsi_frame* d_frames, int num_frames, int dtype,
                                               int max_bands, int max_sam, int max_cem, int* d_status,
                                               hsi_stream_t stream) {
  if (!d_frames || num_frames <= 0 || num_frames > kMaxTableFrames) return HSI_E_INVALID;
  if (max_bands <= 0 || max_bands > HSI_MAX_BANDS || max_sam < 0 || max_cem < 0 || max_sam + max_cem == 0)
    return HSI_E_INVALID;
  if (dtype != HSI_F32 && dtype != HSI_F16) return HSI_E_INVALID;
  ScoreParams p{};
  p.table = d_frames;
  p.num_frames = num_frames;
  p.status = d_status;
  return run_passes(p, dtype, max_bands, max_sam, max_cem, 0, reinterpret_cast<cudaStream_t>(stream));
}
