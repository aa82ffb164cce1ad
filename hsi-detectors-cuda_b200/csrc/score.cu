// score.cu - SAM / CEM filter-bank scoring: one streaming pass over a BSQ cube.
//
// Design (sm_100a):
//  * Persistent CTAs walk a static schedule of 512-pixel tiles over every
//    frame of the launch (one frame, or a batch described by a device table).
//  * One producer warp streams each tile's band planes into a ring of shared
//    memory stages with 1-D bulk copies on the TMA engine (8 bands x 512 px
//    per stage), completing on mbarriers.  Nothing but the copy engine touches
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

#include "common.cuh"

namespace hsi_b200 {
namespace {

constexpr int kGroupThreads = 128;  // one consumer warpgroup
constexpr int kPPT = 4;             // pixels per consumer thread
constexpr int kTile = kGroupThreads * kPPT;
constexpr int kStageBands = 8;
constexpr int kMaxTableFrames = 256;
constexpr int kFiltersPerPass = HSI_MAX_FILTERS_PER_PASS;

template <typename T>
struct CubeTraits;
// Stage ring depth: with two consumer warpgroups two CTAs fit per SM, and
// 12 stages per SM keep ~190 KB of each SM's reads in flight.  With both
// banks in one warpgroup three CTAs fit (the warps hide the packed FMAs'
// latency better), with 4 stages each for FP32.
template <>
struct CubeTraits<float> {
  static constexpr int kStages = 6;
  static constexpr int kStagesFused = 4;
};
template <>
struct CubeTraits<__half> {
  static constexpr int kStages = 10;
  static constexpr int kStagesFused = 7;
};

struct ScoreParams {
  const hsi_frame* table;  // device descriptor table, or null for inline frames
  hsi_frame inline_frames[HSI_MAX_INLINE_FRAMES];
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

__device__ __forceinline__ void named_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

__device__ __forceinline__ int find_frame(const int* prefix, int n, int tile) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}

struct SmemLayout {
  size_t stage_bytes, filt_off, scale_off, bar_off, prefix_off, total;
};

template <typename T>
__host__ __device__ inline SmemLayout smem_layout(int groups, int max_bands, int slots, int stages) {
  SmemLayout l;
  l.stage_bytes = static_cast<size_t>(kStageBands) * kTile * sizeof(T);
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

// Packed FP32 FMA on sm_100: two lanes per instruction, d = a * b + c.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;"
      : "=l"(r)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)),
        "l"(*reinterpret_cast<unsigned long long*>(&c)));
  return *reinterpret_cast<float2*>(&r);
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
  if (nb == kStageBands) {
#pragma unroll
    for (int i = 0; i < kStageBands; ++i) band(i);
  } else {
    for (int i = 0; i < nb; ++i) band(i);
  }
}

__device__ __forceinline__ float angle_of_cos(float c) { return acosf(fminf(fmaxf(c, -1.0f), 1.0f)); }

__device__ __forceinline__ void store4(float* dst, const float v[kPPT], int valid, bool vec) {
  if (vec && valid == kPPT) {
    *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
#pragma unroll
    for (int j = 0; j < kPPT; ++j)
      if (j < valid) dst[j] = v[j];
  }
}

__device__ __forceinline__ void store4i(int32_t* dst, const int32_t v[kPPT], int valid, bool vec) {
  if (vec && valid == kPPT) {
    *reinterpret_cast<int4*>(dst) = make_int4(v[0], v[1], v[2], v[3]);
  } else {
#pragma unroll
    for (int j = 0; j < kPPT; ++j)
      if (j < valid) dst[j] = v[j];
  }
}

__device__ __forceinline__ bool aligned16(const void* p) {
  return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

// SAM epilogue for one thread's 4 pixels starting at frame pixel p.
template <int KG>
__device__ void sam_epilogue(const hsi_frame& F, int pass, int n_f, int64_t p, int valid,
                             const float (&acc)[KG][kPPT], const float (&nrm)[kPPT], const float* scale) {
  {
    const bool first = pass == 0;
    const bool last = pass_count(F.num_sam, pass + 1) == 0;
    const int t0 = pass * kFiltersPerPass;
    float rn[kPPT], best[kPPT];
    int32_t best_t[kPPT];
#pragma unroll
    for (int j = 0; j < kPPT; ++j) {
      rn[j] = nrm[j] > 0.0f ? rsqrtf(nrm[j]) : 0.0f;
      best[j] = -2.0f;
      best_t[j] = -1;
    }
    if (!first) {
#pragma unroll
      for (int j = 0; j < kPPT; ++j) {
        if (j >= valid) continue;
        if (F.sam_best) best[j] = F.sam_best[p + j];
        if (F.sam_best_target) best_t[j] = F.sam_best_target[p + j];
      }
    }
    const bool vec_maps = F.sam_maps && aligned16(F.sam_maps) && (F.map_stride & 3) == 0;
#pragma unroll
    for (int k = 0; k < KG; ++k) {
      if (k < n_f) {
        float c[kPPT];
#pragma unroll
        for (int j = 0; j < kPPT; ++j) {
          c[j] = acc[k][j] * rn[j] * scale[k];
          if (c[j] > best[j]) {
            best[j] = c[j];
            best_t[j] = t0 + k;
          }
        }
        if (F.sam_maps) {
          float a[kPPT];
#pragma unroll
          for (int j = 0; j < kPPT; ++j) a[j] = angle_of_cos(c[j]);
          store4(F.sam_maps + static_cast<int64_t>(t0 + k) * F.map_stride + p, a, valid, vec_maps);
        }
      }
    }
    if (F.sam_best) {
      float out[kPPT];
#pragma unroll
      for (int j = 0; j < kPPT; ++j) out[j] = last ? angle_of_cos(best[j]) : best[j];
      store4(F.sam_best + p, out, valid, aligned16(F.sam_best));
    }
    if (F.sam_best_target) store4i(F.sam_best_target + p, best_t, valid, aligned16(F.sam_best_target));
  }
}

template <int KG>
__device__ void cem_epilogue(const hsi_frame& F, int pass, int n_f, int64_t p, int valid,
                             const float (&acc)[KG][kPPT]) {
  {
    const bool first = pass == 0;
    const int t0 = pass * kFiltersPerPass;
    float best[kPPT];
    int32_t best_t[kPPT];
#pragma unroll
    for (int j = 0; j < kPPT; ++j) {
      best[j] = -INFINITY;
      best_t[j] = -1;
    }
    if (!first) {
#pragma unroll
      for (int j = 0; j < kPPT; ++j) {
        if (j >= valid) continue;
        if (F.cem_best) best[j] = F.cem_best[p + j];
        if (F.cem_best_target) best_t[j] = F.cem_best_target[p + j];
      }
    }
    const bool vec_maps = F.cem_maps && aligned16(F.cem_maps) && (F.map_stride & 3) == 0;
#pragma unroll
    for (int k = 0; k < KG; ++k) {
      if (k < n_f) {
        float r[kPPT];
#pragma unroll
        for (int j = 0; j < kPPT; ++j) {
          r[j] = acc[k][j];
          if (r[j] > best[j]) {
            best[j] = r[j];
            best_t[j] = t0 + k;
          }
        }
        if (F.cem_maps) store4(F.cem_maps + static_cast<int64_t>(t0 + k) * F.map_stride + p, r, valid, vec_maps);
      }
    }
    if (F.cem_best) store4(F.cem_best + p, best, valid, aligned16(F.cem_best));
    if (F.cem_best_target) store4i(F.cem_best_target + p, best_t, valid, aligned16(F.cem_best_target));
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
  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    const int f = find_frame(prefix, nframes, tile);
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

    for (int b0 = 0; b0 < B; b0 += kStageBands) {
      const int nb = B - b0 < kStageBands ? B - b0 : kStageBands;
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
          sam_epilogue<KG>(F, prm.pass, n_f, p, valid, a, n, scale);
        } else {
          cem_epilogue<KG>(F, prm.pass, n_f, p, valid, a);
        }
      }
    }
  }
}

// Fused consumer: one warpgroup scores the SAM and the CEM bank together, so
// each pixel leaves shared memory once for all KS + KC filters.  The bank is
// stored band-major without duplication, [b][KS SAM | KC CEM]; accumulators
// are filter pairs per pixel, (acc_k, acc_k+1) += (x, x) * (f_k, f_k+1), the
// pixel duplicated in a register pair for the packed FMA.
template <typename T, int K>
__device__ __forceinline__ void consume_stage_fused(const T* stage, const float* filt, int nb, int tid,
                                                    float2 (&acc)[K / 2][kPPT], float2 (&nrm)[2]) {
  const T* src = stage + tid * kPPT;
  auto band = [&](int i) {
    float v[kPPT];
    load4<T>(src + i * kTile, v);
    const float2 v01 = make_float2(v[0], v[1]), v23 = make_float2(v[2], v[3]);
    nrm[0] = ffma2(v01, v01, nrm[0]);
    nrm[1] = ffma2(v23, v23, nrm[1]);
    float2 d[kPPT];
#pragma unroll
    for (int j = 0; j < kPPT; ++j) d[j] = make_float2(v[j], v[j]);
    const float* fr = filt + i * K;
#pragma unroll
    for (int k = 0; k < K; k += 4) {
      const float4 f = ld_shared_f4(fr + k);  // (f_k, f_k+1, f_k+2, f_k+3)
      const float2 fa = make_float2(f.x, f.y), fb = make_float2(f.z, f.w);
#pragma unroll
      for (int j = 0; j < kPPT; ++j) {
        acc[k / 2][j] = ffma2(d[j], fa, acc[k / 2][j]);
        acc[k / 2 + 1][j] = ffma2(d[j], fb, acc[k / 2 + 1][j]);
      }
    }
  };
  if (nb == kStageBands) {
#pragma unroll
    for (int i = 0; i < kStageBands; ++i) band(i);
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
  const int nframes = prm.num_frames;
  int cur_frame = -1;
  int n_s = 0, n_c = 0;
  uint32_t it = 0;
  bool aborted = false;
  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    const int f = find_frame(prefix, nframes, tile);
    const hsi_frame& F = frame_at(prm, f);
    const int B = F.bands;
    if (f != cur_frame) {
      named_sync(1, kGroupThreads);
      n_s = pass_count(F.num_sam, prm.pass);
      n_c = pass_count(F.num_cem, prm.pass);
      const int t0 = prm.pass * kFiltersPerPass;
      for (int i = tid; i < B * K; i += kGroupThreads) {
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
      named_sync(1, kGroupThreads);
      cur_frame = f;
    }
    const int64_t P = static_cast<int64_t>(F.height) * F.width;
    const int64_t p0 = static_cast<int64_t>(tile - prefix[f]) * kTile;
    const bool active = n_s > 0 || n_c > 0;

    float2 acc[K / 2][kPPT];
    float2 nrm[2] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
#pragma unroll
    for (int k = 0; k < K / 2; ++k)
#pragma unroll
      for (int j = 0; j < kPPT; ++j) acc[k][j] = make_float2(0.0f, 0.0f);

    for (int b0 = 0; b0 < B; b0 += kStageBands) {
      const int nb = B - b0 < kStageBands ? B - b0 : kStageBands;
      const int slot = static_cast<int>(it % kStages);
      const uint32_t round = it / kStages;
      if (!aborted && !mbar_wait(&full[slot], round & 1u)) {
        record_error(prm.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        aborted = true;
      }
      if (active && !aborted) {
        const T* stage = reinterpret_cast<const T*>(smem + slot * stage_bytes);
        consume_stage_fused<T, K>(stage, filt + b0 * K, nb, tid, acc, nrm);
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
        if (n_s > 0) {
          float a[KS][kPPT];
#pragma unroll
          for (int k = 0; k < KS; ++k)
#pragma unroll
            for (int j = 0; j < kPPT; ++j) a[k][j] = (k & 1) ? acc[k / 2][j].y : acc[k / 2][j].x;
          const float n[kPPT] = {nrm[0].x, nrm[0].y, nrm[1].x, nrm[1].y};
          sam_epilogue<KS>(F, prm.pass, n_s, p, valid, a, n, scale);
        }
        if (n_c > 0) {
          float a[KC][kPPT];
#pragma unroll
          for (int k = 0; k < KC; ++k)
#pragma unroll
            for (int j = 0; j < kPPT; ++j)
              a[k][j] = ((KS + k) & 1) ? acc[(KS + k) / 2][j].y : acc[(KS + k) / 2][j].x;
          cem_epilogue<KC>(F, prm.pass, n_c, p, valid, a);
        }
      }
    }
  }
}

// Both banks in one warpgroup: 4 or 8 filters of each kind.
template <int KS, int KC>
constexpr bool fused_banks() {
  return (KS == 4 || KS == 8) && (KC == 4 || KC == 8);
}

// Kernel: KS SAM filters and KC CEM filters per pass (0 = that warpgroup is
// absent; both in one warpgroup when fused_banks).  Block = (groups * 128 +
// 32) threads; the last warp produces.
template <int KS, int KC>
constexpr int score_groups() {
  return fused_banks<KS, KC>() ? 1 : (KS > 0) + (KC > 0);
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
__global__ void __launch_bounds__(score_groups<KS, KC>() * kGroupThreads + 32, fused_banks<KS, KC>() ? 3 : 1)
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
      mbar_init(&empty[s], kGroups * (kGroupThreads / 32));
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

  if (warp == kGroups * (kGroupThreads / 32)) {
    // ---------------- producer warp ----------------
    if (lane == 0) {
      uint32_t it = 0;
      bool aborted = false;
      uint32_t pending = 0;         // bit s: slot s has copies issued
      uint32_t pending_parity = 0;  // bit s: phase parity of that issue
      for (int tile = blockIdx.x; tile < total_tiles && !aborted; tile += gridDim.x) {
        const int f = find_frame(prefix, nframes, tile);
        const hsi_frame& F = frame_at(prm, f);
        const int64_t P = static_cast<int64_t>(F.height) * F.width;
        const int64_t p0 = static_cast<int64_t>(tile - prefix[f]) * kTile;
        const int npx = static_cast<int>(P - p0 < kTile ? P - p0 : kTile);
        const uint32_t bytes = static_cast<uint32_t>(((npx + 7) & ~7) * sizeof(T));
        const T* cube = static_cast<const T*>(F.cube);
        for (int b0 = 0; b0 < F.bands; b0 += kStageBands) {
          const int nb = F.bands - b0 < kStageBands ? F.bands - b0 : kStageBands;
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
  const int group = warp / (kGroupThreads / 32);  // 0: SAM if KS > 0, else CEM; 1: CEM
  const int tid = threadIdx.x - group * kGroupThreads;
  float* filt = reinterpret_cast<float*>(smem + L.filt_off) + static_cast<size_t>(group) * max_bands * kSlots;
  float* scale = reinterpret_cast<float*>(smem + L.scale_off) + group * kFiltersPerPass;
  if constexpr (fused_banks<KS, KC>()) {
    consumer_loop_fused<T, KS, KC, kStages>(prm, prefix, total_tiles, smem, L.stage_bytes, full, empty, abort_flag,
                                            filt, scale, tid, lane);
    return;
  }
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
// Host side
// ---------------------------------------------------------------------------

int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

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
  const int threads = kGroups * kGroupThreads + 32;
  auto kernel = score_kernel<T, KS, KC>;
  static int configured_bytes = -1;
  static int per_sm = 0;
  if (configured_bytes != static_cast<int>(L.total)) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(L.total));
    if (e != cudaSuccess) return static_cast<int>(e);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, L.total);
    if (e != cudaSuccess) return static_cast<int>(e);
    if (per_sm < 1) per_sm = 1;
    configured_bytes = static_cast<int>(L.total);
  }
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

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API int hsi_score_frames(const hsi_frame* frames, int num_frames, hsi_stream_t stream) {
  if (!frames || num_frames <= 0 || num_frames > HSI_MAX_INLINE_FRAMES) return HSI_E_INVALID;
  ScoreParams p{};
  p.table = nullptr;
  p.num_frames = num_frames;
  p.status = nullptr;
  int max_bands = 0, max_sam = 0, max_cem = 0;
  const int dtype = frames[0].dtype;
  for (int i = 0; i < num_frames; ++i) {
    const int rc = validate_frame(frames[i]);
    if (rc != HSI_OK) return rc;
    if (frames[i].dtype != dtype) return HSI_E_INVALID;
    p.inline_frames[i] = frames[i];
    max_bands = frames[i].bands > max_bands ? frames[i].bands : max_bands;
    max_sam = frames[i].num_sam > max_sam ? frames[i].num_sam : max_sam;
    max_cem = frames[i].num_cem > max_cem ? frames[i].num_cem : max_cem;
  }
  return run_passes(p, dtype, max_bands, max_sam, max_cem, 0, reinterpret_cast<cudaStream_t>(stream));
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
