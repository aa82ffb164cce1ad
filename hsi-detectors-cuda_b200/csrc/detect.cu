// detect.cu - threshold + non-maximum suppression + ordered compaction.
//
// Three launches for a whole batch of score maps, no atomics on the data
// path, so every list comes out in raster order and is identical run to run:
//   1. flags:  per tile of 256 columns x 64 rows of one map, every pixel's
//              pass/fail as warp ballot words (a bitmask in the workspace:
//              one word per 32 pixels of a 2048-pixel row segment).  The
//              map's rows stream through a shared-memory ring (cp.async, four
//              rows ahead).  Per row, each column's first-best score of the
//              (2r+1)-row window (better score, then lower row) is found
//              once; a candidate passes when none of the 2r+1 column bests
//              around it comes first in the window's order (better score,
//              then lower linear index).  Out-of-frame neighbours are NaN,
//              which never win or tie, exactly like the bounds checks of the
//              CPU loop.  Radii above 8 read each candidate's window from
//              global memory instead.  Maps of radius <= 4 whose width is a
//              multiple of 4 (and whose rows therefore start on 16 bytes)
//              take a second kernel with the same steps over 512-column
//              tiles: four columns per thread, 16-byte copies, polarity
//              fixed at compile time;
//   2. scan:   one block per map counts each row segment's passing pixels
//              (popcounts of its mask words), turns the counts into output
//              offsets starting at the caller's *count, and advances *count;
//   3. emit:   one warp per segment writes its detections at offset +
//              in-segment rank, dropping (but having counted) those past
//              capacity; segments whose count is zero cost one load.
// Semantics are the reference CPU path's (src/sam_cpu.cpp:86-138), polarity
// included; the reference GPU kernel (src/detect.cu:43-87) ignores polarity
// and emits in atomic arrival order, both of which this replaces.
#include <cuda.h>

#include <mutex>

#include "common.cuh"
#include "launch_state.h"

namespace hsi_b200 {
namespace {

constexpr int kThreads = 256;                // scan / emit blocks
constexpr int kPerThread = 8;
constexpr int kSeg = kThreads * kPerThread;  // 2048 pixels per row segment
constexpr int kWordsPerSeg = kSeg / 32;      // 64
constexpr int kMaxJobs = 64;
// flags tiles
constexpr int kTileW = 256;                        // columns per tile (8 ballot warps)
constexpr int kTileH = 64;                         // rows per tile
constexpr int kMaxRingR = 8;                       // largest radius streamed through the ring
constexpr int kAhead = 4;                          // rows in flight ahead of the window
constexpr int kRing = 32;                          // ring rows (a power of two >= window + spare + in flight)
static_assert(kRing >= 2 * kMaxRingR + 2 + kAhead, "ring too small for the window");
constexpr int kRingCols = kTileW + 2 * kMaxRingR;  // 272
constexpr int kFlagThreads = 288;                  // >= kRingCols, whole warps
// fast flags tiles (radius <= kFastR, width a multiple of 4)
constexpr int kFastW = 512;                        // columns per tile, four per candidate thread
constexpr int kFastR = 4;                          // largest radius; also the halo of a ring row
constexpr int kFastGroups = kFastW / 4 + 2;        // float4 groups of a ring row (one halo group each side)
constexpr int kFastAhead = 6;                      // rows in flight ahead of the window
constexpr int kFastRing = 16;                      // ring rows
static_assert(kFastRing >= 2 * kFastR + kFastAhead + 2, "fast ring too small for the window");
constexpr int kFastThreads = 160;                  // >= kFastGroups, whole warps

struct Job {
  const float* score;
  const int32_t* target;
  int height, width;
  float threshold;
  int radius;
  int higher;
  int capacity;
  hsi_detection* out;
  uint32_t* count;
  int seg0;          // first segment of this map in the batch
  int segs_per_row;  // ceil(width / kSeg)
  int tile0;         // first flags tile of this map among the maps of its kind
  int tiles_x;       // ceil(width / tile width of its kind)
};

struct Batch {
  Job jobs[kMaxJobs];
  int njobs;
  int total_segs;
  int kind_jobs[2][kMaxJobs];  // job indices of the plain (0) and fast (1) flags kinds, in batch order
  int kind_n[2];
  int kind_tiles[2];
  uint32_t* counts;   // [total_segs]
  uint32_t* offsets;  // [total_segs]
  uint32_t* masks;    // [total_segs * 64]
};

__device__ __forceinline__ int find_job(const Batch& b, int seg) {
  int lo = 0, hi = b.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.jobs[mid].seg0 <= seg) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Job of flags tile `tile` of kind `kind` (0 plain, 1 fast).
__device__ __forceinline__ int find_job_tile(const Batch& b, int kind, int tile) {
  int lo = 0, hi = b.kind_n[kind] - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.jobs[b.kind_jobs[kind][mid]].tile0 <= tile) lo = mid; else hi = mid - 1;
  }
  return b.kind_jobs[kind][lo];
}

__device__ __forceinline__ bool better(float a, float b, bool higher) { return higher ? a > b : a < b; }

__device__ __forceinline__ bool over_threshold(float s, float threshold, bool higher) {
  return higher ? s >= threshold : s <= threshold;  // NaN fails both
}

// Mask word of the 32 pixels of row y starting at column xw (a multiple of 32).
__device__ __forceinline__ uint32_t* mask_word(const Batch& b, const Job& J, int y, int xw) {
  return b.masks + static_cast<int64_t>(J.seg0 + y * J.segs_per_row + xw / kSeg) * kWordsPerSeg + (xw % kSeg) / 32;
}

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// NMS against global memory, for radii too large for the ring.
__device__ bool local_best_global(const float* __restrict__ s, int x, int y, int w, int h, int r, float self,
                                  bool higher) {
  const int64_t self_idx = static_cast<int64_t>(y) * w + x;
  for (int dy = -r; dy <= r; ++dy) {
    const int ny = y + dy;
    if (ny < 0 || ny >= h) continue;
    for (int dx = -r; dx <= r; ++dx) {
      if (dx == 0 && dy == 0) continue;
      const int nx = x + dx;
      if (nx < 0 || nx >= w) continue;
      const int64_t n = static_cast<int64_t>(ny) * w + nx;
      const float o = __ldg(s + n);
      if (better(o, self, higher)) return false;
      if (o == self && n < self_idx) return false;
    }
  }
  return true;
}

// Shared memory of one flags tile.
struct FlagsSmem {
  float ring[kRing][kRingCols];   // score rows, NaN outside the frame
  float2 best[2][kRingCols];      // per column: (first-best score of the window, its row 0 .. 2r as int bits)
  float centre[2][kRingCols];     // per column: the centre row's score
};

// One tile whose window radius R is known at compile time (0 .. kMaxRingR).
template <int R>
__device__ __forceinline__ void flags_tile(const Batch& b, const Job& J, FlagsSmem& sm, int x0, int y0, int y1) {
  constexpr int kCols = kTileW + 2 * R;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const float nan = __int_as_float(0x7fc00000);
  const int W = J.width, H = J.height;
  const bool higher = J.higher != 0;
  const float thr = J.threshold;
  const int cx = x0 - R + t;  // this thread's column in the vertical pass
  const bool col_in = t < kCols && cx >= 0 && cx < W;
  const int last = y1 - 1 + R;  // last row the tile reads
  // One ring row per call: a 4-byte cp.async per in-frame column, NaN stored
  // directly elsewhere, and one commit group per thread per call.
  int next_row = y0 - R;
  auto issue_next = [&]() {
    if (next_row <= last && t < kCols) {
      float* dst = &sm.ring[next_row & (kRing - 1)][t];
      if (col_in && next_row >= 0 && next_row < H)
        cp_async4(dst, J.score + static_cast<int64_t>(next_row) * W + cx);
      else
        *dst = nan;
    }
    cp_async_commit();
    ++next_row;
  };
#pragma unroll
  for (int k = 0; k < 2 * R + kAhead; ++k) issue_next();
  for (int y = y0; y <= y1; ++y) {
    // row y + R + kAhead reuses the slot of row y + R + kAhead - kRing, at
    // most y - R - 2, whose last reader passed the previous barrier
    if (y < y1) issue_next();
    cp_async_wait<kAhead>();  // this thread's copies up to row y + R have landed
    __syncthreads();          // ... and everyone's
    if (y > y0 && t < kTileW) {
      // candidates of row y - 1 against the column bests around them
      const int yh = y - 1, hb = yh & 1;
      const int x = x0 + t;
      bool pass = false;
      if (x < W) {
        const float s = sm.centre[hb][t + R];
        if (over_threshold(s, thr, higher)) {
          pass = true;
#pragma unroll
          for (int dx = -R; dx <= R; ++dx) {
            const float2 vk = sm.best[hb][t + R + dx];
            const float v = vk.x;
            const int k = __float_as_int(vk.y);
            // first in the window's order: better score, or the same score
            // at a lower linear index (an earlier row, or this row to the left)
            if (!isnan(v) && (better(v, s, higher) || (v == s && (k < R || (k == R && dx < 0))))) pass = false;
          }
        }
      }
      const uint32_t word = __ballot_sync(0xffffffffu, pass);
      if (lane == 0 && x0 + 32 * warp < W) *mask_word(b, J, yh, x0 + 32 * warp) = word;
    }
    if (y < y1 && t < kCols) {
      // column t's first-best over rows y - R .. y + R
      float bv = nan;
      int bk = 0;
#pragma unroll
      for (int k = 0; k <= 2 * R; ++k) {
        const float v = sm.ring[(y - R + k) & (kRing - 1)][t];
        if (!isnan(v) && (isnan(bv) || better(v, bv, higher))) {
          bv = v;
          bk = k;
        }
        if (k == R) sm.centre[y & 1][t] = v;
      }
      sm.best[y & 1][t] = make_float2(bv, __int_as_float(bk));
    }
  }
}

// A tile whose radius is too large for the ring: each candidate's window
// read from global memory.
__device__ void flags_tile_global(const Batch& b, const Job& J, int x0, int y0, int y1) {
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int r = J.radius;
  const bool higher = J.higher != 0;
  for (int y = y0; y < y1; ++y) {
    if (t >= kTileW) continue;
    const int x = x0 + t;
    bool pass = false;
    if (x < J.width) {
      const float s = J.score[static_cast<int64_t>(y) * J.width + x];
      pass = over_threshold(s, J.threshold, higher) &&
             local_best_global(J.score, x, y, J.width, J.height, r, s, higher);
    }
    const uint32_t word = __ballot_sync(0xffffffffu, pass);
    if (lane == 0 && x0 + 32 * warp < J.width) *mask_word(b, J, y, x0 + 32 * warp) = word;
  }
}

__global__ void __launch_bounds__(kFlagThreads) flags_kernel(const __grid_constant__ Batch b) {
  __shared__ FlagsSmem sm;
  for (int tile = blockIdx.x; tile < b.kind_tiles[0]; tile += gridDim.x) {
    __syncthreads();  // the previous tile is done with the shared buffers
    const Job& J = b.jobs[find_job_tile(b, 0, tile)];
    const int local = tile - J.tile0;
    const int x0 = (local % J.tiles_x) * kTileW;
    const int y0 = (local / J.tiles_x) * kTileH;
    const int y1 = min(J.height, y0 + kTileH);
    switch (J.radius > 0 ? J.radius : 0) {
      case 0: flags_tile<0>(b, J, sm, x0, y0, y1); break;
      case 1: flags_tile<1>(b, J, sm, x0, y0, y1); break;
      case 2: flags_tile<2>(b, J, sm, x0, y0, y1); break;
      case 3: flags_tile<3>(b, J, sm, x0, y0, y1); break;
      case 4: flags_tile<4>(b, J, sm, x0, y0, y1); break;
      case 5: flags_tile<5>(b, J, sm, x0, y0, y1); break;
      case 6: flags_tile<6>(b, J, sm, x0, y0, y1); break;
      case 7: flags_tile<7>(b, J, sm, x0, y0, y1); break;
      case 8: flags_tile<8>(b, J, sm, x0, y0, y1); break;
      default: flags_tile_global(b, J, x0, y0, y1); break;
    }
  }
}

// Shared memory of one fast flags tile: ring rows as float4 groups starting
// kFastR columns left of the tile, and per group the column bests of the
// window (score, row 0 .. 2r) for two consecutive rows.
struct FastSmem {
  float4 ring[kFastRing][kFastGroups];
  float4 bv[2][kFastGroups];
  int4 bk[2][kFastGroups];
};

template <bool HIGHER>
__device__ __forceinline__ bool better_t(float a, float b) { return HIGHER ? a > b : a < b; }

// Column c's first-best update with the value v of window row k (NaN never
// wins; the first non-NaN value always does).
template <bool HIGHER>
__device__ __forceinline__ void best_update(float v, int k, float& bv, int& bk) {
  if (!isnan(v) && (isnan(bv) || better_t<HIGHER>(v, bv))) {
    bv = v;
    bk = k;
  }
}

// Bits 0..7 of x moved to bits 0, 4, .., 28.
__device__ __forceinline__ uint32_t spread4(uint32_t x) {
  x = (x | (x << 12)) & 0x000F000Fu;
  x = (x | (x << 6)) & 0x03030303u;
  x = (x | (x << 3)) & 0x11111111u;
  return x;
}

// One fast tile: the steps of flags_tile with four adjacent columns per
// thread.  Thread g < kFastGroups copies and reduces ring group g (columns
// x0 - kFastR + 4g ..); thread t < kFastW / 4 tests columns x0 + 4t .. + 3,
// whose windows lie in groups t .. t + 2.  The width is a multiple of 4, so
// a group lies wholly inside or wholly outside the frame.
template <int R, bool HIGHER>
__device__ __forceinline__ void flags_fast_tile(const Batch& b, const Job& J, FastSmem& sm, int x0, int y0, int y1) {
  static_assert(R <= kFastR, "radius above the fast halo");
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const float nan = __int_as_float(0x7fc00000);
  const float4 nan4 = make_float4(nan, nan, nan, nan);
  const int W = J.width, H = J.height;
  const float thr = J.threshold;
  const bool loader = t < kFastGroups;
  const int gx = x0 - kFastR + 4 * t;  // first column of this thread's group
  const bool col_in = loader && gx >= 0 && gx < W;
  const int last = y1 - 1 + R;  // last row the tile reads
  int next_row = y0 - R;
  auto issue_next = [&]() {
    if (next_row <= last && loader) {
      float4* dst = &sm.ring[next_row & (kFastRing - 1)][t];
      if (col_in && next_row >= 0 && next_row < H)
        cp_async16(dst, J.score + static_cast<int64_t>(next_row) * W + gx);
      else
        *dst = nan4;
    }
    cp_async_commit();
    ++next_row;
  };
#pragma unroll
  for (int k = 0; k < 2 * R + kFastAhead; ++k) issue_next();
  for (int y = y0; y <= y1; ++y) {
    // row y + R + kFastAhead reuses the slot of row y + R + kFastAhead -
    // kFastRing <= y - R - 2; the rows still read are y - 1 - R and later
    if (y < y1) issue_next();
    cp_async_wait<kFastAhead>();  // this thread's copies up to row y + R have landed
    __syncthreads();              // ... and everyone's
    if (y > y0 && t < kFastW / 4) {
      // candidates of row y - 1 (its scores are still in the ring) against
      // the column bests around them
      const int yh = y - 1, hb = yh & 1;
      const float4 c4 = sm.ring[yh & (kFastRing - 1)][t + 1];
      const float s[4] = {c4.x, c4.y, c4.z, c4.w};
      float v[12];
      int k[12];
#pragma unroll
      for (int g = 0; g < 3; ++g) {
        const float4 a = sm.bv[hb][t + g];
        const int4 q = sm.bk[hb][t + g];
        v[4 * g] = a.x; v[4 * g + 1] = a.y; v[4 * g + 2] = a.z; v[4 * g + 3] = a.w;
        k[4 * g] = q.x; k[4 * g + 1] = q.y; k[4 * g + 2] = q.z; k[4 * g + 3] = q.w;
      }
      const bool in = x0 + 4 * t < W;
      uint32_t word[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        bool pass = in && (HIGHER ? s[j] >= thr : s[j] <= thr);  // NaN fails both
#pragma unroll
        for (int dx = -R; dx <= R; ++dx) {
          const int o = kFastR + j + dx;
          // first in the window's order: better score, or the same score at
          // a lower linear index (an earlier row, or this row to the left)
          const bool earlier = dx < 0 ? k[o] <= R : k[o] < R;
          if (better_t<HIGHER>(v[o], s[j]) || (v[o] == s[j] && earlier)) pass = false;
        }
        word[j] = __ballot_sync(0xffffffffu, pass);  // bit l: column 4l + j of the warp's 128
      }
      if (lane < 4) {
        // mask word `lane` of the warp: its columns 32 lane + 4i + j come
        // from bit 8 lane + i of word[j]
        uint32_t m = 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j) m |= spread4((word[j] >> (8 * lane)) & 0xffu) << j;
        const int xw = x0 + 128 * warp + 32 * lane;
        if (xw < W) *mask_word(b, J, yh, xw) = m;
      }
    }
    if (y < y1 && loader) {
      // group t's column first-bests over rows y - R .. y + R
      float4 bv = nan4;
      int4 bk = make_int4(0, 0, 0, 0);
#pragma unroll
      for (int k = 0; k <= 2 * R; ++k) {
        const float4 a = sm.ring[(y - R + k) & (kFastRing - 1)][t];
        best_update<HIGHER>(a.x, k, bv.x, bk.x);
        best_update<HIGHER>(a.y, k, bv.y, bk.y);
        best_update<HIGHER>(a.z, k, bv.z, bk.z);
        best_update<HIGHER>(a.w, k, bv.w, bk.w);
      }
      sm.bv[y & 1][t] = bv;
      sm.bk[y & 1][t] = bk;
    }
  }
}

template <bool HIGHER>
__device__ __forceinline__ void flags_fast_dispatch(const Batch& b, const Job& J, FastSmem& sm, int x0, int y0,
                                                    int y1) {
  switch (J.radius > 0 ? J.radius : 0) {
    case 0: flags_fast_tile<0, HIGHER>(b, J, sm, x0, y0, y1); break;
    case 1: flags_fast_tile<1, HIGHER>(b, J, sm, x0, y0, y1); break;
    case 2: flags_fast_tile<2, HIGHER>(b, J, sm, x0, y0, y1); break;
    case 3: flags_fast_tile<3, HIGHER>(b, J, sm, x0, y0, y1); break;
    default: flags_fast_tile<4, HIGHER>(b, J, sm, x0, y0, y1); break;  // the host admits radius <= kFastR only
  }
}

__global__ void __launch_bounds__(kFastThreads) flags_fast_kernel(const __grid_constant__ Batch b) {
  __shared__ FastSmem sm;
  for (int tile = blockIdx.x; tile < b.kind_tiles[1]; tile += gridDim.x) {
    __syncthreads();  // the previous tile is done with the shared buffers
    const Job& J = b.jobs[find_job_tile(b, 1, tile)];
    const int local = tile - J.tile0;
    const int x0 = (local % J.tiles_x) * kFastW;
    const int y0 = (local / J.tiles_x) * kTileH;
    const int y1 = min(J.height, y0 + kTileH);
    if (J.higher)
      flags_fast_dispatch<true>(b, J, sm, x0, y0, y1);
    else
      flags_fast_dispatch<false>(b, J, sm, x0, y0, y1);
  }
}

// Passing pixels of segment `seg` of job J: popcount of its mask words that
// cover pixels of the map (words past the row's end are never written).
__device__ __forceinline__ int seg_words(const Job& J, int local) {
  const int xs = (local % J.segs_per_row) * kSeg;
  const int len = min(kSeg, J.width - xs);
  return (len + 31) / 32;
}

// One block per map: segment counts from the masks, their exclusive scan from
// *count; *count += total.
__global__ void __launch_bounds__(1024) scan_kernel(const __grid_constant__ Batch b) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  const Job& J = b.jobs[blockIdx.x];
  const int segs = J.height * J.segs_per_row;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) s_carry = *J.count;
  __syncthreads();
  for (int chunk = 0; chunk < segs; chunk += 1024) {
    // warp w counts segments chunk + 32 w .. + 31, one per step; lane k
    // keeps the count of segment chunk + 32 w + k (= this thread's)
    uint32_t v = 0u;
    for (int k = 0; k < 32; ++k) {
      const int si = chunk + warp * 32 + k;
      uint32_t c = 0u;
      if (si < segs) {
        const int nw = seg_words(J, si);
        const uint32_t* m = b.masks + static_cast<int64_t>(J.seg0 + si) * kWordsPerSeg;
        c = (lane < nw ? __popc(m[lane]) : 0) + (lane + 32 < nw ? __popc(m[lane + 32]) : 0);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if (lane == k) v = c;
    }
    const int i = chunk + threadIdx.x;
    if (i < segs) b.counts[J.seg0 + i] = v;
    uint32_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = s_warp[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, w, d);
        if (lane >= d) w += o;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t warp_base = warp > 0 ? s_warp[warp - 1] : 0u;
    const uint32_t carry = s_carry;
    if (i < segs) b.offsets[J.seg0 + i] = carry + warp_base + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + s_warp[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *J.count = s_carry;
}

// One warp per segment.  Lane l holds mask words l and l + 32, their
// exclusive prefix of popcounts comes from two shuffle scans, and the warp
// then visits the non-empty words in order with lane = bit, so that the
// detections of one word go to consecutive slots in one coalesced store.
__global__ void __launch_bounds__(kThreads) emit_kernel(const __grid_constant__ Batch b) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (kThreads / 32);
  const uint32_t lt = (1u << lane) - 1u;
  for (int seg = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); seg < b.total_segs; seg += warps) {
    const uint32_t count = b.counts[seg];
    if (count == 0u) continue;  // nothing passed in this segment (the same for the whole warp)
    const Job& J = b.jobs[find_job(b, seg)];
    const int local = seg - J.seg0;
    const int nw = seg_words(J, local);
    const uint32_t* m = b.masks + static_cast<int64_t>(seg) * kWordsPerSeg;
    const uint32_t w0 = lane < nw ? m[lane] : 0u;
    const uint32_t w1 = lane + 32 < nw ? m[lane + 32] : 0u;
    const uint32_t base = b.offsets[seg];
    const uint32_t c0 = __popc(w0), c1 = __popc(w1);
    uint32_t i0 = c0, i1 = c1;  // inclusive scans over the lanes
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o0 = __shfl_up_sync(0xffffffffu, i0, d);
      const uint32_t o1 = __shfl_up_sync(0xffffffffu, i1, d);
      if (lane >= d) {
        i0 += o0;
        i1 += o1;
      }
    }
    const uint32_t first_half = __shfl_sync(0xffffffffu, i0, 31);
    const uint32_t e0 = i0 - c0, e1 = first_half + i1 - c1;  // exclusive prefixes of words lane, lane + 32
    const int y = local / J.segs_per_row;
    const int x0 = (local % J.segs_per_row) * kSeg;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const uint32_t mine = half ? w1 : w0, pre = half ? e1 : e0;
      uint32_t nonempty = __ballot_sync(0xffffffffu, mine != 0u);
      while (nonempty) {
        const int wi = __ffs(nonempty) - 1;
        nonempty &= nonempty - 1u;
        const uint32_t word = __shfl_sync(0xffffffffu, mine, wi);
        const uint32_t wpre = __shfl_sync(0xffffffffu, pre, wi);
        if ((word >> lane) & 1u) {
          const uint32_t slot = base + wpre + __popc(word & lt);
          if (slot < static_cast<uint32_t>(J.capacity)) {
            const int x = x0 + (32 * half + wi) * 32 + lane;
            const int64_t p = static_cast<int64_t>(y) * J.width + x;
            hsi_detection d;
            d.x = x;
            d.y = y;
            d.target = J.target ? J.target[p] : 0;
            d.score = J.score[p];
            J.out[slot] = d;
          }
        }
      }
    }
  }
}

// Row segments of a map; 64-bit, so sizes far past the limits below stay exact.
int64_t segs_of(int height, int width) {
  return static_cast<int64_t>(height) * ((static_cast<int64_t>(width) + kSeg - 1) / kSeg);
}

// Largest segment count of one batch (the kernels index segments in int).
constexpr int64_t kMaxBatchSegs = 0x3fffffff;

size_t ws_bytes_for_segs(int64_t segs) { return static_cast<size_t>(segs) * sizeof(uint32_t) * (2 + kWordsPerSeg) + 256; }

int sm_count() { return device_sm_count(); }

// Blocks of `kernel` resident per SM of the current device at `threads`
// threads (4 if the query fails).
template <typename K>
int resident_blocks(K* kernel, int threads) {
  const int v = device_residency(kernel, threads, 0);
  return v > 0 ? v : 4;
}

int run_batch(const hsi_detect_job* jobs, int n, void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!jobs || n <= 0 || n > kMaxJobs) return HSI_E_INVALID;
  Batch b{};
  int64_t segs = 0, tiles[2] = {0, 0};
  for (int i = 0; i < n; ++i) {
    const hsi_detect_job& j = jobs[i];
    if (!j.score || !j.count || j.height <= 0 || j.width <= 0 || j.capacity < 0) return HSI_E_INVALID;
    if (j.capacity > 0 && !j.out) return HSI_E_INVALID;
    if (j.polarity != HSI_LOWER_IS_BETTER && j.polarity != HSI_HIGHER_IS_BETTER) return HSI_E_INVALID;
    Job& J = b.jobs[i];
    J.score = j.score;
    J.target = j.target;
    J.height = j.height;
    J.width = j.width;
    J.threshold = j.threshold;
    J.radius = j.nms_radius;
    J.higher = j.polarity == HSI_HIGHER_IS_BETTER;
    J.capacity = j.capacity;
    J.out = j.out;
    J.count = j.count;
    J.seg0 = static_cast<int>(segs);
    J.segs_per_row = (j.width + kSeg - 1) / kSeg;
    // fast flags tiles: radius <= kFastR and rows that start on 16 bytes
    const int kind = j.nms_radius <= kFastR && j.width % 4 == 0 &&
                     (reinterpret_cast<uintptr_t>(j.score) & 15u) == 0;
    const int tile_w = kind ? kFastW : kTileW;
    J.tile0 = static_cast<int>(tiles[kind]);
    J.tiles_x = (j.width + tile_w - 1) / tile_w;
    b.kind_jobs[kind][b.kind_n[kind]++] = i;
    segs += segs_of(j.height, j.width);
    tiles[kind] += static_cast<int64_t>(J.tiles_x) * ((j.height + kTileH - 1) / kTileH);
    if (segs > kMaxBatchSegs || tiles[kind] > 0x3fffffff) return HSI_E_CAPACITY;
  }
  if (!ws || ws_bytes < ws_bytes_for_segs(segs)) return HSI_E_WORKSPACE;
  if ((reinterpret_cast<uintptr_t>(ws) & 15u) != 0) return HSI_E_INVALID;
  b.njobs = n;
  b.total_segs = static_cast<int>(segs);
  b.kind_tiles[0] = static_cast<int>(tiles[0]);
  b.kind_tiles[1] = static_cast<int>(tiles[1]);
  uint32_t* p = static_cast<uint32_t*>(ws);
  b.counts = p;
  b.offsets = p + segs;
  b.masks = p + 2 * segs;
  // one wave of resident tiles per flags kind (41 KB of shared memory each),
  // the residency read once per device
  const int per_sm[2] = {resident_blocks(flags_kernel, kFlagThreads),
                         resident_blocks(flags_fast_kernel, kFastThreads)};
  const int64_t emit_blocks = (segs + kThreads / 32 - 1) / (kThreads / 32);  // a warp per segment
  const int grid = static_cast<int>(emit_blocks < 16 * sm_count() ? emit_blocks : 16 * sm_count());
  for (int kind = 0; kind < 2; ++kind) {
    if (tiles[kind] == 0) continue;
    const int64_t wave = static_cast<int64_t>(per_sm[kind]) * sm_count();
    const int flag_grid = static_cast<int>(tiles[kind] < wave ? tiles[kind] : wave);
    if (kind == 0)
      flags_kernel<<<flag_grid, kFlagThreads, 0, s>>>(b);
    else
      flags_fast_kernel<<<flag_grid, kFastThreads, 0, s>>>(b);
  }
  scan_kernel<<<n, 1024, 0, s>>>(b);
  emit_kernel<<<grid, kThreads, 0, s>>>(b);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API size_t hsi_detect_workspace_bytes(int height, int width) {
  if (height <= 0 || width <= 0) return 0;
  const int64_t segs = segs_of(height, width);
  return segs > kMaxBatchSegs ? 0 : ws_bytes_for_segs(segs);
}

extern "C" HSI_API size_t hsi_detect_batch_workspace_bytes(const hsi_detect_job* jobs, int num_jobs) {
  if (!jobs || num_jobs <= 0) return 0;
  int64_t segs = 0;
  for (int i = 0; i < num_jobs; ++i) {
    if (jobs[i].height <= 0 || jobs[i].width <= 0) return 0;
    segs += segs_of(jobs[i].height, jobs[i].width);
    if (segs > kMaxBatchSegs) return 0;
  }
  return ws_bytes_for_segs(segs);
}

extern "C" HSI_API int hsi_detect(const float* d_score, const int32_t* d_target, int height, int width,
                                  float threshold, int nms_radius, int polarity, int capacity,
                                  hsi_detection* d_out, uint32_t* d_count, void* d_workspace,
                                  size_t workspace_bytes, hsi_stream_t stream) {
  hsi_detect_job j;
  j.score = d_score;
  j.target = d_target;
  j.height = height;
  j.width = width;
  j.threshold = threshold;
  j.nms_radius = nms_radius;
  j.polarity = polarity;
  j.capacity = capacity;
  j.out = d_out;
  j.count = d_count;
  return run_batch(&j, 1, d_workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" HSI_API int hsi_detect_batch(const hsi_detect_job* jobs, int num_jobs, void* d_workspace,
                                        size_t workspace_bytes, hsi_stream_t stream) {
  return run_batch(jobs, num_jobs, d_workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
}

// ---- allocation-free detection ------------------------------------------------
//
// For callers that cannot allocate device memory at all -- for example a
// plug-in that a host application hands only its input and output buffers,
// while the application owns every byte of device memory and lets nothing
// else call cudaMalloc -- hsi_detect_noalloc runs the same three launches as
// hsi_detect with its scratch in the file-scope array below instead of a
// caller workspace.  The array is part of the library's device image, so
// every GPU that loads the library holds it (2.06 MiB) until the process
// exits, and every call on one device shares it.
namespace hsi_b200 {
namespace {

constexpr int kNoAllocSegs = HSI_DETECT_NOALLOC_MAX_SEGMENTS;
constexpr size_t kNoAllocBytes = static_cast<size_t>(kNoAllocSegs) * sizeof(uint32_t) * (2 + kWordsPerSeg) + 256;

// Segment counts, offsets and ballot masks of one call.  Every word a call
// reads is written earlier by that same call (flags writes every mask word
// that covers pixels of the map, and scan and emit read no other; scan writes
// the counts and offsets), so nothing here needs to start at zero and stale
// contents from a previous call are never read.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocBytes / sizeof(uint32_t)];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
struct NoAllocAddr {
  unsigned long long context;  // the context the address belongs to (0 = none yet)
  void* addr;                  // device address of the array in that context
};
NoAllocAddr g_noalloc_addr[kNoAllocMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Process-unique id of the current context.  A device reset (or any other
// re-creation of the context) reloads the module, so the array may move; the
// id changes with it, where a context handle could be reused.
int current_context_id(unsigned long long* id) {
  static const CtxGetCurrentFn get_current = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    return cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess
               ? reinterpret_cast<CtxGetCurrentFn>(p)
               : nullptr;
  }();
  static const CtxGetIdFn get_id = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    return cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess
               ? reinterpret_cast<CtxGetIdFn>(p)
               : nullptr;
  }();
  if (!get_current || !get_id) return HSI_E_NO_DEVICE;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return HSI_E_NO_DEVICE;
  return get_id(ctx, id) == CUDA_SUCCESS ? HSI_OK : HSI_E_NO_DEVICE;
}

// Once per device (and again whenever that device's context is re-created),
// with the device current: look up the array's device address (in host code
// its name is only a host-side stand-in).
int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return static_cast<int>(e);
  if (dev < 0 || dev >= kNoAllocMaxDevices) return HSI_E_NO_DEVICE;
  unsigned long long ctx = 0;
  if (current_context_id(&ctx) != HSI_OK) {
    // no context is current before the runtime's first call on this thread:
    // the symbol lookup makes the device's primary context current
    void* addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return static_cast<int>(e);
    const int st = current_context_id(&ctx);
    if (st != HSI_OK) return st;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoAllocAddr& a = g_noalloc_addr[dev];
  if (a.addr == nullptr || a.context != ctx) {
    void* addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return static_cast<int>(e);
    if ((reinterpret_cast<uintptr_t>(addr) & 255u) != 0) return HSI_E_INVALID;
    a.addr = addr;
    a.context = ctx;
  }
  *out = a.addr;
  return HSI_OK;
}

}  // namespace
}  // namespace hsi_b200

extern "C" HSI_API int hsi_detect_noalloc(const float* d_score, const int32_t* d_target, int height, int width,
                                          float threshold, int nms_radius, int polarity, int capacity,
                                          hsi_detection* d_out, uint32_t* d_count, hsi_stream_t stream) {
  if (height <= 0 || width <= 0) return HSI_E_INVALID;
  const int64_t segs = static_cast<int64_t>(height) * ((static_cast<int64_t>(width) + kSeg - 1) / kSeg);
  if (segs > kNoAllocSegs) return HSI_E_CAPACITY;
  void* scratch = nullptr;
  const int st = noalloc_scratch(&scratch);
  if (st != HSI_OK) return st;
  hsi_detect_job j;
  j.score = d_score;
  j.target = d_target;
  j.height = height;
  j.width = width;
  j.threshold = threshold;
  j.nms_radius = nms_radius;
  j.polarity = polarity;
  j.capacity = capacity;
  j.out = d_out;
  j.count = d_count;
  return run_batch(&j, 1, scratch, kNoAllocBytes, reinterpret_cast<cudaStream_t>(stream));
}
