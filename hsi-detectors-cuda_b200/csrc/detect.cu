// detect.cu - threshold + non-maximum suppression + ordered compaction.
//
// Three small launches, no atomics on the data path, so the list comes out in
// raster order and is identical run to run:
//   1. flags:  per 2048-pixel tile, every pixel's pass/fail as a warp ballot
//              word (bitmask in the workspace) and the tile's count;
//   2. scan:   one block turns the tile counts into output offsets, starting
//              at the caller's *d_count, and advances *d_count by the total;
//   3. emit:   each tile writes its detections at its offset + in-tile rank,
//              dropping (but having counted) those past capacity.
// Semantics are the reference CPU path's (src/sam_cpu.cpp:86-138), polarity
// included; the reference GPU kernel (src/detect.cu:43-87) ignores polarity
// and emits in atomic arrival order, both of which this replaces.
#include "common.cuh"

namespace hsi_b200 {
namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr int kTilePixels = kThreads * kPerThread;  // 2048
constexpr int kWordsPerTile = kTilePixels / 32;      // 64

struct DetectWorkspace {
  uint32_t* counts;   // [tiles]
  uint32_t* offsets;  // [tiles]
  uint32_t* masks;    // [tiles * 64]
};

size_t tiles_for(int64_t pixels) { return static_cast<size_t>(div_up<int64_t>(pixels, kTilePixels)); }

size_t workspace_bytes(int64_t pixels) {
  const size_t t = tiles_for(pixels);
  return t * sizeof(uint32_t) * (2 + kWordsPerTile) + 256;
}

DetectWorkspace carve(void* base, int64_t pixels) {
  const size_t t = tiles_for(pixels);
  uint32_t* p = static_cast<uint32_t*>(base);
  return DetectWorkspace{p, p + t, p + 2 * t};
}

__device__ __forceinline__ bool better(float a, float b, bool higher) { return higher ? a > b : a < b; }

__device__ bool local_best(const float* __restrict__ s, int x, int y, int w, int h, int r, float self,
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

__global__ void __launch_bounds__(kThreads) detect_flags_kernel(const float* __restrict__ score, int width,
                                                                int height, float threshold, int radius,
                                                                bool higher, DetectWorkspace ws) {
  const int64_t pixels = static_cast<int64_t>(width) * height;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ uint32_t s_count[kThreads / 32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTilePixels;
  uint32_t mine = 0;
#pragma unroll
  for (int i = 0; i < kPerThread; ++i) {
    const int64_t p = base + i * kThreads + threadIdx.x;
    bool pass = false;
    if (p < pixels) {
      const float s = score[p];
      const bool over = higher ? (s >= threshold) : (s <= threshold);
      if (over) {
        const int x = static_cast<int>(p % width), y = static_cast<int>(p / width);
        pass = radius <= 0 || local_best(score, x, y, width, height, radius, s, higher);
      }
    }
    const uint32_t word = __ballot_sync(0xffffffffu, pass);
    if (lane == 0) {
      ws.masks[static_cast<int64_t>(blockIdx.x) * kWordsPerTile + i * (kThreads / 32) + warp] = word;
      mine += __popc(word);
    }
  }
  if (lane == 0) s_count[warp] = mine;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t total = 0;
    for (int w = 0; w < kThreads / 32; ++w) total += s_count[w];
    ws.counts[blockIdx.x] = total;
  }
}

// Single block: exclusive scan of tile counts starting at *count; *count += total.
__global__ void __launch_bounds__(1024) detect_scan_kernel(int tiles, DetectWorkspace ws, uint32_t* count) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) s_carry = *count;
  __syncthreads();
  for (int chunk = 0; chunk < tiles; chunk += 1024) {
    const int i = chunk + threadIdx.x;
    const uint32_t v = i < tiles ? ws.counts[i] : 0u;
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
      s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t warp_base = warp > 0 ? s_warp[warp - 1] : 0u;
    const uint32_t carry = s_carry;
    if (i < tiles) ws.offsets[i] = carry + warp_base + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + s_warp[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = s_carry;
}

__global__ void __launch_bounds__(kThreads) detect_emit_kernel(const float* __restrict__ score,
                                                               const int32_t* __restrict__ target, int width,
                                                               int capacity, DetectWorkspace ws,
                                                               hsi_detection* __restrict__ out) {
  __shared__ uint32_t s_words[kWordsPerTile];
  __shared__ uint32_t s_prefix[kWordsPerTile];
  const int64_t tile = blockIdx.x;
  if (threadIdx.x < kWordsPerTile) s_words[threadIdx.x] = ws.masks[tile * kWordsPerTile + threadIdx.x];
  __syncthreads();
  if (threadIdx.x < 32) {
    // exclusive prefix of popcounts over the 64 words, two per lane
    const int lane = threadIdx.x;
    const uint32_t a = __popc(s_words[2 * lane]), b = __popc(s_words[2 * lane + 1]);
    uint32_t incl = a + b;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    const uint32_t excl = incl - a - b;
    s_prefix[2 * lane] = excl;
    s_prefix[2 * lane + 1] = excl + a;
  }
  __syncthreads();
  const uint32_t base = ws.offsets[tile];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int i = 0; i < kPerThread; ++i) {
    const int w = i * (kThreads / 32) + warp;
    const uint32_t word = s_words[w];
    if ((word >> lane) & 1u) {
      const uint32_t slot = base + s_prefix[w] + __popc(word & lt);
      if (slot < static_cast<uint32_t>(capacity)) {
        const int64_t p = tile * kTilePixels + static_cast<int64_t>(w) * 32 + lane;
        hsi_detection d;
        d.x = static_cast<int32_t>(p % width);
        d.y = static_cast<int32_t>(p / width);
        d.target = target ? target[p] : 0;
        d.score = score[p];
        out[slot] = d;
      }
    }
  }
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API size_t hsi_detect_workspace_bytes(int height, int width) {
  if (height <= 0 || width <= 0) return 0;
  return workspace_bytes(static_cast<int64_t>(height) * width);
}

extern "C" HSI_API int hsi_detect(const float* d_score, const int32_t* d_target, int height, int width,
                                  float threshold, int nms_radius, int polarity, int capacity,
                                  hsi_detection* d_out, uint32_t* d_count, void* d_workspace,
                                  size_t workspace_bytes_given, hsi_stream_t stream) {
  if (!d_score || !d_count || height <= 0 || width <= 0 || capacity < 0) return HSI_E_INVALID;
  if (capacity > 0 && !d_out) return HSI_E_INVALID;
  if (polarity != HSI_LOWER_IS_BETTER && polarity != HSI_HIGHER_IS_BETTER) return HSI_E_INVALID;
  const int64_t pixels = static_cast<int64_t>(height) * width;
  if (!d_workspace || workspace_bytes_given < workspace_bytes(pixels)) return HSI_E_WORKSPACE;
  if ((reinterpret_cast<uintptr_t>(d_workspace) & 15u) != 0) return HSI_E_INVALID;
  const size_t tiles = tiles_for(pixels);
  if (tiles > 0x7fffffff) return HSI_E_CAPACITY;
  const DetectWorkspace ws = carve(d_workspace, pixels);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const bool higher = polarity == HSI_HIGHER_IS_BETTER;
  detect_flags_kernel<<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(d_score, width, height, threshold,
                                                                      nms_radius, higher, ws);
  detect_scan_kernel<<<1, 1024, 0, s>>>(static_cast<int>(tiles), ws, d_count);
  detect_emit_kernel<<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(d_score, d_target, width, capacity, ws,
                                                                     d_out);
  return static_cast<int>(cudaGetLastError());
}
