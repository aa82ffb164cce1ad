// detect.cu - threshold + non-maximum suppression + ordered compaction.
//
// Three launches for a whole batch of score maps, no atomics on the data
// path, so every list comes out in raster order and is identical run to run:
//   1. flags:  per row segment (up to 2048 pixels of one row), every pixel's
//              pass/fail as warp ballot words (bitmask in the workspace) and
//              the segment's count.  The score rows the NMS window needs are
//              staged in shared memory (radius <= 4; larger radii read global
//              memory), padded with NaN so out-of-frame neighbours never win
//              or tie, exactly like the bounds checks of the CPU loop;
//   2. scan:   one block per map turns segment counts into output offsets,
//              starting at the caller's *count, and advances *count;
//   3. emit:   each segment writes its detections at offset + in-segment
//              rank, dropping (but having counted) those past capacity.
// Semantics are the reference CPU path's (src/sam_cpu.cpp:86-138), polarity
// included; the reference GPU kernel (src/detect.cu:43-87) ignores polarity
// and emits in atomic arrival order, both of which this replaces.
#include <mutex>

#include "common.cuh"

namespace hsi_b200 {
namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr int kSeg = kThreads * kPerThread;  // 2048 pixels per segment
constexpr int kWordsPerSeg = kSeg / 32;      // 64
constexpr int kMaxStagedRadius = 4;
constexpr int kColsPerThread = (kSeg + 2 * kMaxStagedRadius + kThreads - 1) / kThreads;  // 9
// Segments with at most this many threads holding a candidate skip the staged
// window and read their candidates' neighbourhoods from global memory.
constexpr int kSparseThreads = 64;
constexpr int kMaxJobs = 64;

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
};

struct Batch {
  Job jobs[kMaxJobs];
  int njobs;
  int total_segs;
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

__device__ __forceinline__ bool better(float a, float b, bool higher) { return higher ? a > b : a < b; }

// The total order of the suppression window: the better score first (by
// polarity), then the lower linear index; NaN (outside the frame) is last.
// A candidate survives exactly when it is the first of its window.  Inside a
// staged window the position ry * tw + c orders pixels as their linear
// indices do (row first, c < tw), so it stands in for the index.
__device__ __forceinline__ bool lex_first(float av, int ai, float bv, int bi, bool higher) {
  if (isnan(bv)) return !isnan(av);
  if (isnan(av)) return false;
  return better(av, bv, higher) || (av == bv && ai < bi);
}

// NMS against global memory, for radii too large to stage.
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

__global__ void __launch_bounds__(kThreads) flags_kernel(const __grid_constant__ Batch b) {
  // (2r+1) rows x (kSeg + 2r) columns of scores (at least 3 rows: after the
  // vertical pass rows 0 and 1 hold each column's best value and index)
  extern __shared__ float tile[];
  __shared__ uint32_t s_count[kThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int seg = blockIdx.x; seg < b.total_segs; seg += gridDim.x) {
    __syncthreads();  // the previous segment is done with the tile and s_count
    const Job& J = b.jobs[find_job(b, seg)];
    const int local = seg - J.seg0;
    const int y = local / J.segs_per_row;
    const int x0 = (local % J.segs_per_row) * kSeg;
    const int len = min(kSeg, J.width - x0);
    const int r = J.radius > 0 ? J.radius : 0;
    const bool staged = r <= kMaxStagedRadius;
    const bool higher = J.higher != 0;
    const int tw = kSeg + 2 * r;
    float* col_v = tile;                               // tile row 0, after the vertical pass
    int* col_i = reinterpret_cast<int*>(tile + tw);    // tile row 1
    // threshold first: a segment with few candidates checks their windows in
    // global memory (L1/L2), one with many stages the whole window once
    float sv[kPerThread];
    uint32_t over_bits = 0;
#pragma unroll
    for (int i = 0; i < kPerThread; ++i) {
      const int xi = i * kThreads + threadIdx.x;
      sv[i] = 0.0f;
      if (xi < len) {
        sv[i] = J.score[static_cast<int64_t>(y) * J.width + x0 + xi];
        if (higher ? (sv[i] >= J.threshold) : (sv[i] <= J.threshold)) over_bits |= 1u << i;
      }
    }
    const int busy = __syncthreads_count(over_bits != 0);  // threads holding a candidate
    const bool use_tile = r > 0 && staged && busy > kSparseThreads;
    if (use_tile) {
      // row by row, no index division; NaN outside the frame: never better, never equal
      const float nan = __int_as_float(0x7fc00000);
      for (int ry = 0; ry <= 2 * r; ++ry) {
        const int gy = y - r + ry;
        const bool row_in = gy >= 0 && gy < J.height;
        const float* src = J.score + static_cast<int64_t>(row_in ? gy : 0) * J.width;
        float* dst = tile + ry * tw;
        for (int rx = threadIdx.x; rx < len + 2 * r; rx += kThreads) {
          const int gx = x0 - r + rx;
          dst[rx] = row_in && gx >= 0 && gx < J.width ? src[gx] : nan;
        }
      }
      __syncthreads();
      // vertical pass: the first (score, index) of each staged column, kept in
      // registers until every thread has read the tile, then written over its
      // first two rows
      float cv[kColsPerThread];
      int ci[kColsPerThread];
#pragma unroll
      for (int k = 0; k < kColsPerThread; ++k) {
        const int c = threadIdx.x + k * kThreads;
        cv[k] = __int_as_float(0x7fc00000);
        ci[k] = 0;
        if (c < len + 2 * r) {
          cv[k] = tile[c];
          ci[k] = c;
          for (int ry = 1; ry <= 2 * r; ++ry) {
            const int id = ry * tw + c;
            const float v = tile[id];
            if (lex_first(v, id, cv[k], ci[k], higher)) {
              cv[k] = v;
              ci[k] = id;
            }
          }
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kColsPerThread; ++k) {
        const int c = threadIdx.x + k * kThreads;
        if (c < len + 2 * r) {
          col_v[c] = cv[k];
          col_i[c] = ci[k];
        }
      }
      __syncthreads();
    }
    uint32_t mine = 0;
#pragma unroll
    for (int i = 0; i < kPerThread; ++i) {
      const int xi = i * kThreads + threadIdx.x;  // pixel within the segment
      bool pass = false;
      if ((over_bits >> i) & 1u) {
        const int x = x0 + xi;
        const float s = sv[i];
        if (r == 0) {
          pass = true;
        } else if (use_tile) {
          // first of the window = first of the column bests around it
          const int self = r * tw + xi + r;  // tile position of the candidate
          float bv = s;
          int bi = self;
          for (int dx = -r; dx <= r; ++dx) {
            const float v = col_v[xi + r + dx];
            const int id = col_i[xi + r + dx];
            if (lex_first(v, id, bv, bi, higher)) {
              bv = v;
              bi = id;
            }
          }
          pass = bi == self;
        } else {
          pass = local_best_global(J.score, x, y, J.width, J.height, r, s, higher);
        }
      }
      const uint32_t word = __ballot_sync(0xffffffffu, pass);
      if (lane == 0) {
        b.masks[static_cast<int64_t>(seg) * kWordsPerSeg + i * (kThreads / 32) + warp] = word;
        mine += __popc(word);
      }
    }
    if (lane == 0) s_count[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t total = 0;
      for (int w = 0; w < kThreads / 32; ++w) total += s_count[w];
      b.counts[seg] = total;
    }
  }
}

// One block per map: exclusive scan of its segment counts from *count;
// *count += total.
__global__ void __launch_bounds__(1024) scan_kernel(const __grid_constant__ Batch b) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  const Job& J = b.jobs[blockIdx.x];
  const int segs = J.height * J.segs_per_row;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) s_carry = *J.count;
  __syncthreads();
  for (int chunk = 0; chunk < segs; chunk += 1024) {
    const int i = chunk + threadIdx.x;
    const uint32_t v = i < segs ? b.counts[J.seg0 + i] : 0u;
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

__global__ void __launch_bounds__(kThreads) emit_kernel(const __grid_constant__ Batch b) {
  __shared__ uint32_t s_words[kWordsPerSeg];
  __shared__ uint32_t s_prefix[kWordsPerSeg];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int seg = blockIdx.x; seg < b.total_segs; seg += gridDim.x) {
    __syncthreads();
    if (threadIdx.x < kWordsPerSeg) s_words[threadIdx.x] = b.masks[static_cast<int64_t>(seg) * kWordsPerSeg + threadIdx.x];
    __syncthreads();
    if (threadIdx.x < 32) {
      const uint32_t a = __popc(s_words[2 * lane]), c = __popc(s_words[2 * lane + 1]);
      uint32_t incl = a + c;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += o;
      }
      const uint32_t excl = incl - a - c;
      s_prefix[2 * lane] = excl;
      s_prefix[2 * lane + 1] = excl + a;
    }
    __syncthreads();
    const Job& J = b.jobs[find_job(b, seg)];
    const int local = seg - J.seg0;
    const int y = local / J.segs_per_row;
    const int x0 = (local % J.segs_per_row) * kSeg;
    const uint32_t base = b.offsets[seg];
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int i = 0; i < kPerThread; ++i) {
      const int w = i * (kThreads / 32) + warp;
      const uint32_t word = s_words[w];
      if ((word >> lane) & 1u) {
        const uint32_t slot = base + s_prefix[w] + __popc(word & lt);
        if (slot < static_cast<uint32_t>(J.capacity)) {
          const int x = x0 + w * 32 + lane;
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

int segs_of(int height, int width) { return height * ((width + kSeg - 1) / kSeg); }

size_t ws_bytes_for_segs(int64_t segs) { return static_cast<size_t>(segs) * sizeof(uint32_t) * (2 + kWordsPerSeg) + 256; }

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

int run_batch(const hsi_detect_job* jobs, int n, void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!jobs || n <= 0 || n > kMaxJobs) return HSI_E_INVALID;
  Batch b{};
  int64_t segs = 0;
  int max_r = 0;
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
    segs += segs_of(j.height, j.width);
    // staged radii size the shared tile; larger ones read global memory
    if (j.nms_radius <= kMaxStagedRadius && j.nms_radius > max_r) max_r = j.nms_radius;
  }
  if (segs > 0x3fffffff) return HSI_E_CAPACITY;
  if (!ws || ws_bytes < ws_bytes_for_segs(segs)) return HSI_E_WORKSPACE;
  if ((reinterpret_cast<uintptr_t>(ws) & 15u) != 0) return HSI_E_INVALID;
  b.njobs = n;
  b.total_segs = static_cast<int>(segs);
  uint32_t* p = static_cast<uint32_t*>(ws);
  b.counts = p;
  b.offsets = p + segs;
  b.masks = p + 2 * segs;
  const size_t smem = static_cast<size_t>(2 * (max_r > 0 ? max_r : 1) + 1) * (kSeg + 2 * max_r) * sizeof(float);
  static bool configured = false;
  if (!configured) {
    const cudaError_t e = cudaFuncSetAttribute(flags_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>((2 * kMaxStagedRadius + 1) *
                                                                (kSeg + 2 * kMaxStagedRadius) * sizeof(float)));
    if (e != cudaSuccess) return static_cast<int>(e);
    configured = true;
  }
  const int grid = static_cast<int>(segs < 16 * sm_count() ? segs : 16 * sm_count());
  flags_kernel<<<grid, kThreads, smem, s>>>(b);
  scan_kernel<<<n, 1024, 0, s>>>(b);
  emit_kernel<<<grid, kThreads, 0, s>>>(b);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API size_t hsi_detect_workspace_bytes(int height, int width) {
  if (height <= 0 || width <= 0) return 0;
  return ws_bytes_for_segs(segs_of(height, width));
}

extern "C" HSI_API size_t hsi_detect_batch_workspace_bytes(const hsi_detect_job* jobs, int num_jobs) {
  if (!jobs || num_jobs <= 0) return 0;
  int64_t segs = 0;
  for (int i = 0; i < num_jobs; ++i) {
    if (jobs[i].height <= 0 || jobs[i].width <= 0) return 0;
    segs += segs_of(jobs[i].height, jobs[i].width);
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
// reads is written earlier by that same call (flags writes counts and all 64
// mask words of each segment, scan writes offsets), so nothing here needs to
// start at zero and stale contents from a previous call are never read.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocBytes / sizeof(uint32_t)];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kNoAllocMaxDevices];  // device address of the array, per device

// Once per device, with that device current: look up the array's device
// address (in host code its name is only a host-side stand-in) and allow the
// flags kernel its full shared-memory tile on this device.
int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return static_cast<int>(e);
  if (dev < 0 || dev >= kNoAllocMaxDevices) return HSI_E_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_addr[dev] == nullptr) {
    void* addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return static_cast<int>(e);
    if ((reinterpret_cast<uintptr_t>(addr) & 255u) != 0) return HSI_E_INVALID;
    e = cudaFuncSetAttribute(flags_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>((2 * kMaxStagedRadius + 1) * (kSeg + 2 * kMaxStagedRadius) *
                                              sizeof(float)));
    if (e != cudaSuccess) return static_cast<int>(e);
    g_noalloc_addr[dev] = addr;
  }
  *out = g_noalloc_addr[dev];
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
