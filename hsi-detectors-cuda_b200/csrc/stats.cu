// stats.cu - scene moments on the 5th-generation tensor cores, exactly.
//
// Computes, for BSQ frames, the raw first and second moments the detector
// statistics are built from (reference: SpectralMoments, include/hsi/linalg.hpp
// :22-51, accumulated by src/detectors_cpu.cpp:77-93 on the CPU and by the
// never-called src/stats.cu:72-165 on the GPU).
//
// Why integers.  RX/ACE amplify relative covariance errors by the condition
// number of the (loaded) covariance, ~4000 for these scenes, so 1e-4 on the
// scores needs the second moments to ~2e-8.  Measured on B200, FP32
// accumulation on the tensor cores truncates: BF16 hi/lo products with all four
// terms still left a 5e-7..5e-6 bias (RX error 5e-4..3e-3), and even FP32
// CUDA-core FMAs over 1024-pixel chunks gave 1.8e-4.  Integer MMAs accumulate
// exactly.  So:
//   d = x - r (r: per-band reference near the mean, as the reference's shifted
//   accumulation, include/hsi/linalg.hpp:53-90), fixed point
//   q = rint(d * 2^e_b) with -2^22 - 2^15 - 2^7 <= q < 2^22 - 2^15 - 2^7
//   (e_b from a subsample with 4x headroom; a value out of range re-runs the
//   pass with the observed range), balanced signed 8-bit limbs
//   q = L0*2^16 + L1*2^8 + L2 with L0 in [-64, 63], so that D = 2 L0 is an
//   INT8 too, and four exact INT32 accumulators
//     A0 = sum D D^T,  A1 = sum D L1^T,  A2 = sum (L1 L1^T + D L2^T),
//     A3 = sum L1 L2^T
//   (tcgen05.mma kind::i8, three MMAs per K-step, two of them N = 256).  F = 2^30 A0 + 2^24 A1 +
//   2^16 A2 + 2^9 A3 and S = (F + F^T)/2 is sum q q^T except the weight-1
//   products L2 L2^T: their diagonal is added back exactly (the converters
//   count sum L2^2 per band), and of their off-diagonal sums the mean part
//   (sum L2_i)(sum L2_j)/N, which is what is left when the low limbs are not
//   random residues: inputs on a coarse grid (FP16 values, integer counts)
//   give every pixel of a band nearly the same L2.  r is placed on a grid of
//   256 fixed-point steps for the same reason.  The cross terms matter: when
//   outliers set the fixed-point range, typical q carry only ~15 significant
//   bits.
//   A ones-row at band B (q = 2^16) makes the same GEMM produce sum(q) and the
//   pixel count.
//   Every 32768-pixel chunk's accumulators leave TMEM as two exact INT64
//   matrices (sum A0, and sum 2^15 A1 + 2^7 A2 + A3), so the per-CTA partials
//   add up exactly in any order: the moments do not depend on how the pixels
//   were split between CTAs, and come out bit-identical run to run.  They are
//   rebuilt as raw moments in FP64 (src/linalg.cpp:81-103).
//
// Batches.  One launch sequence serves up to kMaxBatch frames of one element
// type: the frames' K-blocks (128 pixels each) form one sequence that the
// persistent GEMM splits evenly over one CTA per SM, so the pipeline runs
// across frame boundaries and a CTA's range meets at most a few frames (each
// meeting is a "piece" with its own partial slot).  The small steps (range
// subsample, reduction, finalisation) each take one launch for all frames.
//
// Kernel roles (one CTA per SM, 22 warps):
//   warp 0       TMA producer: 64-pixel x 128-band boxes, two per K-block,
//                into a 4-deep ring (3 boxes in flight while one converts)
//   warp 1       TMEM allocator + single-thread MMA issuer
//   warps 2-17   converters: FP32 tile -> INT8 limbs D, L1, L2 in the UMMA
//                128-byte-swizzled K-major layout; range check per element
//   warps 18-21  epilogue: INT32 TMEM accumulators -> INT64 partials (once per
//                32768-pixel chunk and at the end of each piece)
// TMEM: columns [0,128) A0, [128,256) A1, [256,384) A2, [384,512) A3.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <atomic>
#include <type_traits>
#include <mutex>

#include "tc.cuh"
#include "launch_state.h"

namespace hsi_b200 {
namespace {

constexpr int kKB = 128;         // pixels per K-block (one INT8 operand row)
constexpr int kBoxPx = 128;      // pixels per TMA box: 512-byte runs of each band plane
constexpr int kHalfPx = 64;      // pixels a converter pass covers (half a K-block)
constexpr int kBoxesPerKB = kKB / kBoxPx;
constexpr int kHalvesPerBox = kBoxPx / kHalfPx;
constexpr int kChunkKB = 256;    // K-blocks per INT32 chunk: 32768 px, no overflow
constexpr int kRows = 128;       // band rows of the GEMM (bands + ones row)
constexpr int kOpStages = 2;
constexpr int kConvWarps = 16;
constexpr int kEpiWarps = 4;
constexpr int kWarpTma = 0;
constexpr int kWarpMma = 1;
constexpr int kWarpConv0 = 2;
constexpr int kWarpEpi0 = kWarpConv0 + kConvWarps;
constexpr int kThreads = (kWarpEpi0 + kEpiWarps) * 32;  // 704
constexpr int kLimbBytes = kRows * kKB;                 // 16 KB per limb tile
constexpr uint32_t kTmemCols = 512;
constexpr int kMaxTensorBands = kRows - 1;  // 127: room for the ones row
constexpr int kMaxCtas = 160;
constexpr int kMaxBatch = 64;               // frames per launch sequence
constexpr int64_t kTensorMinPixels = 32768;
constexpr int64_t kTensorMaxPixels = int64_t(1) << 31;  // TMA pixel coordinates are 32-bit
constexpr int kOnesExp = 16;  // the ones row holds q = 2^16
constexpr size_t kSlotElems = 2 * static_cast<size_t>(kRows) * kRows;  // INT64 H and Lo per piece

// Fixed-point conversion by one FMA: y = x * 2^e + (kMagicQ - r * 2^e).  For
// -2^22 - 0x8080 <= q < 2^22 - 0x8080, y = 1.5 * 2^23 + 0x8080 + q lies in
// [2^23, 2^24), where float spacing is 1, so the FMA's rounding is rint and
// the float's bits are 0x4B000000 + m with m = q + 0x8080 + 2^22.  The limbs
// are m's bytes: L2 = byte0 ^ 0x80, L1 = byte1 ^ 0x80, L0 = byte2 - 64 (the
// 0x80 offsets make the limbs balanced), and D = 2 L0 = (2 byte2) ^ 0x80.
// Any y outside [2^23, 2^24) (q out of range, Inf, NaN) has other bits in
// its top nine: byte 3 differs from 0x4B or bit 23 is set.  The converters
// keep an OR and an AND of the packed high bytes of every four values, which
// detects it with two instructions per four elements.
constexpr float kMagicQ = 12615808.0f;        // 1.5 * 2^23 + 0x8080
constexpr uint32_t kZeroBits = 0x4B408080u;    // y for q = 0 (the limbs of q = 2^16, the ones row: D = 2, L1 = L2 = 0)

// Input stages hold one TMA box (kBoxPx pixels x 128 bands), 128 KB in all.
template <typename T>
constexpr int in_stages() {
  return 131072 / (kRows * kBoxPx * static_cast<int>(sizeof(T)));
}
template <typename T>
constexpr int in_tile_bytes() {
  return kRows * kBoxPx * static_cast<int>(sizeof(T));
}

struct StatsSmem {
  size_t in_off, op_off, bar_off, slot_off, total;
};

template <typename T>
__host__ __device__ inline StatsSmem stats_smem() {
  StatsSmem s;
  size_t off = 0;
  s.in_off = off;
  off += static_cast<size_t>(in_stages<T>()) * in_tile_bytes<T>();
  s.op_off = off;  // 1024-aligned: in tiles are multiples of 1024
  off += static_cast<size_t>(kOpStages) * 3 * kLimbBytes;
  s.bar_off = off;
  off += (2 * 8 + 2 * kOpStages + 3) * sizeof(uint64_t);
  s.slot_off = off;
  off += 16;
  s.total = off + 1024;  // slack to align the dynamic base to 1024
  return s;
}

// Byte offset of byte k of row `row` in a 128B-swizzled K-major tile whose rows
// are 128 bytes (8-row atoms of 1024 bytes).
__device__ __forceinline__ uint32_t sw128_byte(int row, int k) {
  return static_cast<uint32_t>((row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 4) ^ (row & 7))) << 4) + (k & 15));
}

template <typename T>
__device__ __forceinline__ float4 load4f(const T* p);
template <>
__device__ __forceinline__ float4 load4f<float>(const float* p) {
  return *reinterpret_cast<const float4*>(p);
}
template <>
__device__ __forceinline__ float4 load4f<__half>(const __half* p) {
  const uint2 raw = *reinterpret_cast<const uint2*>(p);
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
  return make_float4(a.x, a.y, b.x, b.y);
}

constexpr int kShiftSplit = 16;  // slots per band of the subsample pass, blocks per band of the range pass
constexpr int kShiftItems = 4;   // subsample slots per block
constexpr int kShiftHeld = 4;    // loads per thread and slot issued ahead of the reduction

// Per-frame state of the launch sequence.
struct StatsState {
  float shift[HSI_MAX_BANDS + 1];     // r_b
  int scale_exp[HSI_MAX_BANDS + 1];   // e_b (ones row: kOnesExp)
  int maxdev_bits[HSI_MAX_BANDS + 1]; // max |x_b - r_b| over the frame (float bits, >= 0), after a clamp
  int flags;                          // bit 0: a q was out of range; bit 1: the re-run is armed
  int pad[3];
  unsigned long long l2sq[HSI_MAX_BANDS + 1];  // exact sum of L2^2 per band
  long long l2sum[HSI_MAX_BANDS + 1];          // exact sum of L2 per band
  // subsample pass: per-block sums and counts (fixed slots, summed in a fixed
  // order), range (atomics on the order-independent min / max; cleared first)
  double sub_sum[HSI_MAX_BANDS + 1][kShiftSplit];
  double sub_cnt[HSI_MAX_BANDS + 1][kShiftSplit];
  int sub_lo[HSI_MAX_BANDS + 1];  // float_order of the minimum
  int sub_hi[HSI_MAX_BANDS + 1];
};

// One frame of a launch sequence.
struct FrameStats {
  const void* cube;
  int64_t pixels;
  int64_t stride;
  int64_t kb_begin;        // first K-block of the frame in the batch's sequence
  const float* reference;  // nullable
  double* moments;
  StatsState* state;
  double* fsum;            // [kRows][kRows] F, column-major
  long long* slots;        // nslots partial slots (H then Lo, each [kRows][kRows] column-major)
  int bands;
  int cta_lo;              // first CTA whose K-block range meets this frame
  int nslots;
  int run0;                // bands in the first contiguous run of planes (== bands: one run)
  int64_t run1_plane;      // first plane of the second run, counted from `cube`
};

// Plane of band b: a frame may be a view of two contiguous runs of a cube's
// planes (bands [0, run0) at planes [0, run0), the rest from run1_plane on).
__host__ __device__ __forceinline__ int64_t plane_of(const FrameStats& F, int b) {
  return b < F.run0 ? b : F.run1_plane + (b - F.run0);
}

struct FrameTable {
  FrameStats f[kMaxBatch];
  int n;
  int max_bands;
  int ctas;          // CTAs of the GEMM
  int center_mean;   // reference point r: 1 = subsample mean (FP32 path), 0 = midpoint of its range
  int64_t total_kb;  // K-blocks of all frames
  int* status;       // nullable
};

struct GemmParams {
  CUtensorMap maps[kMaxBatch];
  CUtensorMap maps1[kMaxBatch];  // second run of a two-run frame
  FrameTable t;
  int conditional;  // 1: only frames whose re-run is armed
};

__device__ __forceinline__ int64_t frame_kb(const FrameStats& F) { return div_up<int64_t>(F.pixels, kKB); }

// Index of the frame holding K-block kb (the last frame starting at or before it).
__device__ __forceinline__ int frame_of(const FrameTable& t, int64_t kb) {
  int lo = 0, hi = t.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.f[mid].kb_begin <= kb) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// The pieces of CTA `cta`: its K-block range [kb0, kb1) cut at frame
// boundaries, skipping frames whose re-run is not armed when `conditional`.
// Every role walks the same pieces in the same order.
struct PieceWalk {
  const FrameTable& t;
  int64_t kb0, kb1;
  int conditional;
  __device__ int first() const { return kb0 < kb1 ? frame_of(t, kb0) : t.n; }
  __device__ bool in_range(int f) const { return f < t.n && t.f[f].kb_begin < kb1; }
  __device__ bool skip(int f) const { return conditional && !(t.f[f].state->flags & 2); }
  __device__ int64_t lo(int f) const { return max(kb0, t.f[f].kb_begin); }
  __device__ int64_t hi(int f) const { return min(kb1, t.f[f].kb_begin + frame_kb(t.f[f])); }
};

template <typename T>
__global__ void __launch_bounds__(kThreads, 1) stats_gemm_kernel(const __grid_constant__ GemmParams p) {
  const FrameTable& t = p.t;
  const int64_t kb0 = t.total_kb * blockIdx.x / gridDim.x;
  const int64_t kb1 = t.total_kb * (blockIdx.x + 1) / gridDim.x;
  const PieceWalk walk{t, kb0, kb1, p.conditional};
  {
    // nothing to do (an unarmed re-run): leave before any set-up
    bool any = false;
    for (int f = walk.first(); walk.in_range(f); ++f) any = any || !walk.skip(f);
    if (!any) return;
  }
  constexpr int kInStages = in_stages<T>();
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const StatsSmem L = stats_smem<T>();
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar_off);
  uint64_t* in_full = bars;
  uint64_t* in_empty = in_full + 8;
  uint64_t* op_full = in_empty + 8;
  uint64_t* op_empty = op_full + kOpStages;
  uint64_t* acc_full = op_empty + kOpStages;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* mma_done = acc_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.slot_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.slot_off + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kInStages; ++s) {
      mbar_init(&in_full[s], 1);
      mbar_init(&in_empty[s], kConvWarps);
    }
    for (int s = 0; s < kOpStages; ++s) {
      mbar_init(&op_full[s], kConvWarps);
      mbar_init(&op_empty[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, kEpiWarps);
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == kWarpMma) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kWarpTma) {
    if (lane == 0) {
      uint32_t box = 0, pending = 0, parity = 0;
      bool ok = true;
      for (int f = walk.first(); ok && walk.in_range(f); ++f) {
        if (walk.skip(f)) continue;
        const CUtensorMap* map = &p.maps[f];
        prefetch_tensormap(map);
        const int64_t kbf = t.f[f].kb_begin;
        for (int64_t kb = walk.lo(f); kb < walk.hi(f) && ok; ++kb) {
          for (int half = 0; half < kBoxesPerKB; ++half, ++box) {
            const int s = box % kInStages;
            const uint32_t ph = (box / kInStages) & 1u;
            if (*abort_flag || !mbar_wait(&in_empty[s], ph ^ 1u)) {
              record_error(t.status, HSI_E_TIMEOUT);
              *abort_flag = 1;
              ok = false;
              break;
            }
            unsigned char* dst = smem + L.in_off + static_cast<size_t>(s) * in_tile_bytes<T>();
            const int x = static_cast<int>((kb - kbf) * kKB + half * kBoxPx);
            const FrameStats& Fp = t.f[f];
            if (Fp.run0 < Fp.bands) {
              // two runs: one box each, stacked in the tile's rows
              mbar_arrive_expect_tx(&in_full[s], static_cast<uint32_t>(Fp.bands) * kBoxPx * sizeof(T));
              tma_load_2d(dst, map, x, 0, &in_full[s]);
              tma_load_2d(dst + static_cast<size_t>(Fp.run0) * kBoxPx * sizeof(T), &p.maps1[f], x, 0, &in_full[s]);
            } else {
              mbar_arrive_expect_tx(&in_full[s], in_tile_bytes<T>());
              tma_load_2d(dst, map, x, 0, &in_full[s]);
            }
            pending |= 1u << s;
            parity = (parity & ~(1u << s)) | (ph << s);
          }
        }
      }
      for (int s = 0; s < kInStages; ++s)
        if ((pending >> s) & 1u) mbar_wait(&in_full[s], (parity >> s) & 1u);
    }
  } else if (warp == kWarpMma) {
    if (lane == 0) {
      const uint32_t idesc = idesc_s8_s32(kRows, kRows);
      // D, L1 and L2 are consecutive 128-row tiles, so [D; L1] and [L1; L2] are
      // 256-row B operands: one N = 256 MMA reads its A tile once for two
      // accumulators (A0 | A1 and A2 | A3 are adjacent in TMEM).
      const uint32_t idesc_wide = idesc_s8_s32(kRows, 2 * kRows);
      uint32_t i = 0, chunk = 0;  // K-blocks and chunks issued so far
      bool ok = true;
      for (int f = walk.first(); ok && walk.in_range(f); ++f) {
        if (walk.skip(f)) continue;
        const int64_t lo = walk.lo(f), hi = walk.hi(f);
        for (int64_t kb = lo; kb < hi; ++kb, ++i) {
          const int j = static_cast<int>((kb - lo) % kChunkKB);
          if (j == 0) {
            if (*abort_flag || !mbar_wait(acc_empty, (chunk & 1u) ^ 1u)) {
              record_error(t.status, HSI_E_TIMEOUT);
              *abort_flag = 1;
              ok = false;
              break;
            }
            tc_fence_after();
          }
          const int so = i % kOpStages;
          if (!mbar_wait(&op_full[so], (i / kOpStages) & 1u)) {
            record_error(t.status, HSI_E_TIMEOUT);
            *abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          unsigned char* op = smem + L.op_off + static_cast<size_t>(so) * 3 * kLimbBytes;
          const uint64_t dd = smem_desc_sw128(op);
          const uint64_t d1 = smem_desc_sw128(op + kLimbBytes);
          const uint64_t d2 = smem_desc_sw128(op + 2 * kLimbBytes);
#pragma unroll
          for (int k = 0; k < kKB / 32; ++k) {
            const uint64_t adv = static_cast<uint64_t>(k * 2);  // 32 bytes of K, in 16-byte units
            const uint32_t acc = (j > 0 || k > 0) ? 1u : 0u;
            umma_i8(tmem + 0, dd + adv, dd + adv, idesc_wide, acc);    // A0 | A1 = D [D; L1]^T
            umma_i8(tmem + 256, d1 + adv, d1 + adv, idesc_wide, acc);  // A2 | A3 = L1 [L1; L2]^T
            umma_i8(tmem + 256, dd + adv, d2 + adv, idesc, 1u);        // A2 += D L2^T
          }
          umma_commit(&op_empty[so]);
          if (j == kChunkKB - 1 || kb == hi - 1) {
            umma_commit(acc_full);
            ++chunk;
          }
        }
      }
      // TMEM is freed at the end of the kernel: make sure no MMA of this
      // thread is still running by then (bounded wait).
      if (i > 0) {
        umma_commit(mma_done);
        if (!mbar_wait(mma_done, 0)) record_error(t.status, HSI_E_TIMEOUT);
      }
    }
  } else if (warp < kWarpEpi0) {
    // ---------------- converters ----------------
    // Each input stage is half a K-block (64 pixels).  Warp cw owns 4 band
    // pairs (b, b+4) -- lanes 0-15 the first band, 16-31 the second, 4 pixels
    // per lane -- so one store instruction covers two rows whose swizzled
    // chunks never share a bank.
    const int cw = warp - kWarpConv0;
    constexpr int kSlots = kRows / 2 / kConvWarps;  // 4 band pairs per warp
    const int sub = lane >> 4, lp = (lane & 15) * 4;  // which band of the pair; pixel in the box
    // slot t2 holds band pair cw + 16 t2, i.e. band band0 + 32 t2 (four 8-row
    // swizzle atoms further down: byte offset o0 + 4096 t2); the second half of
    // a K-block sits 64 bytes along, i.e. four 16-byte chunks, which the swizzle
    // maps to o ^ 64
    const int band0 = (cw >> 2) * 8 + (cw & 3) + 4 * sub;
    const uint32_t o0 = sw128_byte(band0, lp);
    uint32_t i = 0;
    bool aborted = false;
    for (int f = walk.first(); !aborted && walk.in_range(f); ++f) {
      if (walk.skip(f)) continue;
      const FrameStats& F = t.f[f];
      const int B = F.bands;
      const int64_t P = F.pixels;
      // Role of each slot for this frame: a band (converted), the ones row, or a
      // row past it.  Rows past the ones row are not written at all: they only
      // reach Gram entries (i, j) with i > B or j > B, which nothing reads, so
      // whatever an earlier K-block or frame left there is harmless.
      float sc[kSlots], off[kSlots];
      bool is_band[kSlots], is_ones[kSlots];
#pragma unroll
      for (int t2 = 0; t2 < kSlots; ++t2) {
        const int b = band0 + 32 * t2;
        is_band[t2] = b < B;
        is_ones[t2] = b == B;
        sc[t2] = 0.0f;
        off[t2] = 0.0f;
        if (b < B) {
          const float s = ldexpf(1.0f, F.state->scale_exp[b]);
          sc[t2] = s;
          off[t2] = kMagicQ - F.state->shift[b] * s;  // exact when r * 2^e stays below 2^23
        }
      }
      // Range check on the packed high bytes: every converted y must have
      // byte 3 == 0x4B (the exponent of [2^23, 2^24)) and bit 23 clear (byte
      // 2 < 0x80).  The OR of the byte pairs catches any extra bit, the AND any
      // missing one; bytes 0-1 of the words hold byte 2 of four values, bytes
      // 2-3 their byte 3.
      uint32_t chk_or = 0x4B4B0000u, chk_and = 0x4B4BFFFFu;
      // sums of L2^2 and of L2 per lane in 32 bits (at most 64 * 8 * 2^14 =
      // 2^23 between flushes), added to the frame's 64-bit counters every 64
      // K-blocks
      unsigned int l2sq[kSlots] = {0u, 0u, 0u, 0u};
      int l2s[kSlots] = {0, 0, 0, 0};
      auto flush_l2 = [&]() {
#pragma unroll
        for (int t2 = 0; t2 < kSlots; ++t2) {
          unsigned long long sq = l2sq[t2];
          long long sm = l2s[t2];
#pragma unroll
          for (int o = 8; o > 0; o >>= 1) {
            sq += __shfl_xor_sync(0xffffffffu, sq, o);
            sm += __shfl_xor_sync(0xffffffffu, sm, o);
          }
          const int b = band0 + 32 * t2;
          if ((lane & 15) == 0 && b < B) {
            if (sq != 0ull) atomicAdd(&F.state->l2sq[b], sq);
            if (sm != 0ll)
              atomicAdd(reinterpret_cast<unsigned long long*>(&F.state->l2sum[b]),
                        static_cast<unsigned long long>(sm));  // two's complement: adds mod 2^64
          }
          l2sq[t2] = 0u;
          l2s[t2] = 0;
        }
      };
      // limbs of four converted values (y bits) of one slot, stored at byte offset o
      auto put = [&](unsigned char* op, uint32_t o, const uint32_t (&y)[4], int t2) {
        const uint32_t p01 = __byte_perm(y[0], y[1], 0x5140), p23 = __byte_perm(y[2], y[3], 0x5140);
        const uint32_t h01 = __byte_perm(y[0], y[1], 0x7362), h23 = __byte_perm(y[2], y[3], 0x7362);
        const uint32_t l2 = __byte_perm(p01, p23, 0x5410) ^ 0x80808080u;
        const uint32_t l1 = __byte_perm(p01, p23, 0x7632) ^ 0x80808080u;
        // byte2 <= 127 in range, so the shift carries nothing across bytes
        const uint32_t dl = (__byte_perm(h01, h23, 0x5410) << 1) ^ 0x80808080u;
        chk_or |= h01 | h23;
        chk_and &= h01 & h23;
        // signed bytes: the limbs are two's-complement INT8
        l2sq[t2] = static_cast<unsigned int>(
            __dp4a(static_cast<int>(l2), static_cast<int>(l2), static_cast<int>(l2sq[t2])));
        l2s[t2] = __dp4a(static_cast<int>(l2), 0x01010101, l2s[t2]);
        *reinterpret_cast<uint32_t*>(op + o) = dl;
        *reinterpret_cast<uint32_t*>(op + kLimbBytes + o) = l1;
        *reinterpret_cast<uint32_t*>(op + 2 * kLimbBytes + o) = l2;
      };
      // One half K-block.  `full`: all 64 pixels lie in the frame (every K-block
      // but a frame's last), so no per-pixel validity test is needed.
      auto convert_half = [&](auto full, const T* in, int sub_off, unsigned char* op, int half, int nvalid) {
#pragma unroll
        for (int t2 = 0; t2 < kSlots; ++t2) {
          const uint32_t o = (o0 + 4096u * t2) ^ (half ? 64u : 0u);
          if (is_band[t2]) {
            const float4 x = load4f<T>(in + (band0 + 32 * t2) * kBoxPx + sub_off + lp);
            const float xv[4] = {x.x, x.y, x.z, x.w};
            uint32_t y[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              y[e] = __float_as_uint(fmaf(xv[e], sc[t2], off[t2]));
              // pixels past the frame convert as q = 0 (a fully unrolled select:
              // no dynamic index into y[])
              if (!decltype(full)::value && e >= nvalid) y[e] = kZeroBits;
            }
            put(op, o, y, t2);
          } else if (is_ones[t2]) {
            // the ones row: q = 2^16 (D = 2, L1 = L2 = 0) for pixels in the frame
            uint32_t dl = 0x02020202u;
            if (!decltype(full)::value) dl = nvalid >= 4 ? dl : (0x02020202u & ((1u << (8 * nvalid)) - 1u));
            *reinterpret_cast<uint32_t*>(op + o) = dl;
            *reinterpret_cast<uint32_t*>(op + kLimbBytes + o) = 0u;
            *reinterpret_cast<uint32_t*>(op + 2 * kLimbBytes + o) = 0u;
          }
        }
      };
      // K-blocks before kb_full hold 128 pixels of the frame each
      const int64_t kb_full = F.kb_begin + P / kKB;
      int since_flush = 0;
      for (int64_t kb = walk.lo(f); kb < walk.hi(f) && !aborted; ++kb, ++i) {
        const int so = i % kOpStages;
        unsigned char* op = smem + L.op_off + static_cast<size_t>(so) * 3 * kLimbBytes;
        const bool full = kb < kb_full;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          const uint32_t box = i * kBoxesPerKB + half / kHalvesPerBox;  // input box of this half
          const int s = box % kInStages;
          const int sub_off = (half % kHalvesPerBox) * kHalfPx;         // its pixels within the box
          if ((sub_off == 0 && !mbar_wait(&in_full[s], (box / kInStages) & 1u)) ||
              (half == 0 && !mbar_wait(&op_empty[so], ((i / kOpStages) & 1u) ^ 1u))) {
            record_error(t.status, HSI_E_TIMEOUT);
            *abort_flag = 1;
            aborted = true;
            break;
          }
          const T* in = reinterpret_cast<const T*>(smem + L.in_off + static_cast<size_t>(s) * in_tile_bytes<T>());
          if (full) {
            convert_half(std::true_type{}, in, sub_off, op, half, 4);
          } else {
            const int64_t gp = (kb - F.kb_begin) * kKB + half * kHalfPx + lp;
            const int nvalid = gp >= P ? 0 : (P - gp >= 4 ? 4 : static_cast<int>(P - gp));
            convert_half(std::false_type{}, in, sub_off, op, half, nvalid);
          }
          __syncwarp();
          if (lane == 0 && sub_off + kHalfPx == kBoxPx) mbar_arrive(&in_empty[s]);
          if (half == 1) {
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&op_full[so]);
          }
        }
        if (++since_flush == 64) {
          flush_l2();
          since_flush = 0;
        }
      }
      // end of the piece: the remaining L2^2 sums and the range check
      flush_l2();
      const bool bad = (chk_or & 0xFFFF8080u) != 0x4B4B0000u || (chk_and >> 16) != 0x4B4Bu;
      if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&F.state->flags, 1);
    }
  } else {
    // ---------------- epilogue ----------------
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int row = q * 32 + lane;
    const uint32_t trow = tmem + (static_cast<uint32_t>(q * 32) << 16);
    uint32_t chunk = 0;
    bool ok = true;
    for (int f = walk.first(); ok && walk.in_range(f); ++f) {
      if (walk.skip(f)) continue;
      const FrameStats& F = t.f[f];
      long long* outH = F.slots + static_cast<size_t>(blockIdx.x - F.cta_lo) * kSlotElems;
      long long* outL = outH + kRows * kRows;
      const int64_t nkb = walk.hi(f) - walk.lo(f);
      const int nch = static_cast<int>(div_up<int64_t>(nkb, kChunkKB));
      for (int c = 0; c < nch; ++c, ++chunk) {
        if (*abort_flag || !mbar_wait(acc_full, chunk & 1u)) {
          record_error(t.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll 1
        for (int cb = 0; cb < kRows / 16; ++cb) {
          const size_t e0 = static_cast<size_t>(16 * cb) * kRows + row;  // column-major
          {
            uint32_t a0[16];
            tmem_ld16(trow + 0 + 16 * cb, a0);
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              long long* d = outH + e0 + static_cast<size_t>(j) * kRows;
              *d = (c == 0 ? 0ll : *d) + static_cast<int>(a0[j]);
            }
          }
          uint32_t a1[16], a2[16], a3[16];
          tmem_ld16(trow + 128 + 16 * cb, a1);
          tmem_ld16(trow + 256 + 16 * cb, a2);
          tmem_ld16(trow + 384 + 16 * cb, a3);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const long long l = (static_cast<long long>(static_cast<int>(a1[j])) << 15) +
                                (static_cast<long long>(static_cast<int>(a2[j])) << 7) +
                                static_cast<long long>(static_cast<int>(a3[j]));
            long long* d = outL + e0 + static_cast<size_t>(j) * kRows;
            *d = (c == 0 ? 0ll : *d) + l;
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kWarpMma) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// Reference point and fixed-point scale per band from a regular subsample
// (about 256 evenly spaced runs of 64 pixels on frames above 512 runs): r = the midpoint of the
// subsample's range (which minimises its largest |x - r|, and, being built
// from a minimum and a maximum, does not depend on the order the blocks
// finish in), e such that that largest |x - r| maps to 2^20 (4x headroom
// below 2^22).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int scale_exp_for(float maxdev) {
  if (!(maxdev > 0.0f)) return 20;
  int e;
  frexpf(maxdev, &e);  // maxdev in [2^(e-1), 2^e)
  int k = 20 - e;      // maxdev * 2^k < 2^20
  return k < -120 ? -120 : (k > 120 ? 120 : k);
}

// Monotone map of a float onto a signed int, so atomicMin/atomicMax order
// floats of either sign.
__device__ __forceinline__ int float_order(float v) {
  const int i = __float_as_int(v);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float order_float(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// One block per frame.
__global__ void shift_init_kernel(const __grid_constant__ FrameTable t) {
  StatsState* st = t.f[blockIdx.x].state;
  for (int b = threadIdx.x; b <= HSI_MAX_BANDS; b += blockDim.x) {
    st->sub_lo[b] = 0x7fffffff;
    st->sub_hi[b] = static_cast<int>(0x80000000u);
  }
}

// Block-wide sum / count (into this block's slot) and min / max (folded into
// the frame's state with atomics).
// Called once per slot by every thread of the block; the leading barrier
// keeps a call's writes behind thread 0's reads of the one before.
__device__ void fold_subsample(double sum, double cnt, float lo, float hi, StatsState* st, int b, int slot) {
  __shared__ double s_sum[8], s_cnt[8];
  __shared__ int s_lo[8], s_hi[8];
  __syncthreads();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    s_sum[warp] = sum;
    s_cnt[warp] = cnt;
    s_lo[warp] = float_order(lo);
    s_hi[warp] = float_order(hi);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ts = s_sum[0], tc = s_cnt[0];
    int tl = s_lo[0], th = s_hi[0];
    for (int w = 1; w < 8; ++w) {
      ts += s_sum[w];
      tc += s_cnt[w];
      tl = min(tl, s_lo[w]);
      th = max(th, s_hi[w]);
    }
    st->sub_sum[b][slot] = ts;
    st->sub_cnt[b][slot] = tc;
    if (tl <= th) {  // the block saw a value other than NaN
      atomicMin(&st->sub_lo[b], tl);
      atomicMax(&st->sub_hi[b], th);
    }
  }
}

// Subsample statistics, grid (bands, kShiftSplit / kShiftItems, frames):
// runs of 64 pixels, about 256 of them per band on frames above 512 runs.
// Each block takes kShiftItems consecutive slots and issues the first
// kShiftHeld loads of every slot before reducing any, so that a block keeps
// 16 loads per thread in flight; each slot's sums are still taken over the
// same runs in the same order, so that the slots hold the same values at any
// kShiftItems.
template <typename T>
__global__ void __launch_bounds__(256) shift_partial_kernel(const __grid_constant__ FrameTable t) {
  const FrameStats& F = t.f[blockIdx.z];
  const int b = blockIdx.x;
  if (b >= F.bands) return;
  const T* plane = static_cast<const T*>(F.cube) + plane_of(F, b) * F.stride;
  const int64_t pixels = F.pixels;
  const int64_t runs = div_up<int64_t>(pixels, 64);
  const int64_t step = runs > 512 ? runs / 256 : 1;  // about 256 runs (16384 pixels) per band
  const int64_t sampled = div_up<int64_t>(runs, step);
  constexpr int kRowGroups = 256 / 64;  // runs a block covers per pass
  const int row = threadIdx.x / 64, col = threadIdx.x & 63;
  float held[kShiftItems][kShiftHeld];
  unsigned valid = 0u;
#pragma unroll
  for (int i = 0; i < kShiftItems; ++i) {
    const int slot = blockIdx.y * kShiftItems + i;
    const int64_t r0 = sampled * slot / kShiftSplit, r1 = sampled * (slot + 1) / kShiftSplit;
    const int64_t first = (r0 + row) * step * 64 + col;  // pixel of this thread's first run
    const int count = static_cast<int>(r1 - r0);          // runs of the slot (at most 32)
#pragma unroll
    for (int k = 0; k < kShiftHeld; ++k) {
      const int64_t px = first + static_cast<int64_t>(kRowGroups * k) * step * 64;
      held[i][k] = 0.0f;
      if (row + kRowGroups * k < count && px < pixels) {
        held[i][k] = static_cast<float>(plane[px]);
        valid |= 1u << (i * kShiftHeld + k);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kShiftItems; ++i) {
    const int slot = blockIdx.y * kShiftItems + i;
    const int64_t r0 = sampled * slot / kShiftSplit, r1 = sampled * (slot + 1) / kShiftSplit;
    double sum = 0.0, cnt = 0.0;
    float lo = INFINITY, hi = -INFINITY;
#pragma unroll
    for (int k = 0; k < kShiftHeld; ++k) {
      if (valid & (1u << (i * kShiftHeld + k))) {
        const float v = held[i][k];
        if (t.center_mean) {
          sum += static_cast<double>(v);
          cnt += 1.0;
        }
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
      }
    }
    // runs past the held ones (slots of more than kRowGroups * kShiftHeld runs)
    for (int64_t run = r0 + row + kRowGroups * kShiftHeld; run < r1; run += kRowGroups) {
      const int64_t px = run * step * 64 + col;
      if (px < pixels) {
        const float v = static_cast<float>(plane[px]);
        if (t.center_mean) {
          sum += static_cast<double>(v);
          cnt += 1.0;
        }
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
      }
    }
    fold_subsample(sum, cnt, lo, hi, F.state, b, slot);
  }
}

// One block per frame: r = the caller's reference, else the midpoint of the
// subsample's range (tensor path) or its mean (FP32 path, whose rounding
// grows with |mean - r|), e such that the subsample's largest |x - r| maps to
// 2^20 (4x headroom below 2^22), r snapped to the 2^-e grid so that inputs on
// that grid (FP16 cubes) convert exactly.
__global__ void __launch_bounds__(256) shift_finalize_kernel(const __grid_constant__ FrameTable t) {
  const FrameStats& F = t.f[blockIdx.x];
  StatsState* st = F.state;
  const int bands = F.bands;
  for (int b = threadIdx.x; b <= HSI_MAX_BANDS; b += blockDim.x) {
    st->maxdev_bits[b] = 0;
    st->l2sq[b] = 0ull;
    st->l2sum[b] = 0ll;
    if (b > bands) {
      st->shift[b] = 0.0f;
      st->scale_exp[b] = 0;
      continue;
    }
    if (b == bands) {
      st->shift[b] = 0.0f;
      st->scale_exp[b] = kOnesExp;
      continue;
    }
    const bool seen = st->sub_lo[b] <= st->sub_hi[b];
    const float slo = order_float(st->sub_lo[b]), shi = order_float(st->sub_hi[b]);
    float r = 0.0f;
    if (F.reference) {
      r = F.reference[b];
    } else if (t.center_mean) {
      double sum = 0.0, cnt = 0.0;
      for (int k = 0; k < kShiftSplit; ++k) {
        sum += st->sub_sum[b][k];
        cnt += st->sub_cnt[b][k];
      }
      r = cnt > 0.0 ? static_cast<float>(sum / cnt) : 0.0f;
    } else if (seen) {
      r = 0.5f * slo + 0.5f * shi;
    }
    const float lo = seen ? slo : r, hi = seen ? shi : r;
    const int e = scale_exp_for(fmaxf(fabsf(hi - r), fabsf(lo - r)) * 1.0000001f);
    // FP32 path: r on the 2^-e grid, so that inputs on that grid (FP16
    // cubes) convert exactly.  Tensor path: r on the 256x coarser grid, so
    // that r * 2^e is a multiple of 256 and adds nothing to the low limb
    // (inputs on a grid of 256 steps -- integer counts, most FP16 values --
    // then have L2 = 0 and exact moments).
    const int g = t.center_mean ? e : e - 8;
    r = ldexpf(rintf(ldexpf(r, g)), -g);
    st->shift[b] = r;
    st->scale_exp[b] = e;
  }
  if (threadIdx.x == 0) st->flags = 0;
}

// After the first GEMM, for frames where a value fell out of range only:
// max |x - r| per band over the whole frame.  Work items are (frame, band,
// slice of 1/kShiftSplit of the pixels), strided over a small grid, so that
// the usual case -- no frame out of range -- costs one flag test per item.
template <typename T>
__global__ void __launch_bounds__(256) range_kernel(const __grid_constant__ FrameTable t) {
  const int per_frame = t.max_bands * kShiftSplit;
  for (int item = blockIdx.x; item < t.n * per_frame; item += gridDim.x) {
    const FrameStats& F = t.f[item / per_frame];
    const int b = (item % per_frame) / kShiftSplit, split = item % kShiftSplit;
    if (b >= F.bands || !(F.state->flags & 1)) continue;
    const T* plane = static_cast<const T*>(F.cube) + plane_of(F, b) * F.stride;
    const int64_t per = div_up<int64_t>(F.pixels, kShiftSplit);
    const int64_t p0 = per * split, p1 = min(F.pixels, p0 + per);
    float lo = INFINITY, hi = -INFINITY;
    for (int64_t px = p0 + threadIdx.x; px < p1; px += blockDim.x) {
      const float v = static_cast<float>(plane[px]);
      lo = fminf(lo, v);
      hi = fmaxf(hi, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0 && hi >= lo) {
      const float r = F.state->shift[b];
      atomicMax(&F.state->maxdev_bits[b], __float_as_int(fmaxf(hi - r, r - lo)));
    }
  }
}

// One block per frame: if a value was out of range, take the range of the
// whole frame and arm the conditional re-run; otherwise leave it disarmed.
__global__ void rescale_kernel(const __grid_constant__ FrameTable t) {
  StatsState* st = t.f[blockIdx.x].state;
  if (!(st->flags & 1)) return;
  for (int b = threadIdx.x; b < t.f[blockIdx.x].bands; b += blockDim.x) {
    const float dev = __int_as_float(st->maxdev_bits[b]);
    const int e = scale_exp_for(dev * 1.0000001f) + 1;  // observed max -> below 2^21
    st->scale_exp[b] = e;
    // keep r on the 256x coarser grid of the new scale (as shift_finalize)
    st->shift[b] = ldexpf(rintf(ldexpf(st->shift[b], e - 8)), -(e - 8));
    st->l2sq[b] = 0ull;  // recounted by the re-run
    st->l2sum[b] = 0ll;
  }
  __syncthreads();
  if (threadIdx.x == 0) st->flags = 2;
}

// Sum the pieces' INT64 partials of each frame (exact, so the order is free)
// and form F = 2^30 H + 2^9 Lo in FP64.  Grid (kRows * kRows / 256, frames).
__global__ void __launch_bounds__(256) stats_reduce_kernel(const __grid_constant__ FrameTable t) {
  const FrameStats& F = t.f[blockIdx.y];
  const int e = blockIdx.x * 256 + threadIdx.x;  // entry in [0, 128*128)
  long long h = 0, l = 0;
  for (int s = 0; s < F.nslots; ++s) {
    const long long* slot = F.slots + static_cast<size_t>(s) * kSlotElems;
    h += slot[e];
    l += slot[kRows * kRows + e];
  }
  F.fsum[e] = ldexp(static_cast<double>(h), 30) + ldexp(static_cast<double>(l), 9);
}

// S = (F + F^T)/2, unscaled -> shifted sums (S1, S2, N) -> raw moments in FP64
// (moments_from_shifted, src/linalg.cpp:81-103).  fsum is column-major:
// fsum[col * 128 + row] = F[row][col].  Output: sum[B], outer[B*B] (full,
// symmetric), count.  Grid (max bands, frames): block (i, f) writes row i.
__global__ void __launch_bounds__(128) stats_finalize_kernel(const __grid_constant__ FrameTable t) {
  const FrameStats& Fr = t.f[blockIdx.y];
  const int B = Fr.bands;
  const int i = blockIdx.x;
  if (i >= B) return;
  __shared__ double s1[kRows];
  __shared__ double r[kRows];
  __shared__ int ex[kRows];
  const double* fsum = Fr.fsum;
  const StatsState* st = Fr.state;
  double* moments = Fr.moments;
  auto F = [&](int row, int col) { return fsum[static_cast<size_t>(col) * kRows + row]; };
  const double N = ldexp(F(B, B), -2 * kOnesExp);
  for (int j = threadIdx.x; j < B; j += blockDim.x) {
    ex[j] = st->scale_exp[j];
    r[j] = static_cast<double>(st->shift[j]);
    s1[j] = ldexp(0.5 * (F(j, B) + F(B, j)), -(st->scale_exp[j] + kOnesExp));
  }
  __syncthreads();
  double* outer = moments + B;
  if (i == 0)
    for (int j = threadIdx.x; j < B; j += blockDim.x) moments[j] = s1[j] + N * r[j];
  // row i, columns j <= i, mirrored, so the matrix is exactly symmetric
  for (int j = threadIdx.x; j <= i; j += blockDim.x) {
    double q = 0.5 * (F(i, j) + F(j, i));
    if (i == j)
      q += static_cast<double>(st->l2sq[i]);  // the weight-1 diagonal, exact
    else  // the mean part of the weight-1 off-diagonal sums
      q += static_cast<double>(st->l2sum[i]) * static_cast<double>(st->l2sum[j]) / N;
    const double s2 = ldexp(q, -(ex[i] + ex[j]));
    const double v = s2 + r[i] * s1[j] + s1[i] * r[j] + N * r[i] * r[j];
    outer[static_cast<size_t>(i) * B + j] = v;
    outer[static_cast<size_t>(j) * B + i] = v;
  }
  if (i == 0 && threadIdx.x == 0) moments[B + B * B] = N;
}

// ---------------------------------------------------------------------------
// Plain FP32 SIMT moments: the comparator path, and the path for B >= 128.
// Each block owns a 64-band x 64-band tile of the lower triangle over a slice
// of pixels, 4x4 register blocks per thread, FP32 sums over each 32-pixel
// staging step flushed into FP64 registers (longer FP32 chains measurably bias
// the covariance), written to per-block partials, then reduced in a fixed
// order.  The shift (and ones row) work as in the tensor path.
// ---------------------------------------------------------------------------
constexpr int kSimtTile = 64;
constexpr int kSimtPx = 32;

template <typename T>
__global__ void __launch_bounds__(256) stats_simt_kernel(const T* __restrict__ cube, int64_t pixels, int64_t stride,
                                                        int bands, const StatsState* __restrict__ st,
                                                        double* __restrict__ partials, int slices) {
  const float* shift = st->shift;
  // blockIdx.x: pixel slice; blockIdx.y: lower-triangle tile pair
  const int tiles = (bands + 1 + kSimtTile - 1) / kSimtTile;  // rows incl. the ones row
  int ti = 0, pair = blockIdx.y;
  while (pair > ti) {
    pair -= ti + 1;
    ++ti;
  }
  const int tj = pair;
  __shared__ float si[kSimtPx][kSimtTile + 4];
  __shared__ float sj[kSimtPx][kSimtTile + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4];
  double dacc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      acc[a][c] = 0.0f;
      dacc[a][c] = 0.0;
    }
  const int64_t per = div_up<int64_t>(pixels, slices);
  const int64_t p0 = per * blockIdx.x, p1 = min(pixels, p0 + per);
  int since_flush = 0;
  for (int64_t base = p0; base < p1; base += kSimtPx) {
    for (int e = threadIdx.x; e < kSimtPx * kSimtTile; e += blockDim.x) {
      const int px = e % kSimtPx, rb = e / kSimtPx;
      const int64_t p = base + px;
      const bool valid = p < p1;
      const int bi = ti * kSimtTile + rb, bj = tj * kSimtTile + rb;
      float vi = 0.0f, vj = 0.0f;
      if (valid) {
        if (bi < bands) vi = static_cast<float>(cube[static_cast<int64_t>(bi) * stride + p]) - shift[bi];
        else if (bi == bands) vi = 1.0f;
        if (bj < bands) vj = static_cast<float>(cube[static_cast<int64_t>(bj) * stride + p]) - shift[bj];
        else if (bj == bands) vj = 1.0f;
      }
      si[px][rb] = vi;
      sj[px][rb] = vj;
    }
    __syncthreads();
#pragma unroll 8
    for (int px = 0; px < kSimtPx; ++px) {
      const float4 a = *reinterpret_cast<const float4*>(&si[px][ty * 4]);
      const float4 b = *reinterpret_cast<const float4*>(&sj[px][tx * 4]);
      const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
    }
    __syncthreads();
    since_flush += kSimtPx;
    if (since_flush >= kSimtPx) {
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          dacc[r][c] += acc[r][c];
          acc[r][c] = 0.0f;
        }
      since_flush = 0;
    }
  }
  // partial layout: [slice][col][row] over the padded (tiles*64)^2 square
  const int n = tiles * kSimtTile;
  double* out = partials + static_cast<size_t>(blockIdx.x) * n * n;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int row = ti * kSimtTile + ty * 4 + r, col = tj * kSimtTile + tx * 4 + c;
      const double v = dacc[r][c] + acc[r][c];
      // F[row][col] for the lower-triangle tile; mirrored so that
      // (F + F^T)/2 yields the full symmetric sum.
      if (ti == tj) {
        out[static_cast<size_t>(col) * n + row] = v;
      } else {
        out[static_cast<size_t>(col) * n + row] = v;
        out[static_cast<size_t>(row) * n + col] = v;
      }
    }
}

__global__ void __launch_bounds__(256) simt_reduce_kernel(const double* __restrict__ partials, int slices, int n,
                                                         double* __restrict__ fsum) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * n) return;
  double t = 0.0;
  for (int c = 0; c < slices; ++c) t += partials[static_cast<size_t>(c) * n * n + e];
  fsum[e] = t;
}

__global__ void __launch_bounds__(256) simt_finalize_kernel(const double* __restrict__ fsum, int n,
                                                           const StatsState* __restrict__ st, int bands,
                                                           double* __restrict__ moments) {
  const float* shift = st->shift;
  __shared__ double s1[HSI_MAX_BANDS];
  __shared__ double r[HSI_MAX_BANDS];
  const int B = bands;
  auto F = [&](int row, int col) { return fsum[static_cast<size_t>(col) * n + row]; };
  const double N = F(B, B);
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    s1[i] = F(i, B);
    r[i] = static_cast<double>(shift[i]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < B; i += blockDim.x) moments[i] = s1[i] + N * r[i];
  for (int e = threadIdx.x; e < B * B; e += blockDim.x) {
    const int i = e / B, j = e % B;
    if (j > i) continue;
    const double v = F(i, j) + r[i] * s1[j] + s1[i] * r[j] + N * r[i] * r[j];
    moments[B + e] = v;
    moments[B + j * B + i] = v;
  }
  if (threadIdx.x == 0) moments[B + B * B] = N;
}

// ---------------------------------------------------------------------------
// Frames of 128..254 bands.  Two contiguous band views of at most 127 bands
// take the exact tensor-core moments as one launch sequence.  Only the cross
// block between them runs on the CUDA cores, each band referenced to its mean
// from the views.  An FP64 assembly gives the frame's raw moments.  The
// CUDA-core work is the h x (B - h) block instead of the whole lower triangle.
// ---------------------------------------------------------------------------
// Mean of band b of a view's raw moments (nb bands), rounded to FP32: the
// reference the cross sums subtract.
__device__ __forceinline__ double view_ref(const double* m, int nb, int b) {
  return static_cast<double>(static_cast<float>(m[b] / m[nb + nb * nb]));
}

// Block (ti, tj) of the cross sums over a pixel slice: rows a = view-1 bands
// [64 ti, 64 ti + 64) (frame bands h + a), columns c = view-0 bands [64 tj, ...).
// FP32 products of mean-referenced values, summed over each 32-pixel step, then
// FP64, as the CUDA-core moments.  Staging is [row][pixel]: a warp loads 32
// consecutive pixels of one band and stores them to 32 consecutive banks; the
// math reads 4 pixels of a row per 128-bit load.  Thread (ty, tx) owns rows
// ty + 16 r and columns tx + 16 c, so the 16 column rows a warp reads at once
// are consecutive, and the row stride of 36 floats puts them on distinct bank
// groups (two wavefronts).
constexpr int kCrossStride = kSimtPx + 4;

template <typename T>
__global__ void __launch_bounds__(256, 3) stats_cross_kernel(const T* __restrict__ cube, int64_t pixels, int64_t stride,
                                                            int h, int n1, const double* __restrict__ m0,
                                                            const double* __restrict__ m1, double* __restrict__ partials,
                                                            int slices, int ct, int nrp, int ncp) {
  const int ti = blockIdx.y / ct, tj = blockIdx.y % ct;
  __shared__ __align__(16) float stage[2 * kSimtTile][kCrossStride];  // rows 0-63: a, 64-127: c
  __shared__ float ref[2 * kSimtTile];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = threadIdx.x; k < 2 * kSimtTile; k += blockDim.x) {
    const int a = ti * kSimtTile + k, c = tj * kSimtTile + (k - kSimtTile);
    ref[k] = k < kSimtTile ? (a < n1 ? static_cast<float>(view_ref(m1, n1, a)) : 0.0f)
                           : (c < h ? static_cast<float>(view_ref(m0, h, c)) : 0.0f);
  }
  // staged rows of this thread: warp + 8 k, k < 16 (k < 8: a rows, then c rows);
  // row a0 + 8 k of view 1 is frame band h + a0 + 8 k, row c0 + 8 k of view 0 band c0 + 8 k
  constexpr int kRowsPerThread = 2 * kSimtTile / 8;
  const int a0 = ti * kSimtTile + warp, c0 = tj * kSimtTile + warp;
  const T* srcA = cube + static_cast<int64_t>(h + a0) * stride;
  const T* srcC = cube + static_cast<int64_t>(c0) * stride;
  const int64_t step8 = 8 * stride;
  __syncthreads();
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4];
  double dacc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      acc[r][c] = 0.0f;
      dacc[r][c] = 0.0;
    }
  const int64_t per = div_up<int64_t>(pixels, slices);
  const int64_t p0 = per * blockIdx.x, p1 = min(pixels, p0 + per);
  float nxt[kRowsPerThread];
  auto fetch = [&](int64_t base) {
    const int64_t p = base + lane;
    const bool in = p < p1;
#pragma unroll
    for (int k = 0; k < kRowsPerThread / 2; ++k) {
      nxt[k] = (in && a0 + 8 * k < n1) ? static_cast<float>(srcA[k * step8 + p]) - ref[warp + 8 * k] : 0.0f;
      nxt[k + kRowsPerThread / 2] =
          (in && c0 + 8 * k < h) ? static_cast<float>(srcC[k * step8 + p]) - ref[kSimtTile + warp + 8 * k] : 0.0f;
    }
  };
  for (int64_t base = p0; base < p1; base += kSimtPx) {
    fetch(base);
#pragma unroll
    for (int k = 0; k < kRowsPerThread; ++k) stage[warp + 8 * k][lane] = nxt[k];
    __syncthreads();
#pragma unroll 2
    for (int q = 0; q < kSimtPx; q += 4) {
      float4 x[4], y[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) x[r] = *reinterpret_cast<const float4*>(&stage[ty + 16 * r][q]);
#pragma unroll
      for (int c = 0; c < 4; ++c) y[c] = *reinterpret_cast<const float4*>(&stage[kSimtTile + tx + 16 * c][q]);
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          acc[r][c] = fmaf(x[r].x, y[c].x, acc[r][c]);
          acc[r][c] = fmaf(x[r].y, y[c].y, acc[r][c]);
          acc[r][c] = fmaf(x[r].z, y[c].z, acc[r][c]);
          acc[r][c] = fmaf(x[r].w, y[c].w, acc[r][c]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        dacc[r][c] += acc[r][c];
        acc[r][c] = 0.0f;
      }
  }
  // partial layout: [slice][column c][row a] over the padded ncp x nrp block
  double* out = partials + static_cast<size_t>(blockIdx.x) * nrp * ncp;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c)
      out[static_cast<size_t>(tj * kSimtTile + tx + 16 * c) * nrp + ti * kSimtTile + ty + 16 * r] = dacc[r][c];
}

// Raw moments [sum (B) | outer (B x B) | N] of the frame from the views' raw
// moments (m0: bands [0, h), m1: bands [h, B)) and the cross sums.  With the
// references r used by the cross kernel,
//   sum_p x_a x_c = C_ac + r_c S_a + r_a S_c - N r_a r_c.
__global__ void __launch_bounds__(256) split_assemble_kernel(const double* __restrict__ m0,
                                                            const double* __restrict__ m1,
                                                            const double* __restrict__ partials, int slices, int h,
                                                            int n1, int nrp, int ncp, double* __restrict__ moments) {
  const int B = h + n1;
  const double N = m0[h + h * h];
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e < B) moments[e] = e < h ? m0[e] : m1[e - h];
  if (e == 0) moments[B + static_cast<int64_t>(B) * B] = N;
  if (e >= static_cast<int64_t>(B) * B) return;
  const int i = static_cast<int>(e / B), j = static_cast<int>(e % B);
  double v;
  if (i < h && j < h) {
    v = m0[h + i * h + j];
  } else if (i >= h && j >= h) {
    v = m1[n1 + (i - h) * n1 + (j - h)];
  } else {
    const int a = i >= h ? i - h : j - h;  // view-1 band
    const int c = i >= h ? j : i;          // view-0 band
    double C = 0.0;
    for (int sl = 0; sl < slices; ++sl) C += partials[static_cast<size_t>(sl) * nrp * ncp + static_cast<size_t>(c) * nrp + a];
    const double ra = view_ref(m1, n1, a), rc = view_ref(m0, h, c);
    v = C + rc * m1[a] + ra * m0[c] - N * ra * rc;
  }
  moments[B + e] = v;
}

// Frames of 128..252 bands with quarters Q0..Q3 of at most 63 bands (q: their
// bounds).  Six exact tensor-core views: Q0 u Q1 and Q2 u Q3 (contiguous) for
// the sums and the diagonal blocks, and Qi u Qj (two runs, i in {0, 1}, j in
// {2, 3}) for the cross blocks.  Every entry of the frame's raw moments is an
// entry of one view's raw moments.
struct QuarterViews {
  const double* m[6];  // raw moments [sum | outer | N] of each view
  int nb[6];           // bands of each view
  int q[5];            // quarter bounds
};

__global__ void __launch_bounds__(256) quarter_assemble_kernel(const __grid_constant__ QuarterViews v,
                                                              double* __restrict__ moments) {
  const int B = v.q[4], h = v.q[2];
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e < B) moments[e] = e < h ? v.m[0][e] : v.m[1][e - h];
  if (e == 0) moments[B + static_cast<int64_t>(B) * B] = v.m[0][v.nb[0] + v.nb[0] * v.nb[0]];
  if (e >= static_cast<int64_t>(B) * B) return;
  const int i = static_cast<int>(e / B), k = static_cast<int>(e % B);
  double val;
  if (i < h && k < h) {
    val = v.m[0][v.nb[0] + i * v.nb[0] + k];
  } else if (i >= h && k >= h) {
    val = v.m[1][v.nb[1] + (i - h) * v.nb[1] + (k - h)];
  } else {
    const int c = i < h ? i : k, a = i < h ? k : i;  // c in Q0 u Q1, a in Q2 u Q3
    const int qc = c < v.q[1] ? 0 : 1, qa = a < v.q[3] ? 2 : 3;
    const int w = 2 + 2 * qc + (qa - 2);
    const int rc = c - v.q[qc], ra = (v.q[qc + 1] - v.q[qc]) + (a - v.q[qa]);
    val = v.m[w][v.nb[w] + rc * v.nb[w] + ra];
  }
  moments[B + e] = val;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

int num_sms() { return device_sm_count(); }

constexpr int kSimtSlices = 96;

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// Tensor path, a group of m frames: m states, m F matrices, and the pieces'
// partial slots (at most one per CTA plus one per frame boundary).
size_t tensor_ws_bytes(int m) {
  return static_cast<size_t>(m) * align256(sizeof(StatsState)) +
         static_cast<size_t>(m) * align256(kRows * kRows * sizeof(double)) +
         static_cast<size_t>(kMaxCtas + m) * kSlotElems * sizeof(long long);
}

size_t simt_ws_bytes(int bands) {
  const int n = ((bands + 1 + kSimtTile - 1) / kSimtTile) * kSimtTile;
  return align256(sizeof(StatsState)) + align256(static_cast<size_t>(kSimtSlices) * n * n * sizeof(double)) +
         align256(static_cast<size_t>(n) * n * sizeof(double));
}

// Split path (128..254 bands): view 0 holds bands [0, h), view 1 bands [h, B).
constexpr int kSplitMaxBands = 2 * kMaxTensorBands;

struct SplitDims {
  int h, n1;     // bands of the two views
  int rt, ct;    // 64-band tiles of the cross block (rows: view 1, columns: view 0)
  int nrp, ncp;  // padded rows and columns
};

SplitDims split_dims(int bands) {
  SplitDims d;
  d.h = (bands + 1) / 2;
  d.n1 = bands - d.h;
  d.rt = (d.n1 + kSimtTile - 1) / kSimtTile;
  d.ct = (d.h + kSimtTile - 1) / kSimtTile;
  d.nrp = d.rt * kSimtTile;
  d.ncp = d.ct * kSimtTile;
  return d;
}

size_t view_moments_bytes(int bands) {
  return align256((static_cast<size_t>(bands) + static_cast<size_t>(bands) * bands + 1) * sizeof(double));
}

// Quarter views serve frames of up to 4 x 63 bands (two quarters per view).
constexpr int kQuarterMaxBands = 4 * 63;

struct QuarterDims {
  int q[5];
  int nb[6];
  int64_t first[6];  // first plane of each view
  int run0[6];
  int64_t run1[6];   // second run's first plane, from the view's first plane
};

QuarterDims quarter_dims(int bands) {
  QuarterDims d;
  const int h = (bands + 1) / 2;
  d.q[0] = 0;
  d.q[1] = (h + 1) / 2;
  d.q[2] = h;
  d.q[3] = h + (bands - h + 1) / 2;
  d.q[4] = bands;
  d.nb[0] = h, d.first[0] = 0, d.run0[0] = h, d.run1[0] = 0;
  d.nb[1] = bands - h, d.first[1] = h, d.run0[1] = bands - h, d.run1[1] = 0;
  for (int i = 0; i < 2; ++i)
    for (int j = 2; j < 4; ++j) {
      const int w = 2 + 2 * i + (j - 2);
      d.run0[w] = d.q[i + 1] - d.q[i];
      d.nb[w] = d.run0[w] + (d.q[j + 1] - d.q[j]);
      d.first[w] = d.q[i];
      d.run1[w] = d.q[j] - d.q[i];
    }
  return d;
}

// The views' tensor-core workspace, their moments, and (two-view form) the cross partials.
size_t split_ws_bytes(int bands) {
  const SplitDims d = split_dims(bands);
  size_t two = tensor_ws_bytes(2) + view_moments_bytes(d.h) + view_moments_bytes(d.n1) +
               align256(static_cast<size_t>(kSimtSlices) * d.nrp * d.ncp * sizeof(double));
  if (bands <= kQuarterMaxBands) {
    const QuarterDims qd = quarter_dims(bands);
    size_t four = tensor_ws_bytes(6);
    for (int w = 0; w < 6; ++w) four += view_moments_bytes(qd.nb[w]);
    if (four > two) two = four;
  }
  return two;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn lookup_encode_fn() {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    return reinterpret_cast<EncodeTiledFn>(p);
  return nullptr;
}

// The driver's entry point is process-wide; a failed lookup is retried.
EncodeTiledFn encode_fn() {
  static std::atomic<EncodeTiledFn> fn{nullptr};
  EncodeTiledFn f = fn.load(std::memory_order_acquire);
  if (!f) {
    f = lookup_encode_fn();
    if (f) fn.store(f, std::memory_order_release);
  }
  return f;
}

FrameStats frame_of_job(const hsi_moments_job& j) {
  FrameStats F{};
  F.cube = j.cube;
  F.pixels = static_cast<int64_t>(j.height) * j.width;
  F.stride = j.plane_stride;
  F.reference = j.reference;
  F.moments = j.moments;
  F.bands = j.bands;
  F.run0 = j.bands;
  return F;
}

template <typename T>
void launch_shift(const FrameTable& t, cudaStream_t s) {
  shift_init_kernel<<<t.n, 256, 0, s>>>(t);
  static_assert(kShiftSplit % kShiftItems == 0, "whole slots per block");
  shift_partial_kernel<T><<<dim3(t.max_bands, kShiftSplit / kShiftItems, t.n), 256, 0, s>>>(t);
  shift_finalize_kernel<<<t.n, 256, 0, s>>>(t);
}

// One launch sequence for m <= kMaxBatch frames of element type T, all on the
// tensor path: shift + scale -> GEMM -> (conditional) range + rescale + GEMM
// re-run -> exact reduction -> finalize.
// run0 / run1_plane (nullable): frames that are two-run views of their cube.
template <typename T>
int launch_tensor_group(const hsi_moments_job* const* jobs, int m, void* workspace, cudaStream_t s,
                        int* status, const int* run0 = nullptr, const int64_t* run1_plane = nullptr) {
  static thread_local GemmParams p;  // large (13 KB): kept off the stack, one per host thread
  p = GemmParams{};
  FrameTable& t = p.t;
  t.n = m;
  t.status = status;
  int64_t total = 0;
  for (int f = 0; f < m; ++f) {
    t.f[f] = frame_of_job(*jobs[f]);
    t.f[f].kb_begin = total;
    total += div_up<int64_t>(t.f[f].pixels, kKB);
    if (t.f[f].bands > t.max_bands) t.max_bands = t.f[f].bands;
    int rc;
    if (run0 && run0[f] < t.f[f].bands) {
      FrameStats& F = t.f[f];
      F.run0 = run0[f];
      F.run1_plane = run1_plane[f];
      const int r1 = F.bands - F.run0;
      const size_t esize = jobs[f]->dtype == HSI_F32 ? 4 : 2;
      rc = encode_cube_map(&p.maps[f], jobs[f]->cube, jobs[f]->dtype, F.pixels, F.run0, F.stride, kBoxPx, F.run0);
      if (rc == HSI_OK)
        rc = encode_cube_map(&p.maps1[f],
                             static_cast<const unsigned char*>(jobs[f]->cube) +
                                 static_cast<size_t>(F.run1_plane) * F.stride * esize,
                             jobs[f]->dtype, F.pixels, r1, F.stride, kBoxPx, r1);
    } else {
      rc = encode_cube_map(&p.maps[f], jobs[f]->cube, jobs[f]->dtype, t.f[f].pixels, t.f[f].bands,
                           t.f[f].stride, kBoxPx, kRows);
    }
    if (rc != HSI_OK) return rc;
  }
  t.total_kb = total;
  int grid = num_sms();
  if (grid > kMaxCtas) grid = kMaxCtas;
  if (total < grid) grid = static_cast<int>(total);
  t.ctas = grid;
  // carve: states, F matrices, slots
  unsigned char* w = static_cast<unsigned char*>(workspace);
  long long* slots =
      reinterpret_cast<long long*>(w + static_cast<size_t>(m) * (align256(sizeof(StatsState)) +
                                                                 align256(kRows * kRows * sizeof(double))));
  int used = 0;
  for (int f = 0; f < m; ++f) {
    FrameStats& F = t.f[f];
    F.state = reinterpret_cast<StatsState*>(w + static_cast<size_t>(f) * align256(sizeof(StatsState)));
    F.fsum = reinterpret_cast<double*>(w + static_cast<size_t>(m) * align256(sizeof(StatsState)) +
                                       static_cast<size_t>(f) * align256(kRows * kRows * sizeof(double)));
    // CTAs c whose range [total*c/grid, total*(c+1)/grid) meets [kb_begin, kb_end)
    const int64_t k0 = F.kb_begin, k1 = F.kb_begin + div_up<int64_t>(F.pixels, kKB);
    int lo = -1, hi = -1;
    for (int c = 0; c < grid; ++c) {
      const int64_t c0 = total * c / grid, c1 = total * (c + 1) / grid;
      if (c1 > k0 && c0 < k1) {
        if (lo < 0) lo = c;
        hi = c;
      }
    }
    F.cta_lo = lo;
    F.nslots = hi - lo + 1;
    F.slots = slots + static_cast<size_t>(used) * kSlotElems;
    used += F.nslots;
  }
  if (used > kMaxCtas + m) return HSI_E_CAPACITY;  // cannot happen: pieces <= CTAs + frames - 1
  const StatsSmem L = stats_smem<T>();
  // set once per device and element type
  const cudaError_t configured = raise_smem_limit(stats_gemm_kernel<T>, static_cast<int>(L.total));
  if (configured != cudaSuccess) return static_cast<int>(configured);
  launch_shift<T>(t, s);
  p.conditional = 0;
  stats_gemm_kernel<T><<<grid, kThreads, L.total, s>>>(p);
  range_kernel<T><<<4 * num_sms(), 256, 0, s>>>(t);
  rescale_kernel<<<m, 128, 0, s>>>(t);
  p.conditional = 1;
  stats_gemm_kernel<T><<<grid, kThreads, L.total, s>>>(p);
  stats_reduce_kernel<<<dim3(kRows * kRows / 256, m), 256, 0, s>>>(t);
  stats_finalize_kernel<<<dim3(t.max_bands, m), 128, 0, s>>>(t);
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int launch_simt_stats(const hsi_moments_job& j, void* workspace, cudaStream_t s) {
  const int B = j.bands;
  const int64_t P = static_cast<int64_t>(j.height) * j.width;
  const int tiles = (B + 1 + kSimtTile - 1) / kSimtTile;
  const int n = tiles * kSimtTile;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  StatsState* state = reinterpret_cast<StatsState*>(w);
  double* partials = reinterpret_cast<double*>(w + align256(sizeof(StatsState)));
  double* fsum = reinterpret_cast<double*>(w + align256(sizeof(StatsState)) +
                                           align256(static_cast<size_t>(kSimtSlices) * n * n * sizeof(double)));
  static thread_local FrameTable t;  // 5.7 KB: kept off the stack, one per host thread
  t = FrameTable{};
  t.n = 1;
  t.max_bands = B;
  t.center_mean = 1;
  t.f[0] = frame_of_job(j);
  t.f[0].state = state;
  launch_shift<T>(t, s);
  const dim3 grid(kSimtSlices, tiles * (tiles + 1) / 2);
  stats_simt_kernel<T><<<grid, 256, 0, s>>>(static_cast<const T*>(j.cube), P, j.plane_stride, B, state, partials,
                                           kSimtSlices);
  simt_reduce_kernel<<<(n * n + 255) / 256, 256, 0, s>>>(partials, kSimtSlices, n, fsum);
  simt_finalize_kernel<<<1, 256, 0, s>>>(fsum, n, state, B, j.moments);
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int launch_quarter_stats(const hsi_moments_job& j, void* workspace, cudaStream_t s) {
  const QuarterDims d = quarter_dims(j.bands);
  unsigned char* w = static_cast<unsigned char*>(workspace) + tensor_ws_bytes(6);
  hsi_moments_job v[6];
  const hsi_moments_job* views[6];
  QuarterViews qv;
  for (int k = 0; k < 6; ++k) {
    v[k] = j;
    v[k].cube = static_cast<const unsigned char*>(j.cube) + static_cast<size_t>(d.first[k]) * j.plane_stride * sizeof(T);
    v[k].bands = d.nb[k];
    v[k].moments = reinterpret_cast<double*>(w);
    v[k].reference = nullptr;
    w += view_moments_bytes(d.nb[k]);
    views[k] = &v[k];
    qv.m[k] = v[k].moments;
    qv.nb[k] = d.nb[k];
  }
  for (int k = 0; k < 5; ++k) qv.q[k] = d.q[k];
  const int rc = launch_tensor_group<T>(views, 6, workspace, s, nullptr, d.run0, d.run1);
  if (rc != HSI_OK) return rc;
  const int64_t BB = static_cast<int64_t>(j.bands) * j.bands;
  quarter_assemble_kernel<<<static_cast<unsigned>((BB + 255) / 256), 256, 0, s>>>(qv, j.moments);
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int launch_split_stats(const hsi_moments_job& j, void* workspace, cudaStream_t s) {
  // all on the tensor cores when quarters fit (a caller's reference points
  // apply to whole bands, so those frames keep the two-view form)
  if (j.bands <= kQuarterMaxBands && !j.reference) return launch_quarter_stats<T>(j, workspace, s);
  const SplitDims d = split_dims(j.bands);
  const int64_t P = static_cast<int64_t>(j.height) * j.width;
  unsigned char* w = static_cast<unsigned char*>(workspace) + tensor_ws_bytes(2);
  double* m0 = reinterpret_cast<double*>(w);
  double* m1 = reinterpret_cast<double*>(w + view_moments_bytes(d.h));
  double* partials = reinterpret_cast<double*>(w + view_moments_bytes(d.h) + view_moments_bytes(d.n1));
  hsi_moments_job v0 = j, v1 = j;
  v0.bands = d.h;
  v0.moments = m0;
  v1.bands = d.n1;
  v1.moments = m1;
  // plane h: 16-byte aligned, as the plane stride is a multiple of 8 elements
  v1.cube = static_cast<const unsigned char*>(j.cube) + static_cast<size_t>(d.h) * j.plane_stride * sizeof(T);
  v1.reference = j.reference ? j.reference + d.h : nullptr;
  const hsi_moments_job* views[2] = {&v0, &v1};
  const int rc = launch_tensor_group<T>(views, 2, workspace, s, nullptr);
  if (rc != HSI_OK) return rc;
  stats_cross_kernel<T><<<dim3(kSimtSlices, d.rt * d.ct), 256, 0, s>>>(
      static_cast<const T*>(j.cube), P, j.plane_stride, d.h, d.n1, m0, m1, partials, kSimtSlices, d.ct, d.nrp,
      d.ncp);
  const int64_t BB = static_cast<int64_t>(j.bands) * j.bands;
  split_assemble_kernel<<<static_cast<unsigned>((BB + 255) / 256), 256, 0, s>>>(m0, m1, partials, kSimtSlices, d.h,
                                                                              d.n1, d.nrp, d.ncp, j.moments);
  return static_cast<int>(cudaGetLastError());
}

int check_job(const hsi_moments_job& j) {
  if (!j.cube || !j.moments || j.height <= 0 || j.width <= 0 || j.bands <= 0 || j.bands > HSI_MAX_BANDS)
    return HSI_E_INVALID;
  if (j.dtype != HSI_F32 && j.dtype != HSI_F16) return HSI_E_INVALID;
  const int64_t P = static_cast<int64_t>(j.height) * j.width;
  if (j.plane_stride < P || (j.plane_stride & 7) != 0) return HSI_E_INVALID;
  if ((reinterpret_cast<uintptr_t>(j.cube) & 15u) != 0) return HSI_E_INVALID;
  return HSI_OK;
}

bool tensor_capable(const hsi_moments_job& j) {
  const int64_t P = static_cast<int64_t>(j.height) * j.width;
  return j.bands <= kMaxTensorBands && P < kTensorMaxPixels;
}

// Default routing: small frames (where the integer path's one approximation,
// the off-diagonal sums of the lowest limbs' products, is largest relative to
// the sums, and the work is cheap) take the FP32 CUDA-core path; larger frames
// of at most 127 bands the tensor path, of 128..254 bands the split path.
bool tensor_default(const hsi_moments_job& j) {
  return tensor_capable(j) && static_cast<int64_t>(j.height) * j.width >= kTensorMinPixels;
}

bool split_default(const hsi_moments_job& j) {
  const int64_t P = static_cast<int64_t>(j.height) * j.width;
  return j.bands > kMaxTensorBands && j.bands <= kSplitMaxBands && P >= kTensorMinPixels && P < kTensorMaxPixels;
}

enum class Route { kDefault, kSimt, kTensor };

std::mutex g_stats_mutex;  // the launch helpers keep their large parameter blocks in statics

int run_jobs(const hsi_moments_job* jobs, int n, void* ws, size_t ws_bytes, cudaStream_t s, Route route) {
  if (!jobs || n <= 0) return HSI_E_INVALID;
  for (int i = 0; i < n; ++i) {
    const int rc = check_job(jobs[i]);
    if (rc != HSI_OK) return rc;
    if (route == Route::kTensor && !tensor_capable(jobs[i])) return HSI_E_CAPACITY;
  }
  if (!ws || ws_bytes < hsi_scene_moments_batch_workspace_bytes(jobs, n)) return HSI_E_WORKSPACE;
  std::lock_guard<std::mutex> lock(g_stats_mutex);
  const hsi_moments_job* group[2][kMaxBatch];
  int count[2] = {0, 0};
  auto flush = [&](int d) -> int {
    if (count[d] == 0) return HSI_OK;
    const int rc = d == 0 ? launch_tensor_group<float>(group[0], count[0], ws, s, nullptr)
                          : launch_tensor_group<__half>(group[1], count[1], ws, s, nullptr);
    count[d] = 0;
    return rc;
  };
  for (int i = 0; i < n; ++i) {
    const hsi_moments_job& j = jobs[i];
    const bool tensor = route == Route::kTensor || (route == Route::kDefault && tensor_default(j));
    int rc = HSI_OK;
    if (tensor) {
      const int d = j.dtype == HSI_F32 ? 0 : 1;
      group[d][count[d]++] = &j;
      if (count[d] == kMaxBatch) rc = flush(d);
    } else if (route == Route::kDefault && split_default(j)) {
      rc = j.dtype == HSI_F32 ? launch_split_stats<float>(j, ws, s) : launch_split_stats<__half>(j, ws, s);
    } else {
      rc = j.dtype == HSI_F32 ? launch_simt_stats<float>(j, ws, s) : launch_simt_stats<__half>(j, ws, s);
    }
    if (rc != HSI_OK) return rc;
  }
  int rc = flush(0);
  if (rc == HSI_OK) rc = flush(1);
  return rc;
}

hsi_moments_job single_job(const void* cube, int height, int width, int bands, int dtype, int64_t stride,
                           double* moments, const float* reference) {
  hsi_moments_job j{};
  j.cube = cube;
  j.plane_stride = stride;
  j.moments = moments;
  j.reference = reference;
  j.height = height;
  j.width = width;
  j.bands = bands;
  j.dtype = dtype;
  return j;
}

}  // namespace

int encode_cube_map(CUtensorMap* map, const void* cube, int dtype, int64_t pixels, int bands, int64_t stride,
                    int box_pixels, int box_bands) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return HSI_E_NO_DEVICE;
  const size_t esize = dtype == HSI_F32 ? 4 : 2;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(pixels), static_cast<cuuint64_t>(bands)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(stride) * esize};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_pixels), static_cast<cuuint32_t>(box_bands)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, dtype == HSI_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                        const_cast<void*>(cube), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HSI_OK : HSI_E_INVALID;
}

// The same map with the 128-byte swizzle: boxes land in shared memory in the
// UMMA "128B swizzle" layout (inner box extent must be 128 bytes; destination
// 1024-byte aligned), ready to be an MMA operand without conversion.
int encode_cube_map_sw128(CUtensorMap* map, const void* cube, int dtype, int64_t pixels, int bands, int64_t stride,
                          int box_pixels, int box_bands) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return HSI_E_NO_DEVICE;
  const size_t esize = dtype == HSI_F32 ? 4 : 2;
  if (static_cast<size_t>(box_pixels) * esize != 128) return HSI_E_INVALID;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(pixels), static_cast<cuuint64_t>(bands)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(stride) * esize};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_pixels), static_cast<cuuint32_t>(box_bands)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, dtype == HSI_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                        const_cast<void*>(cube), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HSI_OK : HSI_E_INVALID;
}

}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API size_t hsi_scene_moments_batch_workspace_bytes(const hsi_moments_job* jobs, int num_jobs) {
  if (!jobs || num_jobs <= 0) return 0;
  size_t need = 0;
  int tensor = 0;
  for (int i = 0; i < num_jobs; ++i) {
    if (jobs[i].bands <= 0 || jobs[i].bands > HSI_MAX_BANDS) return 0;
    // every job may be routed either way (the _tc and _simt entry points force one)
    size_t b = simt_ws_bytes(jobs[i].bands);
    if (jobs[i].bands > kMaxTensorBands && jobs[i].bands <= kSplitMaxBands) {
      const size_t sb = split_ws_bytes(jobs[i].bands);
      if (sb > b) b = sb;
    }
    if (b > need) need = b;
    if (tensor_capable(jobs[i])) ++tensor;
  }
  if (tensor > 0) {
    const size_t b = tensor_ws_bytes(tensor < kMaxBatch ? tensor : kMaxBatch);
    if (b > need) need = b;
  }
  return need;
}

extern "C" HSI_API int hsi_scene_moments_batch(const hsi_moments_job* jobs, int num_jobs, void* d_workspace,
                                               size_t workspace_bytes, hsi_stream_t stream) {
  return run_jobs(jobs, num_jobs, d_workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream),
                  Route::kDefault);
}

extern "C" HSI_API size_t hsi_stats_workspace_bytes(int height, int width, int bands) {
  if (height <= 0 || width <= 0 || bands <= 0 || bands > HSI_MAX_BANDS) return 0;
  const size_t a = tensor_ws_bytes(1), b = simt_ws_bytes(bands);
  const size_t c = bands > kMaxTensorBands && bands <= kSplitMaxBands ? split_ws_bytes(bands) : 0;
  const size_t m = a > b ? a : b;
  return m > c ? m : c;
}

extern "C" HSI_API int hsi_scene_moments(const void* d_cube, int height, int width, int bands, int dtype,
                                         int64_t plane_stride, double* d_moments, const float* d_reference,
                                         void* d_workspace, size_t workspace_bytes, hsi_stream_t stream) {
  const hsi_moments_job j = single_job(d_cube, height, width, bands, dtype, plane_stride, d_moments, d_reference);
  return run_jobs(&j, 1, d_workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream), Route::kDefault);
}

extern "C" HSI_API int hsi_scene_moments_simt(const void* d_cube, int height, int width, int bands, int dtype,
                                              int64_t plane_stride, double* d_moments, const float* d_reference,
                                              void* d_workspace, size_t workspace_bytes, hsi_stream_t stream) {
  const hsi_moments_job j = single_job(d_cube, height, width, bands, dtype, plane_stride, d_moments, d_reference);
  return run_jobs(&j, 1, d_workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream), Route::kSimt);
}

extern "C" HSI_API int hsi_scene_moments_tc(const void* d_cube, int height, int width, int bands, int dtype,
                                            int64_t plane_stride, double* d_moments, const float* d_reference,
                                            void* d_workspace, size_t workspace_bytes, hsi_stream_t stream) {
  const hsi_moments_job j = single_job(d_cube, height, width, bands, dtype, plane_stride, d_moments, d_reference);
  return run_jobs(&j, 1, d_workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream), Route::kTensor);
}
