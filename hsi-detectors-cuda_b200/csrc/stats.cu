// stats.cu - scene moments on the 5th-generation tensor cores, exactly.
//
// Computes, for one BSQ frame, the raw first and second moments the detector
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
//   q = rint(d * 2^e_b) with |q| < 2^22 (e_b from a subsample with 4x headroom;
//   an overflow re-runs the pass with the observed range), balanced signed
//   8-bit limbs q = L0*2^16 + L1*2^8 + L2, and four exact INT32 accumulators
//     A0 = sum L0 L0^T,  A1 = sum L0 L1^T,  A2 = sum (L1 L1^T + 2 L0 L2^T),
//     A3 = sum 2 L1 L2^T
//   (tcgen05.mma kind::i8, seven MMAs per K-step).  F = 2^32 A0 + 2^25 A1 +
//   2^16 A2 + 2^8 A3 in FP64 and S = (F + F^T)/2 is sum q q^T except the
//   weight-1 products L2 L2^T: their diagonal is added back exactly (the
//   converters count sum L2^2 per band), their off-diagonal sums are those of
//   independent rounding residues.  The cross terms matter: when outliers set
//   the fixed-point range, typical q carry only ~15 significant bits.
//   A ones-row at band B (q = 2^16) makes the same GEMM produce sum(q) and the
//   pixel count.  Partial sums of all CTAs are reduced in a fixed order and
//   rebuilt as raw moments in FP64 (src/linalg.cpp:81-103).
//
// Kernel roles (one CTA per SM, 22 warps):
//   warp 0       TMA producer: 64-pixel x 128-band boxes, two per K-block,
//                into a 4-deep ring (3 boxes in flight while one converts)
//   warp 1       TMEM allocator + single-thread MMA issuer
//   warps 2-17   converters: FP32 tile -> INT8 limbs L0, L1, L2 in the UMMA
//                128-byte-swizzled K-major layout; per-band |d| maxima
//   warps 18-21  epilogue: INT32 TMEM accumulators -> FP64 partials (once per
//                32768-pixel chunk, i.e. once per frame at typical sizes)
// TMEM: columns [0,128) A0, [128,256) A1, [256,384) A2, [384,512) A3.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tc.cuh"

namespace hsi_b200 {
namespace {

constexpr int kKB = 128;         // pixels per K-block (one INT8 operand row)
constexpr int kBoxPx = 64;       // pixels per TMA box
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
constexpr int64_t kTensorMinPixels = 32768;
constexpr int kQMax = (1 << 22) - (1 << 16);  // |q| bound of the FMA rounding trick
constexpr int kOnesExp = 16;  // the ones row holds q = 2^16

// Input stages hold one TMA box (half a K-block: 64 pixels x 128 bands).
template <typename T>
constexpr int in_stages() {
  return sizeof(T) == 4 ? 4 : 8;
}
template <typename T>
constexpr int in_tile_bytes() {
  return kRows * kBoxPx * static_cast<int>(sizeof(T));
}

struct StatsSmem {
  size_t in_off, op_off, shift_off, scale_off, bar_off, slot_off, total;
};

template <typename T>
__host__ __device__ inline StatsSmem stats_smem() {
  StatsSmem s;
  size_t off = 0;
  s.in_off = off;
  off += static_cast<size_t>(in_stages<T>()) * in_tile_bytes<T>();
  s.op_off = off;  // 1024-aligned: in tiles are multiples of 1024
  off += static_cast<size_t>(kOpStages) * 3 * kLimbBytes;
  s.shift_off = off;
  off += kRows * sizeof(float);
  s.scale_off = off;
  off += kRows * sizeof(float);
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

// Workspace shared by the launch sequence of one frame.
struct StatsState {
  float shift[HSI_MAX_BANDS + 1];     // r_b
  int scale_exp[HSI_MAX_BANDS + 1];   // e_b (ones row: kOnesExp)
  int maxdev_bits[HSI_MAX_BANDS + 1]; // max |d_b| seen by the GEMM (float bits, >= 0)
  int flags;                          // bit 0: a q was clamped; bit 1: the re-run is armed
  int pad[3];
  unsigned long long l2sq[HSI_MAX_BANDS + 1];  // exact sum of L2^2 per band
  // subsample pass (cleared by a memset before it)
  double sub_sum[HSI_MAX_BANDS + 1];
  double sub_cnt[HSI_MAX_BANDS + 1];
  int sub_lo[HSI_MAX_BANDS + 1];  // float_order of the minimum
  int sub_hi[HSI_MAX_BANDS + 1];
};

struct StatsArgs {
  int64_t pixels;
  int bands;
  StatsState* state;
  double* partials;  // [gridDim.x][kRows][kRows] (column-major per CTA)
  int conditional;   // 1: run only if the re-run is armed
  int* status;
};

template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
    stats_gemm_kernel(const __grid_constant__ CUtensorMap cube_map, const StatsArgs args) {
  if (args.conditional && !(args.state->flags & 2)) return;  // nothing to redo
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
  int* clamp_flag = reinterpret_cast<int*>(smem + L.slot_off + 12);
  float* shift = reinterpret_cast<float*>(smem + L.shift_off);
  float* scale = reinterpret_cast<float*>(smem + L.scale_off);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t P = args.pixels;
  const int B = args.bands;
  const int64_t nkb = div_up<int64_t>(P, kKB);
  const int64_t kb0 = nkb * blockIdx.x / gridDim.x;
  const int64_t kb1 = nkb * (blockIdx.x + 1) / gridDim.x;
  const int n = static_cast<int>(kb1 - kb0);
  const int nchunks = (n + kChunkKB - 1) / kChunkKB;

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
    *clamp_flag = 0;
    fence_barrier_init();
  }
  for (int i = threadIdx.x; i < kRows; i += blockDim.x) {
    shift[i] = args.state->shift[i];
    scale[i] = ldexpf(1.0f, args.state->scale_exp[i]);
  }
  if (warp == kWarpMma) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kWarpTma) {
    if (lane == 0) {
      prefetch_tensormap(&cube_map);
      uint32_t pending = 0, parity = 0;
      for (int i = 0; i < 2 * n; ++i) {
        const int s = i % kInStages;
        const uint32_t ph = (i / kInStages) & 1u;
        if (*abort_flag || !mbar_wait(&in_empty[s], ph ^ 1u)) {
          record_error(args.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        unsigned char* dst = smem + L.in_off + static_cast<size_t>(s) * in_tile_bytes<T>();
        mbar_arrive_expect_tx(&in_full[s], in_tile_bytes<T>());
        tma_load_2d(dst, &cube_map, static_cast<int>(kb0 * kKB + static_cast<int64_t>(i) * kBoxPx), 0, &in_full[s]);
        pending |= 1u << s;
        parity = (parity & ~(1u << s)) | (ph << s);
      }
      for (int s = 0; s < kInStages; ++s)
        if ((pending >> s) & 1u) mbar_wait(&in_full[s], (parity >> s) & 1u);
    }
  } else if (warp == kWarpMma) {
    if (lane == 0) {
      const uint32_t idesc = idesc_s8_s32(kRows, kRows);
      bool issued = false;
      for (int i = 0; i < n && !*abort_flag; ++i) {
        const int chunk = i / kChunkKB, j = i % kChunkKB;
        if (j == 0) {
          if (!mbar_wait(acc_empty, (chunk & 1u) ^ 1u)) {
            record_error(args.status, HSI_E_TIMEOUT);
            *abort_flag = 1;
            break;
          }
          tc_fence_after();
        }
        const int so = i % kOpStages;
        if (!mbar_wait(&op_full[so], (i / kOpStages) & 1u)) {
          record_error(args.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        unsigned char* op = smem + L.op_off + static_cast<size_t>(so) * 3 * kLimbBytes;
        const uint64_t d0 = smem_desc_sw128(op);
        const uint64_t d1 = smem_desc_sw128(op + kLimbBytes);
        const uint64_t d2 = smem_desc_sw128(op + 2 * kLimbBytes);
#pragma unroll
        for (int k = 0; k < kKB / 32; ++k) {
          const uint64_t adv = static_cast<uint64_t>(k * 2);  // 32 bytes of K, in 16-byte units
          const uint32_t acc = (j > 0 || k > 0) ? 1u : 0u;
          umma_i8(tmem + 0, d0 + adv, d0 + adv, idesc, acc);
          umma_i8(tmem + 128, d0 + adv, d1 + adv, idesc, acc);
          umma_i8(tmem + 256, d1 + adv, d1 + adv, idesc, acc);
          umma_i8(tmem + 256, d0 + adv, d2 + adv, idesc, 1u);
          umma_i8(tmem + 256, d0 + adv, d2 + adv, idesc, 1u);
          umma_i8(tmem + 384, d1 + adv, d2 + adv, idesc, acc);
          umma_i8(tmem + 384, d1 + adv, d2 + adv, idesc, 1u);
        }
        umma_commit(&op_empty[so]);
        if (j == kChunkKB - 1 || i == n - 1) umma_commit(acc_full);
        issued = true;
      }
      // TMEM is freed at the end of the kernel: make sure no MMA of this
      // thread is still running by then (bounded wait).
      if (issued) {
        umma_commit(mma_done);
        if (!mbar_wait(mma_done, 0)) record_error(args.status, HSI_E_TIMEOUT);
      }
    }
  } else if (warp < kWarpEpi0) {
    // ---------------- converters ----------------
    // Each input stage is half a K-block (64 pixels).  Warp cw owns 4 band
    // pairs (b, b+4) -- lanes 0-15 the first band, 16-31 the second, 4 pixels
    // per lane -- so one store instruction covers two rows whose swizzled
    // chunks never share a bank.
    // q = rint((x - r) 2^e) comes out of one FMA: adding 1.5*2^23 leaves
    // rint(q) in the low mantissa bits (|q| < 2^22), and w = q + 0x8080 has
    // the balanced limbs as its bytes (low two XOR 0x80, third as is).
    const int cw = warp - kWarpConv0;
    constexpr int kSlots = kRows / 2 / kConvWarps;  // 4 band pairs per warp
    constexpr float kMagic = 12582912.0f;          // 1.5 * 2^23
    const int sub = lane >> 4, lp = (lane & 15) * 4;  // which band of the pair; pixel in the box
    int band[kSlots];
    float sc[kSlots], off[kSlots], xlo[kSlots], xhi[kSlots];
    int l2sq[kSlots];
#pragma unroll
    for (int t = 0; t < kSlots; ++t) {
      const int pair = cw + kConvWarps * t;          // 0..63
      const int b = (pair >> 2) * 8 + (pair & 3) + 4 * sub;
      band[t] = b;
      sc[t] = scale[b];
      off[t] = kMagic - shift[b] * scale[b];  // exact: r sits on the 2^-e grid
      xlo[t] = INFINITY;
      xhi[t] = -INFINITY;
      l2sq[t] = 0;
    }
    const int wbias = __float_as_int(kMagic) - 0x8080;
    bool aborted = false;
    for (int j = 0; j < 2 * n; ++j) {
      const int s = j % kInStages, i = j >> 1, half = j & 1, so = i % kOpStages;
      if (!aborted && (!mbar_wait(&in_full[s], (j / kInStages) & 1u) ||
                       (half == 0 && !mbar_wait(&op_empty[so], ((i / kOpStages) & 1u) ^ 1u)))) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        aborted = true;
      }
      if (aborted) break;
      const T* in = reinterpret_cast<const T*>(smem + L.in_off + static_cast<size_t>(s) * in_tile_bytes<T>());
      unsigned char* op = smem + L.op_off + static_cast<size_t>(so) * 3 * kLimbBytes;
      const int64_t gp = (kb0 + i) * kKB + half * kBoxPx + lp;
      const int nvalid = gp >= P ? 0 : (P - gp >= 4 ? 4 : static_cast<int>(P - gp));
#pragma unroll
      for (int t = 0; t < kSlots; ++t) {
        const int b = band[t];
        int w[4] = {0x8080, 0x8080, 0x8080, 0x8080};  // q = 0
        if (b < B) {
          const float4 x = load4f<T>(in + b * kBoxPx + lp);
          const float xv[4] = {x.x, x.y, x.z, x.w};
          // fully unrolled with a predicate: a loop bounded by nvalid would
          // index w[] dynamically and move it to local memory
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if (e < nvalid) {
              xlo[t] = fminf(xlo[t], xv[e]);
              xhi[t] = fmaxf(xhi[t], xv[e]);
              w[e] = __float_as_int(fmaf(xv[e], sc[t], off[t])) - wbias;
            }
          }
        } else if (b == B) {
#pragma unroll
          for (int e = 0; e < 4; ++e) w[e] = e < nvalid ? (1 << kOnesExp) + 0x8080 : 0x8080;
        }
        const uint32_t p01 = __byte_perm(w[0], w[1], 0x5140), p23 = __byte_perm(w[2], w[3], 0x5140);
        const uint32_t h01 = __byte_perm(w[0], w[1], 0x7362), h23 = __byte_perm(w[2], w[3], 0x7362);
        const uint32_t l2 = __byte_perm(p01, p23, 0x5410) ^ 0x80808080u;
        const uint32_t l1 = __byte_perm(p01, p23, 0x7632) ^ 0x80808080u;
        const uint32_t l0 = __byte_perm(h01, h23, 0x5410);
        l2sq[t] = __dp4a(static_cast<int>(l2), static_cast<int>(l2), l2sq[t]);
        const uint32_t o = sw128_byte(b, half * kBoxPx + lp);
        *reinterpret_cast<uint32_t*>(op + o) = l0;
        *reinterpret_cast<uint32_t*>(op + kLimbBytes + o) = l1;
        *reinterpret_cast<uint32_t*>(op + 2 * kLimbBytes + o) = l2;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&in_empty[s]);
      if (half == 1) {
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&op_full[so]);
      }
    }
    // per band: |x - r| range (for the re-run and for the whitening pass), the
    // clamp check, and the exact sum of L2^2 (reduced over the 16 lanes that
    // share the band)
    bool clamped = false;
#pragma unroll
    for (int t = 0; t < kSlots; ++t) {
      float lo = xlo[t], hi = xhi[t];
      unsigned long long sq = static_cast<unsigned int>(l2sq[t]);
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        sq += __shfl_xor_sync(0xffffffffu, sq, o);
      }
      const int b = band[t];
      const float r = shift[b];
      const float m = hi >= lo ? fmaxf(hi - r, r - lo) : 0.0f;
      if (b < B && !(m * sc[t] <= static_cast<float>(kQMax))) clamped = true;
      if ((lane & 15) == 0 && b < B) {
        atomicMax(&args.state->maxdev_bits[b], __float_as_int(m));
        atomicAdd(&args.state->l2sq[b], sq);
      }
    }
    if (__any_sync(0xffffffffu, clamped) && lane == 0) atomicOr(&args.state->flags, 1);
  } else {
    // ---------------- epilogue ----------------
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int row = q * 32 + lane;
    const uint32_t trow = tmem + (static_cast<uint32_t>(q * 32) << 16);
    double* out = args.partials + static_cast<size_t>(blockIdx.x) * kRows * kRows;
    for (int chunk = 0; chunk < nchunks; ++chunk) {
      if (!mbar_wait(acc_full, chunk & 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
#pragma unroll 1
      for (int cb = 0; cb < kRows / 16; ++cb) {
        uint32_t a0[16], a1[16], a2[16], a3[16];
        tmem_ld16(trow + 0 + 16 * cb, a0);
        tmem_ld16(trow + 128 + 16 * cb, a1);
        tmem_ld16(trow + 256 + 16 * cb, a2);
        tmem_ld16(trow + 384 + 16 * cb, a3);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const double f = ldexp(static_cast<double>(static_cast<int>(a0[j])), 32) +
                           ldexp(static_cast<double>(static_cast<int>(a1[j])), 25) +
                           ldexp(static_cast<double>(static_cast<int>(a2[j])), 16) +
                           ldexp(static_cast<double>(static_cast<int>(a3[j])), 8);
          double* dst = out + static_cast<size_t>(16 * cb + j) * kRows + row;  // column-major
          *dst = chunk == 0 ? f : *dst + f;
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty);
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
// (every 16th run of 64 pixels on large frames): r = subsample mean, e such
// that the subsample's largest |x - r| maps to 2^20 (4x headroom below 2^22).
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

constexpr int kShiftSplit = 16;  // blocks per band of the subsample pass

__global__ void shift_init_kernel(StatsState* st) {
  for (int b = threadIdx.x; b <= HSI_MAX_BANDS; b += blockDim.x) {
    st->sub_sum[b] = 0.0;
    st->sub_cnt[b] = 0.0;
    st->sub_lo[b] = 0x7fffffff;
    st->sub_hi[b] = static_cast<int>(0x80000000u);
  }
}

// Subsample statistics, spread over (bands x kShiftSplit) blocks: runs of 64
// pixels, every 16th run on large frames; partial sums land in the state with
// atomics (the state is cleared by a memset first).
template <typename T>
__global__ void __launch_bounds__(256) shift_partial_kernel(const T* __restrict__ cube, int64_t pixels,
                                                            int64_t stride, int bands, StatsState* st) {
  const int b = blockIdx.x;
  if (b >= bands) return;
  __shared__ double s_sum[8], s_cnt[8];
  __shared__ int s_lo[8], s_hi[8];
  const T* plane = cube + static_cast<int64_t>(b) * stride;
  const int64_t runs = div_up<int64_t>(pixels, 64);
  const int64_t step = runs > 4096 ? 16 : 1;
  const int64_t sampled = div_up<int64_t>(runs, step);
  const int64_t r0 = sampled * blockIdx.y / kShiftSplit, r1 = sampled * (blockIdx.y + 1) / kShiftSplit;
  double sum = 0.0, cnt = 0.0;
  float lo = INFINITY, hi = -INFINITY;
#pragma unroll 4
  for (int64_t run = r0 + threadIdx.x / 64; run < r1; run += blockDim.x / 64) {
    const int64_t p = run * step * 64 + (threadIdx.x & 63);
    if (p < pixels) {
      const float v = static_cast<float>(plane[p]);
      sum += static_cast<double>(v);
      cnt += 1.0;
      lo = fminf(lo, v);
      hi = fmaxf(hi, v);
    }
  }
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
    double ts = 0.0, tc = 0.0;
    int tl = s_lo[0], th = s_hi[0];
    for (int w = 0; w < 8; ++w) {
      ts += s_sum[w];
      tc += s_cnt[w];
      tl = min(tl, s_lo[w]);
      th = max(th, s_hi[w]);
    }
    if (tc > 0.0) {
      atomicAdd(&st->sub_sum[b], ts);
      atomicAdd(&st->sub_cnt[b], tc);
      atomicMin(&st->sub_lo[b], tl);
      atomicMax(&st->sub_hi[b], th);
    }
  }
}

// r = subsample mean (or the caller's reference), e such that the subsample's
// largest |x - r| maps to 2^20 (4x headroom below 2^22), r snapped to the
// 2^-e grid so that inputs on that grid (FP16 cubes) convert exactly.
__global__ void __launch_bounds__(256) shift_finalize_kernel(int bands, const float* __restrict__ given,
                                                             StatsState* st) {
  for (int b = threadIdx.x; b <= HSI_MAX_BANDS; b += blockDim.x) {
    st->maxdev_bits[b] = 0;
    st->l2sq[b] = 0ull;
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
    const double c = st->sub_cnt[b];
    float r = given ? given[b] : (c > 0.0 ? static_cast<float>(st->sub_sum[b] / c) : 0.0f);
    const float lo = c > 0.0 ? order_float(st->sub_lo[b]) : r, hi = c > 0.0 ? order_float(st->sub_hi[b]) : r;
    const int e = scale_exp_for(fmaxf(fabsf(hi - r), fabsf(lo - r)) * 1.0000001f);
    r = ldexpf(rintf(ldexpf(r, e)), -e);
    st->shift[b] = r;
    st->scale_exp[b] = e;
  }
  if (threadIdx.x == 0) st->flags = 0;
}

// After the first GEMM: if a value was clamped, take the range the GEMM
// actually saw and arm the conditional re-run; otherwise leave it disarmed.
__global__ void rescale_kernel(int bands, StatsState* st) {
  if (!(st->flags & 1)) return;
  for (int b = threadIdx.x; b < bands; b += blockDim.x) {
    const float dev = __int_as_float(st->maxdev_bits[b]);
    const int e = scale_exp_for(dev * 1.0000001f) + 1;  // observed max -> below 2^21
    st->scale_exp[b] = e;
    // keep r on the (coarser) new grid so r * 2^e stays an exact integer
    st->shift[b] = ldexpf(rintf(ldexpf(st->shift[b], e)), -e);
    st->l2sq[b] = 0ull;  // recounted by the re-run
  }
  __syncthreads();
  if (threadIdx.x == 0) st->flags = 2;
}

// Sum the CTAs' partial matrices in a fixed order: block = 32 entries, each of
// 8 warps sums a slice of CTAs, then the slices are added in warp order.
__global__ void __launch_bounds__(256) stats_reduce_kernel(const double* __restrict__ partials, int ctas,
                                                          double* __restrict__ fsum) {
  __shared__ double s[8][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x * 32 + lane;  // entry index in [0, 128*128)
  double acc = 0.0;
  const int c0 = ctas * warp / 8, c1 = ctas * (warp + 1) / 8;
  for (int c = c0; c < c1; ++c) acc += partials[static_cast<size_t>(c) * kRows * kRows + e];
  s[warp][lane] = acc;
  __syncthreads();
  if (warp == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += s[w][lane];
    fsum[e] = t;
  }
}

// S = (F + F^T)/2, unscaled -> shifted sums (S1, S2, N) -> raw moments in FP64
// (moments_from_shifted, src/linalg.cpp:81-103).  fsum is column-major:
// fsum[col * 128 + row] = F[row][col].  Output: sum[B], outer[B*B] (full,
// symmetric), count.
__global__ void __launch_bounds__(128) stats_finalize_kernel(const double* __restrict__ fsum,
                                                            const StatsState* __restrict__ st, int bands,
                                                            double* __restrict__ moments) {
  // one block per row i of the output; every block rebuilds the first moments
  __shared__ double s1[kRows];
  __shared__ double r[kRows];
  __shared__ int ex[kRows];
  const int B = bands;
  const int i = blockIdx.x;
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
    if (i == j) q += static_cast<double>(st->l2sq[i]);  // the weight-1 diagonal, exact
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
// Host side
// ---------------------------------------------------------------------------

int num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

constexpr int kSimtSlices = 96;

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

struct StatsWorkspace {
  StatsState* state;
  double* partials;
  double* fsum;
};

size_t tensor_ws_bytes() {
  return align256(sizeof(StatsState)) + align256(static_cast<size_t>(kMaxCtas) * kRows * kRows * sizeof(double)) +
         align256(kRows * kRows * sizeof(double));
}

size_t simt_ws_bytes(int bands) {
  const int n = ((bands + 1 + kSimtTile - 1) / kSimtTile) * kSimtTile;
  return align256(sizeof(StatsState)) + align256(static_cast<size_t>(kSimtSlices) * n * n * sizeof(double)) +
         align256(static_cast<size_t>(n) * n * sizeof(double));
}

StatsWorkspace carve(void* base, size_t partial_bytes) {
  unsigned char* p = static_cast<unsigned char*>(base);
  StatsWorkspace w;
  w.state = reinterpret_cast<StatsState*>(p);
  p += align256(sizeof(StatsState));
  w.partials = reinterpret_cast<double*>(p);
  p += align256(partial_bytes);
  w.fsum = reinterpret_cast<double*>(p);
  return w;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

template <typename T>
void launch_shift(const void* cube, int64_t P, int64_t stride, int B, const float* reference, StatsState* st,
                  cudaStream_t s) {
  shift_init_kernel<<<1, 256, 0, s>>>(st);
  shift_partial_kernel<T><<<dim3(B, kShiftSplit), 256, 0, s>>>(static_cast<const T*>(cube), P, stride, B, st);
  shift_finalize_kernel<<<1, 256, 0, s>>>(B, reference, st);
}

// shift + scale -> GEMM -> (conditional) rescale + GEMM re-run -> reduce -> finalize
template <typename T>
int launch_tensor_stats(const void* cube, int64_t P, int B, int64_t stride, double* moments, const float* reference,
                        void* workspace, cudaStream_t s, int* status) {
  CUtensorMap map;
  const int rc = encode_cube_map(&map, cube, sizeof(T) == 4 ? HSI_F32 : HSI_F16, P, B, stride, kBoxPx, kRows);
  if (rc != HSI_OK) return rc;
  const StatsWorkspace w = carve(workspace, static_cast<size_t>(kMaxCtas) * kRows * kRows * sizeof(double));
  launch_shift<T>(cube, P, stride, B, reference, w.state, s);
  const int64_t nkb = div_up<int64_t>(P, kKB);
  int grid = num_sms();
  if (grid > kMaxCtas) grid = kMaxCtas;
  if (nkb < grid) grid = static_cast<int>(nkb);
  const StatsSmem L = stats_smem<T>();
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(stats_gemm_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(L.total));
    if (e != cudaSuccess) return static_cast<int>(e);
    configured = true;
  }
  StatsArgs a;
  a.pixels = P;
  a.bands = B;
  a.state = w.state;
  a.partials = w.partials;
  a.conditional = 0;
  a.status = status;
  stats_gemm_kernel<T><<<grid, kThreads, L.total, s>>>(map, a);
  rescale_kernel<<<1, 128, 0, s>>>(B, w.state);
  a.conditional = 1;
  stats_gemm_kernel<T><<<grid, kThreads, L.total, s>>>(map, a);
  stats_reduce_kernel<<<kRows * kRows / 32, 256, 0, s>>>(w.partials, grid, w.fsum);
  stats_finalize_kernel<<<B, 128, 0, s>>>(w.fsum, w.state, B, moments);
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int launch_simt_stats(const void* cube, int64_t P, int B, int64_t stride, double* moments, const float* reference,
                      void* workspace, cudaStream_t s) {
  const int tiles = (B + 1 + kSimtTile - 1) / kSimtTile;
  const int n = tiles * kSimtTile;
  const StatsWorkspace w = carve(workspace, static_cast<size_t>(kSimtSlices) * n * n * sizeof(double));
  launch_shift<T>(cube, P, stride, B, reference, w.state, s);
  const dim3 grid(kSimtSlices, tiles * (tiles + 1) / 2);
  stats_simt_kernel<T><<<grid, 256, 0, s>>>(static_cast<const T*>(cube), P, stride, B, w.state, w.partials,
                                           kSimtSlices);
  simt_reduce_kernel<<<(n * n + 255) / 256, 256, 0, s>>>(w.partials, kSimtSlices, n, w.fsum);
  simt_finalize_kernel<<<1, 256, 0, s>>>(w.fsum, n, w.state, B, moments);
  return static_cast<int>(cudaGetLastError());
}

int check_common(const void* cube, int height, int width, int bands, int dtype, int64_t stride, double* moments) {
  if (!cube || !moments || height <= 0 || width <= 0 || bands <= 0 || bands > HSI_MAX_BANDS) return HSI_E_INVALID;
  if (dtype != HSI_F32 && dtype != HSI_F16) return HSI_E_INVALID;
  const int64_t P = static_cast<int64_t>(height) * width;
  if (stride < P || (stride & 7) != 0) return HSI_E_INVALID;
  if ((reinterpret_cast<uintptr_t>(cube) & 15u) != 0) return HSI_E_INVALID;
  return HSI_OK;
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

extern "C" HSI_API size_t hsi_stats_workspace_bytes(int height, int width, int bands) {
  if (height <= 0 || width <= 0 || bands <= 0 || bands > HSI_MAX_BANDS) return 0;
  const size_t a = tensor_ws_bytes(), b = simt_ws_bytes(bands);
  return a > b ? a : b;
}

extern "C" HSI_API int hsi_scene_moments(const void* d_cube, int height, int width, int bands, int dtype,
                                         int64_t plane_stride, double* d_moments, const float* d_reference,
                                         void* d_workspace, size_t workspace_bytes, hsi_stream_t stream) {
  const int rc = check_common(d_cube, height, width, bands, dtype, plane_stride, d_moments);
  if (rc != HSI_OK) return rc;
  if (!d_workspace || workspace_bytes < hsi_stats_workspace_bytes(height, width, bands)) return HSI_E_WORKSPACE;
  const int64_t P = static_cast<int64_t>(height) * width;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // The integer path's one approximation (the off-diagonal sums of the
  // lowest limbs' products) shrinks as 1/sqrt(pixels); small frames, which
  // are also cheap, take the FP32 CUDA-core path.
  if (bands <= kMaxTensorBands && P >= kTensorMinPixels) {
    return dtype == HSI_F32 ? launch_tensor_stats<float>(d_cube, P, bands, plane_stride, d_moments, d_reference,
                                                         d_workspace, s, nullptr)
                            : launch_tensor_stats<__half>(d_cube, P, bands, plane_stride, d_moments, d_reference,
                                                          d_workspace, s, nullptr);
  }
  return dtype == HSI_F32
             ? launch_simt_stats<float>(d_cube, P, bands, plane_stride, d_moments, d_reference, d_workspace, s)
             : launch_simt_stats<__half>(d_cube, P, bands, plane_stride, d_moments, d_reference, d_workspace, s);
}

extern "C" HSI_API int hsi_scene_moments_simt(const void* d_cube, int height, int width, int bands, int dtype,
                                              int64_t plane_stride, double* d_moments, const float* d_reference,
                                              void* d_workspace, size_t workspace_bytes, hsi_stream_t stream) {
  const int rc = check_common(d_cube, height, width, bands, dtype, plane_stride, d_moments);
  if (rc != HSI_OK) return rc;
  if (!d_workspace || workspace_bytes < hsi_stats_workspace_bytes(height, width, bands)) return HSI_E_WORKSPACE;
  const int64_t P = static_cast<int64_t>(height) * width;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return dtype == HSI_F32
             ? launch_simt_stats<float>(d_cube, P, bands, plane_stride, d_moments, d_reference, d_workspace, s)
             : launch_simt_stats<__half>(d_cube, P, bands, plane_stride, d_moments, d_reference, d_workspace, s);
}

extern "C" HSI_API int hsi_scene_moments_tc(const void* d_cube, int height, int width, int bands, int dtype,
                                            int64_t plane_stride, double* d_moments, const float* d_reference,
                                            void* d_workspace, size_t workspace_bytes, hsi_stream_t stream) {
  const int rc = check_common(d_cube, height, width, bands, dtype, plane_stride, d_moments);
  if (rc != HSI_OK) return rc;
  if (bands > kMaxTensorBands) return HSI_E_CAPACITY;
  if (!d_workspace || workspace_bytes < hsi_stats_workspace_bytes(height, width, bands)) return HSI_E_WORKSPACE;
  const int64_t P = static_cast<int64_t>(height) * width;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return dtype == HSI_F32 ? launch_tensor_stats<float>(d_cube, P, bands, plane_stride, d_moments, d_reference,
                                                       d_workspace, s, nullptr)
                          : launch_tensor_stats<__half>(d_cube, P, bands, plane_stride, d_moments, d_reference,
                                                        d_workspace, s, nullptr);
}
