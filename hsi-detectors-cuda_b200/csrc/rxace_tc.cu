// rxace_tc.cu - RX and ACE whitening on the 5th-generation tensor cores.
//
// Per pixel x (reference rx_cpu / ace_best_cpu, src/detectors_cpu.cpp:95-156):
//   z = W (x - mean),  RX = |z|^2,  ACE_t = (z . u_t)^2 / (|u_t|^2 |z|^2),
// with W = L^-1 of the loaded scene covariance and u_t = W (d_t - mean).
// Since z . u_t = (x - mean) . v_t with v_t = W^T u_t, one contraction with the
// augmented matrix A = [W; v_0^T; ...] (N = B + T rows, K = B bands) gives both
// z and the ACE numerators.
//
// Precision.  RX/ACE amplify relative errors by the conditioning of W (its
// rows hold large entries of alternating sign), and the tensor cores' FP32
// accumulation truncates, so the contraction is done in exact integers:
//   data:  d = x - mean (FP32), per pixel p a power-of-two scale 2^t_p that
//          puts its largest |d_b| in [2^21, 2^22); q = rint(d 2^t_p) split into
//          balanced signed bytes q = L0 2^16 + L1 2^8 + L2;
//   rows:  per row n a power-of-two scale 2^f_n with |A_nb| 2^f_n < 2^23 - 2^16,
//          w = rint(A_nb 2^f_n) = M0 2^16 + M1 2^8 + M2 (computed in FP64);
//   MMAs:  tcgen05.mma.kind::i8, INT32 accumulators by limb weight
//          S_k = sum_{a+b=k} La Mb^T for k = 0..3 (the weight-1 pair L2 M2 is
//          dropped: ~2^-32 of the leading term), eight limb products issued as
//          five instructions (three of N = 256 share the A operand);
//   epilogue: z_n = ((S0 256 + S1) 2^16 + (S2 256 + S3)) 2^(8 - f_n - t_p)
//          + (A_n . (mean32 - mean)): both halves are exact int32 sums, then FP32.
// Measured against the FP64 oracle: |RX error| / max(1, RX) and |ACE error|
// are a few 1e-5 at 113 bands (the fixed-point data step and the 24-bit rows).
//
// Kernel roles (one CTA per SM, persistent over 128-pixel tiles):
//   warp 0      TMA producer: 64-pixel x 128-band boxes of the BSQ cube
//   warp 1      TMEM allocator + single-thread MMA issuer
//   warps 2-9   converters: per-pixel scale, limb tiles in the UMMA layout
//   warps 10-17 epilogue: TMEM -> z -> RX, ACE maps, best target
// Two MMA rounds per tile, one per half of the output rows, each into its own
// half of TMEM: round h (rows [64h, 64h + 64)) writes S0 to columns
// [256h, 256h + 64), S1 the next 64, S2 and S3 after them.  The epilogue warps
// of row half h drain round h while the MMAs of the other round run, so the
// tensor cores no longer wait for the whole tile's epilogue.  In shared memory
// the whitener limbs are laid out by row half, [M0 | M1 | M2] of rows 0-63 and
// then of rows 64-127 (8 KB each), so [M0; M1] of a half is one 128-row operand.
#include <cuda_fp16.h>

#include <type_traits>

#include "tc.cuh"
#include "launch_state.h"

namespace hsi_b200 {
namespace {

constexpr int kRows = 128;   // output rows (N): whitener rows + target rows
constexpr int kK = 128;      // bands (K), zero-padded
constexpr int kTilePx = 128; // pixels per tile (M)
constexpr int kBoxPx = 64;   // pixels per TMA box
constexpr int kOpStages = 2;
constexpr int kConvWarps = 8;
constexpr int kEpiWarps = 8;
constexpr int kWarpTma = 0, kWarpMma = 1, kWarpConv0 = 2, kWarpEpi0 = kWarpConv0 + kConvWarps;
constexpr int kThreads = (kWarpEpi0 + kEpiWarps) * 32;  // 576
constexpr int kLimbBytes = kRows * kK;                  // 16 KB per limb tile
constexpr int kMaxTargetsPerPass = HSI_MAX_FILTERS_PER_PASS;
constexpr uint32_t kTmemCols = 512;

template <typename T>
constexpr int in_stages() {
  return sizeof(T) == 4 ? 2 : 4;
}
template <typename T>
constexpr int box_bytes() {
  return kK * kBoxPx * static_cast<int>(sizeof(T));
}

// Per-frame operands written by the prep kernel (workspace) and staged into
// shared memory by every CTA.
struct TcOperands {
  unsigned char limbs[3][kLimbBytes];  // M0 | M1 | M2 tiles, UMMA 128B-swizzled K-major
  float gain[kRows];                   // 2^(8 - f_n) (0 for unused rows)
  float offset[kRows];                 // A_n . (mean32 - mean)
  float mean32[kK];                    // mean rounded to float (0 past B)
  float uu[kMaxTargetsPerPass];        // |u_t|^2 of this pass's targets
};

struct Smem {
  size_t w_off, a_off, in_off, red_off, t_off, ops_off, zz_off, zb_off, bar_off, slot_off, total;
};

template <typename T>
__host__ __device__ inline Smem smem_layout() {
  Smem s;
  size_t off = 0;
  s.w_off = off;                    // 48 KB, 1024-aligned
  off += 3 * kLimbBytes;
  s.a_off = off;                    // kOpStages x 48 KB
  off += static_cast<size_t>(kOpStages) * 3 * kLimbBytes;
  s.in_off = off;
  off += static_cast<size_t>(in_stages<T>()) * box_bytes<T>();
  s.red_off = off;                  // [2][8][64] floats: per-chunk pixel maxima
  off += 2 * kConvWarps * kBoxPx * sizeof(float);
  s.t_off = off;                    // [kOpStages][128] ints: pixel scale exponents
  off += kOpStages * kTilePx * sizeof(int);
  s.ops_off = off;                  // gain, offset, mean32, uu, 1 / uu
  off += (3 * kRows + 2 * kMaxTargetsPerPass) * sizeof(float);
  s.zz_off = off;                   // [2][128] partial |z|^2
  off += 2 * kTilePx * sizeof(float);
  s.zb_off = off;                   // [16][128] ACE numerators
  off += kMaxTargetsPerPass * kTilePx * sizeof(float);
  s.bar_off = off;
  off += (2 * 4 + 2 * kOpStages + 6 + 2 + 8) * sizeof(uint64_t);
  s.slot_off = off;
  off += 16;
  s.total = off + 1024;
  return s;
}

struct TcArgs {
  int64_t pixels;
  int bands;
  int rows;      // B + targets of this pass
  int ntarg;     // targets of this pass
  int t0;        // first target index of this pass
  int first, last;
  const TcOperands* ops;
  float* rx;
  float* ace_best;
  int32_t* ace_target;
  float* ace_maps;
  int64_t map_stride;
  int* status;
};

__device__ __forceinline__ uint32_t sw128_byte(int row, int k) {
  return static_cast<uint32_t>((row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 4) ^ (row & 7))) << 4) + (k & 15));
}

// Two consecutive elements (8- or 4-byte aligned) as floats.
__device__ __forceinline__ float2 load2f(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ float2 load2f(const __half* p) { return __half22float2(*reinterpret_cast<const __half2*>(p)); }


// ---- prep: the augmented matrix in fixed point, FP64 ------------------------
// One block per output row n; thread k = band.
__global__ void __launch_bounds__(128) tc_prep_kernel(const double* __restrict__ stats, int B, int T, int t0,
                                                      int ntarg, TcOperands* __restrict__ ops) {
  const int n = blockIdx.x, k = threadIdx.x;
  const double* mean = stats;
  const double* W = stats + B;
  const double* tw = W + static_cast<size_t>(B) * B;
  const double* tn = tw + static_cast<size_t>(T) * B;
  __shared__ double red[128];
  double a = 0.0;
  if (k < B) {
    if (n < B) {
      a = W[static_cast<size_t>(n) * B + k];
    } else if (n < B + ntarg) {
      const double* u = tw + static_cast<size_t>(t0 + n - B) * B;
      for (int i = k; i < B; ++i) a += W[static_cast<size_t>(i) * B + k] * u[i];
    }
  }
  const double m32 = k < B ? static_cast<double>(static_cast<float>(mean[k])) : 0.0;
  const double dm = k < B ? m32 - mean[k] : 0.0;
  // row maximum
  red[k] = fabs(a);
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (k < s) red[k] = fmax(red[k], red[k + s]);
    __syncthreads();
  }
  const double amax = red[0];
  __syncthreads();
  int f = 0;
  if (amax > 0.0) {
    f = static_cast<int>(floor(log2((8388608.0 - 65536.0) / amax)));
    while (ldexp(amax, f) >= 8388608.0 - 65536.0) --f;  // guard the log2 rounding
  }
  const int w = amax > 0.0 ? static_cast<int>(rint(ldexp(a, f))) : 0;
  const int m2 = ((w + 128) & 255) - 128;
  const int w1 = (w - m2) >> 8;
  const int m1 = ((w1 + 128) & 255) - 128;
  const int m0 = (w1 - m1) >> 8;
  const uint32_t o = sw128_byte(n, k);
  ops->limbs[0][o] = static_cast<unsigned char>(m0 & 255);
  ops->limbs[1][o] = static_cast<unsigned char>(m1 & 255);
  ops->limbs[2][o] = static_cast<unsigned char>(m2 & 255);
  // offset = A_n . (mean32 - mean), FP64
  red[k] = a * dm;
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (k < s) red[k] += red[k + s];
    __syncthreads();
  }
  if (k == 0) {
    ops->gain[n] = amax > 0.0 ? static_cast<float>(ldexp(1.0, 8 - f)) : 0.0f;
    ops->offset[n] = static_cast<float>(red[0]);
  }
  if (n == 0) {
    ops->mean32[k] = static_cast<float>(m32);
    if (k < kMaxTargetsPerPass) ops->uu[k] = k < ntarg ? static_cast<float>(tn[t0 + k]) : 0.0f;
  }
}

// ---- the contraction ------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
    rxace_tc_kernel(const __grid_constant__ CUtensorMap cube_map, const TcArgs args) {
  constexpr int kIn = in_stages<T>();
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const Smem L = smem_layout<T>();
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar_off);
  uint64_t* in_full = bars;
  uint64_t* in_empty = bars + 4;
  uint64_t* op_full = bars + 8;
  uint64_t* op_empty = op_full + kOpStages;
  uint64_t* acc_full = op_empty + kOpStages;  // [2]: one per row half
  uint64_t* acc_empty = acc_full + 2;         // [2]
  uint64_t* w_full = acc_empty + 2;
  uint64_t* mma_done = w_full + 1;
  uint64_t* red_bar = mma_done + 1;   // [2]: converters' per-box maxima written
  uint64_t* pair_bar = red_bar + 2;   // [4][2]: the two epilogue warps of a TMEM lane quarter
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.slot_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.slot_off + 8);
  float* red = reinterpret_cast<float*>(smem + L.red_off);
  int* tvec = reinterpret_cast<int*>(smem + L.t_off);
  float* gain = reinterpret_cast<float*>(smem + L.ops_off);
  float* offset = gain + kRows;
  float* mean32 = offset + kRows;
  float* uu = mean32 + kK;
  float* uinv = uu + kMaxTargetsPerPass;
  float* zzp = reinterpret_cast<float*>(smem + L.zz_off);
  float* zbuf = reinterpret_cast<float*>(smem + L.zb_off);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t P = args.pixels;
  const int64_t ntiles = div_up<int64_t>(P, kTilePx);
  // static persistent schedule: tiles blockIdx.x, blockIdx.x + gridDim.x, ...
  const int n = ntiles > blockIdx.x ? static_cast<int>((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kIn; ++s) {
      mbar_init(&in_full[s], 1);
      mbar_init(&in_empty[s], kConvWarps);
    }
    for (int s = 0; s < kOpStages; ++s) {
      mbar_init(&op_full[s], kConvWarps);
      mbar_init(&op_empty[s], 1 + kEpiWarps);  // MMA done with the limbs + epilogue done with the scales
    }
    for (int h = 0; h < 2; ++h) {
      mbar_init(&acc_full[h], 1);
      mbar_init(&acc_empty[h], kEpiWarps / 2);  // the epilogue warps of that row half
    }
    mbar_init(w_full, 1);
    mbar_init(mma_done, 1);
    for (int b = 0; b < 2; ++b) mbar_init(&red_bar[b], kConvWarps);
    for (int b = 0; b < 8; ++b) mbar_init(&pair_bar[b], 2);
    *abort_flag = 0;
    fence_barrier_init();
  }
  for (int i = threadIdx.x; i < 3 * kRows + kMaxTargetsPerPass; i += blockDim.x) gain[i] = args.ops->gain[i];
  if (threadIdx.x < kMaxTargetsPerPass) {
    const float v = args.ops->uu[threadIdx.x];
    uinv[threadIdx.x] = v > 0.0f ? 1.0f / v : 0.0f;
  }
  if (warp == kWarpMma) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kWarpTma) {
    if (lane == 0) {
      prefetch_tensormap(&cube_map);
      // the whitener limbs, once, by row half: limb l of rows [64h, 64h + 64) at (3h + l) x 8 KB
      mbar_arrive_expect_tx(w_full, 3 * kLimbBytes);
      for (int h = 0; h < 2; ++h)
        for (int l = 0; l < 3; ++l)
          bulk_g2s(smem + L.w_off + (3 * h + l) * (kLimbBytes / 2), args.ops->limbs[l] + h * (kLimbBytes / 2),
                   kLimbBytes / 2, w_full);
      uint32_t pending = 0, parity = 0;
      for (int i = 0; i < 2 * n; ++i) {
        const int s = i % kIn;
        const uint32_t ph = (i / kIn) & 1u;
        if (*abort_flag || !mbar_wait(&in_empty[s], ph ^ 1u)) {
          record_error(args.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        const int64_t tile = blockIdx.x + static_cast<int64_t>(i >> 1) * gridDim.x;
        mbar_arrive_expect_tx(&in_full[s], box_bytes<T>());
        tma_load_2d(smem + L.in_off + static_cast<size_t>(s) * box_bytes<T>(), &cube_map,
                    static_cast<int>(tile * kTilePx + (i & 1) * kBoxPx), 0, &in_full[s]);
        pending |= 1u << s;
        parity = (parity & ~(1u << s)) | (ph << s);
      }
      for (int s = 0; s < kIn; ++s)
        if ((pending >> s) & 1u) mbar_wait(&in_full[s], (parity >> s) & 1u);
      mbar_wait(w_full, 0);
    }
  } else if (warp == kWarpMma) {
    if (lane == 0) {
      const uint32_t id128 = idesc_s8_s32(kTilePx, kRows);      // [M0; M1] of a row half
      const uint32_t id64 = idesc_s8_s32(kTilePx, kRows / 2);   // M2 of a row half
      bool issued = false;
      if (n > 0 && !mbar_wait(w_full, 0)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
      }
      bool ok = true;
      for (int i = 0; i < n && ok && !*abort_flag; ++i) {
        const int so = i % kOpStages;
        if (!mbar_wait(&op_full[so], (i / kOpStages) & 1u)) {
          record_error(args.status, HSI_E_TIMEOUT);
          *abort_flag = 1;
          break;
        }
        unsigned char* a = smem + L.a_off + static_cast<size_t>(so) * 3 * kLimbBytes;
        const uint64_t a0 = smem_desc_sw128(a), a1 = smem_desc_sw128(a + kLimbBytes);
        const uint64_t a2 = smem_desc_sw128(a + 2 * kLimbBytes);
        for (int h = 0; h < 2; ++h) {
          if (!mbar_wait(&acc_empty[h], (i & 1u) ^ 1u)) {
            record_error(args.status, HSI_E_TIMEOUT);
            *abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + 256u * h;  // S0 | S1 | S2 | S3 of this row half, 64 columns each
          const uint64_t bw01 = smem_desc_sw128(smem + L.w_off + 3 * h * (kLimbBytes / 2));      // [M0; M1]
          const uint64_t bw2 = smem_desc_sw128(smem + L.w_off + (3 * h + 2) * (kLimbBytes / 2));  // M2
#pragma unroll
          for (int k = 0; k < kK / 32; ++k) {
            const uint64_t adv = static_cast<uint64_t>(k * 2);  // 32 bytes of K in 16-byte units
            const uint32_t acc = k > 0 ? 1u : 0u;
            umma_i8(d + 128, a2 + adv, bw01 + adv, id128, acc);  // S2 += L2 M0, S3 += L2 M1
            umma_i8(d + 0, a0 + adv, bw01 + adv, id128, acc);    // S0 += L0 M0, S1 += L0 M1
            umma_i8(d + 64, a1 + adv, bw01 + adv, id128, 1u);    // S1 += L1 M0, S2 += L1 M1
            umma_i8(d + 128, a0 + adv, bw2 + adv, id64, 1u);     // S2 += L0 M2
            umma_i8(d + 192, a1 + adv, bw2 + adv, id64, 1u);     // S3 += L1 M2
          }
          umma_commit(&acc_full[h]);
          issued = true;
        }
        if (!ok) break;
        umma_commit(&op_empty[so]);
      }
      if (issued) {
        umma_commit(mma_done);
        if (!mbar_wait(mma_done, 0)) record_error(args.status, HSI_E_TIMEOUT);
      }
    }
  } else if (warp < kWarpEpi0) {
    // ---------------- converters ----------------
    // warp c owns bands [16c, 16c+16); lane l owns box pixels 2l and 2l + 1 (one
    // 64- or 32-bit load per band for both).
    const int c = warp - kWarpConv0;
    constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
    const int wbias = __float_as_int(kMagic) - 0x8080;
    float mu[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) mu[j] = mean32[c * 16 + j];
    bool aborted = false;
    for (int j = 0; j < 2 * n; ++j) {
      const int s = j % kIn, i = j >> 1, half = j & 1, so = i % kOpStages;
      if (!aborted && (!mbar_wait(&in_full[s], (j / kIn) & 1u) ||
                       (half == 0 && !mbar_wait(&op_empty[so], ((i / kOpStages) & 1u) ^ 1u)))) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        aborted = true;
      }
      if (aborted) break;
      const T* in = reinterpret_cast<const T*>(smem + L.in_off + static_cast<size_t>(s) * box_bytes<T>());
      const int64_t tile = blockIdx.x + static_cast<int64_t>(i) * gridDim.x;
      float* r = red + (j & 1) * kConvWarps * kBoxPx;
      float d[2][16];
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) {
        const float2 x = load2f(in + (c * 16 + jj) * kBoxPx + 2 * lane);
        d[0][jj] = x.x - mu[jj];
        d[1][jj] = x.y - mu[jj];
      }
      // pixels past the frame (last tile only) convert as zeros
      const int64_t px0 = tile * kTilePx + half * kBoxPx + 2 * lane;
      if (px0 + 1 >= P) {
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) d[h][jj] = px0 + h < P ? d[h][jj] : 0.0f;
      }
      {
        float m0 = 0.0f, m1 = 0.0f;
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          m0 = fmaxf(m0, fabsf(d[0][jj]));
          m1 = fmaxf(m1, fabsf(d[1][jj]));
        }
        *reinterpret_cast<float2*>(r + c * kBoxPx + 2 * lane) = make_float2(m0, m1);
      }
      // the input box is consumed (values are in registers); maxima published
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&in_empty[s]);
        mbar_arrive(&red_bar[j & 1]);
      }
      if (!mbar_wait(&red_bar[j & 1], (j >> 1) & 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      unsigned char* a = smem + L.a_off + static_cast<size_t>(so) * 3 * kLimbBytes;
      float2 mx = make_float2(0.0f, 0.0f);
#pragma unroll
      for (int cc = 0; cc < kConvWarps; ++cc) {
        const float2 v = *reinterpret_cast<const float2*>(r + cc * kBoxPx + 2 * lane);
        mx.x = fmaxf(mx.x, v.x);
        mx.y = fmaxf(mx.y, v.y);
      }
      // Lane l holds pixels 2l and 2l + 1.  In round it it stores the limbs of
      // pixel 2l + (it ^ ((l >> 2) & 1)): the 32 rows of one store then fall
      // on all eight 16-byte slots of the 128-byte swizzle (row & 7 takes
      // every value), so each 16-byte store of the warp is four conflict-free
      // wavefronts instead of eight.
      const int hflip = (lane >> 2) & 1;
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int h = it ^ hflip;
        const int pl = 2 * lane + h;
        const float m = h ? mx.y : mx.x;
        // 2^t with m 2^t in [2^21, 2^22): |q| <= 2^22, exact through the FMA rounding
        int t = 0;
        if (m > 0.0f) t = min(max(21 - (static_cast<int>((__float_as_uint(m) >> 23) & 255u) - 127), -100), 100);
        const float sc = __int_as_float((t + 127) << 23);
        uint32_t l0[4], l1[4], l2[4];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          int w[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float dv = h ? d[1][g * 4 + e] : d[0][g * 4 + e];
            w[e] = __float_as_int(fmaf(dv, sc, kMagic)) - wbias;
          }
          const uint32_t p01 = __byte_perm(w[0], w[1], 0x5140), p23 = __byte_perm(w[2], w[3], 0x5140);
          const uint32_t h01 = __byte_perm(w[0], w[1], 0x7362), h23 = __byte_perm(w[2], w[3], 0x7362);
          l2[g] = __byte_perm(p01, p23, 0x5410) ^ 0x80808080u;
          l1[g] = __byte_perm(p01, p23, 0x7632) ^ 0x80808080u;
          l0[g] = __byte_perm(h01, h23, 0x5410);
        }
        const int row = half * kBoxPx + pl;
        const uint32_t o = sw128_byte(row, c * 16);
        *reinterpret_cast<uint4*>(a + o) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
        *reinterpret_cast<uint4*>(a + kLimbBytes + o) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
        *reinterpret_cast<uint4*>(a + 2 * kLimbBytes + o) = make_uint4(l2[0], l2[1], l2[2], l2[3]);
        if (c == 0) tvec[so * kTilePx + row] = t;
      }
      if (half == 1) {
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&op_full[so]);
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int e = warp - kWarpEpi0;
    const int q = warp & 3;         // TMEM lane quarter this warp may access
    const int hf = e >> 2;          // row half: rows [64 hf, 64 hf + 64)
    const int px = q * 32 + lane;   // pixel within the tile
    const uint32_t trow = tmem + (static_cast<uint32_t>(q * 32) << 16);
    const int B = args.bands, rows = args.rows, nt = args.ntarg;
    for (int i = 0; i < n; ++i) {
      const int so = i % kOpStages;
      if (!mbar_wait(&acc_full[hf], i & 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      // the scales were published with the limbs (already complete: the MMA waited on it)
      if (!mbar_wait(&op_full[so], (i / kOpStages) & 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      const int t = tvec[so * kTilePx + px];
      __syncwarp();
      if (lane == 0) mbar_arrive(&op_empty[so]);  // scales read
      const float tau = __int_as_float((127 - t) << 23);
      float zz = 0.0f;
#pragma unroll 1
      for (int cb = 0; cb < 4; ++cb) {
        const int n0 = hf * 64 + cb * 16;
        if (n0 >= rows) break;  // warp-uniform
        uint32_t s0[16], s1[16], s2[16], s3[16];
        const uint32_t col = 256u * hf + 16u * cb;  // rows n0.. of this half's S0; S1, S2, S3 64 columns apart
        tmem_ld16(trow + col, s0);
        tmem_ld16(trow + col + 64, s1);
        tmem_ld16(trow + col + 128, s2);
        tmem_ld16(trow + col + 192, s3);
        tmem_wait_ld();
        // all_bands: every row of the block is a whitened band (the common case: no
        // per-row test); otherwise rows past B are ACE numerators, past `rows` unused
        auto block = [&](auto all_bands) {
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            // four rows' gains and offsets per float4 broadcast (n0 is a multiple of 16)
            const float4 gv = *reinterpret_cast<const float4*>(gain + n0 + 4 * v);
            const float4 ov = *reinterpret_cast<const float4*>(offset + n0 + 4 * v);
            const float g[4] = {gv.x, gv.y, gv.z, gv.w}, o[4] = {ov.x, ov.y, ov.z, ov.w};
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
              const int j = 4 * v + jj;
              const int nn = n0 + j;
              // u = S0 2^24 + S1 2^16 + S2 2^8 + S3 as (S0 256 + S1) 2^16 + (S2 256 + S3):
              // |S0| <= 2^20, |S1| < 2^21.6, |S2| < 2^22.3, |S3| <= 2^22 (128 bands of
              // |L0| <= 64, other limbs <= 128 in magnitude), so both halves are exact int32
              const int hi = static_cast<int>(s0[j]) * 256 + static_cast<int>(s1[j]);
              const int lo = static_cast<int>(s2[j]) * 256 + static_cast<int>(s3[j]);
              const float u = fmaf(__int2float_rn(hi), 65536.0f, __int2float_rn(lo));
              const float z = fmaf(u * tau, g[jj], o[jj]);
              if (decltype(all_bands)::value || nn < B) {
                zz = fmaf(z, z, zz);
              } else if (nn < rows) {
                zbuf[(nn - B) * kTilePx + px] = z;
              }
            }
          }
        };
        if (n0 + 16 <= B) {
          block(std::true_type{});
        } else {
          block(std::false_type{});
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[hf]);
      zzp[hf * kTilePx + px] = zz;
      __syncwarp();
      if (lane == 0) mbar_arrive(&pair_bar[q * 2 + 0]);
      if (!mbar_wait(&pair_bar[q * 2 + 0], i & 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      const int64_t tile = blockIdx.x + static_cast<int64_t>(i) * gridDim.x;
      const int64_t p = tile * kTilePx + px;
      if (hf == 0 && p < P) {
        const float rx = zzp[px] + zzp[kTilePx + px];
        if (args.rx && args.first) args.rx[p] = rx;
        if (nt > 0) {
          float best = -1.0f;
          int32_t best_t = -1;
          if (!args.first) {
            if (args.ace_best) best = args.ace_best[p];
            if (args.ace_target) best_t = args.ace_target[p];
          }
          // (z.u)^2 / (|u|^2 |z|^2) as (z.u)^2 (1 / |u|^2) (1 / |z|^2): one division per
          // pixel instead of one per target
          const float rinv = rx > 0.0f ? 1.0f / rx : 0.0f;
          for (int k = 0; k < nt; ++k) {
            float a = 0.0f;
            if (uu[k] > 0.0f && rx > 0.0f) {
              const float zu = zbuf[k * kTilePx + px];
              a = (zu * zu) * (uinv[k] * rinv);
              if (a > best) {
                best = a;
                best_t = args.t0 + k;
              }
            }
            if (args.ace_maps) args.ace_maps[static_cast<int64_t>(args.t0 + k) * args.map_stride + p] = a;
          }
          if (args.ace_best) args.ace_best[p] = args.last ? (best < 0.0f ? 0.0f : fminf(best, 1.0f)) : best;
          if (args.ace_target) args.ace_target[p] = best_t;
        }
      }
      // zzp / zbuf free for the next tile
      __syncwarp();
      if (lane == 0) mbar_arrive(&pair_bar[q * 2 + 1]);
      if (!mbar_wait(&pair_bar[q * 2 + 1], i & 1u)) {
        record_error(args.status, HSI_E_TIMEOUT);
        *abort_flag = 1;
        break;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == kWarpMma) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

size_t tc_ws_bytes() { return (sizeof(TcOperands) + 255) & ~size_t(255); }

int sm_count() { return device_sm_count(); }

template <typename T>
int launch_tc(const void* cube, int64_t P, int B, int64_t stride, const double* stats, int ntargets, float* rx,
              float* ace_best, int32_t* ace_target, float* ace_maps, int64_t map_stride, void* ws, cudaStream_t s) {
  CUtensorMap map;
  const int dt = sizeof(T) == 4 ? HSI_F32 : HSI_F16;
  if (encode_cube_map(&map, cube, dt, P, B, stride, kBoxPx, kK) != 0) return HSI_E_INVALID;
  const Smem L = smem_layout<T>();
  // set once per device and element type
  const cudaError_t configured = raise_smem_limit(rxace_tc_kernel<T>, static_cast<int>(L.total));
  if (configured != cudaSuccess) return static_cast<int>(configured);
  TcOperands* ops = static_cast<TcOperands*>(ws);
  const int per_pass = kRows - B < kMaxTargetsPerPass ? kRows - B : kMaxTargetsPerPass;
  const int passes = ntargets > 0 ? (ntargets + per_pass - 1) / per_pass : 1;
  const int64_t ntiles = div_up<int64_t>(P, kTilePx);
  const int grid = static_cast<int>(ntiles < sm_count() ? ntiles : sm_count());
  for (int pass = 0; pass < passes; ++pass) {
    const int t0 = pass * per_pass;
    const int nt = ntargets > 0 ? (ntargets - t0 < per_pass ? ntargets - t0 : per_pass) : 0;
    tc_prep_kernel<<<kRows, 128, 0, s>>>(stats, B, ntargets, t0, nt, ops);
    TcArgs a;
    a.pixels = P;
    a.bands = B;
    a.rows = B + nt;
    a.ntarg = nt;
    a.t0 = t0;
    a.first = pass == 0;
    a.last = pass == passes - 1;
    a.ops = ops;
    a.rx = rx;
    a.ace_best = ace_best;
    a.ace_target = ace_target;
    a.ace_maps = ace_maps;
    a.map_stride = map_stride;
    a.status = nullptr;
    rxace_tc_kernel<T><<<grid, kThreads, L.total, s>>>(map, a);
  }
  return static_cast<int>(cudaGetLastError());
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API size_t hsi_rx_ace_workspace_bytes(int bands, int num_targets) {
  if (bands <= 0 || num_targets < 0) return 0;
  return tc_ws_bytes();
}

extern "C" HSI_API int hsi_rx_ace(const void* d_cube, int height, int width, int bands, int dtype,
                                  int64_t plane_stride, const double* d_stats64, int num_targets, float* d_rx,
                                  float* d_ace_best, int32_t* d_ace_target, float* d_ace_maps, int64_t map_stride,
                                  void* d_workspace, size_t workspace_bytes, hsi_stream_t stream) {
  if (!d_cube || !d_stats64 || height <= 0 || width <= 0 || bands <= 0) return HSI_E_INVALID;
  if (dtype != HSI_F32 && dtype != HSI_F16) return HSI_E_INVALID;
  if (bands > kK - 1 || num_targets < 0 || num_targets > 64) return HSI_E_CAPACITY;
  const int64_t P = static_cast<int64_t>(height) * width;
  if (plane_stride < P || (plane_stride & 7) != 0) return HSI_E_INVALID;
  if (num_targets > 0 && d_ace_maps && map_stride < P) return HSI_E_INVALID;
  if (!d_workspace || workspace_bytes < tc_ws_bytes()) return HSI_E_WORKSPACE;
  if ((reinterpret_cast<uintptr_t>(d_workspace) & 255u) != 0 || (reinterpret_cast<uintptr_t>(d_cube) & 15u) != 0)
    return HSI_E_INVALID;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (dtype == HSI_F32)
    return launch_tc<float>(d_cube, P, bands, plane_stride, d_stats64, num_targets, d_rx, d_ace_best, d_ace_target,
                            d_ace_maps, map_stride, d_workspace, s);
  return launch_tc<__half>(d_cube, P, bands, plane_stride, d_stats64, num_targets, d_rx, d_ace_best, d_ace_target,
                           d_ace_maps, map_stride, d_workspace, s);
}
