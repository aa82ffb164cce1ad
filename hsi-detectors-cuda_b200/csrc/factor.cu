// factor.cu - detector statistics in FP64 on the device.
//
// From a frame's raw moments (sum, outer, count) and its target library,
// build everything the RX / ACE / CEM scorers index (reference
// build_statistics, src/detector.cpp:47-152, with the FP64 routines of
// src/linalg.cpp:105-162):
//   mean mu = M1/N
//   S = M2/N - mu mu^T + loading I = L L^T     (Cholesky, fails if not PD)
//   W = L^-1                                   (lower, strict upper zero)
//   u_t = W (d_t - mu),  |u_t|^2               (ACE target half)
//   R = M2/N + loading I = C C^T,  x_t = R^-1 d_t,  w_t = x_t / (d_t . x_t)
//                                              (CEM; 0 if d_t . x_t <= 0)
// All arithmetic is FP64, because the factorisation of a nearly rank-6
// covariance needs it.  One cluster of two CTAs per frame: the covariance and
// the correlation chains run at once on two SMs; frames of a batch factor in
// parallel.  Up to 124 bands, the factorisation and the inverse of the factor
// run together with the matrix in registers, one 4x4 tile per thread, in
// panels of four columns (B / 4 steps of two block barriers each), and W
// lands in shared memory as a packed lower triangle.  Above that the
// factorisation and the inverse are blocked (16-column panels, the diagonal
// blocks factored and inverted by one warp in registers), on packed triangles
// in shared memory up to 128 bands; up to 238 bands one packed triangle in
// shared memory turns from the matrix into L and then into W in place (the
// target vectors in the caller's workspace), and beyond that the matrices
// live in the workspace.  The solves use the explicit inverses.
#include <cooperative_groups.h>

#include "common.cuh"
#include "launch_state.h"

namespace hsi_b200 {
namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kSmemMaxBands = 128;
// Shared memory a CTA may hold on sm_100 (opt-in), less the kernel's static
// shared variables and a margin.
constexpr size_t kSmemLimit = 232448 - 64;
// The register-tile path: one thread per 4x4 tile of the lower triangle, up
// to 124 rows (31 * 32 / 2 = 496 tiles).  128 rows would take 528 tiles, and
// a 17th warp would cut the registers a thread may hold below its tile's.
constexpr int kTileMaxBands = 124;
constexpr int kChunk = 16;  // targets per pass through the per-target buffers
constexpr int kNb = 16;     // panel width of the blocked factorisation
constexpr int kLpStride = kNb + 1;  // doubles per panel row in shared memory (spreads the banks)

__host__ __device__ inline size_t tri(int n) { return static_cast<size_t>(n) * (n + 1) / 2; }
__device__ __forceinline__ size_t row_off(int i) { return static_cast<size_t>(i) * (i + 1) / 2; }
// The same offset in 32 bits, for triangles in shared memory (at most 256 rows):
// the in-place path's loops then carry 32-bit shared-memory addresses.
__device__ __forceinline__ unsigned ro32(int i) { return static_cast<unsigned>(i) * static_cast<unsigned>(i + 1) / 2u; }
// doubles of the panel buffer (n rows of kLpStride), which the inverse reuses
// as its block-row buffer (kNb rows of up to n columns)
__host__ __device__ inline size_t lp_elems(int n) {
  const size_t a = static_cast<size_t>(n) * (kNb + 1), b = static_cast<size_t>(kNb) * n;
  return a > b ? a : b;
}

struct FactorArgs {
  int bands, targets;
  double loading;
  const double* moments;  // per frame: sum[B], outer[B*B], count
  int64_t moments_stride;
  const float* library;   // per frame: T x B, or one shared library (stride 0)
  int64_t library_stride;
  double* stats64;        // nullable, packed layout, stride = statistics_elements
  float* stats32;         // nullable, same layout narrowed to float
  float* cem32;           // nullable, T x B per frame (contiguous frames)
  int* status;            // nullable, per frame
  double* scratch;        // global scratch: per frame 2 * tri(B) doubles (B > kSmemMaxBands)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Fill the packed lower triangle with M2/N (- mean mean^T) + loading I.
__device__ void fill_matrix(double* A, const double* outer, const double* mean, double N, double loading, int n,
                            bool centred) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = warp; i < n; i += kWarps) {
    double* ri = A + row_off(i);
    for (int j = lane; j <= i; j += 32) {
      double v = outer[static_cast<size_t>(i) * n + j] / N;
      if (centred) v -= mean[i] * mean[j];
      if (i == j) v += loading;
      ri[j] = v;
    }
  }
  __syncthreads();
}

// The in-place path (kSmemMaxBands < B <= kHybridMaxBands): mean[B], the
// diagonal block's inverse and the packed matrix in shared memory, followed by
// the inverse's block-row buffer (kNb x the last block row's start) when it
// still fits; the target vectors, and that buffer otherwise, in the workspace.
__host__ __device__ inline size_t last_block_row(int n) { return static_cast<size_t>((n - 1) / kNb) * kNb; }
__host__ __device__ inline size_t inplace_core(int n) { return static_cast<size_t>(n) + kNb * kNb + tri(n); }
__host__ __device__ inline bool inplace_tb_in_smem(int n) {
  return sizeof(double) * (inplace_core(n) + kNb * last_block_row(n)) <= kSmemLimit;
}
constexpr int kHybridMaxBands = 238;  // the largest n with inplace_core(n) doubles within kSmemLimit

// ---- blocked Cholesky and triangular inverse (panels of kNb columns) --------
//
// The unblocked factorisation is a chain of n dependent steps, each paying a
// block barrier, a pivot read and an FP64 division.  Blocked, the chain is
// n / kNb panels.  Per panel:
//   1. one warp factors the kNb x kNb diagonal block in registers (shuffles,
//      no barriers) and inverts its factor, V = L_kk^-1, the same way;
//   2. all threads form the panel below it, L_21 = A_21 V^T (independent
//      16-term dot products: the triangular solve becomes a product);
//   3. all threads update the trailing triangle, A_22 -= L_21 L_21^T.
// The inverse W = L^-1 then goes by block rows: W_II = V_II (kept from step
// 1), and W_IJ = -V_II sum_{K=J}^{I-1} L_IK W_KJ for all J < I at once.

// Step 1 (one warp): factor the diagonal block at k0 (kb <= kNb rows) in
// registers, lane l holding row l.  Writes L_kk into A, V = L_kk^-1 into W's
// diagonal block and densely into vs[row * kNb + col].  Sets *bad if a pivot
// is not positive (or NaN).  Not inlined: its 48 doubles of registers would
// otherwise be allocated across the whole kernel, whose other paths then spill.
__device__ __noinline__ void diag_block(double* A, double* W, double* vs, int k0, int kb, int* bad) {
  const int l = threadIdx.x & 31;
  constexpr unsigned kAll = 0xffffffffu;
  double a[kNb];
#pragma unroll
  for (int m = 0; m < kNb; ++m) a[m] = (l < kb && m <= l) ? A[row_off(k0 + l) + k0 + m] : 0.0;
  double rd[kNb];
  bool ok = true;
#pragma unroll
  for (int k = 0; k < kNb; ++k) {
    rd[k] = 0.0;
    if (k < kb) {
      const double akk = __shfl_sync(kAll, a[k], k);
      ok = ok && akk > 0.0;
      const double inv = rsqrt(akk);  // one dependent FP64 op per step instead of a root and a division
      const double sq = akk * inv;
      rd[k] = inv;
      if (l == k) a[k] = sq;
      else if (l > k) a[k] *= inv;
#pragma unroll
      for (int j = k + 1; j < kNb; ++j) {
        const double ljk = __shfl_sync(kAll, a[k], j);
        if (l >= j) a[j] -= a[k] * ljk;
      }
    }
  }
  // V = L^-1, lane l computing column l by forward substitution
  double v[kNb];
#pragma unroll
  for (int i = 0; i < kNb; ++i) {
    double t = i == l ? 1.0 : 0.0;
#pragma unroll
    for (int m = 0; m < i; ++m) t -= __shfl_sync(kAll, a[m], i) * v[m];
    v[i] = (i >= l && i < kb) ? t * rd[i] : 0.0;
  }
  if (l < kb) {
    double* ar = A + row_off(k0 + l) + k0;
#pragma unroll
    for (int m = 0; m < kNb; ++m)
      if (m <= l) ar[m] = a[m];
  }
  __syncwarp();  // L_kk before V over it, when W is A (the in-place path)
  if (l < kNb) {
#pragma unroll
    for (int i = 0; i < kNb; ++i) {
      vs[i * kNb + l] = v[i];
      if (i >= l && i < kb && l < kb) W[row_off(k0 + i) + k0 + l] = v[i];
    }
  }
  if (!ok && l == 0) *bad = 1;
}

// In-place blocked Cholesky of a packed lower triangle (src/linalg.cpp:105-122):
// A holds L on return, and W's diagonal blocks hold their inverses.  Returns
// false -- on every thread -- if a pivot is not positive or is NaN.
// lp: n * kLpStride doubles; vs: kNb * kNb; bad: a shared int.
// Lookahead: while warps 1.. update the trailing triangle below the next
// diagonal block, warp 0 updates that block alone and factors it at once, so
// each panel's serial diagonal work overlaps the previous panel's update.
__device__ bool cholesky_blocked(double* A, double* W, int n, double* lp, double* vs, int* bad) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) *bad = 0;
  __syncthreads();
  if (warp == 0) diag_block(A, W, vs, 0, min(kNb, n), bad);
  __syncthreads();
  for (int k0 = 0; k0 < n; k0 += kNb) {
    if (*bad) return false;
    const int kb = min(kNb, n - k0);
    const int r0 = k0 + kb;
    const int rows = n - r0;
    if (rows == 0) break;
    // panel: lp[i][j] = sum_{m <= j} A[r0 + i][k0 + m] V[j][m]  (kb == kNb here)
    for (int e = threadIdx.x; e < rows * kNb; e += blockDim.x) {
      const int i = e / kNb, j = e % kNb;
      const double* ai = A + row_off(r0 + i) + k0;
      const double* vj = vs + j * kNb;
      double t0 = 0.0, t1 = 0.0;  // two partial sums: half the dependent chain
      int m = 0;
      for (; m + 1 <= j; m += 2) {
        t0 += ai[m] * vj[m];
        t1 += ai[m + 1] * vj[m + 1];
      }
      if (m <= j) t0 += ai[m] * vj[m];
      lp[i * kLpStride + j] = t0 + t1;
    }
    __syncthreads();
    const int nb2 = min(kNb, rows);  // rows of the next diagonal block
    if (warp == 0) {
      // the next diagonal block: its panel rows, its own update, then its factorisation
      for (int e = lane; e < nb2 * kNb; e += 32) {
        const int i = e / kNb, j = e % kNb;
        A[row_off(r0 + i) + k0 + j] = lp[i * kLpStride + j];
      }
      for (int e = lane; e < nb2 * nb2; e += 32) {
        const int i = e / nb2, j = e % nb2;
        if (j > i) continue;
        const double* li = lp + i * kLpStride;
        const double* lj = lp + j * kLpStride;
        double t[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < kNb; ++m) t[m & 3] += li[m] * lj[m];
        A[row_off(r0 + i) + r0 + j] -= (t[0] + t[1]) + (t[2] + t[3]);
      }
      __syncwarp();
      diag_block(A, W, vs, r0, nb2, bad);
    } else {
      // the rest: panel rows past the next block, and their trailing rows
      for (int e = threadIdx.x - 32 + nb2 * kNb; e < rows * kNb; e += blockDim.x - 32) {
        const int i = e / kNb, j = e % kNb;
        A[row_off(r0 + i) + k0 + j] = lp[i * kLpStride + j];
      }
      for (int i = nb2 + warp - 1; i < rows; i += kWarps - 1) {
        const double* li = lp + i * kLpStride;
        double* ai = A + row_off(r0 + i) + r0;
        for (int j = lane; j <= i; j += 32) {
          const double* lj = lp + j * kLpStride;
          double t[4] = {0.0, 0.0, 0.0, 0.0};  // four partial sums: a quarter of the dependent chain
#pragma unroll
          for (int m = 0; m < kNb; ++m) t[m & 3] += li[m] * lj[m];
          ai[j] -= (t[0] + t[1]) + (t[2] + t[3]);
        }
      }
    }
    __syncthreads();
  }
  return true;
}

// The same blocked Cholesky with the matrix alone in shared memory (the
// packed triangle of up to kHybridMaxBands rows, with no room for a panel
// buffer beside it): each panel L_21 = A_21 V^T is formed in place, one
// thread per row with the row's kNb values in registers, and the trailing
// update reads L_21 from A.  The diagonal blocks receive V_kk = L_kk^-1 over
// L_kk (nothing reads L_kk afterwards), so inverse_blocked(A, A, ...) then
// turns A into W in place.
__device__ __forceinline__ bool cholesky_inplace(double* A, int n, double* vs, int* bad) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) *bad = 0;
  __syncthreads();
  if (warp == 0) diag_block(A, A, vs, 0, min(kNb, n), bad);
  __syncthreads();
  for (int k0 = 0; k0 < n; k0 += kNb) {
    if (*bad) return false;
    const int kb = min(kNb, n - k0);
    const int r0 = k0 + kb;
    const int rows = n - r0;
    if (rows == 0) break;
    // panel, in place (kb == kNb here): row i's values are read into registers before any is written
    for (int i = threadIdx.x; i < rows; i += blockDim.x) {
      double* ai = A + ro32(r0 + i) + k0;
      double a[kNb];
#pragma unroll
      for (int m = 0; m < kNb; ++m) a[m] = ai[m];
#pragma unroll
      for (int j = 0; j < kNb; ++j) {
        const double* vj = vs + j * kNb;
        double t0 = 0.0, t1 = 0.0;  // two partial sums: half the dependent chain
#pragma unroll
        for (int m = 0; m <= j; ++m) {
          if (m & 1)
            t1 += a[m] * vj[m];
          else
            t0 += a[m] * vj[m];
        }
        ai[j] = t0 + t1;
      }
    }
    __syncthreads();
    const int nb2 = min(kNb, rows);  // rows of the next diagonal block
    if (warp == 0) {
      // the next diagonal block's own update, then its factorisation
      for (int e = lane; e < nb2 * nb2; e += 32) {
        const int i = e / nb2, j = e % nb2;
        if (j > i) continue;
        const double* li = A + ro32(r0 + i) + k0;
        const double* lj = A + ro32(r0 + j) + k0;
        double t[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < kNb; ++m) t[m & 3] += li[m] * lj[m];
        A[ro32(r0 + i) + r0 + j] -= (t[0] + t[1]) + (t[2] + t[3]);
      }
      __syncwarp();
      diag_block(A, A, vs, r0, nb2, bad);
    } else {
      // the trailing rows past the next block (their columns r0.. only; the
      // panel columns k0.. that warp 0 reads are not written here)
      for (int i = nb2 + warp - 1; i < rows; i += kWarps - 1) {
        const double* li = A + ro32(r0 + i) + k0;
        double* ai = A + ro32(r0 + i) + r0;
        for (int j = lane; j <= i; j += 32) {
          const double* lj = A + ro32(r0 + j) + k0;
          double t[4] = {0.0, 0.0, 0.0, 0.0};  // four partial sums: a quarter of the dependent chain
#pragma unroll
          for (int m = 0; m < kNb; ++m) t[m & 3] += li[m] * lj[m];
          ai[j] -= (t[0] + t[1]) + (t[2] + t[3]);
        }
      }
    }
    __syncthreads();
  }
  return true;
}

// W = L^-1 (both packed lower) by block rows, given L and the inverses of its
// diagonal blocks already in W (src/linalg.cpp:150-162 solves the same system
// column by column).  tb: kNb * n doubles.  Each thread of phase 1 takes one
// column and four rows of the block row, so a W element read from shared
// memory serves four products.
__device__ void inverse_blocked(const double* L, double* W, int n, double* tb) {
  constexpr int kRows = 4;
  for (int i0 = kNb; i0 < n; i0 += kNb) {
    const int ib = min(kNb, n - i0);
    const int groups = (ib + kRows - 1) / kRows;
    // phase 1: tb[r][c] = sum_{m=c}^{i0-1} L[i0 + r][m] W[m][c],  r < ib, c < i0
    for (int e = threadIdx.x; e < groups * i0; e += blockDim.x) {
      const int g = e / i0, c = e % i0;
      double t[kRows][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};  // two partial sums per row
      const double* lr[kRows];
#pragma unroll
      for (int q = 0; q < kRows; ++q) lr[q] = L + row_off(i0 + min(g * kRows + q, ib - 1));
      int m = c;
      for (; m + 1 < i0; m += 2) {
        const double w0 = W[row_off(m) + c], w1 = W[row_off(m + 1) + c];
#pragma unroll
        for (int q = 0; q < kRows; ++q) {
          t[q][0] += lr[q][m] * w0;
          t[q][1] += lr[q][m + 1] * w1;
        }
      }
      if (m < i0) {
        const double w0 = W[row_off(m) + c];
#pragma unroll
        for (int q = 0; q < kRows; ++q) t[q][0] += lr[q][m] * w0;
      }
#pragma unroll
      for (int q = 0; q < kRows; ++q)
        if (g * kRows + q < ib) tb[(g * kRows + q) * i0 + c] = t[q][0] + t[q][1];
    }
    __syncthreads();
    // phase 2: W[i0 + r][c] = -sum_{m <= r} V[r][m] tb[m][c]
    for (int e = threadIdx.x; e < ib * i0; e += blockDim.x) {
      const int r = e / i0, c = e % i0;
      const double* vr = W + row_off(i0 + r) + i0;
      double t0 = 0.0, t1 = 0.0;
      int m = 0;
      for (; m + 1 <= r; m += 2) {
        t0 += vr[m] * tb[m * i0 + c];
        t1 += vr[m + 1] * tb[(m + 1) * i0 + c];
      }
      if (m <= r) t0 += vr[m] * tb[m * i0 + c];
      W[row_off(i0 + r) + c] = -(t0 + t1);
    }
    __syncthreads();
  }
}

// inverse_blocked for the in-place path: W over L in one shared-memory
// triangle (the same sums in the same order, so the same bits), with 32-bit
// shared-memory offsets and the block-row buffer tb in shared memory or the
// workspace.
__device__ __forceinline__ void inverse_inplace(double* A, int n, double* tb) {
  constexpr int kRows = 4;
  for (int i0 = kNb; i0 < n; i0 += kNb) {
    const int ib = min(kNb, n - i0);
    const int groups = (ib + kRows - 1) / kRows;
    for (int e = threadIdx.x; e < groups * i0; e += blockDim.x) {
      const int g = e / i0, c = e % i0;
      double t[kRows][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
      unsigned lr[kRows];
#pragma unroll
      for (int q = 0; q < kRows; ++q) lr[q] = ro32(i0 + min(g * kRows + q, ib - 1));
      int m = c;
      unsigned wm = ro32(m) + c;  // A[m][c]: row m + 1 starts m + 1 doubles after row m
      for (; m + 1 < i0; m += 2) {
        const double w0 = A[wm], w1 = A[wm + m + 1];
        wm += 2 * m + 3;
#pragma unroll
        for (int q = 0; q < kRows; ++q) {
          t[q][0] += A[lr[q] + m] * w0;
          t[q][1] += A[lr[q] + m + 1] * w1;
        }
      }
      if (m < i0) {
        const double w0 = A[wm];
#pragma unroll
        for (int q = 0; q < kRows; ++q) t[q][0] += A[lr[q] + m] * w0;
      }
#pragma unroll
      for (int q = 0; q < kRows; ++q)
        if (g * kRows + q < ib) tb[(g * kRows + q) * i0 + c] = t[q][0] + t[q][1];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ib * i0; e += blockDim.x) {
      const int r = e / i0, c = e % i0;
      const unsigned vr = ro32(i0 + r) + i0;
      double t0 = 0.0, t1 = 0.0;
      int m = 0;
      for (; m + 1 <= r; m += 2) {
        t0 += A[vr + m] * tb[m * i0 + c];
        t1 += A[vr + m + 1] * tb[(m + 1) * i0 + c];
      }
      if (m <= r) t0 += A[vr + m] * tb[m * i0 + c];
      A[ro32(i0 + r) + c] = -(t0 + t1);
    }
    __syncthreads();
  }
}

// ---- register-tile factorisation and inverse (n <= kTileMaxBands) -----------
//
// The right-looking blocked Cholesky and the inverse of its factor together,
// in panels of four columns, with the matrix in registers: thread t owns the
// 4x4 tile (I, K), I >= K, of the lower triangle.  A tile holds A (being
// factored) until its column panel is reached, and R (becoming W = L^-1)
// after it (the recurrences of src/linalg.cpp:105-122 and :150-162, blocked).
// Step J, with D = chol(A_JJ) and Dinv = D^-1 (from the owner of tile (J, J)):
//   phase 1  (J, J):        W_JJ = Dinv
//            (J, K < J):    W_JK = Dinv R_JK           published as W^T rows
//            (I > J, J):    L_IJ = A_IJ Dinv^T          published
//                           R_IJ = -L_IJ Dinv
//   phase 2  (I > J, K > J):  A_IK -= L_IJ L_KJ^T        (rank 4)
//            (I > J, K < J):  R_IK -= L_IJ W_JK
//            then the owner of (J+1, J+1) factors its block for the next step.
// L rows (index >= 4J + 4) and W^T rows (index < 4J) share one published
// panel: phase 2 is the same 64 FMAs for every tile it updates.  Two block
// barriers per step, B / 4 steps.  Rows past n get an identity diagonal, so
// the last panel factors as a full 4x4 block.  The matrix is formed straight
// from the moments (M2/N, centred for the covariance, plus the loading on the
// diagonal).  L itself is not kept: only W is used afterwards.

constexpr int kPanBlock = 18;  // doubles per 4-row block of the panel: 144 bytes, 9 x 16 (conflict-free blocks)
constexpr int kPanDoubles = 32 * kPanBlock;
// the tile path's shared memory: the panel, Dinv, the failure flag
constexpr int kTileShared = kPanDoubles + 16 + 2;

// The Cholesky factor of the 4x4 block a (lower part) with rsqrt pivots, and
// its inverse d (lower, upper zero).  False if a pivot is not positive or NaN.
__device__ __forceinline__ bool factor4(const double (&a)[4][4], double (&d)[4][4]) {
  double l[4][4], s[4];
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double piv = a[c][c];
#pragma unroll
    for (int m = 0; m < c; ++m) piv = fma(-l[c][m], l[c][m], piv);
    ok = ok && piv > 0.0;
    s[c] = rsqrt(piv);
    l[c][c] = piv * s[c];
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      double v = a[r][c];
#pragma unroll
      for (int m = 0; m < c; ++m) v = fma(-l[r][m], l[c][m], v);
      l[r][c] = v * s[c];
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
#pragma unroll
    for (int r = 0; r < c; ++r) d[r][c] = 0.0;
    d[c][c] = s[c];
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      double v = 0.0;
#pragma unroll
      for (int m = c; m < r; ++m) v = fma(l[r][m], d[m][c], v);
      d[r][c] = -s[r] * v;
    }
  }
  return ok;
}

__device__ __forceinline__ double* pan_row(double* pan, int i) { return pan + (i >> 2) * kPanBlock + (i & 3) * 4; }

// sh: kTileShared doubles, 16-byte aligned.  Returns false -- on every thread,
// at the same step -- if a pivot is not positive or is NaN.
__device__ bool chol_inv_tiles(const double* outer, const double* mean, double N, double loading, bool centred,
                               double* W, int n, double* sh) {
  double* pan = sh;
  double* dv = sh + kPanDoubles;
  int* bad = reinterpret_cast<int*>(dv + 16);
  const int t = threadIdx.x;
  const int nt = (n + 3) >> 2;
  const bool own = t < nt * (nt + 1) / 2;
  // tiles by columns: a warp's tiles share a column panel
  int K = 0, first = 0;
  while (K + 1 < nt && first + (nt - K) <= t) first += nt - K++;
  const int I = K + (t - first);
  const int i0 = 4 * I, k0 = 4 * K;
  double x[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + p, k = k0 + q;
      double v = 0.0;
      if (own && i < n && k <= i) {
        v = outer[static_cast<size_t>(i) * n + k] / N;
        if (centred) v -= mean[i] * mean[k];
        if (i == k) v += loading;
      } else if (own && i >= n && i == k) {
        v = 1.0;  // padding: an identity block
      }
      x[p][q] = v;
    }
  if (t == 0) {  // owner of tile (0, 0)
    double d[4][4];
    *bad = factor4(x, d) ? 0 : 1;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) dv[r * 4 + c] = d[r][c];
  }
  __syncthreads();
  for (int J = 0; J < nt; ++J) {
    if (*bad) return false;
    // ---- phase 1: the panel's row and column
    if (own && (I == J || K == J)) {
      double d[4][4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const double2 d01 = *reinterpret_cast<const double2*>(dv + r * 4);
        const double2 d23 = *reinterpret_cast<const double2*>(dv + r * 4 + 2);
        d[r][0] = d01.x, d[r][1] = d01.y, d[r][2] = d23.x, d[r][3] = d23.y;
      }
      if (I == J && K == J) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) x[r][c] = d[r][c];
      } else if (I == J) {
        // W_JK = Dinv R_JK, published as rows k of W^T
        double w[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            double v = 0.0;
#pragma unroll
            for (int m = 0; m <= r; ++m) v = fma(d[r][m], x[m][q], v);
            w[r][q] = v;
          }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          double* row = pan_row(pan, k0 + q);
          *reinterpret_cast<double2*>(row) = make_double2(w[0][q], w[1][q]);
          *reinterpret_cast<double2*>(row + 2) = make_double2(w[2][q], w[3][q]);
#pragma unroll
          for (int r = 0; r < 4; ++r) x[r][q] = w[r][q];
        }
      } else {
        // L_IJ = A_IJ Dinv^T, published; then R_IJ = -L_IJ Dinv
        double l[4][4];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            double v = 0.0;
#pragma unroll
            for (int m = 0; m <= c; ++m) v = fma(x[p][m], d[c][m], v);
            l[p][c] = v;
          }
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          double* row = pan_row(pan, i0 + p);
          *reinterpret_cast<double2*>(row) = make_double2(l[p][0], l[p][1]);
          *reinterpret_cast<double2*>(row + 2) = make_double2(l[p][2], l[p][3]);
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            double v = 0.0;
#pragma unroll
            for (int m = c; m < 4; ++m) v = fma(l[p][m], d[m][c], v);
            x[p][c] = -v;
          }
        }
      }
    }
    __syncthreads();
    // ---- phase 2: rank-4 update of every tile below the panel's row, off its column
    if (own && I > J && K != J) {
      double u[4][4], v[4][4];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const double* ru = pan_row(pan, i0 + p);
        const double* rv = pan_row(pan, k0 + p);
        const double2 u01 = *reinterpret_cast<const double2*>(ru), u23 = *reinterpret_cast<const double2*>(ru + 2);
        const double2 v01 = *reinterpret_cast<const double2*>(rv), v23 = *reinterpret_cast<const double2*>(rv + 2);
        u[p][0] = u01.x, u[p][1] = u01.y, u[p][2] = u23.x, u[p][3] = u23.y;
        v[p][0] = v01.x, v[p][1] = v01.y, v[p][2] = v23.x, v[p][3] = v23.y;
      }
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) x[p][q] = fma(-u[p][c], v[q][c], x[p][q]);
      if (I == J + 1 && K == J + 1) {  // the next diagonal block, now final: factor it
        double d[4][4];
        if (!factor4(x, d)) *bad = 1;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) dv[r * 4 + c] = d[r][c];
      }
    }
    __syncthreads();
  }
  if (own) {
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int i = i0 + p, k = k0 + q;
        if (i < n && k <= i) W[row_off(i) + k] = x[p][q];
      }
  }
  __syncthreads();
  return true;
}

// out[t][i] = sum_{j <= i} M[i][j] v[t][j] (M packed lower), t < nt.
__device__ void lower_matvec(const double* M, const double* v, double* out, int n, int nt) {
  for (int e = threadIdx.x; e < nt * n; e += blockDim.x) {
    const int t = e / n, i = e % n;
    const double* mi = M + row_off(i);
    const double* vt = v + static_cast<size_t>(t) * n;
    double s[4] = {0.0, 0.0, 0.0, 0.0};  // four partial sums: a quarter of the dependent chain
    int j = 0;
    for (; j + 3 <= i; j += 4) {
      s[0] += mi[j] * vt[j];
      s[1] += mi[j + 1] * vt[j + 1];
      s[2] += mi[j + 2] * vt[j + 2];
      s[3] += mi[j + 3] * vt[j + 3];
    }
    for (; j <= i; ++j) s[0] += mi[j] * vt[j];
    out[e] = (s[0] + s[1]) + (s[2] + s[3]);
  }
  __syncthreads();
}

// out[t][i] = sum_{k >= i} M[k][i] v[t][k] (M^T, M packed lower), t < nt.
__device__ void upper_matvec(const double* M, const double* v, double* out, int n, int nt) {
  for (int e = threadIdx.x; e < nt * n; e += blockDim.x) {
    const int t = e / n, i = e % n;
    const double* vt = v + static_cast<size_t>(t) * n;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    int k = i;
    for (; k + 3 < n; k += 4) {
      s[0] += M[row_off(k) + i] * vt[k];
      s[1] += M[row_off(k + 1) + i] * vt[k + 1];
      s[2] += M[row_off(k + 2) + i] * vt[k + 2];
      s[3] += M[row_off(k + 3) + i] * vt[k + 3];
    }
    for (; k < n; ++k) s[0] += M[row_off(k) + i] * vt[k];
    out[e] = (s[0] + s[1]) + (s[2] + s[3]);
  }
  __syncthreads();
}

// One cluster of two CTAs per frame, on two SMs at once:
//   rank 0: covariance S = L L^T -> mean, whitener W = L^-1, ACE vectors;
//   rank 1: correlation R = C C^T -> CEM weights (only when there are targets).
// The chains share nothing but the mean, which each computes.  At the end
// rank 1 writes its result code into rank 0's shared memory and rank 0 writes
// the frame's status: an empty frame or a covariance that is not positive
// definite first (the reference stops there), else the correlation's code.
__global__ void __cluster_dims__(1, 2, 1) __launch_bounds__(kThreads) factor_kernel(const FactorArgs args) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) double smem[];
  __shared__ int s_partner_code;
  __shared__ int s_bad;
  const int f = blockIdx.x;
  const int chain = blockIdx.y;  // 0: covariance, 1: correlation
  const int B = args.bands, T = args.targets;
  const double* mom = args.moments + f * args.moments_stride;
  const float* lib = args.library ? args.library + f * args.library_stride : nullptr;
  const size_t per = static_cast<size_t>(B) + static_cast<size_t>(B) * B + 2 * static_cast<size_t>(T) * B + T;
  double* out64 = args.stats64 ? args.stats64 + f * per : nullptr;
  float* out32 = args.stats32 ? args.stats32 + f * per : nullptr;
  float* cem32 = args.cem32 ? args.cem32 + static_cast<size_t>(f) * T * B : nullptr;
  const bool in_smem = B <= kSmemMaxBands;
  const bool inplace = !in_smem && B <= kHybridMaxBands;
  // smem: mean[B], two chunk buffers of kChunk x B, the panel / block-row
  // buffer, the diagonal block's inverse, then the packed matrices (in the
  // workspace when B is large).  The in-place path keeps only mean, the
  // diagonal block's inverse and one matrix in shared memory.
  double* mean = smem;
  double* vec = mean + B;
  double* buf = vec + static_cast<size_t>(kChunk) * B;
  double* lp = buf + static_cast<size_t>(kChunk) * B;
  double* vs = lp + lp_elems(B);
  double* cbuf = vs + kNb * kNb;  // the tile path's panel, Dinv and flag (kTileShared doubles, 16-byte aligned)
  // the tile path keeps the factor in registers: only W lives in shared memory
  const bool tiles = B <= kTileMaxBands;
  double* ws = args.scratch + (static_cast<size_t>(f) * 2 + chain) * 2 * tri(B);
  double* A = in_smem ? cbuf + kTileShared : ws;
  double* W = tiles ? A : A + tri(B);
  if (inplace) {
    vs = mean + B;
    A = W = vs + kNb * kNb;
    vec = ws;
    buf = vec + static_cast<size_t>(kChunk) * B;
    lp = inplace_tb_in_smem(B) ? A + tri(B) : buf + static_cast<size_t>(kChunk) * B;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t off_tw = static_cast<size_t>(B) + static_cast<size_t>(B) * B;
  const size_t off_tn = off_tw + static_cast<size_t>(T) * B;
  const size_t off_cw = off_tn + T;

  int code = HSI_OK;
  const double N = mom[B + B * B];
  const double* sum = mom;
  const double* outer = mom + B;
  if (!(N > 0.0)) code = HSI_E_EMPTY;
  if (code == HSI_OK && (chain == 0 || T > 0)) {
    for (int i = threadIdx.x; i < B; i += blockDim.x) mean[i] = sum[i] / N;
    __syncthreads();
    // covariance (chain 0) or correlation (chain 1), loaded (src/linalg.cpp:56-79)
    bool factored;
    if (tiles) {
      factored = chol_inv_tiles(outer, mean, N, args.loading, chain == 0, W, B, cbuf);
    } else if (inplace) {
      // pointers taken straight from the shared array, so the inlined loops
      // address shared memory directly
      double* As = smem + B + kNb * kNb;
      fill_matrix(As, outer, mean, N, args.loading, B, chain == 0);
      factored = cholesky_inplace(As, B, smem + B, &s_bad);
      if (factored) {
        if (inplace_tb_in_smem(B))
          inverse_inplace(As, B, As + tri(B));
        else
          inverse_inplace(As, B, lp);
      }
    } else {
      fill_matrix(A, outer, mean, N, args.loading, B, chain == 0);
      factored = cholesky_blocked(A, W, B, lp, vs, &s_bad);
      if (factored) inverse_blocked(A, W, B, lp);
    }
    if (!factored) {
      code = chain == 0 ? HSI_E_NOT_POSITIVE_DEFINITE : HSI_E_CORRELATION_NOT_PD;
    } else {
      if (chain == 0) {
        // outputs: mean, whitener (row-major, upper zero)
        for (int i = threadIdx.x; i < B; i += blockDim.x) {
          if (out64) out64[i] = mean[i];
          if (out32) out32[i] = static_cast<float>(mean[i]);
        }
        for (size_t e = threadIdx.x; e < static_cast<size_t>(B) * B; e += blockDim.x) {
          const int i = static_cast<int>(e / B), j = static_cast<int>(e % B);
          const double v = j <= i ? W[row_off(i) + j] : 0.0;
          if (out64) out64[B + e] = v;
          if (out32) out32[B + e] = static_cast<float>(v);
        }
        // ACE: u_t = W (d_t - mu) and |u_t|^2, kChunk targets at a time
        for (int t0 = 0; t0 < T; t0 += kChunk) {
          const int nt = min(kChunk, T - t0);
          for (int e = threadIdx.x; e < nt * B; e += blockDim.x)
            vec[e] = static_cast<double>(lib[static_cast<size_t>(t0) * B + e]) - mean[e % B];
          __syncthreads();
          lower_matvec(W, vec, buf, B, nt);
          for (int e = threadIdx.x; e < nt * B; e += blockDim.x) {
            if (out64) out64[off_tw + static_cast<size_t>(t0) * B + e] = buf[e];
            if (out32) out32[off_tw + static_cast<size_t>(t0) * B + e] = static_cast<float>(buf[e]);
          }
          for (int t = warp; t < nt; t += kWarps) {
            double q = 0.0;
            for (int i = lane; i < B; i += 32) q += buf[t * B + i] * buf[t * B + i];
            q = warp_sum(q);
            if (lane == 0) {
              if (out64) out64[off_tn + t0 + t] = q;
              if (out32) out32[off_tn + t0 + t] = static_cast<float>(q);
            }
          }
          __syncthreads();
        }
      } else {
        // CEM: y_t = C^-1 d_t, x_t = C^-T y_t = R^-1 d_t, d_t . x_t = |y_t|^2;
        // w_t = x_t / |y_t|^2, 0 if that gain is not positive (src/detector.cpp:128-148)
        for (int t0 = 0; t0 < T; t0 += kChunk) {
          const int nt = min(kChunk, T - t0);
          for (int e = threadIdx.x; e < nt * B; e += blockDim.x)
            vec[e] = static_cast<double>(lib[static_cast<size_t>(t0) * B + e]);
          __syncthreads();
          lower_matvec(W, vec, buf, B, nt);   // y
          upper_matvec(W, buf, vec, B, nt);   // x (d is no longer needed)
          for (int t = warp; t < nt; t += kWarps) {
            double g = 0.0;
            for (int i = lane; i < B; i += 32) g += buf[t * B + i] * buf[t * B + i];
            g = warp_sum(g);
            for (int i = lane; i < B; i += 32) {
              const double w = g > 0.0 ? vec[t * B + i] / g : 0.0;
              const size_t o = static_cast<size_t>(t0 + t) * B + i;
              if (out64) out64[off_cw + o] = w;
              if (out32) out32[off_cw + o] = static_cast<float>(w);
              if (cem32) cem32[o] = static_cast<float>(w);
            }
          }
          __syncthreads();
        }
      }
    }
  }
  // combine the two chains' codes in rank 0 (every thread of both CTAs
  // reaches the cluster barrier: no early returns above)
  cg::cluster_group cluster = cg::this_cluster();
  if (chain == 1 && threadIdx.x == 0) *cluster.map_shared_rank(&s_partner_code, 0) = code;
  cluster.sync();
  if (chain == 0 && threadIdx.x == 0 && args.status) args.status[f] = code != HSI_OK ? code : s_partner_code;
}

size_t smem_bytes(int B, int /*T*/) {
  const size_t vectors =
      static_cast<size_t>(B) + 2 * static_cast<size_t>(kChunk) * B + lp_elems(B) + kNb * kNb + kTileShared;
  if (B <= kTileMaxBands) return sizeof(double) * (vectors + tri(B));
  if (B <= kSmemMaxBands) return sizeof(double) * (vectors + 2 * tri(B));
  if (B <= kHybridMaxBands)
    return sizeof(double) * (inplace_core(B) + (inplace_tb_in_smem(B) ? kNb * last_block_row(B) : 0));
  return sizeof(double) * vectors;
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API size_t hsi_statistics_elements(int bands, int num_targets) {
  if (bands <= 0 || num_targets < 0) return 0;
  return static_cast<size_t>(bands) + static_cast<size_t>(bands) * bands + 2 * static_cast<size_t>(num_targets) * bands +
         num_targets;
}

extern "C" HSI_API size_t hsi_factor_workspace_bytes(int num_frames, int bands) {
  if (num_frames <= 0 || bands <= 0) return 0;
  if (bands <= kSmemMaxBands) return 0;
  // both chains' matrices (A and W) per frame
  return sizeof(double) * 4 * tri(bands) * static_cast<size_t>(num_frames);
}

extern "C" HSI_API int hsi_build_statistics(int num_frames, int bands, int num_targets, double loading,
                                            const double* d_moments, const float* d_library,
                                            int64_t library_stride, double* d_stats64, float* d_stats32,
                                            float* d_cem_weights, int* d_status, void* d_workspace,
                                            size_t workspace_bytes, hsi_stream_t stream) {
  if (num_frames <= 0 || bands <= 0 || bands > HSI_MAX_BANDS || num_targets < 0 || num_targets > 64 || !d_moments)
    return HSI_E_INVALID;
  if (num_targets > 0 && !d_library) return HSI_E_INVALID;
  if (!(loading >= 0.0)) return HSI_E_INVALID;
  const size_t need = hsi_factor_workspace_bytes(num_frames, bands);
  if (need > 0 && (!d_workspace || workspace_bytes < need)) return HSI_E_WORKSPACE;
  FactorArgs a;
  a.bands = bands;
  a.targets = num_targets;
  a.loading = loading;
  a.moments = d_moments;
  a.moments_stride = static_cast<int64_t>(bands) + static_cast<int64_t>(bands) * bands + 1;
  a.library = d_library;
  a.library_stride = library_stride;
  a.stats64 = d_stats64;
  a.stats32 = d_stats32;
  a.cem32 = d_cem_weights;
  a.status = d_status;
  a.scratch = static_cast<double*>(d_workspace);
  const size_t smem = smem_bytes(bands, num_targets);
  if (smem > 227 * 1024) return HSI_E_CAPACITY;
  const cudaError_t e = raise_smem_limit(factor_kernel, static_cast<int>(smem));
  if (e != cudaSuccess) return static_cast<int>(e);
  factor_kernel<<<dim3(num_frames, 2), kThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  return static_cast<int>(cudaGetLastError());
}
