// Shared-memory building blocks for diagonal blocks (order <= 128): Cholesky factor and
// lower-triangular inverse.  A block lives in shared memory as S[i*LDS + j] = element
// (i, j) (row-major, padded row length LDS = 129 so that threads walking down a column
// touch distinct banks).  Blocks of order n are padded to NP = roundup(n, 32) with the
// identity, so every routine works on whole 32 x 32 sub-blocks.  The factor and inverse
// routines are templates on the element type: FP64 for the FP64 drivers, FP32 for the
// diagonal blocks of the mixed-precision factorization (whose working matrix is FP32).
#pragma once
#include "common.cuh"

namespace mo {

constexpr int TRI_MAX = 128;
constexpr int LDS = TRI_MAX + 1;
constexpr int SUB = 32;
constexpr int TRI_THREADS = 256;
// shared memory: the block plus 3 scratch 32 x 33 sub-blocks
constexpr int TRI_SMEM_BYTES = (TRI_MAX * LDS + 4 * SUB * (SUB + 1)) * 8;

__device__ __forceinline__ int round_up32(int n) { return (n + 31) & ~31; }

__device__ __forceinline__ double tri_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float tri_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double tri_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float tri_sqrt(float x) { return sqrtf(x); }

// Load the n x n block at G (column-major, ld) into S as a LOWER triangle:
//   transpose == false: S(i,j) = G(i,j) for i >= j
//   transpose == true : S(i,j) = G(j,i) for i >= j   (reads the upper triangle of G)
// The strict upper part of S is zeroed; rows/cols n..NP-1 become the identity.
// unit_diag forces S(i,i) = 1.  Each thread issues 8 independent loads before its
// shared-memory stores, so a single CTA keeps enough reads in flight.
__device__ inline void tri_load_lower(double *S, const double *G, int64_t ld, int n, bool transpose,
                                      bool unit_diag) {
  const int NP = round_up32(n);
  const int total = NP * NP, step = blockDim.x;
  for (int base = threadIdx.x; base < total; base += 8 * step) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      // e walks G column-major so that consecutive threads read consecutive addresses
      const int e = base + u * step;
      const int i = e % NP, j = e / NP;
      // element of the lower triangle that G(i, j) feeds: (si, sj)
      const int si = transpose ? j : i, sj = transpose ? i : j;
      double x = (si == sj) ? 1.0 : 0.0;
      if (e < total && si < n && sj < n && si >= sj && !(unit_diag && si == sj))
        x = G[i + (int64_t)j * ld];
      v[u] = x;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = base + u * step;
      if (e < total) {
        const int i = e % NP, j = e / NP;
        const int si = transpose ? j : i, sj = transpose ? i : j;
        S[si * LDS + sj] = v[u];
      }
    }
  }
}

// Store the lower triangle of S (n x n) to G: transpose == false -> G(i,j) = S(i,j) for
// i >= j; transpose == true -> G(j,i) = S(i,j) (upper triangle of G).  If full_square,
// the opposite strict triangle of G is written with zeros (used for inverse blocks).
__device__ inline void tri_store_lower(const double *S, double *G, int64_t ld, int n, bool transpose,
                                       bool full_square) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e % n, j = e / n;  // G element (i, j), coalesced in i
    if (transpose) {
      // G(i,j) = S(j,i) when j >= i
      if (j >= i) G[i + (int64_t)j * ld] = S[j * LDS + i];
      else if (full_square) G[i + (int64_t)j * ld] = 0.0;
    } else {
      if (i >= j) G[i + (int64_t)j * ld] = S[i * LDS + j];
      else if (full_square) G[i + (int64_t)j * ld] = 0.0;
    }
  }
}

// S(i, j) -= sum_{k<32} S(i, kb + k) * S(j, kb + k) for the lower triangle (i >= j) of
// rows/cols [r0, NP).  The region is cut into 32 x 32 blocks (bi >= bj); 64 threads own
// one block as an 8 x 8 grid of 4 x 4 micro-tiles whose rows and columns are strided by
// 8, so the 8 rows a warp reads sit in distinct banks.
template <typename T>
__device__ __forceinline__ void tri_syrk_update(T *S, int NP, int r0, int kb) {
  const int nbk = (NP - r0) / SUB;
  const int ntask = nbk * (nbk + 1) / 2;
  const int t = threadIdx.x & 63, tx = t & 7, ty = t >> 3;
  const int nslot = blockDim.x >> 6;
  for (int task = threadIdx.x >> 6; task < ntask; task += nslot) {
    int bi = 0;
    while ((bi + 1) * (bi + 2) / 2 <= task) ++bi;
    const int bj = task - bi * (bi + 1) / 2;
    const int i0 = r0 + bi * SUB + tx, j0 = r0 + bj * SUB + ty;
    T acc[4][4];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[x][y] = T(0);
#pragma unroll 8
    for (int k = 0; k < SUB; ++k) {
      T a[4], b[4];
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        a[x] = S[(i0 + 8 * x) * LDS + kb + k];
        b[x] = S[(j0 + 8 * x) * LDS + kb + k];
      }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
    }
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y)
        if (i0 + 8 * x >= j0 + 8 * y) S[(i0 + 8 * x) * LDS + j0 + 8 * y] -= acc[x][y];
  }
}

// Cholesky of a 32 x 32 lower block held by one warp, lane i holding row i in r[0..31]
// (the reference divides by the square root, calgo/dvec_util.c:230-246; here columns are
// multiplied by reciprocal square roots, equal to rounding).  Two columns per step: every
// lane factors the 2 x 2 diagonal block [a .; b c] itself (l11 = sqrt(a), l21 = b / l11,
// l22 = sqrt(c - l21^2), from three shuffles), forms its row's two multipliers, and the
// pair goes to the other lanes through shared memory, so the dependency chain has one
// shuffle, store, __syncwarp and load per two columns.  The arithmetic is the
// column-by-column algorithm's, in the same order (the second column is updated by the
// first before it is scaled, and each trailing entry takes the first column's product
// before the second's).  The rank-2 updates run on every lane without a lane test: a lane
// only modifies entries right of its diagonal, which are never read, and this keeps the
// unrolled body free of divergent branches.  With `checked`, the loop stops at the first
// NaN pivot and returns its column.  `col` is 4 x 32 elements of shared memory (two
// alternating pairs of multiplier columns).
template <bool checked, typename T>
__device__ __forceinline__ int warp_potrf32(T (&r)[SUB], int lane, double *badv, T *col) {
  int bad = -1;
#pragma unroll
  for (int k = 0; k < SUB; k += 2) {
    const T a = __shfl_sync(0xffffffffu, r[k], k);
    const T b = __shfl_sync(0xffffffffu, r[k], k + 1);
    const T c = __shfl_sync(0xffffffffu, r[k + 1], k + 1);
    const T rs1 = tri_rsqrt(a);
    if (checked) {
      if (isnan(rs1)) {  // uniform: every lane sees the same pivot
        bad = k;
        *badv = a;
        break;
      }
    }
    const T l21 = b * rs1;
    const T d = fma(-l21, l21, c);
    const T rs2 = tri_rsqrt(d);
    if (checked) {
      if (isnan(rs2)) {
        bad = k + 1;
        *badv = d;
        break;
      }
    }
    const T x1 = lane > k ? r[k] * rs1 : T(0);
    const T x2 = lane > k + 1 ? fma(-x1, l21, r[k + 1]) * rs2 : T(0);
    T *c1 = col + ((k >> 1) & 1) * 2 * SUB, *c2 = c1 + SUB;
    c1[lane] = x1;
    c2[lane] = x2;
    __syncwarp();
#pragma unroll
    for (int j = k + 2; j < SUB; ++j) r[j] = fma(-x2, c2[j], fma(-x1, c1[j], r[j]));
    r[k] = lane == k ? tri_sqrt(a) : (lane > k ? x1 : r[k]);
    r[k + 1] = lane == k + 1 ? tri_sqrt(d) : (lane > k + 1 ? x2 : r[k + 1]);
  }
  return bad;
}

// In-place Cholesky of the lower triangle of S (order NP, multiple of 32), right-looking
// over 32-column sub-panels.  The pivot is sqrt(s_kk); when it is NaN (s_kk < 0 or NaN)
// the column index is returned through *bad_col (first failure) and the routine stops.
// Must be called by all threads of the block.  *bad_val receives the failing pivot.
//   (1) 32 x 32 diagonal sub-block: one warp, lane i holds row i in registers; the fast
//       unchecked factor runs first and the checked one reruns only if a pivot was NaN
//   (2) rows below: one thread per row, the 32-wide row segment in registers, scaled by
//       the reciprocal pivots (as LAPACK dpotf2 scales by 1/ajj)
//   (3) trailing lower triangle: register-blocked rank-32 update
template <typename T>
__device__ inline void tri_potrf_lower(T *S, int NP, int *bad_col, double *bad_val) {
  __shared__ int s_bad;
  __shared__ T s_rd[SUB];
  __shared__ T s_col[4 * SUB];
  if (threadIdx.x == 0) s_bad = -1;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int jb = 0; jb < NP; jb += SUB) {
    if (warp == 0) {
      T r[SUB];
#pragma unroll
      for (int j = 0; j < SUB; ++j) r[j] = (j <= lane) ? S[(jb + lane) * LDS + jb + j] : T(0);
      double unused;
      warp_potrf32<false>(r, lane, &unused, s_col);
      T dg = r[0];
#pragma unroll
      for (int j = 1; j < SUB; ++j) dg = (j == lane) ? r[j] : dg;
      if (__ballot_sync(0xffffffffu, isnan(dg)) != 0u) {
        // a pivot failed: redo the sub-block with the stop at the first NaN pivot
#pragma unroll
        for (int j = 0; j < SUB; ++j) r[j] = (j <= lane) ? S[(jb + lane) * LDS + jb + j] : T(0);
        double badv = 0.0;
        const int bad = warp_potrf32<true>(r, lane, &badv, s_col);
        if (lane == 0) {
          s_bad = jb + bad;
          *bad_val = badv;
        }
      }
      s_rd[lane] = T(1) / dg;
#pragma unroll
      for (int j = 0; j < SUB; ++j)
        if (j <= lane) S[(jb + lane) * LDS + jb + j] = r[j];
    }
    __syncthreads();
    if (s_bad >= 0) break;
    // (2) L(i, jb:jb+32) = A(i, jb:jb+32) * L_dd^-T for rows i below the sub-block
    for (int i = jb + SUB + threadIdx.x; i < NP; i += blockDim.x) {
      T v[SUB];
      T *row = S + i * LDS + jb;
#pragma unroll
      for (int k = 0; k < SUB; ++k) v[k] = row[k];
#pragma unroll
      for (int k = 0; k < SUB; ++k) {
        v[k] = v[k] * s_rd[k];
#pragma unroll
        for (int m = k + 1; m < SUB; ++m) v[m] = fma(-v[k], S[(jb + m) * LDS + jb + k], v[m]);
      }
#pragma unroll
      for (int k = 0; k < SUB; ++k) row[k] = v[k];
    }
    __syncthreads();
    // (3) trailing update of the lower triangle
    if (jb + SUB < NP) tri_syrk_update(S, NP, jb + SUB, jb);
    __syncthreads();
  }
  if (threadIdx.x == 0) *bad_col = s_bad;
  __syncthreads();
}

// C(32x32, in W at ldc) = sum over `nk` 32-blocks of P_q(32x32) * Q_q(32x32), where P_q is
// S[prow + r, pcol + 32q + k] and Q_q is S or W data given by pointers; all threads,
// 4 x 4 register micro-tiles (64 per 32 x 32 product).
template <typename T>
__device__ __forceinline__ void tri_small_gemm(T *C, int ldc, const T *P, int ldp, const T *Q,
                                               int ldq, int nk, T sign, int tile,
                                               int ntile_total) {
  (void)ntile_total;
  const int ti = tile / 8, tj = tile % 8;
  T acc[4][4];
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) acc[x][y] = T(0);
  for (int k = 0; k < nk; ++k) {
    T a[4], b[4];
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      a[x] = P[(4 * ti + x) * ldp + k];
      b[x] = Q[k * ldq + 4 * tj + x];
    }
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
  }
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) C[(4 * ti + x) * ldc + 4 * tj + y] = sign * acc[x][y];
}

// In-place inverse of the lower-triangular S (order NP, multiple of 32, non-singular
// diagonal).  W: scratch of 4 * 32 * 33 elements.  Must be called by all threads.
//   X_ii = L_ii^-1 (one warp per diagonal sub-block, one lane per column, registers)
//   X_ij = -X_ii * sum_{k=j}^{i-1} L_ik X_kj   for i > j, block row by block row
template <typename T>
__device__ inline void tri_inverse_lower(T *S, int NP, T *W) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nsub = NP / SUB;
  constexpr int LW = SUB + 1;
  // (1) diagonal sub-blocks, each split in 16 x 16 halves: warp w (< 4) inverts the upper
  //     half of block w and warp w + 4 the lower half, lane c < 16 solving L x = e_c (a
  //     16-long chain instead of 32); then both warps form the off-diagonal half,
  //     X21 = -X22 (L21 X11), through the scratch W
  constexpr int H = SUB / 2;
  const int blk = warp & 3, half = warp >> 2;
  if (blk < nsub) {
    const int b = blk * SUB + half * H;
    // reciprocal pivots, lane i holds 1 / L_ii; the substitution multiplies by them so
    // the serial chain per row is FMAs only
    const T rdi = lane < H ? T(1) / S[(b + lane) * LDS + b + lane] : T(0);
    T x[H];
#pragma unroll
    for (int i = 0; i < H; ++i) {
      const T *lrow = S + (b + i) * LDS + b;
      T s0 = (i == lane) ? T(1) : T(0), s1 = T(0);
#pragma unroll
      for (int m = 0; m + 1 < i; m += 2) {
        s0 = fma(-lrow[m], x[m], s0);
        s1 = fma(-lrow[m + 1], x[m + 1], s1);
      }
      if (i & 1) s0 = fma(-lrow[i - 1], x[i - 1], s0);
      const T rd = __shfl_sync(0xffffffffu, rdi, i);
      x[i] = (i < lane) ? T(0) : (s0 + s1) * rd;
    }
    __syncwarp();
    if (lane < H) {
#pragma unroll
      for (int i = 0; i < H; ++i) S[(b + i) * LDS + b + lane] = x[i];  // column lane
    }
  }
  __syncthreads();
  {
    // thread t of the block's 64: row r = t / 4, columns 4 (t % 4) .. + 3 of the half block
    const int t = (warp >> 2) * 32 + lane, r = t >> 2, c0 = (t & 3) * 4;
    T *Tm = W + blk * H * (H + 1);
    const int b = blk * SUB;
    if (blk < nsub) {
      // T = L21 X11 (X11 lower: k >= column)
      T acc[4] = {T(0), T(0), T(0), T(0)};
      const T *l21 = S + (b + H + r) * LDS + b;
#pragma unroll
      for (int k = 0; k < H; ++k) {
        const T lv = l21[k];
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (k >= c0 + j) acc[j] = fma(lv, S[(b + k) * LDS + b + c0 + j], acc[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) Tm[r * (H + 1) + c0 + j] = acc[j];
    }
    __syncthreads();
    if (blk < nsub) {
      // X21 = -X22 T (X22 lower: k <= row)
      T acc[4] = {T(0), T(0), T(0), T(0)};
      const T *x22 = S + (b + H + r) * LDS + b + H;
#pragma unroll
      for (int k = 0; k < H; ++k) {
        if (k <= r) {
          const T xv = x22[k];
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[j] = fma(xv, Tm[k * (H + 1) + c0 + j], acc[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) S[(b + H + r) * LDS + b + c0 + j] = -acc[j];
    }
  }
  __syncthreads();
  // (2) off-diagonal blocks, block row by block row
  for (int bi = 1; bi < nsub; ++bi) {
    // T_bj = sum_{k=bj}^{bi-1} L(bi,k) X(k,bj) for bj < bi  -> W block bj
    for (int e = threadIdx.x; e < bi * 64; e += blockDim.x) {
      const int bj = e / 64, tile = e % 64;
      tri_small_gemm(W + bj * SUB * LW, LW, S + (bi * SUB) * LDS + bj * SUB, LDS,
                     S + (bj * SUB) * LDS + bj * SUB, LDS, (bi - bj) * SUB, T(1), tile, 64);
    }
    __syncthreads();
    // X(bi,bj) = -X(bi,bi) * T_bj
    for (int e = threadIdx.x; e < bi * 64; e += blockDim.x) {
      const int bj = e / 64, tile = e % 64;
      tri_small_gemm(S + (bi * SUB) * LDS + bj * SUB, LDS, S + (bi * SUB) * LDS + bi * SUB, LDS,
                     W + bj * SUB * LW, LW, SUB, T(-1), tile, 64);
    }
    __syncthreads();
  }
}

}  // namespace mo
