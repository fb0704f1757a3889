// Shared-memory building blocks for diagonal blocks (order <= 128): Cholesky factor and
// lower-triangular inverse.  A block lives in shared memory as S[i*LDS + j] = element
// (i, j) (row-major, padded row length LDS = 129 so that threads walking down a column
// touch distinct banks).  Blocks of order n are padded to NP = roundup(n, 32) with the
// identity, so every routine works on whole 32 x 32 sub-blocks.
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

// Load the n x n block at G (column-major, ld) into S as a LOWER triangle:
//   transpose == false: S(i,j) = G(i,j) for i >= j
//   transpose == true : S(i,j) = G(j,i) for i >= j   (reads the upper triangle of G)
// The strict upper part of S is zeroed; rows/cols n..NP-1 become the identity.
// unit_diag forces S(i,i) = 1.
__device__ inline void tri_load_lower(double *S, const double *G, int64_t ld, int n, bool transpose,
                               bool unit_diag) {
  const int NP = round_up32(n);
  for (int e = threadIdx.x; e < NP * NP; e += blockDim.x) {
    // e walks G column-major so that consecutive threads read consecutive addresses
    int i = e % NP, j = e / NP;
    double v;
    if (transpose) {
      // S(j,i) = G(i,j) when j >= i; thread reads G(i,j) (coalesced in i)
      int si = j, sj = i;
      if (si < n && sj < n) v = (si > sj) ? G[i + (int64_t)j * ld] : (si == sj ? (unit_diag ? 1.0 : G[i + (int64_t)j * ld]) : 0.0);
      else v = (si == sj) ? 1.0 : 0.0;
      S[si * LDS + sj] = v;
    } else {
      if (i < n && j < n) v = (i > j) ? G[i + (int64_t)j * ld] : (i == j ? (unit_diag ? 1.0 : G[i + (int64_t)j * ld]) : 0.0);
      else v = (i == j) ? 1.0 : 0.0;
      S[i * LDS + j] = v;
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

// In-place Cholesky of the lower triangle of S (order NP, multiple of 32), right-looking
// over 32-column sub-panels.  The pivot is sqrt(s_kk); when it is NaN (s_kk < 0 or NaN)
// the column index is returned through *bad_col (first failure) and the routine stops.
// Division (not reciprocal multiplication) scales the column, as the reference does
// (calgo/dvec_util.c:230-246).  Must be called by all threads of the block.
__device__ inline void tri_potrf_lower(double *S, int NP, int *bad_col, double *bad_val) {
  __shared__ int s_bad;
  if (threadIdx.x == 0) s_bad = -1;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int jb = 0; jb < NP; jb += SUB) {
    // (1) factor the 32 x 32 diagonal sub-block with warp 0
    if (warp == 0) {
      for (int k = 0; k < SUB; ++k) {
        const int kk = jb + k;
        if (lane == 0) {
          double a = S[kk * LDS + kk];
          double d = sqrt(a);
          if (isnan(d) && s_bad < 0) {
            s_bad = kk;
            *bad_val = a;
          }
          S[kk * LDS + kk] = d;
        }
        __syncwarp();
        if (s_bad >= 0) break;
        const double d = S[kk * LDS + kk];
        if (lane > k) S[(jb + lane) * LDS + kk] /= d;
        __syncwarp();
        if (lane > k) {
          const double lik = S[(jb + lane) * LDS + kk];
          for (int j = k + 1; j <= lane; ++j)
            S[(jb + lane) * LDS + jb + j] -= lik * S[(jb + j) * LDS + kk];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    if (s_bad >= 0) break;
    // (2) rows below: L(i, jb:jb+32) = A(i, jb:jb+32) * L_dd^-T by row substitution
    for (int i = jb + SUB + threadIdx.x; i < NP; i += blockDim.x) {
      double *row = S + i * LDS + jb;
      for (int k = 0; k < SUB; ++k) {
        const double *lrow = S + (jb + k) * LDS + jb;
        double s = row[k];
        for (int m = 0; m < k; ++m) s -= row[m] * lrow[m];
        row[k] = s / lrow[k];
      }
    }
    __syncthreads();
    // (3) trailing update of the lower triangle: S(i,j) -= sum_k L(i,k) L(j,k)
    const int r0 = jb + SUB, nr = NP - r0;
    const int npairs = nr * (nr + 1) / 2;
    for (int e = threadIdx.x; e < npairs; e += blockDim.x) {
      // e -> (ii >= jj) in the trailing triangle
      int ii = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
      while ((ii + 1) * (ii + 2) / 2 <= e) ++ii;
      while (ii * (ii + 1) / 2 > e) --ii;
      const int jj = e - ii * (ii + 1) / 2;
      const double *li = S + (r0 + ii) * LDS + jb;
      const double *lj = S + (r0 + jj) * LDS + jb;
      double s = 0.0;
#pragma unroll 8
      for (int k = 0; k < SUB; ++k) s = fma(li[k], lj[k], s);
      S[(r0 + ii) * LDS + r0 + jj] -= s;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *bad_col = s_bad;
  __syncthreads();
}

// In-place inverse of the lower-triangular S (order NP, multiple of 32, non-singular
// diagonal).  W: scratch of 4 * 32 * 33 doubles.  Must be called by all threads.
//   X_ii = L_ii^-1 (one warp per diagonal sub-block, one lane per column)
//   X_ij = -X_ii * sum_{k=j}^{i-1} L_ik X_kj   for i > j, block row by block row
__device__ inline void tri_inverse_lower(double *S, int NP, double *W) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nsub = NP / SUB;
  constexpr int LW = SUB + 1;
  // (1) diagonal sub-blocks, warps 0..nsub-1
  if (warp < nsub) {
    const int b = warp * SUB;
    double *w = W + warp * SUB * LW;
    for (int i = 0; i < SUB; ++i) w[i * LW + lane] = 0.0;
    __syncwarp();
    const int c = lane;
    const double xcc = 1.0 / S[(b + c) * LDS + b + c];
    w[c * LW + c] = xcc;
    for (int i = c + 1; i < SUB; ++i) {
      const double *lrow = S + (b + i) * LDS + b;
      double s = 0.0;
      for (int m = c; m < i; ++m) s = fma(lrow[m], w[m * LW + c], s);
      w[i * LW + c] = -s / lrow[i];
    }
    __syncwarp();
    for (int i = 0; i < SUB; ++i) S[(b + i) * LDS + b + lane] = (lane <= i) ? w[i * LW + lane] : 0.0;
  }
  __syncthreads();
  // (2) off-diagonal blocks, block row by block row
  for (int bi = 1; bi < nsub; ++bi) {
    // T_bj = sum_{k=bj}^{bi-1} L(bi,k) X(k,bj) for bj < bi, into W (bi blocks of 32x33)
    const int nel = bi * SUB * SUB;
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
      const int bj = e / (SUB * SUB), r = (e / SUB) % SUB, c = e % SUB;
      const double *lrow = S + (bi * SUB + r) * LDS;  // row of L in block row bi
      double s = 0.0;
      for (int k = bj * SUB + c; k < bi * SUB; ++k) s = fma(lrow[k], S[k * LDS + bj * SUB + c], s);
      W[bj * SUB * LW + r * LW + c] = s;
    }
    __syncthreads();
    // X(bi,bj) = -X(bi,bi) * T_bj
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
      const int bj = e / (SUB * SUB), r = (e / SUB) % SUB, c = e % SUB;
      const double *xrow = S + (bi * SUB + r) * LDS + bi * SUB;
      double s = 0.0;
      for (int q = 0; q <= r; ++q) s = fma(xrow[q], W[bj * SUB * LW + q * LW + c], s);
      S[(bi * SUB + r) * LDS + bj * SUB + c] = -s;
    }
    __syncthreads();
  }
}

}  // namespace mo
