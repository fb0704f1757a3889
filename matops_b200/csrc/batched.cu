// Batched Cholesky / LU factor + solve of many small FP64 systems of uneven order
// (n <= MO_BATCH_MAX_N) in one persistent launch per schedule group, replayed from a CUDA
// graph.  The reference factors one matrix per call (DecomposeCHOL chol.go:116,
// DecomposeLU lu.go:257, SolveCHOL chol.go:147, SolveLU lu.go:320); here each CTA takes
// whole matrices from a work queue ordered by decreasing n^3 (longest job first) and
// runs, for each one:
//
//   Cholesky (lower, right-looking, panel width NB):
//     diag   : NB x NB block in registers of warp 0 (lane i holds row i), column
//              Cholesky by shuffles (reciprocal square root); a NaN pivot stops the matrix
//              with info = column + 1 (the reference panics, chol.go:33-36)
//     panel  : rows below, one thread per row: x = a * L11^-T by forward substitution
//     update : A22 -= L21 L21^T on 64 x 64 lower tiles, K = NB, operands staged in
//              shared memory by cp.async (double-buffered), products on the FP64 tensor
//              pipe (mma.sync m16n8k4, 32 x 16 per warp)
//   LU (partial pivoting, right-looking, panel width NB):
//     panel  : the (n - j) x NB panel in registers (thread t owns logical rows j + t and
//              j + t + 256); per column a block argmax of |a| with ties to the lowest row
//              (pivotIndex, pivot.go:98-107), the row exchange through shared memory,
//              true division by the pivot and the rank-1 update of the panel
//     swaps  : lazy -- a logical-to-physical row map in shared memory; every later access
//              goes through it, and the rows are put in their final order once, at the
//              end, so no strided row exchange touches the matrix per step
//     U12    : one warp per column, unit-lower solve with L11 by shuffles; U12 is also
//              written row-major to the CTA's scratch so the update reads it coalesced
//     update : A22 -= L21 U12 on 64 x 64 tiles as above
//   solve (when B is given): forward and backward substitution per right-hand side,
//     32-row blocks: a warp solves the diagonal block by shuffles, the other rows are
//     updated in axpy form (columns of the factor are read contiguously)
//
// FP64 FMA and the FP64 tensor pipe have the same peak on B200, but one m16n8k4 MMA does
// the work of sixteen warp FMAs, which leaves the issue slots to the loads; the triangular
// and pivoting steps are latency-bound and use warp shuffles to avoid block-wide barriers.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "context.cuh"

namespace mo {
namespace {

constexpr int BT = 256;   // threads per CTA
constexpr int TM = 64;    // update tile (TM x TM)
constexpr int TMP = TM + 4;  // staged row stride: fragment loads (lane 4g + t reads row t,
                             // element g) fall in distinct banks
constexpr int MAXN = MO_BATCH_MAX_N;
constexpr int RPT = MAXN / BT;  // panel rows per thread (LU)

struct BatchParams {
  int count;                 // matrices in this group's queue
  const int *order;          // queue: indices into the arrays below
  int *counter;              // next queue position (reset to 0 before each launch)
  const int *n;              // order of each matrix
  double *const *A;          // device pointers to the matrices
  const int64_t *lda;
  double *const *B;          // right-hand sides (nullptr: factor only)
  const int64_t *ldb;
  int nrhs;
  int64_t *const *piv;       // LU pivots (0-based absolute row, LAPACK convention)
  int *info;                 // per matrix: 0 or column + 1 of the failing pivot
  double *ut;                // LU: per-CTA scratch, NB x MAXN doubles each
};

template <int NB>
struct Smem {
  double As[2][NB][TMP];  // update operands, double-buffered
  double Bs[2][NB][TMP];
  double L11[NB][NB + 1];
  double vec[MAXN];      // solve vector
  double ubuf[NB];       // LU: pivot row
  double sbuf[NB];       // LU: displaced row
  double red_v[BT / 32];
  int red_i[BT / 32];
  int perm[MAXN];        // LU: logical row -> physical row
  int idx, info, pidx, swapped;
};

__device__ __forceinline__ void cp8(double *dst, const double *src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(ok ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// In-register Cholesky of an NB x NB block held by one warp (lane i holds row i; rows and
// columns beyond the block's order are padded with the identity).  Returns the first
// column whose pivot square root is NaN, or -1.
template <int NB>
__device__ __forceinline__ int warp_chol(double (&r)[NB], int lane, double *badv) {
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    const double akk = __shfl_sync(0xffffffffu, r[k], k);
    const double rs = rsqrt(akk);  // one reciprocal square root on the chain per column
    if (isnan(rs)) {  // uniform across the warp
      *badv = akk;
      return k;
    }
    // shuffles and updates use the multiplier lk (zero on lanes <= k): the pivot's square
    // root is off the chain
    const double lk = lane > k ? r[k] * rs : 0.0;
#pragma unroll
    for (int j = k + 1; j < NB; ++j) {
      const double ljk = __shfl_sync(0xffffffffu, lk, j);
      r[j] = fma(-lk, ljk, r[j]);
    }
    r[k] = lane == k ? sqrt(akk) : (lane > k ? lk : r[k]);
  }
  return -1;
}

// block-wide argmax of (v, i): larger v wins, equal v -> lower i.  All threads get the
// winning index.  Uses s.red_* and s.pidx; contains two barriers.
template <int NB>
__device__ __forceinline__ int block_argmax(Smem<NB> &s, double v, int i) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
    if (v2 > v || (v2 == v && i2 < i)) {
      v = v2;
      i = i2;
    }
  }
  if (lane == 0) {
    s.red_v[warp] = v;
    s.red_i[warp] = i;
  }
  __syncthreads();
  if (warp == 0) {
    v = lane < BT / 32 ? s.red_v[lane] : -1.0;
    i = lane < BT / 32 ? s.red_i[lane] : 0x7fffffff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
      const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
      if (v2 > v || (v2 == v && i2 < i)) {
        v = v2;
        i = i2;
      }
    }
    if (lane == 0) s.pidx = i;
  }
  __syncthreads();
  return s.pidx;
}

// Trailing update of one matrix: C -= P * Q on the m2 x m2 trailing block whose first
// logical row and column is j0 (K = kb <= NB columns of the panel starting at column kc).
//   C(i, c) = A[row(j0 + i) + (j0 + c) * ld]
//   P(i, k) = A[row(j0 + i) + (kc + k) * ld]                  (L21)
//   Q(k, c) = LU ? ut[k * MAXN + j0 + c]                        (U12, row-major scratch)
//               : A[(j0 + c) + (kc + k) * ld]                   (L21^T, Cholesky)
// row() is the LU row map (identity for Cholesky).  Cholesky updates only tiles on or
// below the diagonal and, inside diagonal tiles, only elements with row >= column.
// Tile t + 1's operands are staged while tile t is computed.  The products run on the
// FP64 tensor pipe: warp w owns the 32 x 16 block at rows 32 (w & 1), columns 16 (w >> 1)
// of the 64 x 64 tile, as 2 x 2 fragments of mma.sync m16n8k4 (k padded to a multiple of
// 4 with the zeros the staging writes past kb).  Ends with a barrier.
template <bool LU, int NB>
__device__ void trailing_update(Smem<NB> &s, double *A, int64_t ld, int j0, int m2, int kc,
                                int kb, const double *ut) {
  const int nt = (m2 + TM - 1) / TM;
  const int T = LU ? nt * nt : nt * (nt + 1) / 2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int rw = 32 * (warp & 1), cw = 16 * (warp >> 1);
  auto tile_of = [&](int t, int &ti, int &tj) {
    if (LU) {
      ti = t % nt;
      tj = t / nt;
    } else {  // lower tiles, column by column: (tj, ti >= tj)
      int c = 0, rem = t;
      while (rem >= nt - c) {
        rem -= nt - c;
        ++c;
      }
      tj = c;
      ti = c + rem;
    }
  };
  auto row_of = [&](int logical) -> int { return LU ? s.perm[logical] : logical; };
  auto stage = [&](int t, int buf) {
    int ti, tj;
    tile_of(t, ti, tj);
    const int r0 = ti * TM, c0 = tj * TM;
    for (int e = tid; e < TM * NB; e += BT) {
      const int r = e % TM, k = e / TM;
      const bool okr = k < kb && r0 + r < m2;
      const double *src = okr ? A + row_of(j0 + r0 + r) + (int64_t)(kc + k) * ld : A;
      cp8(&s.As[buf][k][r], src, okr);
      const bool okc = k < kb && c0 + r < m2;
      const double *srcq;
      if (LU) srcq = okc ? ut + (int64_t)k * MAXN + j0 + c0 + r : ut;
      else srcq = okc ? A + (j0 + c0 + r) + (int64_t)(kc + k) * ld : A;
      cp8(&s.Bs[buf][k][r], srcq, okc);
    }
  };
  if (T == 0) return;
  stage(0, 0);
  cp_commit();
  for (int t = 0; t < T; ++t) {
    const int buf = t & 1;
    if (t + 1 < T) stage(t + 1, buf ^ 1);
    cp_commit();
    int ti, tj;
    tile_of(t, ti, tj);
    const int r0 = ti * TM, c0 = tj * TM;
    // this thread's C elements (fragment layout): rows rw + 16 mi + g + 8 h,
    // columns cw + 8 ni + 2 t4 + e, accumulator index d[mi][ni][2 h + e]
    double cv[2][2][4];
    int64_t roff[2][2];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = r0 + rw + 16 * mi + g + 8 * h;
        roff[mi][h] = i < m2 ? (int64_t)row_of(j0 + i) : -1;
      }
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int c = c0 + cw + 8 * ni + 2 * t4 + (q & 1);
          const int64_t ro = roff[mi][q >> 1];
          cv[mi][ni][q] = (ro >= 0 && c < m2) ? A[ro + (int64_t)(j0 + c) * ld] : 0.0;
        }
    cp_wait1();
    __syncthreads();
    double d[2][2][4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni)
#pragma unroll
        for (int q = 0; q < 4; ++q) d[mi][ni][q] = 0.0;
    const int ksteps = (kb + 3) >> 2;
#pragma unroll 2
    for (int k4 = 0; k4 < ksteps; ++k4) {
      const int k = 4 * k4 + t4;
      double a[2][2], b[2];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        a[mi][0] = s.As[buf][k][rw + 16 * mi + g];
        a[mi][1] = s.As[buf][k][rw + 16 * mi + g + 8];
      }
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) b[ni] = s.Bs[buf][k][cw + 8 * ni + g];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) dmma_16x8x4(d[mi][ni], a[mi][0], a[mi][1], b[ni]);
    }
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int i = r0 + rw + 16 * mi + g + 8 * (q >> 1);
          const int c = c0 + cw + 8 * ni + 2 * t4 + (q & 1);
          const int64_t ro = roff[mi][q >> 1];
          const bool ok = ro >= 0 && c < m2 && (LU || i >= c);
          if (ok) A[ro + (int64_t)(j0 + c) * ld] = cv[mi][ni][q] - d[mi][ni][q];
        }
    __syncthreads();
  }
  cp_wait0();
}

// In-place lower Cholesky of one n x n matrix; returns 0 or info = column + 1.
template <int NB>
__device__ int chol_matrix(Smem<NB> &s, double *A, int64_t ld, int n) {
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid == 0) s.info = 0;
  for (int j = 0; j < n; j += NB) {
    const int jb = min(NB, n - j);
    if (tid < 32) {
      double r[NB];
#pragma unroll
      for (int k = 0; k < NB; ++k) {
        const bool in = lane < jb && k < jb && k <= lane;
        r[k] = in ? A[(j + lane) + (int64_t)(j + k) * ld] : (lane == k ? 1.0 : 0.0);
      }
      double badv = 0.0;
      const int bad = warp_chol<NB>(r, lane, &badv);
      if (bad >= 0) {
        if (lane == 0) s.info = j + bad + 1;
      } else if (lane < jb) {
#pragma unroll
        for (int k = 0; k < NB; ++k) {
          if (k <= lane && k < jb) A[(j + lane) + (int64_t)(j + k) * ld] = r[k];
          s.L11[lane][k] = r[k];
        }
      }
    }
    __syncthreads();
    if (s.info) return s.info;
    // rows below the diagonal block: x = a * L11^-T
    for (int i = j + jb + tid; i < n; i += BT) {
      double x[NB];
#pragma unroll
      for (int k = 0; k < NB; ++k) x[k] = k < jb ? A[i + (int64_t)(j + k) * ld] : 0.0;
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        if (c < jb) {
          double t = x[c];
#pragma unroll
          for (int k = 0; k < c; ++k) t = fma(-x[k], s.L11[c][k], t);
          x[c] = t / s.L11[c][c];
        }
      }
#pragma unroll
      for (int k = 0; k < NB; ++k)
        if (k < jb) A[i + (int64_t)(j + k) * ld] = x[k];
    }
    __syncthreads();
    const int m2 = n - j - jb;
    if (m2 > 0) trailing_update<false, NB>(s, A, ld, j + jb, m2, j, jb, nullptr);
  }
  return 0;
}

// In-place LU with partial pivoting of one n x n matrix.  piv[k] receives the 0-based row
// exchanged with row k.  Returns 0 or the first column + 1 whose pivot is exactly zero
// (the factorization still completes, as LAPACK's dgetrf does; the reference does not
// check).  On return s.perm holds the row map (logical row r came from physical row
// perm[r] of the input).
template <int NB>
__device__ int lu_matrix(Smem<NB> &s, double *A, int64_t ld, int n, int64_t *piv, double *ut) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int r = tid; r < n; r += BT) s.perm[r] = r;
  if (tid == 0) {
    s.info = 0;
    s.swapped = 0;
  }
  __syncthreads();
  for (int j = 0; j < n; j += NB) {
    const int jb = min(NB, n - j);
    double p[RPT][NB];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int r = j + tid + BT * q;
      const int64_t pr = r < n ? s.perm[r] : 0;
#pragma unroll
      for (int k = 0; k < NB; ++k) p[q][k] = (r < n && k < jb) ? A[pr + (int64_t)(j + k) * ld] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < NB; ++c) {
      if (c >= jb) break;  // uniform
      const int jc = j + c;
      double bv = -1.0;
      int bi = 0x7fffffff;
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int r = j + tid + BT * q;
        if (r < n && r >= jc) {
          const double v = fabs(p[q][c]);
          if (v > bv) {
            bv = v;
            bi = r;
          }
        }
      }
      int pr = block_argmax<NB>(s, bv, bi);
      if (pr >= n) pr = jc;  // no comparable candidate (all NaN): keep the row
      const int po = pr - j;  // owner: thread po % BT, slot po / BT
      if (tid == po % BT) {
        const int q = po / BT;
#pragma unroll
        for (int k = 0; k < NB; ++k) s.ubuf[k] = q ? p[RPT - 1][k] : p[0][k];
      }
      if (pr != jc && tid == c) {
#pragma unroll
        for (int k = 0; k < NB; ++k) s.sbuf[k] = p[0][k];
      }
      __syncthreads();
      if (pr != jc) {
        if (tid == c) {
#pragma unroll
          for (int k = 0; k < NB; ++k) p[0][k] = s.ubuf[k];
        }
        if (tid == po % BT) {
          const int q = po / BT;
#pragma unroll
          for (int k = 0; k < NB; ++k) {
            if (q) p[RPT - 1][k] = s.sbuf[k];
            else p[0][k] = s.sbuf[k];
          }
        }
        if (tid == 0) {
          const int t = s.perm[jc];
          s.perm[jc] = s.perm[pr];
          s.perm[pr] = t;
          s.swapped = 1;
        }
      }
      if (tid == 0) piv[jc] = pr;
      const double u = s.ubuf[c];
      if (u == 0.0 && tid == 0 && s.info == 0) s.info = jc + 1;
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int r = j + tid + BT * q;
        if (r < n && r > jc) {
          const double l = p[q][c] / u;
          p[q][c] = l;
#pragma unroll
          for (int k = c + 1; k < NB; ++k) p[q][k] = fma(-l, s.ubuf[k], p[q][k]);
        }
      }
    }
    __syncthreads();  // row map final for this panel
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int r = j + tid + BT * q;
      if (r < n) {
        const int64_t pr = s.perm[r];
#pragma unroll
        for (int k = 0; k < NB; ++k)
          if (k < jb) A[pr + (int64_t)(j + k) * ld] = p[q][k];
      }
    }
    if (tid < jb) {
#pragma unroll
      for (int k = 0; k < NB; ++k) s.L11[tid][k] = p[0][k];
    }
    __syncthreads();
    // U12 = L11^-1 A12 (unit lower), one warp per column; also row-major into ut
    for (int col = j + jb + warp; col < n; col += BT / 32) {
      const int64_t prow = lane < jb ? s.perm[j + lane] : 0;
      double x = lane < jb ? A[prow + (int64_t)col * ld] : 0.0;
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        const double xc = __shfl_sync(0xffffffffu, x, c);
        if (c < jb && lane > c && lane < jb) x = fma(-s.L11[lane][c], xc, x);
      }
      if (lane < jb) {
        A[prow + (int64_t)col * ld] = x;
        ut[(int64_t)lane * MAXN + col] = x;
      }
    }
    __syncthreads();
    const int m2 = n - j - jb;
    if (m2 > 0) trailing_update<true, NB>(s, A, ld, j + jb, m2, j, jb, ut);
  }
  // put the rows in their final order: row r of the result is physical row perm[r]
  if (s.swapped) {
    constexpr int CH = 8;
    for (int c0 = 0; c0 < n; c0 += CH) {
      double v[RPT][CH];
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int r = tid + BT * q;
        const int64_t pr = r < n ? s.perm[r] : 0;
#pragma unroll
        for (int cc = 0; cc < CH; ++cc)
          v[q][cc] = (r < n && c0 + cc < n) ? A[pr + (int64_t)(c0 + cc) * ld] : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int r = tid + BT * q;
#pragma unroll
        for (int cc = 0; cc < CH; ++cc)
          if (r < n && c0 + cc < n) A[r + (int64_t)(c0 + cc) * ld] = v[q][cc];
      }
      __syncthreads();
    }
  }
  return s.info;
}

// Solve with the factor of one matrix, right-hand side by right-hand side, in 32-row
// blocks.  CHOL: L L^T x = b (SolveCHOL LOWER, chol.go:147-158).  LU: P A = L U, x = U^-1
// L^-1 P b (SolveLU, lu.go:320-334; P b gathered through the row map s.perm).
template <bool LU, int NB>
__device__ void solve_matrix(Smem<NB> &s, const double *A, int64_t ld, int n, double *B,
                             int64_t ldb, int nrhs) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double *y = s.vec;
  for (int rc = 0; rc < nrhs; ++rc) {
    double *b = B + (int64_t)rc * ldb;
    for (int r = tid; r < n; r += BT) y[r] = LU ? b[s.perm[r]] : b[r];
    __syncthreads();
    // forward: L y = b (LU: unit diagonal), axpy form
    for (int j = 0; j < n; j += 32) {
      const int jb = min(32, n - j);
      if (warp == 0) {
        double row[32];
#pragma unroll
        for (int c = 0; c < 32; ++c)
          row[c] = (lane < jb && c <= lane && c < jb) ? A[(j + lane) + (int64_t)(j + c) * ld] : 0.0;
        double yi = lane < jb ? y[j + lane] : 0.0;
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          if (!LU && lane == c) yi = yi / row[c];
          const double yc = __shfl_sync(0xffffffffu, yi, c);
          if (lane > c) yi = fma(-row[c], yc, yi);
        }
        if (lane < jb) y[j + lane] = yi;
      }
      __syncthreads();
      for (int r = j + jb + tid; r < n; r += BT) {
        double t = y[r];
#pragma unroll 8
        for (int c = 0; c < jb; ++c) t = fma(-A[r + (int64_t)(j + c) * ld], y[j + c], t);
        y[r] = t;
      }
      __syncthreads();
    }
    // backward
    const int last = ((n - 1) / 32) * 32;
    for (int j = last; j >= 0; j -= 32) {
      const int jb = min(32, n - j);
      if (!LU) {
        // y_j -= L(j+jb.., j..j+jb)^T y(j+jb..): warp w takes columns w, w+8, w+16, w+24
        // together (four independent loads per row), lanes stride over the rows
        {
          double t[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 2
          for (int r = j + jb + lane; r < n; r += 32) {
            const double yr = y[r];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int c = warp + 8 * u;
              if (c < jb) t[u] = fma(A[r + (int64_t)(j + c) * ld], yr, t[u]);
            }
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t[u] += __shfl_xor_sync(0xffffffffu, t[u], o);
            const int c = warp + 8 * u;
            if (lane == 0 && c < jb) y[j + c] -= t[u];
          }
        }
        __syncthreads();
        if (warp == 0) {
          // L11^T x = y: lane i holds column i of L11 (L(k, i) for k >= i)
          double col[32];
#pragma unroll
          for (int k = 0; k < 32; ++k)
            col[k] = (lane < jb && k >= lane && k < jb) ? A[(j + k) + (int64_t)(j + lane) * ld] : 0.0;
          double xi = lane < jb ? y[j + lane] : 0.0;
#pragma unroll
          for (int c = 31; c >= 0; --c) {
            const double lcc = __shfl_sync(0xffffffffu, col[c], c);
            if (lane == c && c < jb) xi = xi / lcc;
            const double xc = __shfl_sync(0xffffffffu, xi, c);
            if (lane < c && c < jb) xi = fma(-col[c], xc, xi);
          }
          if (lane < jb) y[j + lane] = xi;
        }
        __syncthreads();
      } else {
        if (warp == 0) {
          // U11 x = y: lane i holds row i of U11 (U(i, c) for c >= i)
          double row[32];
#pragma unroll
          for (int c = 0; c < 32; ++c)
            row[c] = (lane < jb && c >= lane && c < jb) ? A[(j + lane) + (int64_t)(j + c) * ld] : 0.0;
          double xi = lane < jb ? y[j + lane] : 0.0;
#pragma unroll
          for (int c = 31; c >= 0; --c) {
            if (lane == c && c < jb) xi = xi / row[c];
            const double xc = __shfl_sync(0xffffffffu, xi, c);
            if (lane < c && c < jb) xi = fma(-row[c], xc, xi);
          }
          if (lane < jb) y[j + lane] = xi;
        }
        __syncthreads();
        // y(0..j) -= U(0..j, j..j+jb) x_j
        for (int r = tid; r < j; r += BT) {
          double t = y[r];
#pragma unroll 8
          for (int c = 0; c < jb; ++c) t = fma(-A[r + (int64_t)(j + c) * ld], y[j + c], t);
          y[r] = t;
        }
        __syncthreads();
      }
    }
    for (int r = tid; r < n; r += BT) b[r] = y[r];
    __syncthreads();
  }
}

template <int KIND, int NB, int MINB>
__global__ void __launch_bounds__(BT, MINB) batch_kernel(BatchParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<NB> &s = *reinterpret_cast<Smem<NB> *>(smem_raw);
  double *ut = p.ut + (size_t)blockIdx.x * NB * MAXN;
  for (;;) {
    if (threadIdx.x == 0) s.idx = atomicAdd(p.counter, 1);
    __syncthreads();
    const int q = s.idx;
    __syncthreads();
    if (q >= p.count) break;
    const int m = p.order[q];
    const int n = p.n[m];
    double *A = p.A[m];
    const int64_t ld = p.lda[m];
    int info;
    if (KIND == MO_BATCH_CHOL) info = chol_matrix<NB>(s, A, ld, n);
    else info = lu_matrix<NB>(s, A, ld, n, p.piv[m], ut);
    if (threadIdx.x == 0) p.info[m] = info;
    const bool solve = p.B != nullptr && (KIND == MO_BATCH_LU || info == 0);
    if (solve) solve_matrix<KIND == MO_BATCH_LU, NB>(s, A, ld, n, p.B[m], p.ldb[m], p.nrhs);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------
// host side: kernel configurations, schedule groups, CUDA graph, autotuner
// ---------------------------------------------------------------------------------------

constexpr int NBUCKETS = MO_BATCH_BUCKETS;
constexpr int NCFG = 2;
const int kBucketMax[NBUCKETS] = {64, 128, 256, MAXN};

struct KernelCfg {
  int nb, minb;
  const void *fn;
  size_t smem;
};

template <int KIND, int NB, int MINB>
KernelCfg make_cfg() {
  return KernelCfg{NB, MINB, (const void *)batch_kernel<KIND, NB, MINB>, sizeof(Smem<NB>)};
}

// configuration c of a kind: 0 = panel 32, 1 = panel 16 (two CTAs per SM)
KernelCfg kernel_cfg(int kind, int c) {
  if (kind == MO_BATCH_CHOL) return c == 0 ? make_cfg<MO_BATCH_CHOL, 32, 2>() : make_cfg<MO_BATCH_CHOL, 16, 2>();
  return c == 0 ? make_cfg<MO_BATCH_LU, 32, 1>() : make_cfg<MO_BATCH_LU, 16, 2>();
}

int bucket_of(int n) {
  for (int b = 0; b < NBUCKETS; ++b)
    if (n <= kBucketMax[b]) return b;
  return NBUCKETS - 1;
}

double work_of(int kind, int n) { return (kind == MO_BATCH_LU ? 2.0 : 1.0) * n * (double)n * n / 3.0; }

int prepare_kernel(const KernelCfg &k, int device, int *occ) {
  MO_CUDA_TRY(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem));
  MO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k.fn, BT, k.smem));
  (void)device;
  if (*occ < 1) return MO_ENOKERNEL;
  return MO_OK;
}

}  // namespace
}  // namespace mo

struct mo_batch {
  mo_ctx *ctx = nullptr;
  int kind = 0, count = 0, nrhs = 0;
  std::vector<int> n;          // orders (host copy)
  int cfg[MO_BATCH_BUCKETS] = {0, 0, 0, 0};
  int *d_n = nullptr;          // orders
  int *d_order = nullptr;      // queues of all groups, back to back
  int *d_counters = nullptr;   // one per group
  double *d_ut = nullptr;      // LU scratch (NB x MAXN doubles per CTA)
  size_t ut_bytes = 0;
  struct Group {
    int cfg, count, offset, grid;
    size_t ut_off;  // doubles
  };
  std::vector<Group> groups;
  double flops = 0.0, bytes = 0.0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<cudaGraphNode_t> knodes;
  std::vector<mo::BatchParams> params;
  bool dirty = true;
};

namespace mo {
namespace {

void release_graph(mo_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->knodes.clear();
}

// groups from the per-bucket configuration: one queue per configuration in use, ordered
// by decreasing n, each with a full persistent grid
int build_groups(mo_batch *b) {
  mo_ctx *ctx = b->ctx;
  std::vector<int> idx[NCFG];
  double work[NCFG] = {0.0, 0.0};
  for (int i = 0; i < b->count; ++i) {
    const int c = b->cfg[bucket_of(b->n[i])];
    idx[c].push_back(i);
    work[c] += work_of(b->kind, b->n[i]);
  }
  (void)work;
  std::vector<int> order;
  b->groups.clear();
  size_t ut_total = 0;
  for (int c = 0; c < NCFG; ++c) {
    if (idx[c].empty()) continue;
    std::stable_sort(idx[c].begin(), idx[c].end(),
                     [&](int x, int y) { return b->n[x] > b->n[y]; });
    const KernelCfg k = kernel_cfg(b->kind, c);
    int occ = 0;
    int rc = prepare_kernel(k, ctx->device, &occ);
    if (rc) return rc;
    const int grid = std::max(1, std::min(ctx->sms * occ, (int)idx[c].size()));
    mo_batch::Group g{c, (int)idx[c].size(), (int)order.size(), grid, ut_total};
    ut_total += (size_t)grid * k.nb * MAXN;
    b->groups.push_back(g);
    order.insert(order.end(), idx[c].begin(), idx[c].end());
  }
  // the group holding the largest matrices runs first
  std::stable_sort(b->groups.begin(), b->groups.end(), [&](const mo_batch::Group &x,
                                                          const mo_batch::Group &y) {
    return b->n[order[x.offset]] > b->n[order[y.offset]];
  });
  if (b->d_order) cudaFree(b->d_order);
  if (b->d_counters) cudaFree(b->d_counters);
  b->d_order = nullptr;
  b->d_counters = nullptr;
  MO_CUDA_TRY(cudaMalloc(&b->d_order, sizeof(int) * std::max<size_t>(1, order.size())));
  MO_CUDA_TRY(cudaMalloc(&b->d_counters, sizeof(int) * NCFG));
  MO_CUDA_TRY(cudaMemcpy(b->d_order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));
  const size_t need = b->kind == MO_BATCH_LU ? ut_total * sizeof(double) : 0;
  if (need > b->ut_bytes) {
    if (b->d_ut) cudaFree(b->d_ut);
    b->d_ut = nullptr;
    b->ut_bytes = 0;
    MO_CUDA_TRY(cudaMalloc(&b->d_ut, need));
    b->ut_bytes = need;
  }
  return MO_OK;
}

BatchParams group_params(mo_batch *b, const mo_batch::Group &g, double *const *A,
                         const int64_t *lda, double *const *B, const int64_t *ldb,
                         int64_t *const *piv, int *info) {
  BatchParams p;
  p.count = g.count;
  p.order = b->d_order + g.offset;
  p.counter = b->d_counters + (&g - b->groups.data());
  p.n = b->d_n;
  p.A = A;
  p.lda = lda;
  p.B = B;
  p.ldb = ldb;
  p.nrhs = b->nrhs;
  p.piv = piv;
  p.info = info;
  p.ut = b->d_ut ? b->d_ut + g.ut_off : nullptr;
  return p;
}

bool same_args(const BatchParams &x, const BatchParams &y) {
  return x.A == y.A && x.lda == y.lda && x.B == y.B && x.ldb == y.ldb && x.piv == y.piv &&
         x.info == y.info;
}

// graph: memset(queue counters) -> one persistent kernel node per group, in sequence
// (each group's kernel fills the whole GPU; groups end with their smallest matrices)
int build_graph(mo_batch *b, const std::vector<BatchParams> &params) {
  release_graph(b);
  MO_CUDA_TRY(cudaGraphCreate(&b->graph, 0));
  cudaMemsetParams ms = {};
  ms.dst = b->d_counters;
  ms.value = 0;
  ms.elementSize = sizeof(int);
  ms.width = NCFG;
  ms.height = 1;
  ms.pitch = 0;
  cudaGraphNode_t mnode;
  MO_CUDA_TRY(cudaGraphAddMemsetNode(&mnode, b->graph, nullptr, 0, &ms));
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    const KernelCfg k = kernel_cfg(b->kind, b->groups[gi].cfg);
    cudaKernelNodeParams kp = {};
    kp.func = const_cast<void *>(k.fn);
    kp.gridDim = dim3(b->groups[gi].grid);
    kp.blockDim = dim3(BT);
    kp.sharedMemBytes = (unsigned)k.smem;
    void *args[] = {const_cast<BatchParams *>(&params[gi])};
    kp.kernelParams = args;
    cudaGraphNode_t kn;
    cudaGraphNode_t dep = b->knodes.empty() ? mnode : b->knodes.back();
    MO_CUDA_TRY(cudaGraphAddKernelNode(&kn, b->graph, &dep, 1, &kp));
    b->knodes.push_back(kn);
  }
  MO_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->params = params;
  b->dirty = false;
  return MO_OK;
}

int update_graph(mo_batch *b, const std::vector<BatchParams> &params) {
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    const KernelCfg k = kernel_cfg(b->kind, b->groups[gi].cfg);
    cudaKernelNodeParams kp = {};
    kp.func = const_cast<void *>(k.fn);
    kp.gridDim = dim3(b->groups[gi].grid);
    kp.blockDim = dim3(BT);
    kp.sharedMemBytes = (unsigned)k.smem;
    void *args[] = {const_cast<BatchParams *>(&params[gi])};
    kp.kernelParams = args;
    MO_CUDA_TRY(cudaGraphExecKernelNodeSetParams(b->exec, b->knodes[gi], &kp));
  }
  b->params = params;
  return MO_OK;
}

int batch_run(mo_batch *b, double *const *A, const int64_t *lda, double *const *B,
              const int64_t *ldb, int64_t *const *piv, int *info) {
  mo_ctx *ctx = b->ctx;
  int rc;
  if (b->dirty || b->groups.empty()) {
    if ((rc = build_groups(b))) return rc;
    release_graph(b);
  }
  std::vector<BatchParams> params;
  for (const auto &g : b->groups) params.push_back(group_params(b, g, A, lda, B, ldb, piv, info));
  if (!b->exec) {
    if ((rc = build_graph(b, params))) return rc;
  } else {
    bool same = true;
    for (size_t i = 0; i < params.size(); ++i) same = same && same_args(params[i], b->params[i]);
    if (!same && (rc = update_graph(b, params))) return rc;
  }
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_BATCH);
  MO_CUDA_TRY(cudaGraphLaunch(b->exec, ctx->stream));
  prof_end(ctx, ps, b->flops, b->bytes);
  return MO_OK;
}

// synthetic matrices for the autotuner: uniform[-1, 1] entries from a hash of (matrix,
// row, column); symmetric with n added to the diagonal (positive definite) for Cholesky
__global__ void tune_fill_kernel(double *buf, const int64_t *off, const int *n, int kind) {
  const int m = blockIdx.y;
  const int nm = n[m];
  double *A = buf + off[m];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)nm * nm;
       e += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(e % nm), j = (int)(e / nm);
    if (kind == MO_BATCH_CHOL && i < j) {
      const int t = i;
      i = j;
      j = t;
    }
    uint64_t h = ((uint64_t)m * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)i << 32 | (uint32_t)j);
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    double v = (double)(h >> 11) * 0x1.0p-53 * 2.0 - 1.0;
    if (kind == MO_BATCH_CHOL && i == j) v += nm;
    A[e] = v;
  }
}

// Time every configuration on a sample of each size bucket of the plan (synthetic
// matrices of the plan's own orders) and keep the fastest per bucket.
int batch_tune(mo_batch *b, int reps, double *ms_out) {
  mo_ctx *ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  reps = std::max(1, reps);
  for (int bk = 0; bk < NBUCKETS; ++bk) {
    std::vector<int> sizes;
    for (int i = 0; i < b->count; ++i)
      if (bucket_of(b->n[i]) == bk) sizes.push_back(b->n[i]);
    if (sizes.empty()) continue;
    std::sort(sizes.begin(), sizes.end(), [](int x, int y) { return x > y; });
    const int S = std::min<int>((int)sizes.size(), 4 * ctx->sms);
    std::vector<int> ns(S);
    for (int s = 0; s < S; ++s) ns[s] = sizes[(size_t)s * sizes.size() / S];
    std::vector<int64_t> off(S), lds(S), boff(S);
    int64_t tot = 0, btot = 0;
    for (int s = 0; s < S; ++s) {
      off[s] = tot;
      lds[s] = ns[s];
      tot += (int64_t)ns[s] * ns[s];
      boff[s] = btot;
      btot += (int64_t)ns[s] * std::max(1, b->nrhs);
    }
    std::vector<int> order(S);
    for (int s = 0; s < S; ++s) order[s] = s;
    // device buffers: pristine + work matrices, B, pivots, pointer arrays, scratch
    size_t ut_need = 0;
    int occs[NCFG];
    for (int c = 0; c < NCFG; ++c) {
      const KernelCfg k = kernel_cfg(b->kind, c);
      int rc = prepare_kernel(k, ctx->device, &occs[c]);
      if (rc) return rc;
      ut_need = std::max(ut_need, (size_t)std::min(S, ctx->sms * occs[c]) * k.nb * MAXN);
    }
    char *mem = nullptr;
    const size_t bytes = 2 * tot * 8 + btot * 8 + tot * 8 /*piv*/ + S * (3 * 8 + 8 + 8 + 4 + 4 + 4) +
                         ut_need * 8 + 4096;
    MO_CUDA_TRY(cudaMalloc(&mem, bytes));
    int rc = MO_OK;
    do {
      char *p = mem;
      auto take = [&](size_t nb) {
        char *r = p;
        p += (nb + 255) & ~(size_t)255;
        return r;
      };
      double *pristine = (double *)take(tot * 8), *work = (double *)take(tot * 8);
      double *Bbuf = (double *)take(btot * 8);
      int64_t *pivbuf = (int64_t *)take(tot * 8);
      double **dA = (double **)take(S * 8), **dB = (double **)take(S * 8);
      int64_t **dP = (int64_t **)take(S * 8);
      int64_t *dlda = (int64_t *)take(S * 8), *doff = (int64_t *)take(S * 8);
      int *dn = (int *)take(S * 4), *dorder = (int *)take(S * 4), *dinfo = (int *)take(S * 4);
      int *dcounter = (int *)take(4);
      double *dut = (double *)take(ut_need * 8);
      std::vector<double *> hA(S), hB(S);
      std::vector<int64_t *> hP(S);
      for (int s = 0; s < S; ++s) {
        hA[s] = work + off[s];
        hB[s] = Bbuf + boff[s];
        hP[s] = pivbuf + off[s];
      }
      if (cudaMemcpy(dA, hA.data(), S * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(dB, hB.data(), S * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(dP, hP.data(), S * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(dlda, lds.data(), S * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(doff, off.data(), S * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(dn, ns.data(), S * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(dorder, order.data(), S * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = MO_ECUDA;
        break;
      }
      tune_fill_kernel<<<dim3(16, S), 256, 0, st>>>(pristine, doff, dn, b->kind);
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      double best = INFINITY;
      int best_c = b->cfg[bk];
      for (int c = 0; c < NCFG && !rc; ++c) {
        const KernelCfg k = kernel_cfg(b->kind, c);
        BatchParams prm;
        prm.count = S;
        prm.order = dorder;
        prm.counter = dcounter;
        prm.n = dn;
        prm.A = dA;
        prm.lda = dlda;
        prm.B = b->nrhs > 0 ? dB : nullptr;
        prm.ldb = dlda;
        prm.nrhs = b->nrhs;
        prm.piv = dP;
        prm.info = dinfo;
        prm.ut = dut;
        const int grid = std::min(S, ctx->sms * occs[c]);
        double t_min = INFINITY;
        for (int r = 0; r <= reps && !rc; ++r) {
          cudaMemcpyAsync(work, pristine, tot * 8, cudaMemcpyDeviceToDevice, st);
          cudaMemsetAsync(Bbuf, 0, btot * 8, st);
          cudaMemsetAsync(dcounter, 0, 4, st);
          cudaEventRecord(e0, st);
          void *args[] = {&prm};
          if (cudaLaunchKernel(k.fn, dim3(grid), dim3(BT), args, k.smem, st) != cudaSuccess) {
            rc = MO_ECUDA;
            break;
          }
          cudaEventRecord(e1, st);
          if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = MO_ECUDA;
            break;
          }
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e0, e1);
          if (r > 0) t_min = std::min(t_min, (double)ms);
        }
        if (ms_out) ms_out[bk * NCFG + c] = t_min;
        if (t_min < best) {
          best = t_min;
          best_c = c;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      b->cfg[bk] = best_c;
    } while (false);
    cudaStreamSynchronize(st);
    cudaFree(mem);
    if (rc) return rc;
  }
  b->dirty = true;
  return MO_OK;
}

}  // namespace
}  // namespace mo

using namespace mo;

extern "C" int mo_batch_create(mo_ctx *ctx, int kind, int count, const int32_t *n, int nrhs,
                               mo_batch **out) {
  int rc = enter(ctx);
  if (rc) return rc;
  if (!out || count < 0 || nrhs < 0 || (count > 0 && !n)) return MO_EINVAL;
  if (kind != MO_BATCH_CHOL && kind != MO_BATCH_LU) return MO_EINVAL;
  for (int i = 0; i < count; ++i)
    if (n[i] < 1 || n[i] > MO_BATCH_MAX_N) return MO_EBATCHN;
  mo_batch *b = new mo_batch;
  b->ctx = ctx;
  b->kind = kind;
  b->count = count;
  b->nrhs = nrhs;
  b->n.assign(n, n + count);
  for (int i = 0; i < count; ++i) {
    const double ni = n[i];
    b->flops += work_of(kind, n[i]) + (nrhs ? 2.0 * ni * ni * nrhs : 0.0);
    b->bytes += 16.0 * ni * ni + 16.0 * ni * nrhs;
  }
  // default schedule: panel 16 for n <= 64, panel 32 above (the autotuner may change it)
  b->cfg[0] = 1;
  if (cudaMalloc(&b->d_n, sizeof(int) * std::max(1, count)) != cudaSuccess ||
      (count > 0 && cudaMemcpy(b->d_n, n, sizeof(int) * count, cudaMemcpyHostToDevice) != cudaSuccess)) {
    if (b->d_n) cudaFree(b->d_n);
    delete b;
    return MO_ENOMEM;
  }
  *out = b;
  return MO_OK;
}

extern "C" int mo_batch_destroy(mo_batch *b) {
  if (!b) return MO_EINVAL;
  enter(b->ctx);
  cudaStreamSynchronize(b->ctx->stream);
  release_graph(b);
  if (b->d_n) cudaFree(b->d_n);
  if (b->d_order) cudaFree(b->d_order);
  if (b->d_counters) cudaFree(b->d_counters);
  if (b->d_ut) cudaFree(b->d_ut);
  delete b;
  return MO_OK;
}

extern "C" int mo_batch_run(mo_batch *b, double *const *A, const int64_t *lda, double *const *B,
                            const int64_t *ldb, int64_t *const *piv, int *info) {
  if (!b) return MO_EINVAL;
  int rc = enter(b->ctx);
  if (rc) return rc;
  if (b->count == 0) return MO_OK;
  if (!A || !lda || !info || (b->kind == MO_BATCH_LU && !piv)) return MO_EINVAL;
  if (B && !ldb) return MO_EINVAL;
  if (b->nrhs == 0) B = nullptr;
  return batch_run(b, A, lda, B, B ? ldb : nullptr, piv, info);
}

extern "C" int mo_batch_tune(mo_batch *b, int reps, double *ms) {
  if (!b) return MO_EINVAL;
  int rc = enter(b->ctx);
  if (rc) return rc;
  if (ms)
    for (int i = 0; i < MO_BATCH_BUCKETS * NCFG; ++i) ms[i] = -1.0;
  return batch_tune(b, reps, ms);
}

extern "C" int mo_batch_schedule(mo_batch *b, int *cfg, int set) {
  if (!b || !cfg) return MO_EINVAL;
  if (set) {
    for (int i = 0; i < MO_BATCH_BUCKETS; ++i)
      if (cfg[i] < 0 || cfg[i] >= NCFG) return MO_EINVAL;
    for (int i = 0; i < MO_BATCH_BUCKETS; ++i) b->cfg[i] = cfg[i];
    b->dirty = true;
  } else {
    for (int i = 0; i < MO_BATCH_BUCKETS; ++i) cfg[i] = b->cfg[i];
  }
  return MO_OK;
}
