// Symmetric indefinite LDL^T factorizations and solves (ldlnp.go, ldl.go, ldlbk.go,
// ldlbks.go): DecomposeLDLnoPiv / SolveLDLnoPiv (no interchanges), DecomposeLDL /
// SolveLDL (1 x 1 pivots, the largest remaining diagonal entry, interchanges applied to
// whole rows) and DecomposeBK / SolveBK (Bunch-Kaufman 1 x 1 and 2 x 2 pivots, LAPACK
// DSYTF2 / DSYTRS, interchanges inside the part not yet factored).
//
// Device form: one cooperative kernel per factorization runs the reference's unblocked
// right-looking sweep over the whole matrix in place.  Per column: the pivot search as
// per-CTA partial maxima summed in a fixed order after a bounded grid barrier (every CTA
// reaches the same decision), the symmetric interchange spread over all threads, and the
// rank-1 or rank-2 update of the lower triangle left, one warp per column.  The column's
// multipliers are written one step later by CTA 0 (the update still reads the unscaled
// column).  The element updates keep the reference's operation order (a_ij + x_i (alpha
// x_j) with separate multiply and add), so the pivot decisions see the same values.
// UPPER storage is handled by the same code on the index-reversed matrix (element (i, j)
// at (n-1-i, n-1-j)): the reference's UPPER sweeps run from the bottom-right corner and
// are the LOWER sweeps of the reversed matrix, with ties in the pivot search going to the
// smallest ORIGINAL index (the reference's IAMax, calgo/dvec_util.c:164).
//
// Solves: SolveLDLnoPiv / SolveLDL as the reference composes them (row interchanges, two
// unit-triangular solves on the TRSM engine, the diagonal scaling); SolveBK by a
// kernel that follows ldlbks.go's two sweeps (interchange, rank-1 / rank-2
// update of the rows of B below, 1 x 1 / 2 x 2 diagonal solve; then the transposed sweep
// back up), on the reversed problem for UPPER.
#include <algorithm>

#include "context.cuh"

namespace mo {
namespace {

constexpr int kLdlThreads = 256;
constexpr double kBkAlpha = 0.6403882032022075;  // (1 + sqrt(17)) / 8, ldlbk.go:16

enum LdlMode : int { kLdlNoPiv = 0, kLdlDiag = 1, kLdlBK = 2 };

// the working lower triangle: element (i, j), i >= j, of A or of the index-reversed A
struct SymView {
  double *d;
  int64_t ld;
  int n;
  int rev;
  __device__ __forceinline__ double *at(int i, int j) const {
    return rev ? d + (n - 1 - i) + (int64_t)(n - 1 - j) * ld : d + i + (int64_t)j * ld;
  }
};

struct LdlScratch {
  double *val;         // [2][grid] per-CTA partial maxima
  int *idx;            // [2][grid] their indices
  unsigned *bar;       // grid-barrier arrival counter (zeroed before the launch)
  int *abort_flag;
};

__device__ bool ldl_grid_barrier(unsigned *counter, unsigned target, int *status,
                                 int *abort_flag) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
    int ok = 1;
    for (unsigned i = 0;; ++i) {
      if (*(volatile unsigned *)counter >= target) break;
      if (*(volatile int *)abort_flag) {
        ok = 0;
        break;
      }
      if (i > MO_SPIN_LIMIT) {
        set_status(status, MO_EDEVTIMEOUT);
        atomicExch(abort_flag, 1);
        ok = 0;
        break;
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Loads of the matrix inside the sweep bypass L1: other CTAs wrote it since this SM may
// last have cached the line (only L2 is coherent across SMs)
__device__ __forceinline__ double ldg(const double *p) { return __ldcg(p); }

// (value, index) order of the pivot searches: the larger value wins; equal values go to
// the smaller original index (smaller i directly, larger i on the reversed matrix); NaN
// never wins (the reference's strict comparisons skip it)
__device__ __forceinline__ bool ldl_better(double v, int i, double bv, int bi, int rev) {
  if (!(v >= 0.0)) return false;
  if (v > bv) return true;
  return v == bv && (rev ? i > bi : i < bi);
}

// CTA-wide (value, index) maximum into (s_v, s_i) of thread 0's view; every thread returns
// with the CTA's result after the final barrier
__device__ void ldl_cta_max(double v, int i, int rev, double *s_v, int *s_i) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_down_sync(0xffffffffu, v, o);
    const int i2 = __shfl_down_sync(0xffffffffu, i, o);
    if (ldl_better(v2, i2, v, i, rev)) {
      v = v2;
      i = i2;
    }
  }
  if (lane == 0) {
    s_v[warp] = v;
    s_i[warp] = i;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bv = s_v[0];
    int bi = s_i[0];
    for (int w = 1; w < kLdlThreads / 32; ++w)
      if (ldl_better(s_v[w], s_i[w], bv, bi, rev)) {
        bv = s_v[w];
        bi = s_i[w];
      }
    s_v[0] = bv;
    s_i[0] = bi;
  }
  __syncthreads();
}

// every CTA's partials of the current search, reduced in CTA order (same result in all)
__device__ void ldl_grid_max(const LdlScratch &sc, int par, int rev, double *s_v, int *s_i,
                             double *out_v, int *out_i) {
  double v = -1.0;
  int i = 0x7fffffff;
  if (rev) i = -1;
  for (int g = threadIdx.x; g < (int)gridDim.x; g += kLdlThreads) {
    const double gv = __ldcg(&sc.val[par * gridDim.x + g]);
    const int gi = __ldcg(&sc.idx[par * gridDim.x + g]);
    if (ldl_better(gv, gi, v, i, rev)) {
      v = gv;
      i = gi;
    }
  }
  ldl_cta_max(v, i, rev, s_v, s_i);
  *out_v = s_v[0];
  *out_i = s_i[0];
  __syncthreads();
}

// The unblocked right-looking sweep (MODE: no interchanges, diagonal pivoting or
// Bunch-Kaufman) over the lower triangle of A (the reversed matrix for UPPER storage).
// ipiv in the reference's encoding at ORIGINAL positions: 1-based partner (DecomposeLDL: 0
// for none; DecomposeBK: the row itself for none), negative for both rows of a 2 x 2
// block.  info: k + 1 for a zero diagonal pivot at step k (DecomposeLDL only).
template <int MODE>
__global__ void __launch_bounds__(kLdlThreads, 1)
    ldl_kernel(SymView A, int64_t *ipiv, LdlScratch sc, int *status, int *info) {
  __shared__ double s_v[kLdlThreads / 32];
  __shared__ int s_i[kLdlThreads / 32];
  const int n = A.n, G = gridDim.x, tid = threadIdx.x, cta = blockIdx.x;
  const int gt = cta * kLdlThreads + tid, GT = G * kLdlThreads;
  const int lane = tid & 31, gw = cta * (kLdlThreads / 32) + (tid >> 5);
  const int GW = G * (kLdlThreads / 32);
  const int rev = A.rev;
  unsigned bars = 0;
  int searches = 0;
  // multipliers of the previous step, written by CTA 0 after the next barrier
  int pk = -1, pnp = 0;
  double p_a11 = 1.0, p_i00 = 0.0, p_i11 = 0.0, p_scale = 0.0;
  auto orig = [&](int i) { return rev ? n - 1 - i : i; };
  auto barrier = [&]() -> bool {
    ++bars;
    return ldl_grid_barrier(sc.bar, bars * (unsigned)G, status, sc.abort_flag);
  };
  auto flush = [&]() {
    if (cta == 0 && pk >= 0) {
      for (int i = pk + pnp + tid; i < n; i += kLdlThreads) {
        if (pnp == 1) {
          double *x = A.at(i, pk);
          *x = ldg(x) / p_a11;  // InvScale (true division)
        } else {
          double *c0 = A.at(i, pk), *c1 = A.at(i, pk + 1);
          const double v0 = ldg(c0), v1 = ldg(c1);
          *c0 = __dmul_rn(p_scale, __dadd_rn(__dmul_rn(v0, p_i00), -v1));
          *c1 = __dmul_rn(p_scale, __dadd_rn(-v0, __dmul_rn(v1, p_i11)));
        }
      }
    }
    pk = -1;
  };
  // one grid-wide (value, index) maximum: each thread offers its candidates through `f`
  auto grid_search = [&](auto &&f, double *mv, int *mi) -> bool {
    double v = -1.0;
    int bi = rev ? -1 : 0x7fffffff;
    f(v, bi);
    ldl_cta_max(v, bi, rev, s_v, s_i);
    const int par = searches & 1;
    ++searches;
    if (tid == 0) {
      sc.val[par * G + cta] = s_v[0];
      sc.idx[par * G + cta] = s_i[0];
    }
    if (!barrier()) return false;
    ldl_grid_max(sc, par, rev, s_v, s_i, mv, mi);
    return true;
  };

  int k = 0;
  while (k < n) {
    if (k > 0 && !barrier()) return;  // the previous update is complete
    flush();
    int np = 1, r = 0;  // pivot block size; partner offset below k (0: none)
    if (MODE == kLdlDiag) {
      double mv;
      int mi;
      if (!grid_search(
              [&](double &v, int &bi) {
                for (int i = k + gt; i < n; i += GT) {
                  const double a = fabs(ldg(A.at(i, i)));
                  if (ldl_better(a, i, v, bi, rev)) {
                    v = a;
                    bi = i;
                  }
                }
              },
              &mv, &mi))
        return;
      r = (mv >= 0.0 && mi >= k && mi < n) ? mi - k : 0;
      if (rev && !(mv >= 0.0)) r = n - 1 - k;  // all NaN: the reference's IAMax gives 0
      if (cta == 0 && tid == 0) ipiv[orig(k)] = r > 0 ? orig(k + r) + 1 : 0;
      if (r > 0) {
        // rows / columns k and p of the whole lower triangle (pivot.go:145-162)
        const int p = k + r, n1 = k, n2 = r - 1, n3 = n - p - 1;
        for (int t = gt; t < n1 + n2 + n3 + 1; t += GT) {
          double *x, *y;
          if (t < n1) {
            x = A.at(k, t);
            y = A.at(p, t);
          } else if (t < n1 + n2) {
            const int u = k + 1 + (t - n1);
            x = A.at(u, k);
            y = A.at(p, u);
          } else if (t < n1 + n2 + n3) {
            const int i = p + 1 + (t - n1 - n2);
            x = A.at(i, k);
            y = A.at(i, p);
          } else {
            x = A.at(k, k);
            y = A.at(p, p);
          }
          const double tv = ldg(x);
          *x = ldg(y);
          *y = tv;
        }
        if (!barrier()) return;
      }
    } else if (MODE == kLdlBK && k < n - 1) {
      double rmax;
      int ri;
      if (!grid_search(
              [&](double &v, int &bi) {
                for (int i = k + 1 + gt; i < n; i += GT) {
                  const double a = fabs(ldg(A.at(i, k)));
                  if (ldl_better(a, i, v, bi, rev)) {
                    v = a;
                    bi = i;
                  }
                }
              },
              &rmax, &ri))
        return;
      if (!(rmax >= 0.0)) {  // all NaN: IAMax gives the first row below
        ri = rev ? n - 1 : k + 1;
        rmax = fabs(ldg(A.at(ri, k)));
      }
      const double amax = fabs(ldg(A.at(k, k)));
      if (!(amax >= kBkAlpha * rmax)) {
        // |a(ri, ri)| is read before the next barrier: once every CTA has passed it, the
        // first ones may already be interchanging (ri, ri) with another diagonal entry
        const double arr = fabs(ldg(A.at(ri, ri)));
        double qmax;
        int qi;
        if (!grid_search(
                [&](double &v, int &bi) {
                  // row ri left of its diagonal (from column k) and column ri below it
                  const int m1 = ri - k, m2 = n - ri - 1;
                  for (int t = gt; t < m1 + m2; t += GT) {
                    const double a = t < m1 ? fabs(ldg(A.at(ri, k + t))) : fabs(ldg(A.at(ri + 1 + t - m1, ri)));
                    const int it = t < m1 ? k + t : ri + 1 + t - m1;
                    if (ldl_better(a, it, v, bi, rev)) {
                      v = a;
                      bi = it;
                    }
                  }
                },
                &qmax, &qi))
          return;
        if (!(qmax >= 0.0)) qmax = 0.0;
        if (!(amax >= kBkAlpha * rmax * (rmax / qmax))) {
          r = ri - k;
          np = arr >= kBkAlpha * qmax ? 1 : 2;
        }
      }
      if (cta == 0 && tid == 0) {
        const int64_t pv = orig(k + r) + 1;
        if (np == 1) {
          ipiv[orig(k)] = pv;
        } else {
          ipiv[orig(k)] = -pv;
          ipiv[orig(k + 1)] = -pv;
        }
      }
      if (r != 0 && r != np - 1) {
        // ldlbk.go:48-76 within the part left: rows / columns src = k + np - 1 and dst
        const int src = k + np - 1, dst = k + r;
        const int n2 = dst - src - 1, n3 = n - dst - 1, extra = np == 2 ? 1 : 0;
        for (int t = gt; t < n2 + n3 + 1 + extra; t += GT) {
          double *x, *y;
          if (t < n2) {
            x = A.at(src + 1 + t, src);
            y = A.at(dst, src + 1 + t);
          } else if (t < n2 + n3) {
            const int i = dst + 1 + (t - n2);
            x = A.at(i, src);
            y = A.at(i, dst);
          } else if (t == n2 + n3) {
            x = A.at(src, src);
            y = A.at(dst, dst);
          } else {
            x = A.at(k + 1, k);
            y = A.at(dst, k);
          }
          const double tv = ldg(x);
          *x = ldg(y);
          *y = tv;
        }
        if (!barrier()) return;
      }
    } else if (MODE == kLdlBK) {
      if (cta == 0 && tid == 0) ipiv[orig(k)] = orig(k) + 1;
    }
    if (np == 1) {
      const double a11 = ldg(A.at(k, k));
      if (MODE == kLdlDiag && a11 == 0.0) {
        if (cta == 0 && tid == 0) *info = k + 1;
        return;
      }
      const double alpha = -1.0 / a11;
      // A22 += a21 (alpha a21^T), lower triangle: a_ij + x_i (alpha x_j)
      for (int j = k + 1 + gw; j < n; j += GW) {
        const double cf = __dmul_rn(alpha, ldg(A.at(j, k)));
        for (int i = j + lane; i < n; i += 32) {
          double *a = A.at(i, j);
          *a = __dadd_rn(ldg(a), __dmul_rn(ldg(A.at(i, k)), cf));
        }
      }
      pk = k;
      pnp = 1;
      p_a11 = a11;
    } else {
      const double a = ldg(A.at(k, k)), b = ldg(A.at(k + 1, k)), d = ldg(A.at(k + 1, k + 1));
      const double i00 = d / b, i11 = a / b;
      double scale = 1.0 / __dadd_rn(__dmul_rn(a / b, d / b), -1.0);
      scale /= b;
      // A22 -= (a21 E^-1) a21^T with the unscaled a21 (ldlbk.go:289-313)
      for (int j = k + 2 + gw; j < n; j += GW) {
        const double cj0 = ldg(A.at(j, k)), cj1 = ldg(A.at(j, k + 1));
        for (int i = j + lane; i < n; i += 32) {
          const double ci0 = ldg(A.at(i, k)), ci1 = ldg(A.at(i, k + 1));
          const double l0 = __dmul_rn(scale, __dadd_rn(__dmul_rn(ci0, i00), -ci1));
          const double l1 = __dmul_rn(scale, __dadd_rn(-ci0, __dmul_rn(ci1, i11)));
          double *e = A.at(i, j);
          *e = __dadd_rn(ldg(e), -1.0 * __dadd_rn(__dmul_rn(l0, cj0), __dmul_rn(l1, cj1)));
        }
      }
      pk = k;
      pnp = 2;
      p_i00 = i00;
      p_i11 = i11;
      p_scale = scale;
    }
    k += np;
  }
  if (!barrier()) return;
  flush();
}

constexpr int kBkSolveThreads = 256;

// sum over the CTA in a fixed order (every thread gets the result)
__device__ double bk_block_sum(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < kBkSolveThreads / 32; ++w) t += red[w];
  return t;
}

// ldlbks.go:15-156 (unblkSolveBKLower, both sweeps) for the columns of B, one CTA per
// column (the columns are independent; no grid-wide synchronization), on the working
// (reversed for UPPER) indices.  ipiv holds the reference's values at ORIGINAL positions.
__global__ void __launch_bounds__(kBkSolveThreads) ldl_bk_solve_kernel(SymView A, double *B,
                                                                       int64_t ldb, int nrhs,
                                                                       const int64_t *ipiv) {
  __shared__ double red[2][kBkSolveThreads / 32];
  const int n = A.n, rev = A.rev, tid = threadIdx.x, c = blockIdx.x;
  if (c >= nrhs) return;
  double *bc = B + (int64_t)c * ldb;
  auto brow = [&](int i) -> double * { return bc + (rev ? n - 1 - i : i); };
  // pivot of working step k in working indices (1-based, negative for a 2 x 2 block)
  auto piv = [&](int k) -> int64_t {
    const int64_t p = ipiv[rev ? n - 1 - k : k];
    if (p > 0) return (rev ? (int64_t)n - p : p - 1) + 1;
    const int64_t q = -p - 1;
    return -((rev ? (int64_t)n - 1 - q : q) + 1);
  };
  auto swap_rows = [&](int x, int y) {
    if (tid == 0 && x != y && x >= 0 && x < n && y >= 0 && y < n) {
      const double t = *brow(x);
      *brow(x) = *brow(y);
      *brow(y) = t;
    }
    __syncthreads();
  };
  // sweep 1: D^-1 L^-1 with the interchanges of each step (ldlbks.go:72-118)
  for (int k = 0; k < n;) {
    const int64_t pk = piv(k);
    if (pk > 0) {
      if (pk != k + 1) swap_rows(k, (int)pk - 1);
      const double bk = *brow(k);
      for (int i = k + 1 + tid; i < n; i += kBkSolveThreads)
        *brow(i) = __dadd_rn(*brow(i), -(*A.at(i, k) * bk));
      __syncthreads();
      if (tid == 0) *brow(k) = bk / *A.at(k, k);
      __syncthreads();
      k += 1;
    } else {
      if (k + 1 >= n) return;  // a 2 x 2 block cannot start at the last row
      if (pk != -(k + 1)) swap_rows(k + 1, (int)(-pk) - 1);
      const double b = *A.at(k + 1, k);
      const double apb = *A.at(k, k) / b, dpb = *A.at(k + 1, k + 1) / b;
      double scale = __dadd_rn(__dmul_rn(apb, dpb), -1.0);
      scale *= b;
      const double s0 = *brow(k), s1 = *brow(k + 1);
      for (int i = k + 2 + tid; i < n; i += kBkSolveThreads)
        *brow(i) = __dadd_rn(*brow(i), -__dadd_rn(__dmul_rn(*A.at(i, k), s0), __dmul_rn(*A.at(i, k + 1), s1)));
      __syncthreads();
      if (tid == 0) {
        *brow(k) = __dadd_rn(__dmul_rn(dpb, s0), -s1) / scale;
        *brow(k + 1) = __dadd_rn(__dmul_rn(apb, s1), -s0) / scale;
      }
      __syncthreads();
      k += 2;
    }
  }
  // sweep 2: L^-T with the interchanges undone from the last step (ldlbks.go:119-146)
  for (int nc = n; nc > 0;) {
    const int64_t pl = piv(nc - 1);
    if (pl > 0) {
      const int k = nc - 1;
      double acc = 0.0;
      for (int i = k + 1 + tid; i < n; i += kBkSolveThreads)
        acc = __dadd_rn(acc, __dmul_rn(*A.at(i, k), *brow(i)));
      acc = bk_block_sum(acc, red[0]);
      if (tid == 0) *brow(k) = __dadd_rn(*brow(k), -acc);
      __syncthreads();
      if (pl != nc) swap_rows(k, (int)pl - 1);
      nc -= 1;
    } else {
      const int k = nc - 2;
      if (k < 0) return;
      double a0 = 0.0, a1 = 0.0;
      for (int i = k + 2 + tid; i < n; i += kBkSolveThreads) {
        const double bi = *brow(i);
        a0 = __dadd_rn(a0, __dmul_rn(*A.at(i, k), bi));
        a1 = __dadd_rn(a1, __dmul_rn(*A.at(i, k + 1), bi));
      }
      a0 = bk_block_sum(a0, red[0]);
      a1 = bk_block_sum(a1, red[1]);
      if (tid == 0) {
        *brow(k) = __dadd_rn(*brow(k), -a0);
        *brow(k + 1) = __dadd_rn(*brow(k + 1), -a1);
      }
      __syncthreads();
      if (piv(k) != -nc) swap_rows(k + 1, (int)(-piv(k)) - 1);
      nc -= 2;
    }
  }
}

// pivot.go:63-78 (applyRowPivots, offset 0) on the columns of B, one thread per column:
// forward k = 0.., backward k = ..0; ipiv[k] > 0 swaps rows k and ipiv[k] - 1
__global__ void ldl_row_pivots_kernel(double *B, int64_t ldb, int nrhs, const int64_t *ipiv,
                                      int n, int forward) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nrhs) return;
  double *bc = B + (int64_t)c * ldb;
  for (int t = 0; t < n; ++t) {
    const int k = forward ? t : n - 1 - t;
    const int64_t p = ipiv[k];
    if (p > 0 && p <= n && p - 1 != k) {
      const double x = bc[k];
      bc[k] = bc[p - 1];
      bc[p - 1] = x;
    }
  }
}

// diag.go:85-128 (SolveDiag, LEFT, D = the diagonal of A): row k of B times 1 / A(k, k)
__global__ void ldl_solve_diag_kernel(double *B, int64_t ldb, int n, int nrhs, const double *A,
                                      int64_t lda) {
  const int i = blockIdx.x * 256 + threadIdx.x, c = blockIdx.y;
  if (i >= n || c >= nrhs) return;
  B[i + (int64_t)c * ldb] *= 1.0 / A[i + (int64_t)i * lda];
}

}  // namespace

// DecomposeLDLnoPiv / DecomposeLDL / DecomposeBK on the device: one cooperative sweep.
// Returns MO_OK, or k + 1 for DecomposeLDL's zero pivot at step k (synchronizes then).
size_t ldl_scratch_bytes(int sms) { return (size_t)2 * sms * (sizeof(double) + sizeof(int)) + 512; }

int ldl_factor(mo_ctx *ctx, View A, int64_t *ipiv, int mode, bool upper, char *scratch = nullptr) {
  const int n = A.rows;
  if (n == 0) return MO_OK;
  const int grid = std::max(1, std::min(ctx->sms, n / 32));
  const size_t bytes = ldl_scratch_bytes(grid);
  char *ws = scratch;
  int rc = MO_OK;
  if (!ws && (rc = workspace(ctx, bytes, (void **)&ws))) return rc;
  LdlScratch sc;
  sc.val = (double *)ws;
  sc.idx = (int *)(ws + (size_t)2 * grid * sizeof(double));
  char *tailp = ws + (((size_t)2 * grid * (sizeof(double) + sizeof(int)) + 255) & ~(size_t)255);
  sc.bar = (unsigned *)tailp;
  sc.abort_flag = (int *)(tailp + 64);
  int *info = (int *)(tailp + 128);
  MO_CUDA_TRY(cudaMemsetAsync(tailp, 0, 256, ctx->stream));
  SymView v{A.d, A.ld, n, upper ? 1 : 0};
  int *status = &control(ctx)->status;
  void *args[] = {&v, &ipiv, &sc, &status, &info};
  const void *fn = mode == kLdlNoPiv ? (const void *)ldl_kernel<kLdlNoPiv>
                   : mode == kLdlDiag ? (const void *)ldl_kernel<kLdlDiag>
                                      : (const void *)ldl_kernel<kLdlBK>;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_PANEL);
  MO_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kLdlThreads), args, 0, ctx->stream));
  prof_end(ctx, ps, (double)n * n * n / 3.0, 16.0 * n * (double)n * n / 3.0);
  MO_CUDA_TRY(cudaGetLastError());
  if (mode != kLdlDiag) return MO_OK;
  int h_info = 0;
  MO_CUDA_TRY(cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return h_info;
}

// SolveBK's device part: B (n x nrhs) := A^-1 B with DecomposeBK's factor and ipiv
int ldl_bk_solve(mo_ctx *ctx, View B, View A, const int64_t *ipiv, bool upper) {
  if (B.rows == 0 || B.cols == 0) return MO_OK;
  SymView v{A.d, A.ld, A.rows, upper ? 1 : 0};
  ldl_bk_solve_kernel<<<B.cols, kBkSolveThreads, 0, ctx->stream>>>(v, B.d, B.ld, B.cols, ipiv);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// SolveLDLnoPiv / SolveLDL's device part (ldlnp.go:251-266, ldl.go:486-510): interchanges
// (when ipiv), two unit-triangular solves and the diagonal scaling, in the reference's order
int ldl_solve(mo_ctx *ctx, View B, View A, const int64_t *ipiv, bool upper) {
  const int n = A.rows;
  if (B.rows == 0 || B.cols == 0) return MO_OK;
  const int tri = upper ? MO_UPPER : MO_LOWER;
  auto pivots = [&](bool forward) -> int {
    if (!ipiv) return MO_OK;
    ldl_row_pivots_kernel<<<(B.cols + 127) / 128, 128, 0, ctx->stream>>>(B.d, B.ld, B.cols, ipiv,
                                                                         n, forward ? 1 : 0);
    MO_CUDA_TRY(cudaGetLastError());
    return MO_OK;
  };
  int rc = pivots(!upper);
  if (!rc) rc = trsm(ctx, B, A, MO_LEFT | tri | MO_UNIT, 1.0);
  if (rc) return rc;
  ldl_solve_diag_kernel<<<dim3((n + 255) / 256, B.cols), 256, 0, ctx->stream>>>(B.d, B.ld, n,
                                                                                B.cols, A.d, A.ld);
  MO_CUDA_TRY(cudaGetLastError());
  if ((rc = trsm(ctx, B, A, MO_LEFT | tri | MO_UNIT | MO_TRANSA, 1.0))) return rc;
  return pivots(upper);
}

namespace {

// X(:, c) *= 1 / d_c (SolveDiag RIGHT, diag.go:97-102) or, with W, W(:, c) = X(:, c) d_c
// (MultDiag RIGHT, diag.go:38-44); d the diagonal of the factored block (stride ldd + 1)
__global__ void ldl_cols_kernel(double *X, int64_t ldx, int rows, const double *D, int64_t ldd,
                                double *W, int64_t ldw) {
  const int i = blockIdx.x * 256 + threadIdx.x, c = blockIdx.y;
  if (i >= rows) return;
  const double d = D[c + (int64_t)c * ldd];
  if (W)
    W[i + (int64_t)c * ldw] = X[i + (int64_t)c * ldx] * d;
  else
    X[i + (int64_t)c * ldx] *= 1.0 / d;
}

}  // namespace

// DecomposeLDLnoPiv blocked as ldlnp.go:104-205 does it with nb = 128: the diagonal block by
// the sweep, the block column by a unit-triangular solve and D^-1, the rest of the matrix
// by one engine update in its triangle mode (UpdateTrm's A22 -= L21 (L21 D)^T)
int ldl_nopiv_blocked(mo_ctx *ctx, View A, bool upper) {
  const int n = A.rows, NB = 128;
  const size_t wbytes = ((size_t)n * NB * 8 + 255) & ~(size_t)255;
  const size_t ibytes = (size_t)NB * NB * 8;
  char *ws = nullptr;
  int rc = workspace(ctx, wbytes + ibytes + ldl_scratch_bytes(ctx->sms), (void **)&ws);
  if (rc) return rc;
  double *W = (double *)ws, *inv = (double *)(ws + wbytes);
  char *scr = ws + wbytes + ibytes;
  auto cols = [&](View X, const View &D, double *w) -> int {
    if (X.rows == 0 || X.cols == 0) return MO_OK;
    ldl_cols_kernel<<<dim3((X.rows + 255) / 256, X.cols), 256, 0, ctx->stream>>>(
        X.d, X.ld, X.rows, D.d, D.ld, w, X.rows);
    MO_CUDA_TRY(cudaGetLastError());
    return MO_OK;
  };
  GemmOpts o;
  o.mode = upper ? kSyrkUpper : kSyrkLower;
  if (!upper) {
    for (int kb = 0; kb < n; kb += NB) {
      const int bo = std::min(NB, n - kb), rest = n - kb - bo;
      const View A11 = A.sub(kb, kb, bo, bo);
      if ((rc = ldl_factor(ctx, A11, nullptr, kLdlNoPiv, false, scr))) return rc;
      if (rest == 0) break;
      const View A21 = A.sub(kb + bo, kb, rest, bo);
      if ((rc = trsm_with_scratch(ctx, A21, A11, MO_RIGHT | MO_LOWER | MO_UNIT | MO_TRANSA, 1.0,
                                  inv)))
        return rc;
      if ((rc = cols(A21, A11, nullptr)) || (rc = cols(A21, A11, W))) return rc;
      if ((rc = gemm_ex(ctx, A.sub(kb + bo, kb + bo, rest, rest), A21, false,
                        View{W, rest, bo, rest}, true, -1.0, 1.0, o)))
        return rc;
    }
  } else {
    for (int e = n; e > 0; e -= NB) {
      const int bo = std::min(NB, e), s0 = e - bo;
      const View A11 = A.sub(s0, s0, bo, bo);
      if ((rc = ldl_factor(ctx, A11, nullptr, kLdlNoPiv, true, scr))) return rc;
      if (s0 == 0) break;
      const View A01 = A.sub(0, s0, s0, bo);
      if ((rc = trsm_with_scratch(ctx, A01, A11, MO_RIGHT | MO_UPPER | MO_UNIT | MO_TRANSA, 1.0,
                                  inv)))
        return rc;
      if ((rc = cols(A01, A11, nullptr)) || (rc = cols(A01, A11, W))) return rc;
      if ((rc = gemm_ex(ctx, A.sub(0, 0, s0, s0), A01, false, View{W, s0, bo, s0}, true, -1.0,
                        1.0, o)))
        return rc;
    }
  }
  return MO_OK;
}

}  // namespace mo

using mo::View;

namespace {

int ldl_tri(int flags, bool *upper) {
  // LOWER selects the lower triangle (the reference tests LOWER first), otherwise upper
  *upper = (flags & MO_LOWER) == 0;
  return MO_OK;
}

}  // namespace

extern "C" {

// ldlnp.go:211-235
int mo_decompose_ldl_nopiv(mo_ctx *ctx, mo_matrix Am, mo_matrix Wm, int flags, int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A;
  if ((rc = mo::to_view(Am, A))) return rc;
  if (A.rows != A.cols) return MO_ENOTSQUARE;
  if (!(A.cols < nb || nb == 0) && Wm.data == nullptr) return MO_ELDLWORK;
  bool upper;
  ldl_tri(flags, &upper);
  // one sweep for small orders, the blocked form (ldlnp.go:104) above
  return A.rows > 256 ? mo::ldl_nopiv_blocked(ctx, A, upper) : mo::ldl_factor(ctx, A, nullptr, 0, upper);
}

// ldlnp.go:251-266
int mo_solve_ldl_nopiv(mo_ctx *ctx, mo_matrix Bm, mo_matrix Am, int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View B, A;
  if ((rc = mo::to_view(Bm, B)) || (rc = mo::to_view(Am, A))) return rc;
  if (!(flags & (MO_LOWER | MO_UPPER))) return MO_OK;
  if (A.rows != A.cols || B.rows != A.rows) return MO_EABSIZE;
  return mo::ldl_solve(ctx, B, A, nullptr, (flags & MO_UPPER) != 0);
}

// ldl.go:439-466
int mo_decompose_ldl(mo_ctx *ctx, mo_matrix Am, mo_matrix Wm, int64_t *ipiv, int64_t npiv,
                     int flags, int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A;
  if ((rc = mo::to_view(Am, A))) return rc;
  (void)Wm;
  (void)nb;
  if (A.rows != A.cols) return MO_ENOTSQUARE;
  if (npiv > 0 && !ipiv) return MO_EINVAL;
  if (npiv > 0) MO_CUDA_TRY(cudaMemsetAsync(ipiv, 0, (size_t)npiv * sizeof(int64_t), ctx->stream));
  if (npiv < A.rows) return MO_EPIVLEN;
  bool upper;
  ldl_tri(flags, &upper);
  rc = mo::ldl_factor(ctx, A, ipiv, 1, upper);
  return rc > 0 ? MO_EZERODIAG : rc;
}

// ldl.go:486-510
int mo_solve_ldl(mo_ctx *ctx, mo_matrix Bm, mo_matrix Am, const int64_t *ipiv, int64_t npiv,
                 int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View B, A;
  if ((rc = mo::to_view(Bm, B)) || (rc = mo::to_view(Am, A))) return rc;
  if (!(flags & (MO_LOWER | MO_UPPER))) return MO_OK;
  if (A.rows != A.cols || B.rows != A.rows) return MO_EABSIZE;
  if (npiv < A.rows) return MO_EPIVLEN;
  return mo::ldl_solve(ctx, B, A, ipiv, (flags & MO_UPPER) != 0);
}

// ldlbk.go:1114-1140
int mo_decompose_bk(mo_ctx *ctx, mo_matrix Am, mo_matrix Wm, int64_t *ipiv, int64_t npiv,
                    int flags, int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A;
  if ((rc = mo::to_view(Am, A))) return rc;
  if (npiv > 0 && !ipiv) return MO_EINVAL;
  if (npiv > 0) MO_CUDA_TRY(cudaMemsetAsync(ipiv, 0, (size_t)npiv * sizeof(int64_t), ctx->stream));
  const bool blocked = !(A.cols < nb || nb == 0);
  if (Wm.data == nullptr || (blocked ? Wm.cols < nb + 1 : Wm.cols < 2) || Wm.rows < A.rows)
    return MO_EBKWORK;
  if (A.rows != A.cols) return MO_ENOTSQUARE;
  if (npiv < A.rows) return MO_EPIVLEN;
  if (!(flags & (MO_LOWER | MO_UPPER))) return MO_OK;
  return mo::ldl_factor(ctx, A, ipiv, 2, (flags & MO_LOWER) == 0);
}

// ldlbks.go:303-318
int mo_solve_bk(mo_ctx *ctx, mo_matrix Bm, mo_matrix Am, const int64_t *ipiv, int64_t npiv,
                int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View B, A;
  if ((rc = mo::to_view(Bm, B)) || (rc = mo::to_view(Am, A))) return rc;
  if (!(flags & (MO_LOWER | MO_UPPER))) return MO_OK;
  if (A.rows != A.cols || B.rows != A.rows) return MO_EABSIZE;
  if (npiv < A.rows) return MO_EPIVLEN;
  return mo::ldl_bk_solve(ctx, B, A, ipiv, (flags & MO_LOWER) == 0);
}

}  // extern "C"
