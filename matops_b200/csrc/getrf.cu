// LU factorization with partial pivoting (DecomposeLU) and the row interchanges used by
// SolveLU, on the device.
//
// Reference: lu.go:173-231 (blockedLUpiv, left-looking Crout variant), lu.go:103-171
// (unblockedLUpiv), pivot.go:27-61 (swapRows/applyPivots), pivot.go:98-107 (pivotIndex:
// first row holding the strict maximum of |x|; a NaN never wins unless it sits on the
// diagonal, where the scan starts).  The factors do not depend on left- vs right-looking
// order except through rounding, so the device runs the right-looking form:
//   panel   : cooperative kernel, every CTA owns a slice of panel rows in shared memory,
//             one grid barrier per column (candidate rows are published with the local
//             argmax, so every CTA picks the pivot itself)
//   laswp   : apply the panel's interchanges to the columns left and right of it
//   trsm    : U12 = L11^-1 A12 (unit lower inverse + in-place GEMM)
//   update  : A22 -= L21 U12 on the FP64 tensor pipe
#include <algorithm>
#include <climits>
#include <utility>

#include "context.cuh"
#include "tri.cuh"

namespace mo {
int trtri_blocks(mo_ctx *ctx, View A, int N, bool trans, bool lower_eff, bool unit, double *inv);

namespace {

constexpr int PANEL_THREADS = 256;
constexpr int MAX_PANEL_W = 128;

struct PanelScratch {
  // double-buffered per-CTA candidates: value, index, NaN-on-diagonal flag, row values
  double *cand_val;   // [2][nblk]
  int *cand_idx;      // [2][nblk]
  double *cand_row;   // [2][nblk][W]
  double *rowj;       // [2][W]  current contents of panel row j (published by its owner)
  int *diag_nan;      // [2]
  unsigned *barrier;  // monotonically increasing arrival counter
};

__device__ __forceinline__ bool better(double v, int i, double bv, int bi) {
  return v > bv || (v == bv && i < bi);
}

// Bounded grid barrier over `nblk` co-resident CTAs (cooperative launch).  Returns false
// after recording MO_EDEVTIMEOUT.
__device__ bool grid_barrier(unsigned *counter, unsigned target, int *status, int *abort_flag) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
    int ok = 1;
    unsigned i = 0;
    while (true) {
      unsigned v = *(volatile unsigned *)counter;
      if (v >= target) break;
      if (*(volatile int *)abort_flag) {
        ok = 0;
        break;
      }
      if (++i > MO_SPIN_LIMIT) {
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

// Factor the m x W panel P (column-major, ld) in place; piv[j] = row0 + pivot position.
// Each CTA owns rows [b*R, min((b+1)*R, m)) in shared memory (row-major, stride W+1).
__global__ void __launch_bounds__(PANEL_THREADS)
    lu_panel_kernel(double *P, int64_t ld, int m, int W, int R, int64_t *piv, int64_t row0,
                    PanelScratch sc, int *status, int *abort_flag) {
  extern __shared__ double S[];
  const int nblk = gridDim.x, b = blockIdx.x;
  const int LDW = W + 1;
  const int rbeg = b * R, rend = min(m, rbeg + R), nr = max(0, rend - rbeg);
  __shared__ double s_prow[MAX_PANEL_W];
  __shared__ double s_oldj[MAX_PANEL_W];
  __shared__ double red_v[PANEL_THREADS / 32];
  __shared__ int red_i[PANEL_THREADS / 32];
  __shared__ int red_q[PANEL_THREADS / 32];

  for (int e = threadIdx.x; e < nr * W; e += blockDim.x) {
    const int r = e % nr, c = e / nr;
    S[r * LDW + c] = P[(rbeg + r) + (int64_t)c * ld];
  }
  __syncthreads();

  const int kmax = min(m, W);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // (row, column) work of the update: G consecutive lanes per row
  int G = 32;
  while (G > 1 && G * nr > (int)blockDim.x) G >>= 1;
  for (int j = 0; j < kmax; ++j) {
    const int par = j & 1;
    // (a) local argmax of |column j| over owned positions >= j; every warp then combines
    // the warps' partials itself (no second barrier)
    double bv = -1.0;
    int bi = INT_MAX;
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
      const int gi = rbeg + r;
      if (gi < j) continue;
      double v = fabs(S[r * LDW + j]);
      if (isnan(v)) v = -1.0;  // NaN never wins off the diagonal
      if (better(v, gi, bv, bi)) {
        bv = v;
        bi = gi;
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (better(ov, oi, bv, bi)) {
        bv = ov;
        bi = oi;
      }
    }
    if (lane == 0) {
      red_v[wid] = bv;
      red_i[wid] = bi;
    }
    __syncthreads();
    bv = lane < nw ? red_v[lane] : -1.0;
    bi = lane < nw ? red_i[lane] : INT_MAX;
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (better(ov, oi, bv, bi)) {
        bv = ov;
        bi = oi;
      }
    }
    // (b) publish the candidate and its row and, if owned here, row j
    if (threadIdx.x == 0) {
      sc.cand_val[par * nblk + b] = bv;
      sc.cand_idx[par * nblk + b] = bi;
    }
    {
      double *crow = sc.cand_row + ((size_t)par * nblk + b) * W;
      if (bi != INT_MAX)
        for (int c = threadIdx.x; c < W; c += blockDim.x) crow[c] = S[(bi - rbeg) * LDW + c];
      if (j >= rbeg && j < rend) {
        for (int c = threadIdx.x; c < W; c += blockDim.x) sc.rowj[par * W + c] = S[(j - rbeg) * LDW + c];
        if (threadIdx.x == 0) sc.diag_nan[par] = isnan(S[(j - rbeg) * LDW + j]) ? 1 : 0;
      }
    }
    if (!grid_barrier(sc.barrier, (unsigned)(j + 1) * nblk, status, abort_flag)) return;
    // (c) every CTA selects the pivot: largest value, lowest index; NaN on the diagonal wins.
    // The candidates are read in parallel (one per thread) and reduced like the local
    // argmax, so the selection costs one L2 round trip, not one per CTA.
    int p, wb;
    {
      double v = -2.0;
      int pi = INT_MAX, wq = INT_MAX;
      for (int q = threadIdx.x; q < nblk; q += blockDim.x) {
        const double cv = __ldcg(sc.cand_val + par * nblk + q);
        const int ci = __ldcg(sc.cand_idx + par * nblk + q);
        if (ci != INT_MAX && better(cv, ci, v, pi)) {
          v = cv;
          pi = ci;
          wq = q;
        }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, pi, off);
        const int oq = __shfl_xor_sync(0xffffffffu, wq, off);
        if (better(ov, oi, v, pi)) {
          v = ov;
          pi = oi;
          wq = oq;
        }
      }
      if (lane == 0) {
        red_v[wid] = v;
        red_i[wid] = pi;
        red_q[wid] = wq;
      }
      __syncthreads();
      v = lane < nw ? red_v[lane] : -2.0;
      pi = lane < nw ? red_i[lane] : INT_MAX;
      wq = lane < nw ? red_q[lane] : INT_MAX;
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, pi, off);
        const int oq = __shfl_xor_sync(0xffffffffu, wq, off);
        if (better(ov, oi, v, pi)) {
          v = ov;
          pi = oi;
          wq = oq;
        }
      }
      p = pi;
      wb = pi == INT_MAX ? -1 : wq;
      if (__ldcg(sc.diag_nan + par)) {
        p = j;
        wb = -1;
      }
      if (p == INT_MAX) p = j;  // no comparable candidate: keep the row
    }
    // (d) the pivot row (U row) and the old row j, into shared memory
    for (int c = threadIdx.x; c < W; c += blockDim.x) {
      const double oj = __ldcg(sc.rowj + par * W + c);
      s_oldj[c] = oj;
      s_prow[c] = (wb >= 0) ? __ldcg(sc.cand_row + ((size_t)par * nblk + wb) * W + c) : oj;
    }
    if (b == 0 && threadIdx.x == 0) piv[j] = row0 + p;
    __syncthreads();
    // (e) interchange rows j and p (pivot.go:27-35 on the panel columns), l = a_ij / u_jj
    // (true division, mvec.go:422 InvScale) and the rank-1 update of the owned rows below j,
    // in one pass: row j takes the pivot row; the row at p is read from the old row j
    if (p != j && j >= rbeg && j < rend)
      for (int c = threadIdx.x; c < W; c += blockDim.x) S[(j - rbeg) * LDW + c] = s_prow[c];
    const double ujj = s_prow[j];
    const int r0 = max(0, j + 1 - rbeg);  // first owned row below j
    const int grp = threadIdx.x / G, gl = threadIdx.x % G;
    // the lanes of this thread's group (G divides 32; every lane of a group runs the same
    // iterations)
    const unsigned gmask = G == 32 ? 0xffffffffu : ((1u << G) - 1u) << (lane & ~(G - 1));
    for (int r = r0 + grp; r < nr; r += blockDim.x / G) {
      double *row = S + r * LDW;
      const bool swapped = p != j && rbeg + r == p;
      const double *src = swapped ? s_oldj : row;
      const double l = src[j] / ujj;
      __syncwarp(gmask);  // the group has read src[j] before it is overwritten
      if (swapped)
        for (int c = gl; c < j; c += G) row[c] = src[c];
      if (gl == 0) row[j] = l;
      for (int c = j + 1 + gl; c < W; c += G) row[c] = fma(-l, s_prow[c], src[c]);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nr * W; e += blockDim.x) {
    const int r = e % nr, c = e / nr;
    P[(rbeg + r) + (int64_t)c * ld] = S[r * LDW + c];
  }
}

// Apply interchanges rows (r0+s) <-> piv[s] (absolute rows of A), s = 0..ns-1 in order,
// to columns [0, ncols) of A; one thread per column.  Out-of-range pivots are reported.
__global__ void laswp_kernel(double *A, int64_t ld, int rows, int ncols, const int64_t *piv,
                             int ns, int64_t r0, int *status) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  double *col = A + (int64_t)c * ld;
  for (int s = 0; s < ns; ++s) {
    const int64_t p = piv[s];
    const int64_t q = r0 + s;
    if (p <= 0 || p == q) continue;  // pivot.go:57: entries <= 0 are skipped
    if (p >= rows || q >= rows) {
      if (c == 0) set_status(status, MO_EINVAL);
      continue;
    }
    const double t = col[q];
    col[q] = col[p];
    col[p] = t;
  }
}

// The net effect of the interchanges rows (r0 + s) <-> piv[s], s = 0 .. ns - 1 in order
// (pivot.go:55-61, entries <= 0 skipped) on the rows they touch: rows r0 .. r0 + ns - 1 and
// the distinct pivot rows beyond them.  One warp simulates the swaps on row labels and
// writes the moves dst[i] <- src[i] (i < *count), so that one pass of loads and one of
// stores applies all of them to any set of columns.  ns <= MAX_PANEL_W.
__global__ void __launch_bounds__(32) swap_map_kernel(const int64_t *piv, int ns, int64_t r0,
                                                      int rows, int *dst, int *src, int *count,
                                                      int *status) {
  __shared__ int lab[2 * MAX_PANEL_W];   // source row now held at each position
  __shared__ int ext[MAX_PANEL_W];       // rows beyond the block, in order of first use
  __shared__ int next;
  const int lane = threadIdx.x;
  for (int i = lane; i < ns; i += 32) lab[i] = (int)(r0 + i);
  if (lane == 0) next = 0;
  __syncwarp();
  for (int s = 0; s < ns; ++s) {
    const int64_t p = piv[s];
    const int64_t q = r0 + s;
    if (p <= 0 || p == q) continue;
    if (p >= rows || q >= rows) {
      if (lane == 0) set_status(status, MO_EINVAL);
      continue;
    }
    int pos;
    if (p < r0 + ns) {
      pos = (int)(p - r0);
    } else {
      const int ne = next;
      int found = -1;
      for (int b = 0; b < ne; b += 32) {
        const unsigned hit = __ballot_sync(0xffffffffu, b + lane < ne && ext[b + lane] == (int)p);
        if (hit) {
          found = b + __ffs(hit) - 1;
          break;
        }
      }
      if (found < 0) {
        found = ne;
        if (lane == 0) {
          ext[ne] = (int)p;
          lab[ns + ne] = (int)p;
          next = ne + 1;
        }
      }
      pos = ns + found;
    }
    __syncwarp();
    if (lane == 0) {
      const int t = lab[s];
      lab[s] = lab[pos];
      lab[pos] = t;
    }
    __syncwarp();
  }
  const int total = ns + next;
  for (int i = lane; i < total; i += 32) {
    dst[i] = i < ns ? (int)(r0 + i) : ext[i - ns];
    src[i] = lab[i];
  }
  if (lane == 0) *count = total;
}

// swap_map_kernel for panels whose rows [r0, rows) fit a shared-memory table (label per
// position, touched flag): the pivots are read in parallel, one thread applies the swaps
// to the table in order (a few shared-memory operations each, no warp-wide search), and
// the moves are written in the same form and order as swap_map_kernel's.
constexpr int kSwapTableMax = 32768;
__global__ void __launch_bounds__(256) swap_map_table_kernel(const int64_t *piv, int ns, int64_t r0,
                                                             int rows, int *dst, int *src,
                                                             int *count, int *status) {
  extern __shared__ int tb[];
  const int span = rows - (int)r0;
  int *lab = tb;                                             // [span]
  int *ext = lab + span;                                     // [MAX_PANEL_W]
  int *pv = ext + MAX_PANEL_W;                               // [MAX_PANEL_W]
  unsigned char *touched = reinterpret_cast<unsigned char *>(pv + MAX_PANEL_W);  // [span]
  __shared__ int next;
  for (int i = threadIdx.x; i < span; i += blockDim.x) {
    lab[i] = (int)r0 + i;
    touched[i] = 0;
  }
  for (int i = threadIdx.x; i < ns; i += blockDim.x) {
    const int64_t p = piv[i];
    // -1: skipped (pivot.go:57, entries <= 0, or no exchange); -2: out of range
    pv[i] = (p <= 0 || p == r0 + i) ? -1 : ((p >= rows || p < r0 || r0 + i >= rows) ? -2 : (int)(p - r0));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int ne = 0;
    bool bad = false;
    for (int s2 = 0; s2 < ns; ++s2) {
      const int pi = pv[s2];
      if (pi == -1) continue;
      if (pi == -2) {
        bad = true;
        continue;
      }
      const int t = lab[s2];
      lab[s2] = lab[pi];
      lab[pi] = t;
      if (pi >= ns && !touched[pi]) {
        touched[pi] = 1;
        ext[ne++] = pi;
      }
    }
    if (bad) set_status(status, MO_EINVAL);
    next = ne;
  }
  __syncthreads();
  const int total = ns + next;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int pos = i < ns ? i : ext[i - ns];
    dst[i] = (int)r0 + pos;
    src[i] = lab[pos];
  }
  if (threadIdx.x == 0) *count = total;
}

// A[dst[i], c] = A_old[src[i], c] for the moves of swap_map_kernel, columns [0, ncols): a
// CTA takes 32 columns, loads every source row of them into shared memory (lanes along the
// rows, so the contiguous block rows are read 256 bytes at a time), then stores.
__global__ void __launch_bounds__(256) laswp_map_kernel(double *A, int64_t ld, int ncols,
                                                        const int *dst, const int *src,
                                                        const int *count) {
  extern __shared__ double vals[];  // [count][32]
  const int cnt = *count;
  const int c0 = blockIdx.x * 32;
  const int nc = min(32, ncols - c0);
  for (int e = threadIdx.x; e < cnt * nc; e += blockDim.x) {
    const int i = e % cnt, c = e / cnt;
    vals[c * cnt + i] = A[src[i] + (int64_t)(c0 + c) * ld];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < cnt * nc; e += blockDim.x) {
    const int i = e % cnt, c = e / cnt;
    A[dst[i] + (int64_t)(c0 + c) * ld] = vals[c * cnt + i];
  }
}

// All interchanges rows s <-> piv[s] (s = 0 .. ns - 1, in order) on a few columns of B
// (SolveLU's applyPivots): one CTA per column, the column in shared memory, one thread
// applying the swaps in order.
__global__ void __launch_bounds__(256) laswp_cols_kernel(double *B, int64_t ld, int rows,
                                                         const int64_t *piv, int ns, int *status) {
  extern __shared__ double col[];
  double *g = B + (int64_t)blockIdx.x * ld;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) col[i] = g[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < ns; ++s) {
      const int64_t p = piv[s];
      if (p <= 0 || p == s) continue;
      if (p >= rows || s >= rows) {
        if (blockIdx.x == 0) set_status(status, MO_EINVAL);
        continue;
      }
      const double t = col[s];
      col[s] = col[p];
      col[p] = t;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < rows; i += blockDim.x) g[i] = col[i];
}

// piv[i] = v for i in [lo, hi)
__global__ void fill_pivots_kernel(int64_t *piv, int64_t lo, int64_t hi, int64_t v) {
  const int64_t i = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < hi) piv[i] = v;
}

struct CtrlView {
  int status;
  int info;
  double bad;
};

}  // namespace

int laswp(mo_ctx *ctx, View A, int c0, int c1, const int64_t *piv, int ns, int64_t r0) {
  if (c1 <= c0 || ns <= 0) return MO_OK;
  const int nc = c1 - c0;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_LASWP);
  laswp_kernel<<<(nc + 127) / 128, 128, 0, ctx->stream>>>(
      A.at(0, c0), A.ld, A.rows, nc, piv, ns, r0,
      &reinterpret_cast<CtrlView *>(ctx->d_status)->status);
  prof_end(ctx, ps, 0.0, 4.0 * 8.0 * ns * (double)nc);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// SolveLU's applyPivots(B, pivots) (lu.go:322, pivot.go:55-61)
int laswp_forward(mo_ctx *ctx, View B, const int64_t *piv, int64_t npiv) {
  if (B.rows == 0 || B.cols == 0 || npiv <= 0) return MO_OK;
  if (npiv > INT_MAX) return MO_EINVAL;
  const size_t smem = (size_t)B.rows * sizeof(double);
  if (smem > 200 * 1024) return laswp(ctx, B, 0, B.cols, piv, (int)npiv, 0);
  if (int rc = mo_smem_attr((const void *)laswp_cols_kernel, (int)smem)) return rc;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_LASWP);
  laswp_cols_kernel<<<B.cols, 256, smem, ctx->stream>>>(
      B.d, B.ld, B.rows, piv, (int)npiv,
      &reinterpret_cast<CtrlView *>(ctx->d_status)->status);
  prof_end(ctx, ps, 0.0, 16.0 * B.rows * (double)B.cols);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// the panel's interchanges on columns [c0, c1) of A through the move list of swap_map_kernel
int laswp_moves(mo_ctx *ctx, View A, int c0, int c1, const int *dst, const int *src,
                const int *count, int max_moves) {
  if (c1 <= c0) return MO_OK;
  const int nc = c1 - c0;
  const size_t smem = (size_t)max_moves * 32 * sizeof(double);
  if (int rc = mo_smem_attr((const void *)laswp_map_kernel, (int)smem)) return rc;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_LASWP);
  laswp_map_kernel<<<(nc + 31) / 32, 256, smem, ctx->stream>>>(A.at(0, c0), A.ld, nc, dst, src,
                                                               count);
  prof_end(ctx, ps, 0.0, 16.0 * max_moves * (double)nc);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

int getrf(mo_ctx *ctx, View A, int64_t *piv, int64_t npiv, int ref_nb) {
  const int m = A.rows, n = A.cols, mn = min(m, n);
  int *status = &reinterpret_cast<CtrlView *>(ctx->d_status)->status;
  // panel width and rows per CTA: keep the panel slice <= ~200 KB of shared memory
  int W = MAX_PANEL_W;
  const int max_blocks = ctx->sms;
  auto rows_per_block = [&](int) {
    int nblk = min(max_blocks, max(1, (m + 63) / 64));
    return std::pair<int, int>((m + nblk - 1) / nblk, nblk);
  };
  auto smem_for = [](int R, int w) { return (size_t)R * (w + 1) * sizeof(double); };
  auto rb = rows_per_block(W);
  while (smem_for(rb.first, W) > 200 * 1024 && W > 8) {
    W /= 2;
    rb = rows_per_block(W);
  }
  if (smem_for(rb.first, W) > 200 * 1024) return MO_EINVAL;  // > ~3.2M rows
  const int R = rb.first, nblk = rb.second;
  // later (shorter) panels may use up to 64 rows per CTA
  const size_t smem = smem_for(std::max(R, 64), W);
  MO_CUDA_TRY(cudaFuncSetAttribute(lu_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  int occ = 0;
  MO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, lu_panel_kernel, PANEL_THREADS,
                                                            smem));
  if (occ * ctx->sms < nblk) return MO_EINVAL;

  // workspace: panel scratch + L11 inverse
  const size_t sz_val = 2 * nblk * sizeof(double), sz_idx = 2 * nblk * sizeof(int);
  const size_t sz_row = (size_t)2 * nblk * W * sizeof(double), sz_rowj = 2 * W * sizeof(double);
  const size_t inv_bytes = 2 * 128 * 128 * sizeof(double);  // two panels' L11 inverses
  const size_t sz_moves = 2 * (2 * MAX_PANEL_W) * sizeof(int) + 64;
  const size_t total = inv_bytes + sz_val + sz_row + sz_rowj + sz_idx + 64 + 64 + sz_moves;
  char *ws = nullptr;
  int rc = workspace(ctx, total, (void **)&ws);
  if (rc) return rc;
  double *inv = (double *)ws, *inv_b = inv + 128 * 128;
  PanelScratch sc;
  char *q = ws + inv_bytes;
  sc.cand_val = (double *)q;
  q += sz_val;
  sc.cand_row = (double *)q;
  q += sz_row;
  sc.rowj = (double *)q;
  q += sz_rowj;
  sc.cand_idx = (int *)q;
  q += sz_idx;
  sc.diag_nan = (int *)q;
  q += 16;
  sc.barrier = (unsigned *)q;
  q += 16;
  int *abort_flag = (int *)q;
  q += 32;
  int *mv_dst = (int *)q, *mv_src = mv_dst + 2 * MAX_PANEL_W, *mv_count = mv_src + 2 * MAX_PANEL_W;

  // one panel: factor A[k:m, k:k+b], then apply its interchanges left and right of it
  auto panel = [&](int k, int b) -> int {
    MO_CUDA_TRY(cudaMemsetAsync(sc.barrier, 0, 32, ctx->stream));  // barrier + abort flag
    View Pv = A.sub(k, k, m - k, b);
    const int pm = m - k;
    int pblk = min(nblk, max(1, (pm + 63) / 64));
    int pR = (pm + pblk - 1) / pblk;
    int64_t *pv = piv + k;
    int64_t row0 = k;
    double *pd = Pv.d;
    int64_t pld = Pv.ld;
    int pw = b;
    void *args[] = {&pd, &pld, (void *)&pm, &pw, &pR, &pv, &row0, &sc, &status, &abort_flag};
    ProfScope ps;
    prof_begin(ctx, ps, MO_PROF_PANEL);
    MO_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)lu_panel_kernel, dim3(pblk),
                                            dim3(PANEL_THREADS), args, smem, ctx->stream));
    prof_end(ctx, ps, (double)pm * b * b - (double)b * b * b / 3.0, 16.0 * pm * b);
    // interchanges on the columns left and right of the panel, as one move list
    if (k > 0 || k + b < n) {
      ProfScope pms;
      prof_begin(ctx, pms, MO_PROF_LASWP);
      if (m - k <= kSwapTableMax) {
        const size_t tsm = (size_t)(m - k) * 5 + 2 * MAX_PANEL_W * sizeof(int) + 16;
        int r2 = mo_smem_attr((const void *)swap_map_table_kernel, (int)tsm);
        if (r2) return r2;
        swap_map_table_kernel<<<1, 256, tsm, ctx->stream>>>(piv + k, b, k, m, mv_dst, mv_src,
                                                            mv_count, status);
      } else {
        swap_map_kernel<<<1, 32, 0, ctx->stream>>>(piv + k, b, k, m, mv_dst, mv_src, mv_count,
                                                   status);
      }
      prof_end(ctx, pms, 0.0, 8.0 * b);
      MO_CUDA_TRY(cudaGetLastError());
    }
    int r2 = laswp_moves(ctx, A, 0, k, mv_dst, mv_src, mv_count, 2 * b);
    if (!r2) r2 = laswp_moves(ctx, A, k + b, n, mv_dst, mv_src, mv_count, 2 * b);
    return r2;
  };
  // Panels in pairs: the second panel's columns are brought up to date with the first
  // (its U12 block and a (m - k2) x b1 x b0 update), the second is factored, and then the
  // rows of the first two block rows right of the pair become U (two small products and
  // one b1-row update between them) and the rest of the matrix takes ONE update with
  // K = b0 + b1: the trailing matrix is read and written once per pair, not per panel.
  for (int k = 0; k < mn; k += 2 * W) {
    const int b0 = min(W, mn - k);
    if ((rc = panel(k, b0))) return rc;
    const int k2 = k + b0;
    const int b1 = k2 < mn ? min(W, mn - k2) : 0;
    const int c_rest = n - k2 - b1;  // columns right of the pair
    if (n - k2 > 0) {
      if ((rc = trtri_blocks(ctx, A.sub(k, k, b0, b0), b0, false, true, true, inv))) return rc;
    }
    if (b1 == 0) {
      // single last panel: U12 and the update of what is right of it
      const int rest_c = n - k2;
      if (rest_c > 0) {
        View A12 = A.sub(k, k2, b0, rest_c);
        if ((rc = gemm(ctx, A12, View{inv, b0, b0, 128}, false, A12, false, 1.0, 0.0))) return rc;
        const int rest_r = m - k2;
        if (rest_r > 0 && (rc = gemm(ctx, A.sub(k2, k2, rest_r, rest_c), A.sub(k2, k, rest_r, b0),
                                     false, A12, false, -1.0, 1.0)))
          return rc;
      }
      continue;
    }
    // the second panel's columns: U01 = inv0 A01, A[k2:m, P1] -= L[k2:m, P0] U01
    {
      View U01 = A.sub(k, k2, b0, b1);
      if ((rc = gemm(ctx, U01, View{inv, b0, b0, 128}, false, U01, false, 1.0, 0.0))) return rc;
      if ((rc = gemm(ctx, A.sub(k2, k2, m - k2, b1), A.sub(k2, k, m - k2, b0), false, U01, false,
                     -1.0, 1.0)))
        return rc;
    }
    if ((rc = panel(k2, b1))) return rc;
    if (c_rest <= 0) continue;
    const int kc = k2 + b1;
    if ((rc = trtri_blocks(ctx, A.sub(k2, k2, b1, b1), b1, false, true, true, inv_b))) return rc;
    // rows k..k2 of the columns right of the pair: U0T = inv0 A0T
    View U0T = A.sub(k, kc, b0, c_rest);
    if ((rc = gemm(ctx, U0T, View{inv, b0, b0, 128}, false, U0T, false, 1.0, 0.0))) return rc;
    // rows k2..kc: A1T -= L10 U0T, then U1T = inv1 A1T
    View U1T = A.sub(k2, kc, b1, c_rest);
    if ((rc = gemm(ctx, U1T, A.sub(k2, k, b1, b0), false, U0T, false, -1.0, 1.0))) return rc;
    if ((rc = gemm(ctx, U1T, View{inv_b, b1, b1, 128}, false, U1T, false, 1.0, 0.0))) return rc;
    // the rest: A[kc:m, kc:n] -= L[kc:m, k:kc] U[k:kc, kc:n]  (K = b0 + b1)
    const int rest_r = m - kc;
    if (rest_r > 0 && (rc = gemm(ctx, A.sub(kc, kc, rest_r, c_rest), A.sub(kc, k, rest_r, b0 + b1),
                                 false, A.sub(k, kc, b0 + b1, c_rest), false, -1.0, 1.0)))
      return rc;
  }
  // The reference's blocked path (mlen > nb, nb != 0) leaves the pivot entries past
  // min(rows, cols) inside the last block equal to that block's start row (lu.go:216-219).
  if (ref_nb > 0 && mn > ref_nb && npiv > mn) {
    int64_t k_last = 0;
    for (int64_t k = 0; k < m && k < n;) {
      k_last = k;
      k += (k + ref_nb > n) ? n - k : ref_nb;
    }
    const int64_t hi = std::min<int64_t>(npiv, k_last + ref_nb);
    if (hi > mn) {
      ProfScope ps;
      prof_begin(ctx, ps, MO_PROF_OTHER);
      fill_pivots_kernel<<<(unsigned)((hi - mn + 255) / 256), 256, 0, ctx->stream>>>(piv, mn, hi,
                                                                                     k_last);
      prof_end(ctx, ps, 0.0, 8.0 * (hi - mn));
    }
    MO_CUDA_TRY(cudaGetLastError());
  }
  return MO_OK;
}

}  // namespace mo
