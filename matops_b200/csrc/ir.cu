// Mixed-precision Cholesky solve with FP64 iterative refinement (mo_dsposv_ir).
//
// The factor L comes from lpchol.cu (split-product GEMMs on an FP32 copy of A).  Everything
// that decides the accuracy runs in FP64 on the device:
//   residual   r = b - A x      sym_apply_kernel reads only the stored triangle of A (or the
//                               GEMM engine on a full FP64 copy, for many right-hand sides)
//   correction d = M^-1 r       M = L L^T: two triangular solves with the FP32 L in FP64
//                               arithmetic, in 1024-row block steps (lpsolve.cu) from order
//                               kBlockSolveMinN, else 64-row steps (trsm_few.cu)
//              or d = GMRES(A, r) left-preconditioned by M^-1, restarted after
//                               kGmresMax iterations, classical Gram-Schmidt applied twice
//   update     x += d
//   stop       berr = |r|_inf / (|A|_inf |x|_inf + |b|_inf) <= tol (max over columns)
// Classic refinement converges while kappa(A) * u_factor << 1; GMRES-IR (Carson and
// Higham, SIAM J. Sci. Comput. 40 (2018) A817-A847) extends this to kappa(A) near
// u_factor^-2.  If the low-precision factorization meets a non-positive pivot, it is
// redone on A + s*diag(A) (the shift of Higham and Pranesh, SIAM J. Sci. Comput. 43 (2021)
// A258-A277) with s growing 8x per retry.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "lpchol.cuh"

namespace mo {
int potrf(mo_ctx *ctx, View A, bool upper, int *d_info, double *d_bad, double *inv);
int trsm_few_f32(mo_ctx *ctx, View B, const float *L, int64_t ldl, int N, bool trans,
                 const double *inv_L, int *flag_buf, const int *skip);

namespace {

constexpr int RR = 32;    // rows of A per CTA in sym_apply
constexpr int RT = 32;    // tile depth
constexpr int RQ = 256 / RR;  // depth groups per tile (threads per row)
constexpr int RD = RT / RQ;   // depth indices per group and tile
constexpr int RU = RT * RR / 256;  // tile elements per thread
constexpr int RNR = 16;   // right-hand sides per launch
static_assert(RR == 32 && RNR == 16 && RQ == 8, "sym_apply_kernel's thread layout");
constexpr int kGmresMax = 60;
constexpr int DOT_ROWS = 1024;

// Y = Bv + sa * op|A| X for symmetric A stored as its lower (UP == false) or upper
// triangle; ABS uses |A|.  CTA b owns rows r0 = RR b .. r0 + RR - 1.  It reads its row
// strip L(r0.., 0..r0+RR) (masked to j <= r) and its column strip L(r0.., r0..)^T (masked
// to i > r), so every stored element is read twice over the grid and never mirrored in
// memory.  Tiles are 32 deep, staged in shared memory from loads that are coalesced in
// either storage; the next tile is fetched into registers while the current one is used.
// Warp q accumulates RD of each tile's 32 depth indices, each thread a 4 x 4 block (4 rows,
// 4 right-hand sides) in registers; the RQ partial sums per row are added at the end in
// fixed order.
// 32-row strips give n / 32 CTAs (two or more per SM at the orders that matter).
struct SymArgs {
  const double *A;
  int64_t lda;
  int n;
  const double *X;
  int64_t ldx;
  const double *Bv;  // may be null (0)
  int64_t ldb;
  double *Y;
  int64_t ldy;
  int nr;
  double sa;
  const int *skip;  // optional: return at once when the word is set
};

template <bool UP, bool ABS>
__global__ void __launch_bounds__(256) sym_apply_kernel(SymArgs p) {
  if (p.skip && *(volatile const int *)p.skip) return;
  // the tile buffers and, after the last tile, the cross-q reduction share one block
  __shared__ __align__(16) double buf[RQ * RR * (RNR + 1) > RT * (RR + 2) + RT * (RNR + 2)
                                          ? RQ * RR * (RNR + 1)
                                          : RT * (RR + 2) + RT * (RNR + 2)];
  // even row strides: the products read their operands as 16-byte pairs (the tile stores
  // that walk down a column then meet 2-way bank conflicts, a few per thread and tile)
  double(*T)[RR + 2] = reinterpret_cast<double(*)[RR + 2]>(buf);
  double(*Xs)[RNR + 2] = reinterpret_cast<double(*)[RNR + 2]>(buf + RT * (RR + 2));
  double(*red)[RR][RNR + 1] = reinterpret_cast<double(*)[RR][RNR + 1]>(buf);
  // thread = (depth group q = warp, 4 rows 4 rq.., 4 right-hand sides 4 cq..)
  const int q = threadIdx.x >> 5, rq = threadIdx.x & 7, cq = (threadIdx.x >> 3) & 3;
  const int r0 = blockIdx.x * RR;
  const int n = p.n;
  const int t1 = (min(r0 + RR, n) + RT - 1) / RT;
  const int ntile = t1 + (n - r0 + RT - 1) / RT;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[i][c] = 0.0;
  double av[RU], xv[2];
  auto fetch = [&](int t) {
    const bool ph1 = t < t1;
    const int base = ph1 ? t * RT : r0 + (t - t1) * RT;
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int e = threadIdx.x + u * 256;
      int a, b;
      bool use;
      int row, col;
      if (ph1) {  // L(r0 + b, base + a), j <= r
        if (!UP) { b = e % RR; a = e / RR; } else { a = e % RT; b = e / RT; }
        row = r0 + b;
        col = base + a;
        use = row < n && col <= row;
      } else {    // L(base + a, r0 + b), i > r
        if (!UP) { a = e % RT; b = e / RT; } else { b = e % RR; a = e / RR; }
        row = base + a;
        col = r0 + b;
        use = row < n && col < n && row > col;
      }
      const double v = use ? (UP ? p.A[col + (int64_t)row * p.lda] : p.A[row + (int64_t)col * p.lda])
                           : 0.0;
      av[u] = ABS ? fabs(v) : v;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int e = threadIdx.x + u * 256;
      const int a = e % RT, c = e / RT;
      const int row = base + a;
      xv[u] = (row < n && c < p.nr) ? p.X[row + (int64_t)c * p.ldx] : 0.0;
    }
  };
  auto stash = [&](int t) {
    const bool ph1 = t < t1;
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int e = threadIdx.x + u * 256;
      int a, b;
      if (ph1) {
        if (!UP) { b = e % RR; a = e / RR; } else { a = e % RT; b = e / RT; }
      } else {
        if (!UP) { a = e % RT; b = e / RT; } else { b = e % RR; a = e / RR; }
      }
      T[a][b] = av[u];
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int e = threadIdx.x + u * 256;
      Xs[e % RT][e / RT] = xv[u];
    }
  };
  if (ntile > 0) fetch(0);
  for (int t = 0; t < ntile; ++t) {
    __syncthreads();  // the previous tile is no longer read
    stash(t);
    __syncthreads();
    if (t + 1 < ntile) fetch(t + 1);
#pragma unroll
    for (int jj = 0; jj < RD; ++jj) {
      const double2 a01 = *reinterpret_cast<const double2 *>(&T[RD * q + jj][4 * rq]);
      const double2 a23 = *reinterpret_cast<const double2 *>(&T[RD * q + jj][4 * rq + 2]);
      const double2 x01 = *reinterpret_cast<const double2 *>(&Xs[RD * q + jj][4 * cq]);
      const double2 x23 = *reinterpret_cast<const double2 *>(&Xs[RD * q + jj][4 * cq + 2]);
      const double a[4] = {a01.x, a01.y, a23.x, a23.y}, x[4] = {x01.x, x01.y, x23.x, x23.y};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[i][c] = fma(a[i], x[c], acc[i][c]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int c = 0; c < 4; ++c) red[q][4 * rq + i][4 * cq + c] = acc[i][c];
  __syncthreads();
  for (int e = threadIdx.x; e < RR * RNR; e += 256) {
    const int rr = e % RR, c = e / RR;
    const int row = r0 + rr;
    if (row < n && c < p.nr) {
      double s = red[0][rr][c];
#pragma unroll
      for (int qq = 1; qq < RQ; ++qq) s += red[qq][rr][c];
      const double b = p.Bv ? p.Bv[row + (int64_t)c * p.ldb] : 0.0;
      p.Y[row + (int64_t)c * p.ldy] = fma(p.sa, s, b);
    }
  }
}

// out[c] = max_r |V(r, c)| (out zeroed by the caller; non-negative doubles order like
// their bit patterns, so the maximum is exact and independent of the order)
__global__ void colmax_kernel(const double *V, int64_t ld, int n, int nr, double *out) {
  const int c = blockIdx.y;
  double m = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    m = fmax(m, fabs(V[r + (int64_t)c * ld]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0)
    atomicMax(reinterpret_cast<unsigned long long *>(out + c),
              (unsigned long long)__double_as_longlong(m));
}

// partial[blk * pstride + i * nr + c] = sum over rows of chunk blk of V_i(r, c) * W(r, c)
// (V_i = V + i * vstride, all n x nr with leading dimension n)
__global__ void __launch_bounds__(256) dots_kernel(const double *V, int64_t vstride, int nv,
                                                   const double *W, int n, int nr,
                                                   double *partial, int pstride,
                                                   const int *skip) {
  if (skip && *(volatile const int *)skip) return;
  __shared__ double s[8][kGmresMax + 2];
  const int c = blockIdx.y, blk = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double w[4];
  int rows[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    rows[k] = blk * DOT_ROWS + threadIdx.x + 256 * k;
    w[k] = rows[k] < n ? W[rows[k] + (int64_t)c * n] : 0.0;
  }
  for (int i = 0; i < nv; ++i) {
    const double *vi = V + i * vstride + (int64_t)c * n;
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (rows[k] < n) t = fma(vi[rows[k]], w[k], t);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) s[warp][i] = t;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nv; i += 256) {
    double t = 0.0;
    for (int w8 = 0; w8 < 8; ++w8) t += s[w8][i];
    partial[(size_t)blk * pstride + i * nr + c] = t;
  }
}

// h[i * nr + c] (+)= sum over chunks (fixed order); with `root`, h = sqrt of the sum
__global__ void dots_reduce_kernel(const double *partial, int pstride, int nblk, int nv, int nr,
                                   double *h, bool root, const int *skip) {
  if (skip && *(volatile const int *)skip) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nv * nr) return;
  double t = 0.0;
  for (int b = 0; b < nblk; ++b) t += partial[(size_t)b * pstride + e];
  h[e] = root ? sqrt(t) : t;
}

// W(r, c) += sign * sum_{i < nv} V_i(r, c) * h[i * nr + c]
__global__ void vupdate_kernel(double *W, const double *V, int64_t vstride, int nv,
                               const double *h, int n, int nr, double sign, const int *skip) {
  if (skip && *(volatile const int *)skip) return;
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= n) return;
  double t = 0.0;
  for (int i = 0; i < nv; ++i) t = fma(V[i * vstride + r + (int64_t)c * n], h[i * nr + c], t);
  W[r + (int64_t)c * n] = fma(sign, t, W[r + (int64_t)c * n]);
}

// dst(r, c) = src(r, c) / s[c]  (0 where s[c] == 0)
__global__ void vscale_kernel(double *dst, const double *src, const double *s, int n, int nr,
                              const int *skip) {
  if (skip && *(volatile const int *)skip) return;
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= n) return;
  const double d = s[c];
  dst[r + (int64_t)c * n] = d > 0.0 ? src[r + (int64_t)c * n] / d : 0.0;
}

// copy between an n x nr view (ld) and a packed n x nr block (ld n)
__global__ void vcopy_kernel(double *dst, int64_t ldd, const double *src, int64_t lds, int n,
                             int nr) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r < n && c < nr) dst[r + (int64_t)c * ldd] = src[r + (int64_t)c * lds];
}

__global__ void vfill_kernel(double *dst, double v, int64_t count) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < count) dst[e] = v;
}

// S = the symmetric matrix whose lower (UP == false) or upper triangle A stores, written in
// full (n x n, ld n); 32 x 32 tiles through shared memory so both the reads of the stored
// triangle and the mirrored writes are coalesced
template <bool UP>
__global__ void sym_full_kernel(const double *A, int64_t lda, int n, double *S) {
  __shared__ double T[32][33];
  const int bi = blockIdx.x, bj = blockIdx.y;  // tile row, tile column of S
  if (UP ? bi > bj : bi < bj) return;          // tiles on the stored side write both copies
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int r = ty; r < 32; r += 8) {
    const int i = bi * 32 + tx, j = bj * 32 + r;
    double v = 0.0;
    if (i < n && j < n) {
      const bool stored = UP ? i <= j : i >= j;
      v = stored ? A[i + (int64_t)j * lda] : A[j + (int64_t)i * lda];
    }
    T[r][tx] = v;
    if (i < n && j < n) S[i + (int64_t)j * n] = v;
  }
  if (bi == bj) return;
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {  // mirrored tile: S(j, i) = S(i, j)
    const int i = bj * 32 + tx, j = bi * 32 + r;
    if (i < n && j < n) S[i + (int64_t)j * n] = T[tx][r];
  }
}

// out[j] = sum_i |S(i, j)| (= the row sums, S symmetric); one CTA per column
__global__ void __launch_bounds__(256) abs_colsum_kernel(const double *S, int n, double *out) {
  __shared__ double red[8];
  const int j = blockIdx.x;
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) t += fabs(S[i + (int64_t)j * n]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0.0;
    for (int w = 0; w < 8; ++w) u += red[w];
    out[j] = u;
  }
}


// GMRES bookkeeping on the device, one thread per right-hand side c (column-major state,
// LDR = kGmresMax + 1 rows per Hessenberg column):
//   column j of the Hessenberg matrix = h1 + h2 (the two Gram-Schmidt passes) and |w|,
//   the earlier Givens rotations applied to it, a new rotation zeroing its subdiagonal, and
//   g (the rotated right-hand side) updated; |g[j+1]| / beta is the preconditioned residual
//   ratio.  When the largest ratio is <= tau (or j is the last iteration), *done := 1 and
//   *m := j + 1.  Nothing happens once *done is set.
struct GmresState {
  double *R;      // nr x kGmresMax x LDR
  double *cs, *sn;  // nr x kGmresMax
  double *g;      // nr x LDR
  double *beta;   // nr
  int *done;      // [0] done flag, [1] iterations used
};
constexpr int LDR = kGmresMax + 1;

__global__ void __launch_bounds__(256) gmres_start_kernel(GmresState st, const double *beta, int nr) {
  for (int c = threadIdx.x; c < nr; c += blockDim.x) {
    st.beta[c] = beta[c];
    st.g[(size_t)c * LDR] = beta[c];
    for (int i = 1; i < LDR; ++i) st.g[(size_t)c * LDR + i] = 0.0;
  }
  if (threadIdx.x == 0) {
    st.done[0] = 0;
    st.done[1] = 0;
  }
}

__global__ void __launch_bounds__(256) gmres_givens_kernel(GmresState st, const double *h1,
                                                          const double *h2, const double *hn,
                                                          int j, int nr, double tau, int last) {
  if (*(volatile const int *)st.done) return;
  __shared__ double red[256];
  double worst = 0.0;
  for (int c = threadIdx.x; c < nr; c += blockDim.x) {
    double *Rc = st.R + ((size_t)c * kGmresMax + j) * LDR;
    double *cs = st.cs + (size_t)c * kGmresMax, *sn = st.sn + (size_t)c * kGmresMax;
    double *g = st.g + (size_t)c * LDR;
    for (int i = 0; i <= j; ++i) Rc[i] = h1[(size_t)i * nr + c] + h2[(size_t)i * nr + c];
    Rc[j + 1] = hn[c];
    for (int i = 0; i < j; ++i) {
      const double a = Rc[i], b = Rc[i + 1];
      Rc[i] = cs[i] * a + sn[i] * b;
      Rc[i + 1] = -sn[i] * a + cs[i] * b;
    }
    const double a = Rc[j], b = Rc[j + 1];
    const double rr = hypot(a, b);
    const double cc = rr > 0.0 ? a / rr : 1.0, ss = rr > 0.0 ? b / rr : 0.0;
    cs[j] = cc;
    sn[j] = ss;
    Rc[j] = rr;
    Rc[j + 1] = 0.0;
    const double gj = g[j];
    g[j + 1] = -ss * gj;
    g[j] = cc * gj;
    if (st.beta[c] > 0.0) worst = fmax(worst, fabs(g[j + 1]) / st.beta[c]);
  }
  red[threadIdx.x] = worst;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0 && (red[0] <= tau || last)) {
    st.done[1] = j + 1;
    st.done[0] = 1;
  }
}

// y = R^-1 g (m x m upper triangular per column), written as h[i * nr + c]
__global__ void __launch_bounds__(256) gmres_backsolve_kernel(GmresState st, int m, int nr,
                                                             double *y) {
  for (int c = threadIdx.x; c < nr; c += blockDim.x) {
    const double *g = st.g + (size_t)c * LDR;
    for (int i = m - 1; i >= 0; --i) {
      double t = g[i];
      for (int k = i + 1; k < m; ++k)
        t -= st.R[((size_t)c * kGmresMax + k) * LDR + i] * y[(size_t)k * nr + c];
      const double dii = st.R[((size_t)c * kGmresMax + i) * LDR + i];
      y[(size_t)i * nr + c] = dii != 0.0 ? t / dii : 0.0;
    }
  }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------

struct Solver {
  mo_ctx *ctx;
  View A;
  bool upper;
  int n, nr;  // nr: right-hand sides (all columns)
  LpChol f;
  double *b, *x, *r, *d;  // n x nr packed
  double *V;              // (kGmresMax + 1) blocks of n x nr
  double *h, *h2;         // Gram-Schmidt coefficients, (kGmresMax + 1) x nr each
  double *scal;           // per-column scalars (nr)
  double *partial;        // dot partial sums
  double *norms;          // [0, nr): |r|, [nr, 2nr): |x|, [2nr, 3nr): |b|, 3nr: |A|
  int *flags;             // trsm_few block flags
  GmresState gs;          // device-side Hessenberg, rotations and convergence words
  const int *skip = nullptr;  // set while GMRES iterations run: their convergence word
  int nblk_dot, pstride;
  double *S = nullptr;    // full symmetric copy of A (many right-hand sides only)
  LpSolve ls;             // block solves with the factor (orders >= kBlockSolveMinN)
  bool blocked = false;
};

// from this order on the refinement solves take n / 1024 block steps (lpsolve.cu) instead
// of the few-RHS kernel's n / 64 dependent steps
constexpr int kBlockSolveMinN = 2048;

// products with A through the FP64 GEMM engine on the symmetric copy pay off above this
// many right-hand sides (one 128-column tile pass against a 16-column pass per group)
constexpr int kGemmResidualMinRhs = 33;

dim3 vgrid(int n, int nr) { return dim3((n + 255) / 256, nr); }

int sym_apply(Solver &s, const double *X, int64_t ldx, const double *Bv, double *Y, double sa,
              bool abs_a, int nr) {
  mo_ctx *ctx = s.ctx;
  if (s.S) {
    if (abs_a) {  // row sums of |A| (X is the ones vector)
      ProfScope ps;
      prof_begin(ctx, ps, MO_PROF_IR);
      abs_colsum_kernel<<<s.n, 256, 0, ctx->stream>>>(s.S, s.n, Y);
      prof_end(ctx, ps, (double)s.n * s.n, 8.0 * s.n * (double)s.n);
      MO_CUDA_TRY(cudaGetLastError());
      return MO_OK;
    }
    if (Bv) {
      vcopy_kernel<<<vgrid(s.n, nr), 256, 0, ctx->stream>>>(Y, s.n, Bv, s.n, s.n, nr);
      MO_CUDA_TRY(cudaGetLastError());
    }
    const View Yv{Y, s.n, nr, s.n}, Sv{s.S, s.n, s.n, s.n},
        Xv{const_cast<double *>(X), s.n, nr, ldx};
    GemmOpts o;
    o.skip = s.skip;  // inside GMRES: iterations past convergence return at once
    return gemm_ex(ctx, Yv, Sv, false, Xv, false, sa, Bv ? 1.0 : 0.0, o);
  }
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_IR);
  for (int c0 = 0; c0 < nr; c0 += RNR) {
    SymArgs p;
    p.A = s.A.d;
    p.lda = s.A.ld;
    p.n = s.n;
    p.X = X + (int64_t)c0 * ldx;
    p.ldx = ldx;
    p.Bv = Bv ? Bv + (int64_t)c0 * s.n : nullptr;
    p.ldb = s.n;
    p.Y = Y + (int64_t)c0 * s.n;
    p.ldy = s.n;
    p.nr = std::min(RNR, nr - c0);
    p.sa = sa;
    p.skip = s.skip;
    const int grid = (s.n + RR - 1) / RR;
    if (s.upper) {
      if (abs_a) sym_apply_kernel<true, true><<<grid, 256, 0, ctx->stream>>>(p);
      else sym_apply_kernel<true, false><<<grid, 256, 0, ctx->stream>>>(p);
    } else {
      if (abs_a) sym_apply_kernel<false, true><<<grid, 256, 0, ctx->stream>>>(p);
      else sym_apply_kernel<false, false><<<grid, 256, 0, ctx->stream>>>(p);
    }
  }
  prof_end(ctx, ps, 2.0 * s.n * (double)s.n * nr,
           8.0 * s.n * (double)s.n * ((nr + RNR - 1) / RNR) + 24.0 * s.n * nr);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

int colmax(Solver &s, const double *V, int64_t ld, int n, int nr, double *out) {
  MO_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double) * nr, s.ctx->stream));
  colmax_kernel<<<dim3(std::min(64, (n + 255) / 256), nr), 256, 0, s.ctx->stream>>>(V, ld, n,
                                                                                   nr, out);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// D = M^-1 D in place (D: packed n x nr): L^-1 then L^-T with the FP32 factor (FP64
// arithmetic): block solves for large orders, else the few-RHS kernel with right-hand
// sides in groups of 64
int precond(Solver &s, double *D) {
  if (s.blocked) return lp_solve_apply(s.ctx, s.ls, D, s.nr, s.skip);
  for (int c0 = 0; c0 < s.nr; c0 += 64) {
    const View B{D + (int64_t)c0 * s.n, s.n, std::min(64, s.nr - c0), s.n};
    int rc = trsm_few_f32(s.ctx, B, s.f.W, s.f.ldw, s.n, false, s.f.inv, s.flags, s.skip);
    if (!rc) rc = trsm_few_f32(s.ctx, B, s.f.W, s.f.ldw, s.n, true, s.f.inv, s.flags, s.skip);
    if (rc) return rc;
  }
  return MO_OK;
}

// h(0..nv-1, :) = V_0..nv-1^T W per column; root: h = sqrt(W^T W) (nv = 1, V = W)
int dots(Solver &s, const double *V, int nv, const double *W, double *h, bool root) {
  cudaStream_t st = s.ctx->stream;
  ProfScope ps;
  prof_begin(s.ctx, ps, MO_PROF_IR);
  dots_kernel<<<dim3(s.nblk_dot, s.nr), 256, 0, st>>>(V, (int64_t)s.n * s.nr, nv, W, s.n, s.nr,
                                                      s.partial, s.pstride, s.skip);
  const int m = nv * s.nr;
  dots_reduce_kernel<<<(m + 127) / 128, 128, 0, st>>>(s.partial, s.pstride, s.nblk_dot, nv, s.nr,
                                                      h, root, s.skip);
  prof_end(s.ctx, ps, 2.0 * s.n * (double)s.nr * nv, 8.0 * s.n * (double)s.nr * (nv + 1));
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

int vupdate(Solver &s, double *W, const double *V, int nv, const double *h, double sign) {
  ProfScope ps;
  prof_begin(s.ctx, ps, MO_PROF_IR);
  vupdate_kernel<<<vgrid(s.n, s.nr), 256, 0, s.ctx->stream>>>(W, V, (int64_t)s.n * s.nr, nv, h,
                                                              s.n, s.nr, sign, s.skip);
  prof_end(s.ctx, ps, 2.0 * s.n * (double)s.nr * nv, 8.0 * s.n * (double)s.nr * (nv + 2));
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// d = GMRES(A, r) preconditioned on the left by M^-1, at most kGmresMax iterations, until
// every column's preconditioned residual has dropped by tau; *its receives the iterations.
// The Hessenberg matrix, the Givens rotations and the convergence test live on the device
// (gmres_givens_kernel); the host enqueues iterations up to kGmresLag ahead of the last
// test it has seen (read through pinned memory and one event per iteration, without
// stopping the stream), and iterations enqueued past convergence return at once (their
// kernels test the same device word).
constexpr int kGmresLag = 2;

int gmres_slots(mo_ctx *ctx) {
  if (!ctx->h_gmres) MO_CUDA_TRY(cudaHostAlloc((void **)&ctx->h_gmres, 64 * sizeof(int) * 2, 0));
  while ((int)ctx->gmres_ev.size() < kGmresMax) {
    cudaEvent_t e;
    MO_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->gmres_ev.push_back(e);
  }
  return MO_OK;
}

// budget_s > 0: once the iterations completed so far took longer than budget_s seconds
// (host clock), the next one enqueued is the last
int gmres(Solver &s, double tau, int *its, double budget_s) {
  const auto t0 = std::chrono::steady_clock::now();
  const int n = s.n, nr = s.nr;
  const int64_t vs = (int64_t)n * nr;
  mo_ctx *ctx = s.ctx;
  cudaStream_t st = ctx->stream;
  int rc;
  if ((rc = gmres_slots(ctx))) return rc;
  MO_CUDA_TRY(cudaMemcpyAsync(s.d, s.r, sizeof(double) * vs, cudaMemcpyDeviceToDevice, st));
  if ((rc = precond(s, s.d))) return rc;
  if ((rc = dots(s, s.d, 1, s.d, s.scal, true))) return rc;  // beta = |M^-1 r|_2
  vscale_kernel<<<vgrid(n, nr), 256, 0, st>>>(s.V, s.d, s.scal, n, nr, nullptr);
  gmres_start_kernel<<<1, 256, 0, st>>>(s.gs, s.scal, nr);
  MO_CUDA_TRY(cudaGetLastError());
  int *hd = ctx->h_gmres;  // hd[2 j], hd[2 j + 1]: done word and count after iteration j
  s.skip = s.gs.done;
  int m = 0;
  bool final = false;
  for (int j = 0; j < kGmresMax; ++j) {
    // the convergence test of iteration j - kGmresLag, once the device has passed it
    if (j - kGmresLag >= 0) {
      const int q = j - kGmresLag;
      MO_CUDA_TRY(cudaEventSynchronize(ctx->gmres_ev[q]));
      if (hd[2 * q]) break;
      final = budget_s > 0.0 &&
              std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > budget_s;
    }
    double *vj = s.V + j * vs, *w = s.V + (j + 1) * vs;
    if ((rc = sym_apply(s, vj, n, nullptr, w, 1.0, false, nr))) return rc;  // w = A v_j
    if ((rc = precond(s, w))) return rc;                                     // w = M^-1 w
    // classical Gram-Schmidt, applied twice (h = h1 + h2)
    if ((rc = dots(s, s.V, j + 1, w, s.h, false))) return rc;
    if ((rc = vupdate(s, w, s.V, j + 1, s.h, -1.0))) return rc;
    if ((rc = dots(s, s.V, j + 1, w, s.h2, false))) return rc;
    if ((rc = vupdate(s, w, s.V, j + 1, s.h2, -1.0))) return rc;
    if ((rc = dots(s, w, 1, w, s.scal, true))) return rc;  // |w|_2
    vscale_kernel<<<vgrid(n, nr), 256, 0, st>>>(w, w, s.scal, n, nr, s.skip);
    gmres_givens_kernel<<<1, 256, 0, st>>>(s.gs, s.h, s.h2, s.scal, j, nr, tau,
                                           j == kGmresMax - 1 || final);
    MO_CUDA_TRY(cudaGetLastError());
    MO_CUDA_TRY(cudaMemcpyAsync(hd + 2 * j, s.gs.done, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    MO_CUDA_TRY(cudaEventRecord(ctx->gmres_ev[j], st));
    if (final) break;
  }
  s.skip = nullptr;
  MO_CUDA_TRY(cudaMemcpyAsync(hd, s.gs.done, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  MO_CUDA_TRY(cudaStreamSynchronize(st));
  m = hd[1];
  if (m <= 0) return MO_EDEVTIMEOUT;  // the last iteration always sets the count
  // y = R^-1 g per column (device), d = V y
  gmres_backsolve_kernel<<<1, 256, 0, st>>>(s.gs, m, nr, s.h);
  MO_CUDA_TRY(cudaGetLastError());
  MO_CUDA_TRY(cudaMemsetAsync(s.d, 0, sizeof(double) * vs, st));
  if ((rc = vupdate(s, s.d, s.V, m, s.h, 1.0))) return rc;
  *its = m;
  return MO_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// workspace bytes for order n, nr right-hand sides
size_t ir_bytes(int n, int nr, int prec, bool gmres_possible, int sms) {
  const size_t vec = align256((size_t)n * nr * 8);
  const int nblk_dot = (n + DOT_ROWS - 1) / DOT_ROWS;
  size_t b = align256(lp_chol_bytes(n, prec)) + 4 * vec;
  if (nr >= kGemmResidualMinRhs) b += align256((size_t)n * n * 8);
  if (n >= kBlockSolveMinN) b += align256(lp_solve_bytes(n, nr, sms));
  if (gmres_possible) b += (kGmresMax + 1) * vec;
  b += 2 * align256((size_t)(kGmresMax + 1) * nr * 8) + align256((size_t)nr * 8);
  if (gmres_possible)
    b += align256((size_t)nr * kGmresMax * (kGmresMax + 1) * 8) + 2 * align256((size_t)nr * kGmresMax * 8) +
         align256((size_t)nr * (kGmresMax + 1) * 8) + align256((size_t)nr * 8) + 256;
  b += align256((size_t)nblk_dot * (kGmresMax + 2) * nr * 8);
  b += align256((size_t)(3 * nr + 1) * 8) + align256((size_t)(128 * ((n + 63) / 64) + 64) * 4) + 4096;
  return b;
}

// The FP64 path (potrf + two triangular solves) for a copy of A; returns info like
// mo_decompose_chol
int fp64_solve(mo_ctx *ctx, const View &A, bool upper, const View &X, const double *b) {
  const int n = A.rows;
  double *tmp = nullptr;
  MO_CUDA_TRY(cudaMalloc(&tmp, (size_t)n * n * sizeof(double)));
  int rc = MO_OK;
  do {
    if (cudaMemcpy2DAsync(tmp, (size_t)n * 8, A.d, (size_t)A.ld * 8, (size_t)n * 8, n,
                          cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess) {
      rc = MO_ECUDA;
      break;
    }
    const View T{tmp, n, n, n};
    double *inv = nullptr;
    if ((rc = workspace(ctx, 128 * 128 * sizeof(double), (void **)&inv))) break;
    Control *cb = control(ctx);
    if (cudaMemsetAsync(&cb->info, 0, sizeof(Control) - offsetof(Control, info), ctx->stream) !=
        cudaSuccess) {
      rc = MO_ECUDA;
      break;
    }
    if ((rc = potrf(ctx, T, upper, &cb->info, &cb->bad, inv))) break;
    Control h;
    if (cudaMemcpy(&h, cb, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = MO_ECUDA;
      break;
    }
    if (h.info > 0) {
      rc = h.info;
      break;
    }
    vcopy_kernel<<<vgrid(n, X.cols), 256, 0, ctx->stream>>>(X.d, X.ld, b, n, n, X.cols);
    if (upper) {
      rc = trsm(ctx, X, T, MO_UPPER | MO_TRANSA, 1.0);
      if (!rc) rc = trsm(ctx, X, T, MO_UPPER, 1.0);
    } else {
      rc = trsm(ctx, X, T, MO_LOWER, 1.0);
      if (!rc) rc = trsm(ctx, X, T, MO_LOWER | MO_TRANSA, 1.0);
    }
    if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = MO_ECUDA;
  } while (false);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(tmp);
  return rc;
}

// berr per column from the device norms; returns the max (0 for all-zero columns)
double backward_error(Solver &s, std::vector<double> &nh) {
  double worst = 0.0;
  const double an = nh[3 * s.nr];
  for (int c = 0; c < s.nr; ++c) {
    const double den = an * nh[s.nr + c] + nh[2 * s.nr + c];
    const double e = den > 0.0 ? nh[c] / den : (nh[c] > 0.0 ? INFINITY : 0.0);
    worst = std::max(worst, e);
  }
  return worst;
}

int dsposv(mo_ctx *ctx, const View &X, const View &A, const View &B, bool upper, int prec,
           int method_flags, double tol, int maxit, mo_ir_info &info) {
  const int n = A.rows, nr = B.cols;
  const int method = method_flags & 0xff;
  const bool fallback_ok = (method_flags & MO_IR_NO_FALLBACK) == 0;
  cudaStream_t st = ctx->stream;
  Solver s;
  s.ctx = ctx;
  s.A = A;
  s.upper = upper;
  s.n = n;
  s.nr = nr;
  const bool gm = method != MO_IR_CLASSIC;
  // BF16x3 under MO_IR_AUTO may move to the TF32x3 factor (see below): room for either
  const bool may_switch = prec == kLpBf16x3 && method == MO_IR_AUTO;
  const int ws_prec = may_switch ? kLpTf32x3 : prec;
  const size_t need = ir_bytes(n, nr, ws_prec, gm, ctx->sms);
  if (need > ctx->ws_ir_bytes) {
    MO_CUDA_TRY(cudaStreamSynchronize(st));
    if (ctx->ws_ir) cudaFree(ctx->ws_ir);
    ctx->ws_ir = nullptr;
    ctx->ws_ir_bytes = 0;
    MO_CUDA_TRY(cudaMalloc(&ctx->ws_ir, need));
    ctx->ws_ir_bytes = need;
  }
  char *p = (char *)ctx->ws_ir;
  auto take = [&](size_t bytes) {
    char *r = p;
    p += align256(bytes);
    return r;
  };
  void *chol_mem = take(lp_chol_bytes(n, ws_prec));
  lp_chol_setup(n, prec, chol_mem, s.f);
  info.prec = prec == kLpBf16x3 ? MO_PREC_BF16X3 : MO_PREC_TF32X3;
  const size_t vec = (size_t)n * nr * 8;
  s.b = (double *)take(vec);
  s.x = (double *)take(vec);
  s.r = (double *)take(vec);
  s.d = (double *)take(vec);
  // GMRES basis: kGmresMax + 1 blocks of n x nr, packed with stride n * nr
  s.V = gm ? (double *)take((kGmresMax + 1) * align256(vec)) : nullptr;
  s.h = (double *)take((size_t)(kGmresMax + 1) * nr * 8);
  s.h2 = (double *)take((size_t)(kGmresMax + 1) * nr * 8);
  s.scal = (double *)take((size_t)nr * 8);
  if (gm) {
    s.gs.R = (double *)take((size_t)nr * kGmresMax * (kGmresMax + 1) * 8);
    s.gs.cs = (double *)take((size_t)nr * kGmresMax * 8);
    s.gs.sn = (double *)take((size_t)nr * kGmresMax * 8);
    s.gs.g = (double *)take((size_t)nr * (kGmresMax + 1) * 8);
    s.gs.beta = (double *)take((size_t)nr * 8);
    s.gs.done = (int *)take(256);
  }
  s.nblk_dot = (n + DOT_ROWS - 1) / DOT_ROWS;
  s.pstride = (kGmresMax + 2) * nr;
  s.partial = (double *)take((size_t)s.nblk_dot * s.pstride * 8);
  s.norms = (double *)take((size_t)(3 * nr + 1) * 8);
  s.flags = (int *)take((size_t)(128 * ((n + 63) / 64) + 64) * 4);
  if (n >= kBlockSolveMinN) {
    lp_solve_setup(n, nr, ctx->sms, take(lp_solve_bytes(n, nr, ctx->sms)), s.ls);
    s.blocked = true;
  }
  int rc;
  if (nr >= kGemmResidualMinRhs) s.S = (double *)take((size_t)n * n * 8);
  // The refinement's inputs -- the full symmetric FP64 copy of A (many right-hand sides),
  // b, |b|_inf and |A|_inf -- are memory-bound passes over A that nothing in the
  // factorization needs: they run on a third stream beside it and are joined before the
  // first refinement step.
  cudaStream_t side = nullptr;
  if ((rc = side_stream(ctx, &side))) return rc;
  if ((rc = stream_wait(ctx, side, st, ctx->ev_side_fork))) return rc;
  {
    StreamSwap sw(ctx, side);
    if (s.S) {
      const dim3 tg((n + 31) / 32, (n + 31) / 32);
      ProfScope ps;
      prof_begin(ctx, ps, MO_PROF_IR);
      if (upper) sym_full_kernel<true><<<tg, 256, 0, side>>>(A.d, A.ld, n, s.S);
      else sym_full_kernel<false><<<tg, 256, 0, side>>>(A.d, A.ld, n, s.S);
      prof_end(ctx, ps, 0.0, 8.0 * n * (double)n * 1.5);
      MO_CUDA_TRY(cudaGetLastError());
    }
    // b, |b|, |A|_inf (row sums of |A| through the same symmetric kernel, with x = 1)
    vcopy_kernel<<<vgrid(n, nr), 256, 0, side>>>(s.b, n, B.d, B.ld, n, nr);
    vfill_kernel<<<(n + 255) / 256, 256, 0, side>>>(s.d, 1.0, n);
    if ((rc = sym_apply(s, s.d, n, nullptr, s.r, 1.0, true, 1))) return rc;
    if ((rc = colmax(s, s.r, n, n, 1, s.norms + 3 * nr))) return rc;
    if ((rc = colmax(s, s.b, n, n, nr, s.norms + 2 * nr))) return rc;
  }
  // low-precision factorization, shifted on breakdown
  Control *cb = control(ctx);
  auto first_shift = [](int p) { return p == kLpBf16x3 ? 0x1p-15 : 0x1p-22; };
  double shift = 0.0;
  bool factored = false;
  double t_fact = 0.0;  // host seconds of the last factorization attempt
  for (int attempt = 0; attempt < 5; ++attempt) {
    const auto f0 = std::chrono::steady_clock::now();
    MO_CUDA_TRY(cudaMemsetAsync(&cb->info, 0, sizeof(Control) - offsetof(Control, info), st));
    if ((rc = lp_chol_convert(ctx, s.f, A, upper, shift)) ||
        (rc = lp_chol_factor(ctx, s.f, &cb->info, &cb->bad))) {
      stream_wait(ctx, st, side, ctx->ev_side_join);
      return rc;
    }
    Control h;
    MO_CUDA_TRY(cudaMemcpyAsync(&h, cb, sizeof(h), cudaMemcpyDeviceToHost, st));
    MO_CUDA_TRY(cudaStreamSynchronize(st));
    t_fact = std::chrono::duration<double>(std::chrono::steady_clock::now() - f0).count();
    if (h.status) {
      cudaMemset(&cb->status, 0, sizeof(int));
      stream_wait(ctx, st, side, ctx->ev_side_join);  // later work waits for the side stream
      return h.status;
    }
    if (h.info == 0) {
      factored = true;
      break;
    }
    if (may_switch && s.f.prec == kLpBf16x3) {
      // the BF16x3 factor (about 16 significant bits) broke down: kappa(A) is beyond what
      // it can precondition well, so refactor with the TF32x3 split (FP32 accuracy), unshifted
      lp_chol_setup(n, kLpTf32x3, chol_mem, s.f);
      info.prec = MO_PREC_TF32X3;
      shift = 0.0;
    } else {
      shift = shift == 0.0 ? first_shift(s.f.prec) : shift * 8.0;
    }
    info.shifts += 1;
  }
  info.shift = factored ? shift : 0.0;
  if ((rc = stream_wait(ctx, st, side, ctx->ev_side_join))) return rc;  // refinement inputs
  if (factored && s.blocked && (rc = lp_solve_prepare(ctx, s.f, s.ls))) return rc;
  std::vector<double> nh(3 * nr + 1);
  double prev = INFINITY;
  bool use_gmres = method == MO_IR_GMRES;
  int stall = 0;
  // the FP64 path (factor + solve) costs about kFp64OverLp times the split-product factor
  // (measured at n = 16384: 73.5 ms against about 20 ms); a refinement whose projected
  // remaining cost exceeds that is abandoned for the fallback
  constexpr double kFp64OverLp = 3.0;
  auto t_step0 = std::chrono::steady_clock::now();
  if (factored) {
    MO_CUDA_TRY(cudaMemsetAsync(s.x, 0, vec, st));
    for (int it = 0;; ++it) {
      if (it == 0) MO_CUDA_TRY(cudaMemcpyAsync(s.r, s.b, vec, cudaMemcpyDeviceToDevice, st));
      else if ((rc = sym_apply(s, s.x, n, s.b, s.r, -1.0, false, nr))) return rc;
      if ((rc = colmax(s, s.r, n, n, nr, s.norms))) return rc;
      if ((rc = colmax(s, s.x, n, n, nr, s.norms + nr))) return rc;
      MO_CUDA_TRY(cudaMemcpyAsync(nh.data(), s.norms, nh.size() * 8, cudaMemcpyDeviceToHost, st));
      MO_CUDA_TRY(cudaStreamSynchronize(st));
      const double berr = backward_error(s, nh);
      if (it < MO_IR_HISTORY) info.history[it] = berr;
      info.berr = berr;
      if (berr <= tol) {
        info.converged = 1;
        break;
      }
      if (it >= maxit || !std::isfinite(berr)) break;
      const auto now = std::chrono::steady_clock::now();
      const double t_step = std::chrono::duration<double>(now - t_step0).count();
      t_step0 = now;
      // GMRES-IR steps so far: project the steps still needed from the last reduction and
      // fall back once they would cost more than the FP64 path
      if (fallback_ok && method == MO_IR_AUTO && it > 0 && info.method == MO_IR_GMRES &&
          berr < prev) {
        const double need = std::ceil(std::log(tol / berr) / std::log(berr / prev));
        if (need * t_step > kFp64OverLp * t_fact) {
          info.abandoned = 1;
          break;
        }
      }
      // a step that did not reduce berr 20x: switch to GMRES-IR (auto), else count stalls.
      // A classic step that did not even reduce it 3x says kappa(A) u_factor is near 1: GMRES
      // would then need more iterations than the FP64 path costs (measured at n = 16384,
      // 16 right-hand sides: 25-27 iterations for a 0.42 reduction, 6-10 for 0.05-0.13), so
      // the auto mode goes to the fallback at once.
      if (it > 0 && berr > 0.05 * prev) {
        if (method == MO_IR_AUTO && !use_gmres) {
          if (fallback_ok && berr > 0.3 * prev) {
            info.abandoned = 1;
            break;
          }
          use_gmres = true;
        } else if (berr > 0.5 * prev && ++stall >= 2) {
          break;
        }
      }
      prev = berr;
      if (use_gmres) {
        int its = 0;
        // a GMRES step may take as long as the FP64 path would (then the refinement has at
        // most doubled the cost of solving in FP64 outright)
        const double budget = fallback_ok && method == MO_IR_AUTO ? kFp64OverLp * t_fact : 0.0;
        if ((rc = gmres(s, 1e-10, &its, budget))) return rc;
        info.gmres_iters += its;
        info.method = MO_IR_GMRES;
      } else {
        MO_CUDA_TRY(cudaMemcpyAsync(s.d, s.r, vec, cudaMemcpyDeviceToDevice, st));
        if ((rc = precond(s, s.d))) return rc;
        info.method = MO_IR_CLASSIC;
      }
      vfill_kernel<<<(nr + 255) / 256, 256, 0, st>>>(s.scal, 1.0, nr);
      // x += d  (as x += V_0 h with V_0 = d, h = 1 per column)
      if ((rc = vupdate(s, s.x, s.d, 1, s.scal, 1.0))) return rc;
      info.iters += 1;
    }
    MO_CUDA_TRY(cudaStreamSynchronize(st));
  }
  if (info.converged || (!fallback_ok && factored)) {
    vcopy_kernel<<<vgrid(n, nr), 256, 0, st>>>(X.d, X.ld, s.x, n, n, nr);
    MO_CUDA_TRY(cudaGetLastError());
    MO_CUDA_TRY(cudaStreamSynchronize(st));
    return MO_OK;
  }
  if (!fallback_ok) return MO_EINVAL;
  // FP64 factorization and solve
  info.fallback = 1;
  if ((rc = fp64_solve(ctx, A, upper, X, s.b)) != MO_OK) return rc;
  // report the backward error of the FP64 solution
  vcopy_kernel<<<vgrid(n, nr), 256, 0, st>>>(s.x, n, X.d, X.ld, n, nr);
  if ((rc = sym_apply(s, s.x, n, s.b, s.r, -1.0, false, nr))) return rc;
  if ((rc = colmax(s, s.r, n, n, nr, s.norms))) return rc;
  if ((rc = colmax(s, s.x, n, n, nr, s.norms + nr))) return rc;
  MO_CUDA_TRY(cudaMemcpyAsync(nh.data(), s.norms, nh.size() * 8, cudaMemcpyDeviceToHost, st));
  MO_CUDA_TRY(cudaStreamSynchronize(st));
  info.berr = backward_error(s, nh);
  info.converged = info.berr <= tol;
  return MO_OK;
}

}  // namespace
}  // namespace mo

extern "C" int mo_dsposv_ir(mo_ctx *ctx, mo_matrix Xm, mo_matrix Am, mo_matrix Bm, int flags,
                            int prec, int method, double tol, int maxit, mo_ir_info *info) {
  using namespace mo;
  int rc = enter(ctx);
  if (rc) return rc;
  View X, A, B;
  if ((rc = to_view(Xm, X)) || (rc = to_view(Am, A)) || (rc = to_view(Bm, B))) return rc;
  if (A.rows != A.cols) return MO_ENOTSQUARE;
  if (B.rows != A.rows || X.rows != B.rows || X.cols != B.cols) return MO_ESIZE;
  if (prec != MO_PREC_BF16X3 && prec != MO_PREC_TF32X3) return MO_EINVAL;
  const int m = method & 0xff;
  if (m != MO_IR_AUTO && m != MO_IR_CLASSIC && m != MO_IR_GMRES) return MO_EINVAL;
  if (maxit < 0 || !(tol >= 0.0)) return MO_EINVAL;
  mo_ir_info local;
  mo_ir_info &inf = info ? *info : local;
  std::memset(&inf, 0, sizeof(inf));
  if (A.rows == 0 || B.cols == 0) {
    inf.converged = 1;
    return MO_OK;
  }
  const int lp = prec == MO_PREC_BF16X3 ? kLpBf16x3 : kLpTf32x3;
  return dsposv(ctx, X, A, B, (flags & MO_UPPER) != 0, lp, method, tol, maxit, inf);
}
