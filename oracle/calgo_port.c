/*
 * oracle/calgo_port.c -- TEST INFRASTRUCTURE ONLY (the oracle), never product code.
 *
 * Plain-C restatement of the arithmetic of the reference's C kernels (hrautila/matops
 * calgo/) that lie on the GEMM / SYRK / TRSM / Cholesky / LU path.  The reference uses
 * SSE micro-kernels with packing buffers; this restatement keeps every semantic that
 * changes results (where beta is applied and how beta==0/1 are special-cased, alpha
 * applied after a blocked triangular solve, true division by pivots / diagonals, the
 * SYRK beta quirk) and replaces the micro-kernels by scalar loops.  Summation order
 * inside a dot product therefore differs from the SSE code; results agree to rounding.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load this code,
 * and only as the checker.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "calgo_iface.h"

#define MAX_VP_ROWS 196 /* calgo/cmops.h:28 */
#define MAX_VP_COLS 68  /* calgo/cmops.h:29 */

#define AT(M, i, j) ((M)->md[(long)(i) + (long)(j) * (M)->step])

/* calgo/vec_scale.c:114-140 (dscale_tile): f==1 -> untouched, f==0 -> zeros, else scale */
static void scale_tile(double *X, int ldX, double f, int M, int N) {
  if (f == 1.0) return;
  for (int j = 0; j < N; j++)
    for (int i = 0; i < M; i++) X[i + (long)j * ldX] = (f == 0.0) ? 0.0 : X[i + (long)j * ldX] * f;
}

/* calgo/vec_scale.c:94-111 (dscale_vec) */
static void scale_vec(double *X, int inc, double f, int N) {
  if (f == 1.0) return;
  for (int i = 0; i < N; i++) X[(long)i * inc] = (f == 0.0) ? 0.0 : X[(long)i * inc] * f;
}

static inline double opA(const mdata_t *A, int flags, int i, int p) {
  return (flags & MTX_TRANSA) ? AT(A, p, i) : AT(A, i, p);
}
static inline double opB(const mdata_t *B, int flags, int p, int j) {
  return (flags & MTX_TRANSB) ? AT(B, j, p) : AT(B, p, j);
}

/* C[R:E, S:L] += alpha * sum_{p in [p0,p1)} opA(i,p) opB(p,j), one partial sum per panel
 * (calgo/dmmat_gemm.c:309-360, the panel step _dblock_mult_gepp) */
static void panel_update(mdata_t *C, const mdata_t *A, const mdata_t *B, double alpha, int flags,
                         int p0, int p1, int S, int L, int R, int E) {
  for (int j = S; j < L; j++)
    for (int i = R; i < E; i++) {
      double s = 0.0;
      for (int p = p0; p < p1; p++) s += opA(A, flags, i, p) * opB(B, flags, p, j);
      AT(C, i, j) += alpha * s;
    }
}

/* calgo/dmmat_gemm.c:364-415: C = beta*C + alpha*op(A)*op(B) on rows [R,E) and columns
 * [S,L); beta is applied per NB column block before its k-panels of length vlen. */
void dmult_mm_blocked3(mdata_t *C, const mdata_t *A, const mdata_t *B, double alpha,
                       double beta, int flags, int P, int S, int L, int R, int E, int vlen,
                       int NB, int MB) {
  (void)MB;
  if (L - S <= 0 || E - R <= 0) return;
  if (NB > MAX_VP_ROWS || NB <= 0) NB = MAX_VP_ROWS;
  if (vlen > MAX_VP_ROWS || vlen <= 0) vlen = MAX_VP_ROWS;
  for (int j = S; j < L; j += NB) {
    int nJ = L - j < NB ? L - j : NB;
    scale_tile(&AT(C, R, j), C->step, beta, E - R, nJ);
    for (int k = 0; k < P; k += vlen) {
      int nP = P - k < vlen ? P - k : vlen;
      panel_update(C, A, B, alpha, flags, k, k + nP, j, j + nJ, R, E);
    }
  }
}

/* calgo/dmmat_rank.c:62-127 (dmmat_rank_blk) with _dmmat_rank_diag (:18-57).
 * Diagonal NB x NB blocks: the triangle (upper if flags&UPPER, else lower) gets
 * beta*C + alpha*op(A)op(A)^T.  Off-diagonal blocks (left of the diagonal block when
 * flags&LOWER, right of it otherwise) get alpha*... added WITHOUT beta: the reference
 * applies beta only inside the diagonal blocks, so only beta==1 gives BLAS SYRK. */
void dmmat_rank_blk(mdata_t *C, const mdata_t *A, double alpha, double beta, int flags, int P,
                    int S, int E, int vlen, int NB) {
  (void)vlen;
  if (E - S <= 0 || P <= 0) return;
  if (NB > MAX_VP_COLS || NB <= 0) NB = MAX_VP_COLS;
  if (NB > E - S) NB = E - S;
  /* op(A)(i,p): A(i,p) normally, A(p,i) with TRANSA; C += alpha*op(A)*op(A)^T */
  int ta = flags & MTX_TRANSA ? MTX_TRANSA : 0;
  for (int i = S; i < E; i += NB) {
    int nI = E - i < NB ? E - i : NB;
    /* 1. diagonal block, row by row (dmmat_rank.c:28-56) */
    for (int r = 0; r < nI; r++) {
      int c0 = (flags & MTX_UPPER) ? r : 0;
      int c1 = (flags & MTX_UPPER) ? nI : r + 1;
      for (int c = c0; c < c1; c++) {
        double *cij = &AT(C, i + r, i + c);
        *cij = (beta == 1.0) ? *cij : (beta == 0.0 ? 0.0 : *cij * beta);
        double s = 0.0;
        for (int p = 0; p < P; p++) s += opA(A, ta, i + r, p) * opA(A, ta, i + c, p);
        *cij += alpha * s;
      }
    }
    /* 2. off-diagonal block (dmmat_rank.c:96-104 / :113-121), no beta */
    int cs = (flags & MTX_LOWER) ? 0 : i + nI;
    int ce = (flags & MTX_LOWER) ? i : E;
    for (int c = cs; c < ce; c++)
      for (int r = 0; r < nI; r++) {
        double s = 0.0;
        for (int p = 0; p < P; p++) s += opA(A, ta, i + r, p) * opA(A, ta, c, p);
        AT(C, i + r, c) += alpha * s;
      }
  }
}

/* Triangular solves on B's columns [S,E) (LEFT) or rows [S,E) (RIGHT) with the N x N
 * triangle of A.  calgo/dmmat_solve.c:864-908 dispatches to eight blocked variants
 * (:464-862) that solve with alpha == 1 and scale by alpha at the end; the diagonal
 * is divided (not multiplied by a reciprocal) unless UNIT (e.g. :171, :203).
 * Upper is chosen iff flags&UPPER, right side iff flags&RIGHT. */
void dmmat_solve_blk(mdata_t *B, const mdata_t *A, double alpha, int flags, int N, int S, int E,
                     int NB) {
  (void)NB;
  if (E - S <= 0) return;
  int unit = flags & MTX_UNIT, upper = flags & MTX_UPPER, tr = flags & MTX_TRANSA;
  /* effective triangle of op(A): lower unless (upper xor trans) */
  int lower_eff = upper ? (tr != 0) : (tr == 0);
#define OPA(i, j) (tr ? AT(A, j, i) : AT(A, i, j))
  if (flags & MTX_RIGHT) {
    /* X * op(A) = B, rows r in [S,E): x_j = (b_j - sum_{k} x_k opA(k,j)) / opA(j,j) */
    for (int r = S; r < E; r++) {
      if (lower_eff) {
        /* op(A) lower: column j depends on k > j -> go backwards */
        for (int j = N - 1; j >= 0; j--) {
          double s = AT(B, r, j);
          for (int k = j + 1; k < N; k++) s -= AT(B, r, k) * OPA(k, j);
          AT(B, r, j) = unit ? s : s / OPA(j, j);
        }
      } else {
        for (int j = 0; j < N; j++) {
          double s = AT(B, r, j);
          for (int k = 0; k < j; k++) s -= AT(B, r, k) * OPA(k, j);
          AT(B, r, j) = unit ? s : s / OPA(j, j);
        }
      }
    }
    if (alpha != 1.0)
      for (int j = 0; j < N; j++) scale_vec(&AT(B, S, j), 1, alpha, E - S);
  } else {
    /* op(A) X = B, columns c in [S,E) */
    for (int c = S; c < E; c++) {
      if (lower_eff) {
        for (int i = 0; i < N; i++) {
          double s = AT(B, i, c);
          for (int k = 0; k < i; k++) s -= OPA(i, k) * AT(B, k, c);
          AT(B, i, c) = unit ? s : s / OPA(i, i);
        }
      } else {
        for (int i = N - 1; i >= 0; i--) {
          double s = AT(B, i, c);
          for (int k = i + 1; k < N; k++) s -= OPA(i, k) * AT(B, k, c);
          AT(B, i, c) = unit ? s : s / OPA(i, i);
        }
      }
    }
    if (alpha != 1.0) scale_tile(&AT(B, 0, S), B->step, alpha, N, E - S);
  }
#undef OPA
}

/* calgo/dmvec_rank.c:239-262 (dmvec_symv_rank, SYR): for columns c in [S,L)
 * lower: rows c..L-1 ; upper: rows 0..c ; A(r,c) += x(r) * (alpha*x(c)) */
void dmvec_symv_rank(mdata_t *A, const mvec_t *X, double alpha, int flags, int S, int L,
                     int NB) {
  (void)NB;
  if (L - S <= 0) return;
  for (int c = S; c < L; c++) {
    double cf = alpha * X->md[(long)c * X->inc];
    int r0 = (flags & MTX_UPPER) ? 0 : c;
    int r1 = (flags & MTX_UPPER) ? c + 1 : L;
    for (int r = r0; r < r1; r++) AT(A, r, c) += X->md[(long)r * X->inc] * cf;
  }
}

/* 0: the transposed GEMV scales y by beta once per MB-row block of A (the reference's
 * calgo/dmvec_gemv.c:368-395); 1: once in all (BLAS semantics, or_gemv_beta_once) */
static int gemv_beta_once = 0;
int or_gemv_beta_once(int on) {
  int old = gemv_beta_once;
  gemv_beta_once = on;
  return old;
}

/* calgo/dmvec_gemv.c:353-427 (dmult_gemv_blocked).  Non-transposed: per MB row block,
 * y = beta*y (dscale_vec semantics), then y += alpha*A[:,S:L]*x.  Transposed (y[R:E] +=
 * alpha*A[S:L,R:E]^T x[S:L]): per MB block of A's rows S..L-1 the WHOLE of y[R:E] is first
 * scaled by beta (calgo/dmvec_gemv.c:379-393), so y ends as beta^nblocks*y + ... when
 * beta != 1 and L-S > MB. */
void dmult_gemv_blocked(mvec_t *Y, const mdata_t *A, const mvec_t *X, double alpha, double beta,
                        int flags, int S, int L, int R, int E, int vlen, int MB) {
  (void)vlen;
  if (L - S <= 0 || E - R <= 0) return;
  if (flags & MTX_TRANSA) {
    if (MB <= 0) MB = L - S;
    for (int i = S; i < L; i += MB) {
      const int nI = L - i < MB ? L - i : MB;
      if (beta != 1.0 && (!gemv_beta_once || i == S))
        scale_vec(&Y->md[(long)R * Y->inc], Y->inc, beta, E - R);
      for (int r = R; r < E; r++) {
        double s = 0.0;
        for (int c = i; c < i + nI; c++) s += AT(A, c, r) * X->md[(long)c * X->inc];
        Y->md[(long)r * Y->inc] += alpha * s;
      }
    }
    return;
  }
  if (MB <= 0) MB = E - R;
  for (int i = R; i < E; i += MB) {
    int nI = E - i < MB ? E - i : MB;
    if (beta != 1.0) scale_vec(&Y->md[(long)i * Y->inc], Y->inc, beta, nI);
    for (int r = i; r < i + nI; r++) {
      double s = 0.0;
      for (int c = S; c < L; c++) s += AT(A, r, c) * X->md[(long)c * X->inc];
      Y->md[(long)r * Y->inc] += alpha * s;
    }
  }
}

/* calgo/dmvec_solve.c:165-222 (dmvec_solve_blocked, TRSV): forward substitution when
 * flags&LOWER, backward otherwise; TRANSA is not consulted by the reference. */
void dmvec_solve_blocked(mvec_t *X, const mdata_t *A, int flags, int N, int NB) {
  (void)NB;
  int unit = flags & MTX_UNIT;
  double *x = X->md;
  long inc = X->inc;
  if (flags & MTX_LOWER) {
    for (int i = 0; i < N; i++) {
      double s = x[i * inc];
      for (int k = 0; k < i; k++) s -= AT(A, i, k) * x[k * inc];
      x[i * inc] = unit ? s : s / AT(A, i, i);
    }
  } else {
    for (int i = N - 1; i >= 0; i--) {
      double s = x[i * inc];
      for (int k = i + 1; k < N; k++) s -= AT(A, i, k) * x[k * inc];
      x[i * inc] = unit ? s : s / AT(A, i, i);
    }
  }
}

/* calgo/dvec_util.c:46-67 (dvec_dot): alpha * sum x*y */
double dvec_dot(const mvec_t *X, const mvec_t *Y, double alpha, int N) {
  double s = 0.0;
  for (int i = 0; i < N; i++) s += X->md[(long)i * X->inc] * Y->md[(long)i * Y->inc];
  return alpha * s;
}

/* calgo/dvec_util.c:230-246 (dvec_invscal): x /= alpha, true division */
void dvec_invscal(mvec_t *X, double alpha, int N) {
  for (int i = 0; i < N; i++) X->md[(long)i * X->inc] /= alpha;
}

/* calgo/dvec_util.c:200-225 (dvec_swap) */
void dvec_swap(mvec_t *X, mvec_t *Y, int N) {
  for (int i = 0; i < N; i++) {
    double t = X->md[(long)i * X->inc];
    X->md[(long)i * X->inc] = Y->md[(long)i * Y->inc];
    Y->md[(long)i * Y->inc] = t;
  }
}

/* ---------------- the rest of the level-3 surface ---------------- */

/* element (i, j) of the symmetric matrix whose UPPER (flags & MTX_UPPER) or LOWER triangle A
 * stores (calgo/dmmat_symm.c:253-390 reads only that triangle) */
static inline double sym_at(const mdata_t *A, int flags, int i, int j) {
  const int up = (flags & MTX_UPPER) != 0;
  if (up ? i <= j : i >= j) return AT(A, i, j);
  return AT(A, j, i);
}

/* calgo/dmmat_symm.c:253-390 (dmult_symm_blocked2): C[R:E, S:L] = beta*C + alpha*A*B
 * without MTX_RIGHT, else beta*C + alpha*op(B)*A (op(B) = B^T with MTX_TRANSB); A (P x P)
 * symmetric.  With no side bit the reference's kernel mixes its two branches (the loop of
 * the right side, calgo/dmmat_symm.c:287, and the left-side diagonal-block product,
 * :239-244), which is A*B for orders up to its block size 68; this restatement gives A*B.
 * The left branch reads B untransposed whatever MTX_TRANSB says (the reference's kernel
 * never consults it there). */
void dmult_symm_blocked2(mdata_t *C, const mdata_t *A, const mdata_t *B, double alpha,
                         double beta, int flags, int P, int S, int L, int R, int E, int vlen,
                         int NB, int MB) {
  (void)vlen; (void)NB; (void)MB;
  if (L - S <= 0 || E - R <= 0) return;
  scale_tile(&AT(C, R, S), C->step, beta, E - R, L - S);
  for (int j = S; j < L; j++)
    for (int i = R; i < E; i++) {
      double s = 0.0;
      for (int p = 0; p < P; p++) {
        if (!(flags & MTX_RIGHT)) s += sym_at(A, flags, i, p) * AT(B, p, j);
        else s += ((flags & MTX_TRANSB) ? AT(B, p, i) : AT(B, i, p)) * sym_at(A, flags, p, j);
      }
      AT(C, i, j) += alpha * s;
    }
}

/* element (i, k) of op(A) for the triangular A of TRMM (flags: UPPER / LOWER, TRANSA, UNIT) */
static inline double tri_op(const mdata_t *A, int flags, int i, int k) {
  const int r = (flags & MTX_TRANSA) ? k : i, c = (flags & MTX_TRANSA) ? i : k;
  const int up = (flags & MTX_UPPER) != 0;
  if (up ? r > c : r < c) return 0.0;
  if (r == c && (flags & MTX_UNIT)) return 1.0;
  return AT(A, r, c);
}

/* calgo/dmmat_trid.c:780-830 (dmmat_trmm_blk): B = alpha*op(A)*B (columns S..E-1 of B) or
 * alpha*B*op(A) with MTX_RIGHT (rows S..E-1 of B); A is N x N triangular */
void dmmat_trmm_blk(mdata_t *B, const mdata_t *A, double alpha, int flags, int N, int S, int E,
                    int NB) {
  (void)NB;
  if (E - S <= 0 || N <= 0) return;
  double *t = malloc(sizeof(double) * N);
  for (int v = S; v < E; v++) {
    /* v: a column of B (left) or a row of B (right) */
    for (int i = 0; i < N; i++) {
      double s = 0.0;
      for (int k = 0; k < N; k++) {
        if (flags & MTX_RIGHT) s += AT(B, v, k) * tri_op(A, flags, k, i);
        else s += tri_op(A, flags, i, k) * AT(B, k, v);
      }
      t[i] = alpha * s;
    }
    for (int i = 0; i < N; i++) {
      if (flags & MTX_RIGHT) AT(B, v, i) = t[i];
      else AT(B, i, v) = t[i];
    }
  }
  free(t);
}

static inline int in_tri(int flags, int i, int j) {
  return (flags & MTX_UPPER) ? i <= j : i >= j;
}

/* calgo/dmmat_rank.c:132-235 (dmmat_rank2_blk): the triangle of C[S:E, S:E] gets
 * alpha*(A*B^T + B*A^T) (alpha*(A^T*B + B^T*A) with MTX_TRANSA).  beta is applied inside the
 * NB x NB diagonal blocks only (dmmat_rank.c:167, 196), and without MTX_TRANSA a second time
 * before the second product (dmmat_rank.c:228): the diagonal blocks become
 * beta^2 C + beta alpha A B^T + alpha B A^T there.  Off the diagonal blocks beta is not
 * applied.  NB as in dmmat_rank.c:146-154. */
void dmmat_rank2_blk(mdata_t *C, const mdata_t *A, const mdata_t *B, double alpha, double beta,
                     int flags, int P, int S, int E, int vlen, int NB) {
  (void)vlen;
  if (E - S <= 0 || P <= 0) return;
  if (NB > MAX_VP_COLS || NB <= 0) NB = MAX_VP_COLS;
  if (NB > E - S) NB = E - S;
  const int ta = (flags & MTX_TRANSA) != 0;
  for (int j = S; j < E; j++)
    for (int i = S; i < E; i++) {
      if (!in_tri(flags, i, j)) continue;
      double ab = 0.0, ba = 0.0;
      for (int p = 0; p < P; p++) {
        const double ai = ta ? AT(A, p, i) : AT(A, i, p), aj = ta ? AT(A, p, j) : AT(A, j, p);
        const double bi = ta ? AT(B, p, i) : AT(B, i, p), bj = ta ? AT(B, p, j) : AT(B, j, p);
        ab += ai * bj;
        ba += bi * aj;
      }
      const int diag = (i - S) / NB == (j - S) / NB;
      double c = AT(C, i, j);
      if (diag) c = (beta == 0.0) ? 0.0 : (beta == 1.0 ? c : beta * c);
      c += alpha * ab;
      if (diag && !ta) c = (beta == 0.0) ? 0.0 : (beta == 1.0 ? c : beta * c);
      c += alpha * ba;
      AT(C, i, j) = c;
    }
}

/* calgo/dmmat_rank.c:292-355 (dmmat_trmupd_blk): the triangle of C[S:E, S:E] =
 * beta*C + alpha*op(A)*op(B), beta applied inside the NB x NB diagonal blocks only
 * (_dmmat_trmupd_diag); NB as in dmmat_rank.c:306-314 */
void dmmat_trmupd_blk(mdata_t *C, const mdata_t *A, const mdata_t *B, double alpha, double beta,
                      int flags, int P, int S, int E, int vlen, int NB) {
  (void)vlen;
  if (E - S <= 0 || P <= 0) return;
  if (NB > MAX_VP_COLS || NB <= 0) NB = MAX_VP_COLS;
  if (NB > E - S) NB = E - S;
  for (int j = S; j < E; j++)
    for (int i = S; i < E; i++) {
      if (!in_tri(flags, i, j)) continue;
      double s = 0.0;
      for (int p = 0; p < P; p++) s += opA(A, flags, i, p) * opB(B, flags, p, j);
      double c = AT(C, i, j);
      if ((i - S) / NB == (j - S) / NB) c = (beta == 0.0) ? 0.0 : (beta == 1.0 ? c : beta * c);
      AT(C, i, j) = c + alpha * s;
    }
}

/* calgo/dmvec_rank.c:128-148 (dmvec_rank): A[R:E, S:L] += alpha * x * y^T */
void dmvec_rank(mdata_t *A, const mvec_t *X, const mvec_t *Y, double alpha, int S, int L, int R,
                int E, int NB, int MB) {
  (void)NB; (void)MB;
  for (int j = S; j < L; j++) {
    const double yj = Y->md[(long)j * Y->inc];
    for (int i = R; i < E; i++) AT(A, i, j) += alpha * X->md[(long)i * X->inc] * yj;
  }
}

/* calgo/dvec_util.c:250-264 (dvec_scal): X *= alpha */
void dvec_scal(mvec_t *X, double alpha, int N) {
  for (int i = 0; i < N; i++) X->md[(long)i * X->inc] *= alpha;
}

/* calgo/dvec_util.c:120-141 (dvec_nrm2): sqrt of the sum of squares, no scaling */
double dvec_nrm2(const mvec_t *X, int N) {
  double s = 0.0;
  for (int i = 0; i < N; i++) {
    const double x = X->md[(long)i * X->inc];
    s += x * x;
  }
  return sqrt(s);
}

/* calgo/dmmat_plus.c:86-116 (dmmat_scale_plus): A = alpha*A + beta*op(B) over rows R..E-1
 * and columns S..L-1 of A (op per MTX_TRANSB; with MTX_TRANSA the same on A^T); alpha == 0
 * does not read A */
void dmmat_scale_plus(mdata_t *A, const mdata_t *B, double alpha, double beta, int flags,
                      int S, int L, int R, int E) {
  if (L - S <= 0 || E - R <= 0) return;
  const int ta = (flags & MTX_TRANSA) != 0, tb = (flags & MTX_TRANSB) != 0;
  for (int j = S; j < L; j++)
    for (int i = R; i < E; i++) {
      /* element (i, j) of op_A(A) and of op_B(B) */
      double *a = ta ? &AT(A, j, i) : &AT(A, i, j);
      const double b = tb ? AT(B, j, i) : AT(B, i, j);
      *a = alpha == 0.0 ? beta * b : alpha * *a + beta * b;
    }
}

/* calgo/dmvec_trid.c:209-230 (dmvec_trid_unb): X = op(A)*X for the N x N upper (MTX_UPPER)
 * or lower triangle of A, unit diagonal with MTX_UNIT, op = transpose with MTX_TRANSA or
 * MTX_TRANS */
void dmvec_trid_unb(mvec_t *X, const mdata_t *A, int flags, int N) {
  if (N <= 0) return;
  const int unit = (flags & MTX_UNIT) != 0, upper = (flags & MTX_UPPER) != 0;
  const int tr = (flags & (MTX_TRANSA | MTX_TRANS)) != 0;
  double *x = X->md;
  const long inc = X->inc;
  /* effective upper: x_i depends on x_j with j >= i, so compute i upward */
  if (upper != tr) {
    for (int i = 0; i < N; i++) {
      double s = unit ? x[i * inc] : 0.0;
      for (int j = i + unit; j < N; j++) s += (upper ? AT(A, i, j) : AT(A, j, i)) * x[j * inc];
      x[i * inc] = s;
    }
  } else {
    for (int i = N - 1; i >= 0; i--) {
      double s = unit ? x[i * inc] : 0.0;
      for (int j = 0; j <= i - unit; j++) s += (upper ? AT(A, j, i) : AT(A, i, j)) * x[j * inc];
      x[i * inc] = s;
    }
  }
}

/* calgo/dmvec_rank.c:263-285 (dmvec_trmv_upd): columns S..L-1 of the lower (rows j..L-1) or,
 * with MTX_UPPER, upper (rows 0..j) triangle of A += alpha x y^T, as a_ij += x_i (alpha y_j) */
void dmvec_trmv_upd(mdata_t *A, const mvec_t *X, const mvec_t *Y, double alpha, int flags, int S,
                    int L, int NB) {
  (void)NB;
  for (int j = S; j < L; j++) {
    const double cf = alpha * Y->md[(long)j * Y->inc];
    const int i0 = (flags & MTX_UPPER) ? 0 : j, i1 = (flags & MTX_UPPER) ? j + 1 : L;
    for (int i = i0; i < i1; i++) AT(A, i, j) += X->md[(long)i * X->inc] * cf;
  }
}
