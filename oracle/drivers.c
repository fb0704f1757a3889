/*
 * oracle/drivers.c -- TEST INFRASTRUCTURE ONLY (the oracle), never product code.
 *
 * C restatement of the Go layer of hrautila/matops on the level-3 / Cholesky / LU path:
 * the BLAS-3 wrappers of mmult.go (Mult with its goroutine worker split, SolveTrm,
 * RankUpdateSym), the level-1/2 wrappers of mvec.go used inside the panels, pivot.go,
 * chol.go and lu.go, with the FLAME partitioning of partition.go turned into index
 * arithmetic.  The same file is linked against oracle/calgo_port.c (this repository's
 * restatement of the C kernels) and against the reference's own calgo C files (oracle/_ref).
 *
 * A FloatMatrix view (hrautila/matrix, not vendored) is column-major storage with a
 * leading index; FloatArray()[0] is the view's (0,0) (inferred from mmult.go:228-233).
 *
 * Return codes mirror the Go error values: 0 = nil error, negative = the error string
 * listed at OR_E*, positive k+1 = the panic "illegal value at k" of chol.go:34-36.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include "calgo_iface.h"

enum {
  OR_OK = 0,
  OR_ESIZE = -1,        /* "Mult: size mismatch"             mmult.go:224 */
  OR_ENOTSQUARE = -2,   /* "A not a square matrix"           chol.go:119 */
  OR_EPIVLEN = -3,      /* "pivot array < min(A.Rows(),A.Cols())" lu.go:260-262 */
  OR_ECNOTSQUARE = -4,  /* "C not a square matrix"           mmult.go:428 */
  OR_EABSIZE = -5,      /* "A, B size mismatch"              mmult.go:406 */
  OR_ENOTVECTOR = -6,   /* "X not a vector." / "Y not a vector."  mvec.go:34-37 */
  OR_ESYMSIZE = -7      /* "MultSym: size mismatch"          mmult.go:290 */
};

/* package globals, mmult.go:33-41 */
static int vpLen = 196, nB = 68, mB = 68;
static int nWorker = 1;
static const int64_t limitOne = 200LL * 200 * 200;

typedef struct { double *d; int r, c, ld; } fm;

static inline fm sub(fm A, int i, int j, int nr, int nc) {
  fm s = {A.d + (intptr_t)i + (intptr_t)j * A.ld, nr, nc, A.ld};
  return s;
}
static inline fm sub2(fm A, int i, int j) { return sub(A, i, j, A.r - i, A.c - j); }
static inline int is_vector(fm X) { return X.r == 1 || X.c == 1; }
static inline int imin(int a, int b) { return a < b ? a : b; }

typedef struct { int64_t *p; int n; } pv;
static inline pv pslice(pv P, int a, int b) { pv s = {P.p + a, b - a}; return s; }

/* ---------------- mvec.go wrappers used by the panels ---------------- */

/* mvec.go:422-436 */
static void InvScale(fm X, double alpha) {
  int n = X.r * X.c;
  if (n == 0 || !is_vector(X)) return;
  mvec_t x = {X.d, X.c != 1 ? X.ld : 1};
  dvec_invscal(&x, alpha, n);
}

/* mvec.go:67-95 (MVRankUpdate): A += alpha * x * y^T for row or column vectors x, y */
static int MVRankUpdate(fm A, fm X, fm Y, double alpha) {
  if (A.r == 0 || A.c == 0) return OR_OK;
  if (!is_vector(Y) || !is_vector(X)) return OR_ENOTVECTOR;
  mdata_t a = {A.d, A.ld};
  mvec_t x = {X.d, X.r == 1 ? X.ld : 1}, y = {Y.d, Y.r == 1 ? Y.ld : 1};
  dmvec_rank(&a, &x, &y, alpha, 0, A.c, 0, A.r, 0, 0);
  return OR_OK;
}

/* mvec.go:439-453 (Scale) */
static void Scale(fm X, double alpha) {
  int n = X.r * X.c;
  if (n == 0 || !is_vector(X)) return;
  mvec_t x = {X.d, X.c != 1 ? X.ld : 1};
  dvec_scal(&x, alpha, n);
}

/* mvec.go:101-121 */
static int MVRankUpdateSym(fm A, fm X, double alpha, int flags) {
  if (A.r == 0 || A.c == 0) return OR_OK;
  if (!is_vector(X)) return OR_ENOTVECTOR;
  mdata_t a = {A.d, A.ld};
  mvec_t x = {X.d, X.r == 1 ? X.ld : 1};
  dmvec_symv_rank(&a, &x, alpha, flags, 0, A.c, nB);
  return OR_OK;
}

/* mvec.go:203-222 (alpha is not used by the reference) */
static int MVSolveTrm(fm X, fm A, double alpha, int flags) {
  (void)alpha;
  if (A.r == 0 || A.c == 0) return OR_OK;
  if (!is_vector(X)) return OR_ENOTVECTOR;
  mdata_t a = {A.d, A.ld};
  mvec_t x = {X.d, X.r == 1 ? X.ld : 1};
  dmvec_solve_blocked(&x, &a, flags, A.c, nB);
  return OR_OK;
}

/* mvec.go:28-60 */
static int MVMult(fm Y, fm A, fm X, double alpha, double beta, int flags) {
  if (A.r == 0 || A.c == 0) return OR_OK;
  if (!is_vector(Y) || !is_vector(X)) return OR_ENOTVECTOR;
  mdata_t a = {A.d, A.ld};
  mvec_t y = {Y.d, Y.r == 1 ? Y.ld : 1};
  mvec_t x = {X.d, X.r == 1 ? X.ld : 1};
  dmult_gemv_blocked(&y, &a, &x, alpha, beta, flags, 0, X.r * X.c, 0, Y.r * Y.c, vpLen, mB);
  return OR_OK;
}

/* mvec.go:274-297 with calgo/cmops.go:517-537 (N<=0 -> 0) */
static double Dot(fm X, fm Y, double alpha) {
  if (!is_vector(X) || !is_vector(Y)) return NAN;
  int n = X.r * X.c;
  if (n <= 0) return 0.0;
  mvec_t x = {X.d, X.c != 1 ? X.ld : 1};
  mvec_t y = {Y.d, Y.c != 1 ? Y.ld : 1};
  return dvec_dot(&x, &y, alpha, n);
}

/* mvec.go:456-482 */
static void Swap(fm X, fm Y) {
  if (X.r * X.c == 0 || Y.r * Y.c == 0) return;
  if (!is_vector(X) || !is_vector(Y)) return;
  mvec_t x = {X.d, X.c != 1 ? X.ld : 1};
  mvec_t y = {Y.d, Y.c != 1 ? Y.ld : 1};
  dvec_swap(&x, &y, X.r * X.c);
}

/* ---------------- pivot.go ---------------- */

/* pivot.go:27-35 */
static void swapRows(fm A, int src, int dst) {
  if (src == dst || A.r == 0) return;
  Swap(sub(A, src, 0, 1, A.c), sub(A, dst, 0, 1, A.c));
}

/* pivot.go:55-61: forward order, entries <= 0 skipped */
static void applyPivots(fm A, pv p) {
  for (int k = 0; k < p.n; k++)
    if (p.p[k] > 0) swapRows(A, (int)p.p[k], k);
}

/* pivot.go:98-107: first index of the strict maximum of |x|, scanning from row 0 */
static void pivotIndex(fm A, pv p) {
  double max = fabs(A.d[0]);
  for (int k = 1; k < A.r; k++) {
    double v = fabs(A.d[k]);
    if (v > max) {
      p.p[0] = k;
      max = v;
    }
  }
}

/* ---------------- mmult.go BLAS-3 wrappers ---------------- */

/* mmult.go:105-110 */
static int blockIndex4(int i, int r, int sz) {
  if (i == r) return sz;
  int v = (int)((int64_t)i * sz / r);
  return v - (v & 0x3);
}

/* mmult.go:137-167 */
static void divideWork(int rows, int cols, int workers, int *colW, int *rowW) {
  int nwsqrt = (int)sqrt((double)workers);
  int issquare = nwsqrt * nwsqrt == workers;
  if (workers == 2 || (workers & 0x1) != 0) {
    if (cols > rows) { *colW = workers; *rowW = 1; }
    else { *rowW = workers; *colW = 1; }
  } else if (issquare) {
    *colW = nwsqrt; *rowW = nwsqrt;
  } else {
    if (cols > rows) { *rowW = 2; *colW = workers / 2; }
    else { *colW = 2; *rowW = workers / 2; }
  }
}

typedef struct {
  mdata_t C, A, B;
  double alpha, beta;
  int flags, P, S, L, R, E;
} mult_task;

static void *mult_worker(void *arg) {
  mult_task *t = (mult_task *)arg;
  dmult_mm_blocked3(&t->C, &t->A, &t->B, t->alpha, t->beta, t->flags, t->P, t->S, t->L, t->R,
                    t->E, vpLen, nB, mB);
  return NULL;
}

/* mmult.go:198-256 */
int or_mult_fm(fm C, fm A, fm B, double alpha, double beta, int flags) {
  int ar = A.r, ac = A.c, br = B.r, bc = B.c, cr = C.r, cc = C.c, ok, empty;
  switch (flags & (MTX_TRANSA | MTX_TRANSB)) {
    case MTX_TRANSA | MTX_TRANSB: empty = ac == 0 || br == 0; ok = cr == ac && cc == br && ar == bc; break;
    case MTX_TRANSA: empty = ac == 0 || bc == 0; ok = cr == ac && cc == bc && ar == br; break;
    case MTX_TRANSB: empty = ar == 0 || br == 0; ok = cr == ar && cc == br && ac == bc; break;
    default: empty = ar == 0 || bc == 0; ok = cr == ar && cc == bc && ac == br;
  }
  if (empty) return OR_OK;
  if (!ok) return OR_ESIZE;
  int64_t psize = (int64_t)C.r * C.c * (int64_t)A.c;
  int P = (flags & MTX_TRANSA) ? A.r : A.c;
  mult_task base = {{C.d, C.ld}, {A.d, A.ld}, {B.d, B.ld}, alpha, beta, flags, P, 0, C.c, 0, C.r};
  if (nWorker <= 1 || psize <= limitOne) {
    mult_worker(&base);
    return OR_OK;
  }
  int colW, rowW;
  divideWork(C.r, C.c, nWorker, &colW, &rowW);
  int nt = colW * rowW;
  mult_task *tasks = (mult_task *)malloc(sizeof(mult_task) * nt);
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nt);
  int t = 0;
  /* mmult.go:171-188 (scheduleWork) */
  for (int k = 0; k < colW; k++)
    for (int l = 0; l < rowW; l++, t++) {
      tasks[t] = base;
      tasks[t].S = blockIndex4(k, colW, C.c);
      tasks[t].L = blockIndex4(k + 1, colW, C.c);
      tasks[t].R = blockIndex4(l, rowW, C.r);
      tasks[t].E = blockIndex4(l + 1, rowW, C.r);
      pthread_create(&th[t], NULL, mult_worker, &tasks[t]);
    }
  for (t = 0; t < nt; t++) pthread_join(th[t], NULL);
  free(tasks);
  free(th);
  return OR_OK;
}

/* mmult.go:388-422 */
int or_solve_trm_fm(fm B, fm A, double alpha, int flags) {
  int ok = 1, empty = 0, br = B.r, bc = B.c, ar = A.r, ac = A.c;
  switch (flags & (MTX_LEFT | MTX_RIGHT)) {
    case MTX_LEFT: empty = br == 0; ok = br == ac && ac == ar; break;
    case MTX_RIGHT: empty = bc == 0; ok = bc == ar && ac == ar; break;
  }
  if (empty) return OR_OK;
  if (!ok) return OR_EABSIZE;
  int E = (flags & MTX_RIGHT) ? br : bc;
  /* calgo/cmops.go:195-215 (DSolveBlk): N == 0 or an empty range returns */
  if (ac == 0 || E <= 0) return OR_OK;
  mdata_t b = {B.d, B.ld}, a = {A.d, A.ld};
  dmmat_solve_blk(&b, &a, alpha, flags, ac, 0, E, nB);
  return OR_OK;
}

/* mmult.go:426-445 */
int or_rank_update_sym_fm(fm C, fm A, double alpha, double beta, int flags) {
  if (C.r != C.c) return OR_ECNOTSQUARE;
  int P = (flags & MTX_TRANSA) ? A.r : A.c;
  /* calgo/cmops.go:219-240 (DSymmRankBlk) */
  if (P == 0 || C.r <= 0) return OR_OK;
  mdata_t c = {C.d, C.ld}, a = {A.d, A.ld};
  dmmat_rank_blk(&c, &a, alpha, beta, flags, P, 0, C.r, vpLen, nB);
  return OR_OK;
}

/* ---------------- the rest of mmult.go's level-3 surface ---------------- */

/* mmult.go:266-330 (MultSym); errors.New("MultSym: size mismatch") -> OR_ESYMSIZE */
int or_mult_sym_fm(fm C, fm A, fm B, double alpha, double beta, int flags) {
  int ok, empty;
  int ar = A.r, ac = A.c, br = B.r, bc = B.c, cr = C.r, cc = C.c;
  switch (flags & (MTX_TRANSA | MTX_TRANSB)) {
  case MTX_TRANSA | MTX_TRANSB:
    empty = ac == 0 || br == 0;
    ok = ar == ac && cr == ac && cc == br && ar == bc;
    break;
  case MTX_TRANSA:
    empty = ac == 0 || bc == 0;
    ok = ar == ac && cr == ac && cc == bc && ar == br;
    break;
  case MTX_TRANSB:
    empty = ar == 0 || br == 0;
    ok = ar == ac && cr == ar && cc == br && ac == bc;
    break;
  default:
    empty = ar == 0 || bc == 0;
    ok = ar == ac && cr == ar && cc == bc && ac == br;
  }
  if (empty) return OR_OK;
  if (!ok) return OR_ESYMSIZE;
  mdata_t c = {C.d, C.ld}, a = {A.d, A.ld}, b = {B.d, B.ld};
  /* the worker split of mmult.go:311-321 partitions C only; one call covers it */
  dmult_symm_blocked2(&c, &a, &b, alpha, beta, flags, A.c, 0, C.c, 0, C.r, vpLen, nB, mB);
  return OR_OK;
}

/* mmult.go:338-375 (MultTrm) */
int or_mult_trm_fm(fm B, fm A, double alpha, int flags) {
  int ok = 1, empty = 0;
  switch (flags & (MTX_LEFT | MTX_RIGHT)) {
  case MTX_LEFT:
    empty = B.r == 0 || B.c == 0;
    ok = B.r == A.c && A.c == A.r;
    break;
  case MTX_RIGHT:
    empty = B.c == 0 || B.r == 0;
    ok = B.c == A.r && A.c == A.r;
    break;
  }
  if (empty) return OR_OK;
  if (!ok) return OR_EABSIZE;
  int E = (flags & MTX_RIGHT) ? B.r : B.c;
  if (A.c == 0 || E <= 0) return OR_OK; /* calgo/cmops.go:153-155 */
  mdata_t b = {B.d, B.ld}, a = {A.d, A.ld};
  dmmat_trmm_blk(&b, &a, alpha, flags, A.c, 0, E, nB);
  return OR_OK;
}

/* mmult.go:453-475 (RankUpdate2Sym) */
int or_rank_update2_sym_fm(fm C, fm A, fm B, double alpha, double beta, int flags) {
  if (C.r != C.c) return OR_ECNOTSQUARE;
  int P = (flags & MTX_TRANSA) ? A.r : A.c;
  if (P == 0 || C.r == 0) return OR_OK; /* calgo/cmops.go:252-254 */
  mdata_t c = {C.d, C.ld}, a = {A.d, A.ld}, b = {B.d, B.ld};
  dmmat_rank2_blk(&c, &a, &b, alpha, beta, flags, P, 0, C.r, vpLen, nB);
  return OR_OK;
}

/* mmult.go:501-523 (UpdateTrm) */
int or_update_trm_fm(fm C, fm A, fm B, double alpha, double beta, int flags) {
  if (C.r != C.c) return OR_ECNOTSQUARE;
  int P = (flags & MTX_TRANSA) ? A.r : A.c;
  if (P == 0 || C.r == 0) return OR_OK; /* calgo/cmops.go:281-283 */
  mdata_t c = {C.d, C.ld}, a = {A.d, A.ld}, b = {B.d, B.ld};
  dmmat_trmupd_blk(&c, &a, &b, alpha, beta, flags, P, 0, C.r, vpLen, nB);
  return OR_OK;
}

/* ---------------- trinv.go ---------------- */

/* trinv.go:16-49 (unblockedInverseLower) */
static void unblockedInverseLower(fm A) {
  for (int k = 0; k < A.r; k++) {
    fm a10t = sub(A, k, 0, 1, k), a11 = sub(A, k, k, 1, 1);
    fm A20 = sub(A, k + 1, 0, A.r - k - 1, k), a21 = sub(A, k + 1, k, A.r - k - 1, 1);
    double aval = a11.d[0];
    InvScale(a21, -aval);
    MVRankUpdate(A20, a21, a10t, 1.0);
    InvScale(a10t, aval);
    a11.d[0] = 1.0 / aval;
  }
}

/* trinv.go:51-84 (unblockedInverseUpper) */
static void unblockedInverseUpper(fm A) {
  for (int k = 0; k < A.r; k++) {
    fm a01 = sub(A, 0, k, k, 1), a11 = sub(A, k, k, 1, 1);
    fm A02 = sub(A, 0, k + 1, k, A.c - k - 1), a12t = sub(A, k, k + 1, 1, A.c - k - 1);
    double aval = a11.d[0];
    InvScale(a12t, -aval);
    MVRankUpdate(A02, a01, a12t, 1.0);
    InvScale(a01, aval);
    a11.d[0] = 1.0 / aval;
  }
}

/* trinv.go:86-114 (unblockedInverseUnitLower) */
static void unblockedInverseUnitLower(fm A) {
  for (int k = 0; k < A.r; k++) {
    fm a10t = sub(A, k, 0, 1, k);
    fm A20 = sub(A, k + 1, 0, A.r - k - 1, k), a21 = sub(A, k + 1, k, A.r - k - 1, 1);
    Scale(a21, -1.0);
    MVRankUpdate(A20, a21, a10t, 1.0);
  }
}

/* trinv.go:116-144 (unblockedInverseUnitUpper) */
static void unblockedInverseUnitUpper(fm A) {
  for (int k = 0; k < A.r; k++) {
    fm a01 = sub(A, 0, k, k, 1);
    fm A02 = sub(A, 0, k + 1, k, A.c - k - 1), a12t = sub(A, k, k + 1, 1, A.c - k - 1);
    Scale(a12t, -1.0);
    MVRankUpdate(A02, a01, a12t, 1.0);
  }
}

/* trinv.go:146-181 (blockedInverseLower, libflame variant 3) */
static void blockedInverseLower(fm A, int flags, int nb) {
  for (int k = 0; k < A.r; ) {
    int b = (k + nb > A.c) ? A.c - k : nb; /* partition.go:252-254 */
    fm A10 = sub(A, k, 0, b, k), A11 = sub(A, k, k, b, b);
    fm A20 = sub(A, k + b, 0, A.r - k - b, k), A21 = sub(A, k + b, k, A.r - k - b, b);
    or_solve_trm_fm(A21, A11, -1.0, flags | MTX_RIGHT);
    or_mult_fm(A20, A21, A10, 1.0, 1.0, MTX_NOTRANS);
    or_solve_trm_fm(A10, A11, 1.0, flags);
    if (flags & MTX_UNIT) unblockedInverseUnitLower(A11);
    else unblockedInverseLower(A11);
    k += b;
  }
}

/* trinv.go:183-217 (blockedInverseUpper, libflame variant 1) */
static void blockedInverseUpper(fm A, int flags, int nb) {
  for (int k = 0; k < A.r; ) {
    int b = (k + nb > A.c) ? A.c - k : nb;
    fm A00 = sub(A, 0, 0, k, k), A01 = sub(A, 0, k, k, b), A11 = sub(A, k, k, b, b);
    or_mult_trm_fm(A01, A00, 1.0, flags);
    or_solve_trm_fm(A01, A11, -1.0, flags | MTX_RIGHT);
    if (flags & MTX_UNIT) unblockedInverseUnitUpper(A11);
    else unblockedInverseUpper(A11);
    k += b;
  }
}

/* trinv.go:219-243 (InverseTrm) */
int or_inverse_trm_fm(fm A, int flags, int nb) {
  if (nb == 0 || A.c < nb) {
    if (flags & MTX_UNIT) {
      if (flags & MTX_LOWER) unblockedInverseUnitLower(A);
      else unblockedInverseUnitUpper(A);
    } else {
      if (flags & MTX_LOWER) unblockedInverseLower(A);
      else unblockedInverseUpper(A);
    }
  } else {
    if (flags & MTX_LOWER) blockedInverseLower(A, flags, nb);
    else blockedInverseUpper(A, flags, nb);
  }
  return OR_OK;
}

/* ---------------- chol.go ---------------- */

/* chol.go:17-56 (unblockedCHOL); returns k+1 for the panic at absolute column k */
static int unblockedCHOL(fm A, int flags, int nr) {
  for (int k = 0; k < A.r; k++) {
    fm a11 = sub(A, k, k, 1, 1);
    double aval = sqrt(a11.d[0]);
    if (isnan(aval)) return nr + k + 1;
    a11.d[0] = aval;
    fm A22 = sub2(A, k + 1, k + 1);
    if (flags & MTX_LOWER) {
      fm a21 = sub(A, k + 1, k, A.r - k - 1, 1);
      InvScale(a21, aval);
      MVRankUpdateSym(A22, a21, -1.0, flags);
    } else {
      fm a12 = sub(A, k, k + 1, 1, A.c - k - 1);
      InvScale(a12, aval);
      MVRankUpdateSym(A22, a12, -1.0, flags);
    }
  }
  return OR_OK;
}

/* chol.go:58-94 (blockedCHOL), block steps whose first column k lies in [k0, k1) */
static int blockedCHOL_steps(fm A, int flags, int nb, int k0, int k1) {
  for (int k = k0; k < A.r && k < A.c && k < k1; ) {
    int b = (k + nb > A.c) ? A.c - k : nb;
    fm A11 = sub(A, k, k, b, b);
    int err = unblockedCHOL(A11, flags, k);
    if (err > 0) return err; /* the Go code panics here */
    fm A22 = sub2(A, k + b, k + b);
    if (flags & MTX_LOWER) {
      fm A21 = sub(A, k + b, k, A.r - k - b, b);
      or_solve_trm_fm(A21, A11, 1.0, MTX_RIGHT | MTX_LOWER | MTX_TRANSA);
      or_rank_update_sym_fm(A22, A21, -1.0, 1.0, MTX_LOWER);
    } else {
      fm A12 = sub(A, k, k + b, b, A.c - k - b);
      or_solve_trm_fm(A12, A11, 1.0, MTX_UPPER | MTX_TRANSA);
      or_rank_update_sym_fm(A22, A12, -1.0, 1.0, MTX_UPPER | MTX_TRANSA);
    }
    k += b;
  }
  return OR_OK;
}

static int blockedCHOL(fm A, int flags, int nb) {
  return blockedCHOL_steps(A, flags, nb, 0, A.c);
}

/* chol.go:116-127 */
int or_decompose_chol_fm(fm A, int flags, int nb) {
  if (A.c != A.r) return OR_ENOTSQUARE;
  if (A.c < nb || nb == 0) return unblockedCHOL(A, flags, 0);
  return blockedCHOL(A, flags, nb);
}

/* chol.go:147-158 */
void or_solve_chol_fm(fm B, fm A, int flags) {
  if (flags & MTX_UPPER) {
    or_solve_trm_fm(B, A, 1.0, MTX_UPPER | MTX_TRANSA);
    or_solve_trm_fm(B, A, 1.0, MTX_UPPER);
  } else if (flags & MTX_LOWER) {
    or_solve_trm_fm(B, A, 1.0, MTX_LOWER);
    or_solve_trm_fm(B, A, 1.0, MTX_LOWER | MTX_TRANSA);
  }
}

/* ---------------- lu.go ---------------- */

/* lu.go:103-171 (unblockedLUpiv): left-looking column step */
static int unblockedLUpiv(fm A, pv p) {
  int k = 0;
  for (; k < A.r && k < A.c; k++) {
    fm A00 = sub(A, 0, 0, k, k);
    fm a01 = sub(A, 0, k, k, 1);
    fm a10 = sub(A, k, 0, 1, k);
    fm a11 = sub(A, k, k, 1, 1);
    fm A20 = sub(A, k + 1, 0, A.r - k - 1, k);
    fm a21 = sub(A, k + 1, k, A.r - k - 1, 1);
    fm a1 = sub(A, 0, k, A.r, 1);
    pv p0 = pslice(p, 0, k);
    pv p1 = pslice(p, k, imin(k + 1, p.n));
    if (p1.n == 0) return OR_EPIVLEN; /* the Go code would index past the slice */

    applyPivots(a1, p0);
    MVSolveTrm(a01, A00, 1.0, MTX_LOWER | MTX_UNIT);
    a11.d[0] += Dot(a10, a01, -1.0);
    MVMult(a21, A20, a01, -1.0, 1.0, MTX_NOTRANS);

    fm aB1 = sub(A, k, k, A.r - k, 1);
    pivotIndex(aB1, p1);
    applyPivots(aB1, p1);
    InvScale(a21, a11.d[0]);
    fm AB0 = sub(A, k, 0, A.r - k, k);
    applyPivots(AB0, p1);
    p1.p[0] += k;
  }
  if (k < A.c) {
    fm ATR = sub(A, 0, k, k, A.c - k);
    fm ATL = sub(A, 0, 0, k, k);
    applyPivots(ATR, p);
    or_solve_trm_fm(ATR, ATL, 1.0, MTX_LEFT | MTX_UNIT | MTX_LOWER);
  }
  return OR_OK;
}

/* lu.go:173-231 (blockedLUpiv): left-looking (Crout) blocked variant */
static int blockedLUpiv(fm A, pv p, int nb) {
  int k = 0;
  while (k < A.r && k < A.c) {
    int b = (k + nb > A.c) ? A.c - k : nb;                  /* partition.go:252-254 */
    int pb = (k + nb > p.n) ? p.n - k : nb;                  /* partition.go:386-388 */
    fm A00 = sub(A, 0, 0, k, k);
    fm A01 = sub(A, 0, k, k, b);
    fm A10 = sub(A, k, 0, b, k);
    fm A11 = sub(A, k, k, b, b);
    fm A20 = sub(A, k + b, 0, A.r - k - b, k);
    fm A21 = sub(A, k + b, k, A.r - k - b, b);
    fm A1 = sub(A, 0, k, A.r, b);
    pv p0 = pslice(p, 0, k);
    pv p1 = pslice(p, k, k + pb);

    applyPivots(A1, p0);
    or_solve_trm_fm(A01, A00, 1.0, MTX_LOWER | MTX_UNIT);
    or_mult_fm(A11, A10, A01, -1.0, 1.0, MTX_NOTRANS);
    or_mult_fm(A21, A20, A01, -1.0, 1.0, MTX_NOTRANS);

    fm AB1 = sub(A, k, k, A.r - k, A11.c);
    unblockedLUpiv(AB1, p1);
    fm AB0 = sub(A, k, 0, A.r - k, k);
    applyPivots(AB0, p1);
    for (int i = 0; i < p1.n; i++) p1.p[i] += k;
    k += b;
  }
  if (k < A.c) {
    fm ATR = sub(A, 0, k, k, A.c - k);
    fm ATL = sub(A, 0, 0, k, k);
    applyPivots(ATR, p);
    or_solve_trm_fm(ATR, ATL, 1.0, MTX_LEFT | MTX_UNIT | MTX_LOWER);
  }
  return OR_OK;
}

/* lu.go:257-272 */
int or_decompose_lu_fm(fm A, pv p, int nb) {
  int mlen = imin(A.r, A.c);
  if (p.n < mlen) return OR_EPIVLEN;
  for (int k = 0; k < p.n; k++) p.p[k] = 0;
  if (mlen <= nb || nb == 0) return unblockedLUpiv(A, p);
  return blockedLUpiv(A, p, nb);
}

/* lu.go:320-331 */
int or_solve_lu_fm(fm B, fm A, pv p, int flags) {
  applyPivots(B, p);
  if (flags & MTX_TRANSA) {
    or_solve_trm_fm(B, A, 1.0, MTX_LOWER | MTX_UNIT | MTX_TRANSA);
    or_solve_trm_fm(B, A, 1.0, MTX_UPPER | MTX_TRANSA);
  } else {
    or_solve_trm_fm(B, A, 1.0, MTX_LOWER | MTX_UNIT);
    or_solve_trm_fm(B, A, 1.0, MTX_UPPER);
  }
  return OR_OK;
}

/* ---------------- house.go, qrwy.go, qrwym.go: QR with the compact WY form ---------------- */

enum {
  OR_EWORKSMALL = -13, /* "work space too small" qrwy.go:526 / "workspace too small" qrwym.go:667 */
  OR_ENOWORK = -14,    /* "workspace not defined"           qrwym.go:652 */
  OR_ECQSIZE = -15,    /* "C*Q: C.Cols != A.Rows"           qrwym.go:656 */
  OR_ETSMALL = -16     /* "reflector matrix T too small"    qrwy.go:550 */
};

/* mvec.go:362-376 (Norm2) over calgo/dvec_util.c:120 */
static double Norm2(fm X) {
  if (!is_vector(X)) return NAN;
  mvec_t x = {X.d, X.c != 1 ? X.ld : 1};
  return dvec_nrm2(&x, X.r * X.c);
}

/* mmult.go:478-490 (ScalePlus): A = alpha*A + beta*op(B) */
static void ScalePlus(fm A, fm B, double alpha, double beta, int flags) {
  mdata_t a = {A.d, A.ld}, b = {B.d, B.ld};
  dmmat_scale_plus(&a, &b, alpha, beta, flags, 0, A.c, 0, A.r);
}

/* mvec.go:226-245 (MVMultTrm): X = op(A)*X, A triangular */
static int MVMultTrm(fm X, fm A, int flags) {
  if (A.r == 0 || A.c == 0) return OR_OK;
  if (X.r != 1 && X.c != 1) return OR_ENOTVECTOR;
  mdata_t a = {A.d, A.ld};
  mvec_t x = {X.d, X.r == 1 ? X.ld : 1};
  dmvec_trid_unb(&x, &a, flags, A.c);
  return OR_OK;
}

/* element k of a row or column vector view */
static inline double *vel(fm X, int k) { return X.c == 1 ? X.d + k : X.d + (intptr_t)k * X.ld; }

/* house.go:18-32 (sqrtX2Y2, LAPACK dlapy2) */
static double sqrtX2Y2(double x, double y) {
  const double xa = fabs(x), ya = fabs(y);
  const double w = xa > ya ? xa : ya, z = xa < ya ? xa : ya;
  if (z == 0.0) return w;
  return w * sqrt(1.0 + (z / w) * (z / w));
}

/* house.go:55-78 (computeHouseholder, LAPACK dlarfg): reflector of [a11; x]; x becomes v,
 * a11 becomes beta, *tau the scalar factor (0 when x is zero) */
static void computeHouseholder(fm a11, fm x, fm tau) {
  const double nx = Norm2(x);
  if (nx == 0.0) {
    tau.d[0] = 0.0;
    return;
  }
  const double alpha = a11.d[0];
  const double sign = signbit(alpha) ? -1.0 : 1.0;
  const double beta = -sign * sqrtX2Y2(alpha, nx);
  InvScale(x, alpha - beta);
  tau.d[0] = (beta - alpha) / beta;
  a11.d[0] = beta;
}

/* house.go:97-122 (applyHouseholder, side LEFT): [a1; A2] = H*[a1; A2] with
 * w1 = tau*(a1 + A2^T v), a1 -= w1, A2 -= v*w1 */
static void applyHouseholderLeft(fm tau, fm v, fm a1, fm A2) {
  const double t = tau.d[0];
  if (t == 0.0) return;
  const int n = a1.r * a1.c;
  double *buf = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  for (int k = 0; k < n; k++) buf[k] = *vel(a1, k);
  fm w1 = {buf, 1, n, 1};
  MVMult(w1, A2, v, 1.0, 1.0, MTX_TRANSA);
  Scale(w1, t);
  for (int k = 0; k < n; k++) *vel(a1, k) -= buf[k];
  MVRankUpdate(A2, v, w1, -1.0);
  free(buf);
}

/* t01 = T00 * (-tau * (a10^T + A20^T a21)): column j of the block reflector
 * (qrwy.go:61-70 and :121-129) */
static void qr_t_column(fm T, int j, double tauval, fm a10, fm A20, fm a21) {
  fm t01 = sub(T, 0, j, j, 1), T00 = sub(T, 0, 0, j, j);
  for (int k = 0; k < j; k++) *vel(t01, k) = *vel(a10, k);
  MVMult(t01, A20, a21, -tauval, -tauval, MTX_TRANSA);
  MVMultTrm(t01, T00, MTX_UPPER);
}

/* qrwy.go:91-140 (unblockedQRT) */
static void unblockedQRT(fm A, fm T) {
  for (int j = 0; j < A.r && j < A.c; j++) {
    fm a11 = sub(A, j, j, 1, 1), a21 = sub(A, j + 1, j, A.r - j - 1, 1);
    fm a12 = sub(A, j, j + 1, 1, A.c - j - 1), A22 = sub(A, j + 1, j + 1, A.r - j - 1, A.c - j - 1);
    fm t11 = sub(T, j, j, 1, 1);
    computeHouseholder(a11, a21, t11);
    applyHouseholderLeft(t11, a21, a12, A22);
    const double tauval = t11.d[0];
    if (tauval != 0.0) qr_t_column(T, j, tauval, sub(A, j, 0, 1, j), sub(A, j + 1, 0, A.r - j - 1, j), a21);
  }
}

/* qrwy.go:146-181 (unblockedQR): tau(j) per reflector, no T */
static void unblockedQR(fm A, fm tau) {
  for (int j = 0; j < A.r && j < A.c && j < tau.r; j++) {
    fm a11 = sub(A, j, j, 1, 1), a21 = sub(A, j + 1, j, A.r - j - 1, 1);
    fm a12 = sub(A, j, j + 1, 1, A.c - j - 1), A22 = sub(A, j + 1, j + 1, A.r - j - 1, A.c - j - 1);
    fm tau1 = sub(tau, j, 0, 1, 1);
    computeHouseholder(a11, a21, tau1);
    applyHouseholderLeft(tau1, a21, a12, A22);
  }
}

/* qrwy.go:29-84 (unblkQRBlockReflector, LAPACK dlarft): T from the reflectors in A and tau */
static void unblkQRBlockReflector(fm T, fm A, fm tau) {
  for (int j = 0; j < A.r && j < A.c && j < tau.r; j++) {
    const double tauval = tau.d[j];
    if (tauval != 0.0) {
      T.d[j + (intptr_t)j * T.ld] = tauval;
      qr_t_column(T, j, tauval, sub(A, j, 0, 1, j), sub(A, j + 1, 0, A.r - j - 1, j),
                  sub(A, j + 1, j, A.r - j - 1, 1));
    }
  }
}

/* qrwy.go:266-303 (updateWithQT): [C1; C2] = Q^T [C1; C2] (transpose) or Q [C1; C2] with
 * Q = I - Y T Y^T, Y = [Y1 (unit lower); Y2] */
static void updateWithQT(fm C1, fm C2, fm Y1, fm Y2, fm T, fm W, int transpose) {
  ScalePlus(W, C1, 0.0, 1.0, MTX_TRANSB);
  or_mult_trm_fm(W, Y1, 1.0, MTX_LOWER | MTX_UNIT | MTX_RIGHT);
  or_mult_fm(W, C2, Y2, 1.0, 1.0, MTX_TRANSA);
  int tflags = MTX_UPPER | MTX_RIGHT;
  if (!transpose) tflags |= MTX_TRANSA;
  or_mult_trm_fm(W, T, 1.0, tflags);
  or_mult_fm(C2, Y2, W, -1.0, 1.0, MTX_TRANSB);
  or_mult_trm_fm(W, Y1, 1.0, MTX_LOWER | MTX_UNIT | MTX_TRANSA | MTX_RIGHT);
  ScalePlus(C1, W, 1.0, -1.0, MTX_TRANSB);
}

/* qrwy.go:315-348 (updateWithQTRight): [C1 C2] = [C1 C2] Q^T (transpose) or [C1 C2] Q */
static void updateWithQTRight(fm C1, fm C2, fm Y1, fm Y2, fm T, fm W, int transpose) {
  ScalePlus(W, C1, 0.0, 1.0, MTX_NOTRANS);
  or_mult_trm_fm(W, Y1, 1.0, MTX_LOWER | MTX_UNIT | MTX_RIGHT);
  or_mult_fm(W, C2, Y2, 1.0, 1.0, MTX_NOTRANS);
  int tflags = MTX_UPPER | MTX_RIGHT;
  if (transpose) tflags |= MTX_TRANSA;
  or_mult_trm_fm(W, T, 1.0, tflags);
  or_mult_fm(C2, W, Y2, -1.0, 1.0, MTX_TRANSB);
  or_mult_trm_fm(W, Y1, 1.0, MTX_LOWER | MTX_UNIT | MTX_RIGHT | MTX_TRANSA);
  ScalePlus(C1, W, 1.0, -1.0, MTX_NOTRANS);
}

/* qrwy.go:433-453 (updateQRTReflector): T = -T1 * (Y10^T Y11 + Y20^T Y21) * T2 */
static void updateQRTReflector(fm T, fm Y10, fm Y20, fm Y11, fm Y21, fm T1, fm T2) {
  if (Y10.c == 0) return;
  ScalePlus(T, Y10, 0.0, 1.0, MTX_TRANSB);
  or_mult_trm_fm(T, Y11, 1.0, MTX_LOWER | MTX_UNIT | MTX_RIGHT);
  or_mult_fm(T, Y20, Y21, 1.0, 1.0, MTX_TRANSA);
  or_mult_trm_fm(T, T1, -1.0, MTX_UPPER);
  or_mult_trm_fm(T, T2, 1.0, MTX_UPPER | MTX_RIGHT);
}

/* qrwy.go:351-427 (blockedQRT); the partitions of partition.go clip the block to the
 * columns left (repartition2x2to3x3, pBOTTOMRIGHT) */
static void blockedQRT(fm A, fm T, fm W, int nb) {
  for (int k = 0; k < A.r && k < A.c; ) {
    const int b = imin(nb, A.c - k), bt = imin(nb, T.c - k), bw = imin(nb, W.r - k);
    fm A10 = sub(A, k, 0, b, k), A11 = sub(A, k, k, b, b), A12 = sub(A, k, k + b, b, A.c - k - b);
    fm A20 = sub(A, k + b, 0, A.r - k - b, k), A21 = sub(A, k + b, k, A.r - k - b, b);
    fm A22 = sub(A, k + b, k + b, A.r - k - b, A.c - k - b);
    fm T00 = sub(T, 0, 0, k, k), T01 = sub(T, 0, k, k, bt), T11 = sub(T, k, k, bt, bt);
    fm W2 = sub(W, k + bw, 0, W.r - k - bw, W.c);
    fm AL = sub(A, k, k, A.r - k, imin(nb, A.c - k));
    unblockedQRT(AL, T11);
    updateWithQT(A12, A22, A11, A21, T11, W2, 1);
    updateQRTReflector(T01, A10, A20, A11, A21, T00, T11);
    k += b;
  }
}

/* qrwy.go:188-259 (blockedQR): DGEQRF with a scratch T per block; tau from its diagonal */
static void blockedQR(fm A, fm tau, fm Twork, fm W, int nb) {
  for (int k = 0; k < A.r && k < A.c; ) {
    const int b = imin(nb, A.c - k), bw = imin(nb, W.r - k);
    fm A11 = sub(A, k, k, b, b), A12 = sub(A, k, k + b, b, A.c - k - b);
    fm A21 = sub(A, k + b, k, A.r - k - b, b), A22 = sub(A, k + b, k + b, A.r - k - b, A.c - k - b);
    fm W2 = sub(W, k + bw, 0, W.r - k - bw, W.c);
    fm AL = sub(A, k, k, A.r - k, imin(nb, A.c - k));
    unblockedQRT(AL, Twork);
    const int tb = imin(nb, tau.r - k);
    for (int i = 0; i < tb; i++) tau.d[k + i] = Twork.d[i + (intptr_t)i * Twork.ld];
    updateWithQT(A12, A22, A11, A21, Twork, W2, 1);
    k += b;
  }
}

/* qrwy.go:474-497 (DecomposeQR) */
int or_decompose_qr_fm(fm A, fm tau, fm W, int nb) {
  if (nb == 0 || A.c <= nb) {
    unblockedQR(A, tau);
    return OR_OK;
  }
  double *tw = (double *)calloc((size_t)nb * nb, sizeof(double));
  double *wa = NULL;
  if (W.d == NULL) {
    wa = (double *)calloc((size_t)A.c * nb, sizeof(double));
    W = (fm){wa, A.c, nb, A.c};
  } else if (W.c < nb || W.r < A.c) {
    free(tw);
    return OR_EWORKSMALL;
  }
  blockedQR(A, tau, (fm){tw, nb, nb, nb}, sub(W, 0, 0, A.c, nb), nb);
  free(tw);
  free(wa);
  return OR_OK;
}

/* qrwy.go:517-538 (DecomposeQRT) */
int or_decompose_qrt_fm(fm A, fm T, fm W, int nb) {
  if (nb == 0 || A.c <= nb) {
    unblockedQRT(A, T);
    return OR_OK;
  }
  double *wa = NULL;
  if (W.d == NULL) {
    wa = (double *)calloc((size_t)A.c * nb, sizeof(double));
    W = (fm){wa, A.c, nb, A.c};
  } else if (W.c < nb || W.r < A.c) {
    return OR_EWORKSMALL;
  }
  blockedQRT(A, T, sub(W, 0, 0, A.c, nb), nb);
  free(wa);
  return OR_OK;
}

/* qrwy.go:546-556 (BuildT) */
int or_build_t_fm(fm T, fm A, fm tau) {
  if (T.c < A.c || T.r < A.c) return OR_ETSMALL;
  unblkQRBlockReflector(T, A, tau);
  return OR_OK;
}

/* qrwym.go:382-462 (blockedMultQTLeft) */
static void blockedMultQTLeft(fm C, fm A, fm T, fm W, int nb, int flags) {
  if (flags & MTX_TRANS) {
    /* top-left to bottom-right: Q^T C */
    int kc = 0;
    for (int k = 0; k < A.r && k < A.c; ) {
      const int b = imin(nb, A.c - k), bt = imin(nb, T.c - k);
      const int bc = imin(b, C.r - kc);
      fm A11 = sub(A, k, k, b, b), A21 = sub(A, k + b, k, A.r - k - b, b);
      fm T11 = sub(T, k, k, bt, bt);
      fm C1 = sub(C, kc, 0, bc, C.c), C2 = sub(C, kc + bc, 0, C.r - kc - bc, C.c);
      updateWithQT(C1, C2, A11, A21, T11, sub(W, 0, 0, C1.c, b), 1);
      k += b;
      kc += bc;
    }
  } else {
    /* bottom-right to top-left: Q C; the A and C partitions start mb = rows - cols above
     * the bottom, T's at its own bottom-right corner */
    const int mb = A.r - A.c;
    int ka = A.r - mb, kt = T.r, nc = C.r - mb;
    int ca = A.c;
    while (ka > 0 && ca > 0) {
      const int b = imin(nb, ka), bt = imin(nb, kt);
      const int bc = imin(b, nc);
      fm A11 = sub(A, ka - b, ka - b, b, b), A21 = sub(A, ka, ka - b, A.r - ka, b);
      fm T11 = sub(T, kt - bt, kt - bt, bt, bt);
      fm C1 = sub(C, nc - bc, 0, bc, C.c), C2 = sub(C, nc, 0, C.r - nc, C.c);
      updateWithQT(C1, C2, A11, A21, T11, sub(W, 0, 0, C1.c, b), 0);
      ka -= b;
      ca -= b;
      kt -= bt;
      nc -= bc;
    }
  }
}

/* qrwym.go:469-566 (blockedMultQTRight) */
static void blockedMultQTRight(fm C, fm A, fm T, fm W, int nb, int flags) {
  if (flags & MTX_TRANS) {
    /* bottom-right to top-left: C Q^T */
    const int mb = A.r - A.c, cb = C.c - A.c;
    int ka = A.r - mb, kt = T.r, kc = C.c - cb;
    int ca = A.c;
    while (ka > 0 && ca > 0) {
      const int b = imin(nb, ka), bt = imin(nb, kt), bc = imin(b, kc);
      fm A11 = sub(A, ka - b, ka - b, b, b), A21 = sub(A, ka, ka - b, A.r - ka, b);
      fm T11 = sub(T, kt - bt, kt - bt, bt, bt);
      fm C1 = sub(C, 0, kc - bc, C.r, bc), C2 = sub(C, 0, kc, C.r, C.c - kc);
      updateWithQTRight(C1, C2, A11, A21, T11, sub(W, 0, 0, C1.r, b), 1);
      ka -= b;
      ca -= b;
      kt -= bt;
      kc -= bc;
    }
  } else {
    /* top-left to bottom-right: C Q */
    int kc = 0;
    for (int k = 0; k < A.r && k < A.c; ) {
      const int b = imin(nb, A.c - k), bt = imin(nb, T.c - k), bc = imin(b, C.c - kc);
      fm A11 = sub(A, k, k, b, b), A21 = sub(A, k + b, k, A.r - k - b, b);
      fm T11 = sub(T, k, k, bt, bt);
      fm C1 = sub(C, 0, kc, C.r, bc), C2 = sub(C, 0, kc + bc, C.r, C.c - kc - bc);
      updateWithQTRight(C1, C2, A11, A21, T11, sub(W, 0, 0, C1.r, b), 0);
      k += b;
      kc += bc;
    }
  }
}

/* qrwym.go:646-688 (MultQT); W.d == NULL stands for a nil workspace */
int or_mult_qt_fm(fm C, fm A, fm T, fm W, int flags, int nb) {
  if (nb == 0) nb = T.c;
  if (W.d == NULL) return OR_ENOWORK;
  if (flags & MTX_RIGHT) {
    if (C.c != A.r) return OR_ECQSIZE;
    if (W.c < nb || W.r < C.r) return OR_EWORKSMALL;
    blockedMultQTRight(C, A, T, sub(W, 0, 0, C.r, nb), nb, flags);
  } else {
    if (W.c < nb || W.r < C.c) return OR_EWORKSMALL;
    blockedMultQTLeft(C, A, T, sub(W, 0, 0, C.c, nb), nb, flags);
  }
  return OR_OK;
}

/* qrwym.go:784-819 (SolveQRT).  With MTX_TRANS the rows of B below the first A.c are
 * cleared before Q is applied (the reference's intent, qrwym.go:795-797). */
int or_solve_qrt_fm(fm B, fm A, fm T, fm W, int flags, int nb) {
  fm R = sub(A, 0, 0, A.c, A.c), BT = sub(B, 0, 0, A.c, B.c);
  if (flags & MTX_TRANS) {
    int rc = or_solve_trm_fm(BT, R, 1.0, MTX_LEFT | MTX_UPPER | MTX_TRANSA);
    fm BB = sub(B, A.c, 0, B.r - A.c, B.c);
    for (int j = 0; j < BB.c; j++)
      for (int i = 0; i < BB.r; i++) BB.d[i + (intptr_t)j * BB.ld] = 0.0;
    (void)rc;
    return or_mult_qt_fm(B, A, T, W, MTX_LEFT, nb);
  }
  int rc = or_mult_qt_fm(B, A, T, W, MTX_LEFT | MTX_TRANS, nb);
  if (rc) return rc;
  return or_solve_trm_fm(BT, R, 1.0, MTX_LEFT | MTX_UPPER);
}

/* house.go:152-183 (applyHHTo2x1, side LEFT) with the caller's w1 */
static void applyHHTo2x1Left(double tval, fm v, fm a1, fm A2, fm w1) {
  if (tval == 0.0) return;
  const int n = a1.r * a1.c;
  for (int k = 0; k < n; k++) *vel(w1, k) = *vel(a1, k);
  MVMult(w1, A2, v, 1.0, 1.0, MTX_TRANSA);
  Scale(w1, tval);
  for (int k = 0; k < n; k++) *vel(a1, k) -= *vel(w1, k);
  MVRankUpdate(A2, v, w1, -1.0);
}

/* qrwyk.go:20-90 (unblockedBuildQ, LAPACK DORG2R): Q = H(0)...H(k-1) in place from the last
 * column to the first; tau(j) is element j of tau (a column vector) counted from its end as
 * the reference's partitions do.  "zero the upper part" (a01.SetIndexes(0.0)) is taken to
 * clear the column above the diagonal (DORG2R). */
static void unblockedBuildQ(fm A, fm tau, fm w) {
  int k = A.c, nt = tau.r * tau.c;
  while (k > 0 && nt > 0) {
    const int j = k - 1;
    const double t = *vel(tau, nt - 1);
    fm a21 = sub(A, j + 1, j, A.r - j - 1, 1), a12 = sub(A, j, j + 1, 1, A.c - j - 1);
    fm A22 = sub(A, j + 1, j + 1, A.r - j - 1, A.c - j - 1);
    applyHHTo2x1Left(t, a21, a12, A22, sub(w, 0, 0, 1, A.c - j - 1));
    Scale(a21, -t);
    A.d[j + (intptr_t)j * A.ld] = 1.0 - t;
    for (int i = 0; i < j; i++) A.d[i + (intptr_t)j * A.ld] = 0.0;
    k--;
    nt--;
  }
}

/* qrwyk.go:93-150 (blockedBuildQ, DORGQR) and :153-229 (blockedBuildQT): blocks of nb
 * columns from the bottom-right; T11 from tau by unblkQRBlockReflector (BuildQ) or from T's
 * diagonal block (BuildQT), the trailing columns take Q_b, the block's own columns the
 * unblocked form */
static void blockedBuildQ_(fm A, fm tau, fm T, fm W, int nb) {
  double *twork = NULL;
  fm Tk = {NULL, 0, 0, 1};
  if (!T.d) {
    twork = (double *)calloc((size_t)nb * nb, sizeof(double));
    Tk = (fm){twork, nb, nb, nb};
  }
  int k = A.c, nt = T.d ? T.r : tau.r * tau.c;
  while (k > 0 && A.r > 0) {
    const int b = imin(nb, k), bt = T.d ? imin(nb, nt) : imin(nb, nt);
    fm A11 = sub(A, k - b, k - b, b, b), A12 = sub(A, k - b, k, b, A.c - k);
    fm A21 = sub(A, k, k - b, A.r - k, b), A22 = sub(A, k, k, A.r - k, A.c - k);
    fm AL = sub(A, k - b, k - b, A.r - k + b, b);
    fm T11, tau1;
    double *diag = NULL;
    if (T.d) {
      T11 = sub(T, nt - bt, nt - bt, bt, bt);
      diag = (double *)malloc(sizeof(double) * (bt > 0 ? bt : 1));
      for (int i = 0; i < bt; i++) diag[i] = T11.d[i + (intptr_t)i * T11.ld];
      tau1 = (fm){diag, bt, 1, bt > 0 ? bt : 1};
    } else {
      tau1 = sub(tau, nt - bt, 0, bt, 1);
      T11 = sub(Tk, 0, 0, b, b);
      unblkQRBlockReflector(T11, AL, tau1);
    }
    updateWithQT(A12, A22, A11, A21, T11, sub(W, 0, 0, A12.c, b), 0);
    unblockedBuildQ(AL, tau1, sub(W, 0, 0, 1, b));
    for (int j = k - b; j < k; j++)
      for (int i = 0; i < k - b; i++) A.d[i + (intptr_t)j * A.ld] = 0.0;
    free(diag);
    k -= b;
    nt -= bt;
  }
  free(twork);
}

/* qrwyk.go:232-267 (BuildQ) */
int or_build_q_fm(fm A, fm tau, fm W, int nb) {
  if (nb != 0 && W.d == NULL) return OR_ENOWORK;
  if (nb != 0 && (W.c < nb || W.r < A.c)) return OR_EWORKSMALL;
  if (A.r < A.c) return OR_EABSIZE;
  if (nb == 0) {
    double *w = (double *)calloc((size_t)(A.c > 0 ? A.c : 1), sizeof(double));
    unblockedBuildQ(A, tau, (fm){w, 1, A.c, 1});
    free(w);
  } else {
    blockedBuildQ_(A, tau, (fm){NULL, 0, 0, 1}, sub(W, 0, 0, A.c, nb), nb);
  }
  return OR_OK;
}

/* qrwyk.go:278-293 (BuildQT) */
int or_build_qt_fm(fm A, fm T, fm W, int nb) {
  if (nb == 0) nb = A.c;
  if (W.d == NULL) return OR_ENOWORK;
  if (W.c < nb || W.r < A.c) return OR_EWORKSMALL;
  if (A.r < A.c) return OR_EABSIZE;
  blockedBuildQ_(A, (fm){NULL, 0, 0, 1}, T, sub(W, 0, 0, A.c, nb), nb);
  return OR_OK;
}

/* ---------------- ldlnp.go, ldl.go, ldlbk.go, ldlbks.go: symmetric indefinite LDL^T ------- */

/* mvec.go:163-190 (MVUpdateTrm): the lower (MTX_LOWER) or upper triangle of
 * A += alpha x y^T by calgo/dmvec_rank.c:263 (dmvec_trmv_upd) */
static int MVUpdateTrm(fm A, fm X, fm Y, double alpha, int flags) {
  if (A.r == 0 || A.c == 0) return OR_OK;
  if (!is_vector(Y) || !is_vector(X)) return OR_ENOTVECTOR;
  mdata_t a = {A.d, A.ld};
  mvec_t x = {X.d, X.r == 1 ? X.ld : 1}, y = {Y.d, Y.r == 1 ? Y.ld : 1};
  dmvec_trmv_upd(&a, &x, &y, alpha, flags, 0, A.c, nB);
  return OR_OK;
}

/* mvec.go:405-419 (IAMax) over calgo/dvec_util.c:164: first index of the largest |x| */
static int IAMax(fm X) {
  const int n = X.r * X.c;
  if (n <= 1) return 0;
  double mx = 0.0;
  int ix = 0;
  for (int i = 0; i < n; i++) {
    const double v = fabs(*vel(X, i));
    if (v > mx) {
      mx = v;
      ix = i;
    }
  }
  return ix;
}

/* the diagonal of a square view as a vector (FloatMatrix.Diag) */
static fm diagv(fm A) {
  fm d = {A.d, 1, A.r < A.c ? A.r : A.c, A.ld + 1};
  return d;
}

static void swap_el(double *a, double *b) {
  const double t = *a;
  *a = *b;
  *b = t;
}

/* pivot.go:145-190 (applyPivotSym): symmetric interchange of row/column 0 of AR with
 * row/column `index`, AL the factored columns left (LOWER) of AR */
static void applyPivotSymLower(fm AL, fm AR, int index) {
  for (int c = 0; c < AL.c; c++) swap_el(AL.d + (intptr_t)c * AL.ld, AL.d + index + (intptr_t)c * AL.ld);
  for (int i = 1; i < index; i++) swap_el(AR.d + i, AR.d + index + (intptr_t)i * AR.ld);
  for (int i = index + 1; i < AR.r; i++) swap_el(AR.d + i, AR.d + i + (intptr_t)index * AR.ld);
  swap_el(AR.d, AR.d + index + (intptr_t)index * AR.ld);
}

/* applyPivotSym UPPER (pivot.go:163-183): AL = [ATL ATR] full rows, AR = [a11 a12]; the
 * last row/column of ATL (colno) with `index` */
static void applyPivotSymUpper(fm A, int colno, int index) {
  /* S1 (row colno right of the diagonal) <-> row index, same columns */
  for (int c = colno + 1; c < A.c; c++)
    swap_el(A.d + colno + (intptr_t)c * A.ld, A.d + index + (intptr_t)c * A.ld);
  for (int i = index + 1; i < colno; i++)
    swap_el(A.d + i + (intptr_t)colno * A.ld, A.d + index + (intptr_t)i * A.ld);
  for (int i = 0; i < index; i++)
    swap_el(A.d + i + (intptr_t)index * A.ld, A.d + i + (intptr_t)colno * A.ld);
  swap_el(A.d + colno + (intptr_t)colno * A.ld, A.d + index + (intptr_t)index * A.ld);
}

/* ldlnp.go:23-58 / :64-97 */
static void unblkLDLnoPiv(fm A, int upper) {
  const int n = A.r;
  for (int s = 0; s < n; s++) {
    const int k = upper ? n - 1 - s : s;
    const double a11 = A.d[k + (intptr_t)k * A.ld];
    if (!upper) {
      fm a21 = sub(A, k + 1, k, n - k - 1, 1), A22 = sub(A, k + 1, k + 1, n - k - 1, n - k - 1);
      MVUpdateTrm(A22, a21, a21, -1.0 / a11, MTX_LOWER);
      InvScale(a21, a11);
    } else {
      fm a01 = sub(A, 0, k, k, 1), A00 = sub(A, 0, 0, k, k);
      MVUpdateTrm(A00, a01, a01, -1.0 / a11, MTX_UPPER);
      InvScale(a01, a11);
    }
  }
}

/* ldl.go:25-88 (unblkLowerLDL) / :297-349 (unblkUpperLDL): 1x1 pivots, the largest |diagonal|
 * of the part left; ipiv[k] = 1-based partner or 0.  Returns 1 on a zero pivot. */
static int unblkLDL(fm A, int64_t *ipiv, int upper) {
  const int n = A.r;
  for (int s = 0; s < n; s++) {
    if (!upper) {
      const int k = s;
      fm ABR = sub(A, k, k, n - k, n - k), ABL = sub(A, k, 0, n - k, k);
      const int imax = IAMax(diagv(ABR));
      if (imax > 0) {
        applyPivotSymLower(ABL, ABR, imax);
        ipiv[k] = imax + k + 1;
      } else {
        ipiv[k] = 0;
      }
      const double a11 = A.d[k + (intptr_t)k * A.ld];
      if (a11 == 0.0) return 1;
      fm a21 = sub(A, k + 1, k, n - k - 1, 1), A22 = sub(A, k + 1, k + 1, n - k - 1, n - k - 1);
      MVUpdateTrm(A22, a21, a21, -1.0 / a11, MTX_LOWER);
      InvScale(a21, a11);
    } else {
      const int k = n - 1 - s;  /* ATL is A[0:k+1, 0:k+1] */
      fm ATL = sub(A, 0, 0, k + 1, k + 1);
      const int imax = IAMax(diagv(ATL));
      if (imax < k) {
        applyPivotSymUpper(A, k, imax);
        ipiv[k] = imax + 1;
      } else {
        ipiv[k] = 0;
      }
      const double a11 = A.d[k + (intptr_t)k * A.ld];
      if (a11 == 0.0) return 1;
      fm a01 = sub(A, 0, k, k, 1), A00 = sub(A, 0, 0, k, k);
      MVUpdateTrm(A00, a01, a01, -1.0 / a11, MTX_UPPER);
      InvScale(a01, a11);
    }
  }
  return 0;
}

#define BK_ALPHA 0.6403882032022075 /* ldlbk.go:16, (1 + sqrt(17)) / 8 */

/* ldlbk.go:107-207 (findBKPivot, LOWER): A is the part left (ABR) */
static void findBKPivotLower(fm A, int *r_out, int *np_out) {
  *r_out = 0;
  *np_out = 1;
  if (A.r == 1) return;
  const double amax = fabs(A.d[0]);
  const int r = IAMax(sub(A, 1, 0, A.r - 1, 1)) + 1;
  const double rmax = fabs(A.d[r]);
  if (amax >= BK_ALPHA * rmax) return;
  int q = IAMax(sub(A, r, 0, 1, r));
  double qmax = fabs(A.d[r + (intptr_t)q * A.ld]);
  if (r < A.r - 1) {
    fm qrow = sub(A, r + 1, r, A.r - r - 1, 1);
    q = IAMax(qrow);
    const double qmax2 = fabs(*vel(qrow, q));
    if (qmax2 > qmax) qmax = qmax2;
  }
  if (amax >= BK_ALPHA * rmax * (rmax / qmax)) return;
  *r_out = r;
  *np_out = fabs(A.d[r + (intptr_t)r * A.ld]) >= BK_ALPHA * qmax ? 1 : 2;
}

/* ldlbk.go:164-205 (findBKPivot, UPPER): A is ATL; r = -1 for no interchange */
static void findBKPivotUpper(fm A, int *r_out, int *np_out) {
  *r_out = -1;
  *np_out = 1;
  if (A.r == 1) return;
  const int last = A.r - 1;
  const double amax = fabs(A.d[last + (intptr_t)last * A.ld]);
  const int r = IAMax(sub(A, 0, last, last, 1));
  const double rmax = fabs(A.d[r + (intptr_t)last * A.ld]);
  if (amax >= BK_ALPHA * rmax) return;
  double qmax = 0.0;
  if (r > 0) {
    fm qc = sub(A, 0, r, r, 1);
    const int q = IAMax(qc);
    qmax = fabs(*vel(qc, q));
  }
  fm qrow = sub(A, r, r + 1, 1, last - r);
  const int q = IAMax(qrow);
  const double qmax2 = fabs(*vel(qrow, q));
  if (qmax2 > qmax) qmax = qmax2;
  if (amax >= BK_ALPHA * rmax * (rmax / qmax)) return;
  *r_out = r;
  *np_out = fabs(A.d[r + (intptr_t)r * A.ld]) >= BK_ALPHA * qmax ? 1 : 2;
}

/* ldlbk.go:48-76 (applyBKPivotSym LOWER): within AR, rows/columns src and dst (src < dst) */
static void applyBKPivotSymLower(fm AR, int src, int dst) {
  for (int t = 0; t < dst - src - 1; t++)
    swap_el(AR.d + (src + 1 + t) + (intptr_t)src * AR.ld, AR.d + dst + (intptr_t)(src + 1 + t) * AR.ld);
  for (int i = dst + 1; i < AR.r; i++)
    swap_el(AR.d + i + (intptr_t)src * AR.ld, AR.d + i + (intptr_t)dst * AR.ld);
  swap_el(AR.d + src + (intptr_t)src * AR.ld, AR.d + dst + (intptr_t)dst * AR.ld);
}

/* ldlbk.go:77-104 (applyBKPivotSym UPPER): within AR (= ATL), src > dst */
static void applyBKPivotSymUpper(fm AR, int src, int dst) {
  for (int t = 0; t < src - dst - 1; t++)
    swap_el(AR.d + (dst + 1 + t) + (intptr_t)src * AR.ld, AR.d + dst + (intptr_t)(dst + 1 + t) * AR.ld);
  for (int i = 0; i < dst; i++)
    swap_el(AR.d + i + (intptr_t)src * AR.ld, AR.d + i + (intptr_t)dst * AR.ld);
  swap_el(AR.d + src + (intptr_t)src * AR.ld, AR.d + dst + (intptr_t)dst * AR.ld);
}

/* the 2 x 2 pivot step of ldlbk.go:289-313 / :415-436: cwrk = the two columns c, then
 * c = scale * cwrk * [[i00, -1], [-1, i11]] (Mult, beta 0) and the triangle of A22 -=
 * c cwrk^T (UpdateTrm, beta 1) */
static void bk_two_by_two(fm c, fm A22, double *cw, int m, double i00, double i11, double scale,
                          int tri) {
  fm W = {cw, m, 2, m > 0 ? m : 1};
  for (int i = 0; i < m; i++) {
    cw[i] = c.d[i];
    cw[m + i] = c.d[i + (intptr_t)c.ld];
  }
  double inv[4] = {i00, -1.0, -1.0, i11};
  fm E = {inv, 2, 2, 2};
  or_mult_fm(c, W, E, scale, 0.0, MTX_NOTRANS);
  or_update_trm_fm(A22, c, W, -1.0, 1.0, tri | MTX_TRANSB);
}

/* ldlbk.go:212-330 (unblkDecompBKLower) and :335-455 (unblkDecompBKUpper), LAPACK DSYTF2 */
static void unblkDecompBK(fm A, int64_t *ipiv, int upper) {
  const int n = A.r;
  double *cw = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  int done = 0;
  while (done < n) {
    int r, np;
    if (!upper) {
      const int k = done;
      fm ABR = sub(A, k, k, n - k, n - k);
      findBKPivotLower(ABR, &r, &np);
      if (r != 0 && r != np - 1) {
        applyBKPivotSymLower(ABR, np - 1, r);
        if (np == 2) swap_el(ABR.d + 1, ABR.d + r);
      }
      if (np == 1) {
        const double a11 = ABR.d[0];
        fm a21 = sub(A, k + 1, k, n - k - 1, 1), A22 = sub(A, k + 1, k + 1, n - k - 1, n - k - 1);
        MVUpdateTrm(A22, a21, a21, -1.0 / a11, MTX_LOWER);
        InvScale(a21, a11);
        ipiv[k] = r + k + 1;
      } else {
        const double a = ABR.d[0], b = ABR.d[1], d = ABR.d[1 + (intptr_t)ABR.ld];
        const double i00 = d / b, i11 = a / b;
        double scale = 1.0 / ((a / b) * (d / b) - 1.0);
        scale /= b;
        const int m = n - k - 2;
        fm a21 = sub(A, k + 2, k, m, 2), A22 = sub(A, k + 2, k + 2, m, m);
        bk_two_by_two(a21, A22, cw, m, i00, i11, scale, MTX_LOWER);
        ipiv[k] = -(r + k + 1);
        ipiv[k + 1] = ipiv[k];
      }
    } else {
      const int s = n - done; /* ATL is s x s */
      fm ATL = sub(A, 0, 0, s, s);
      const int nr = s - 1;
      findBKPivotUpper(ATL, &r, &np);
      if (r != -1) {
        applyBKPivotSymUpper(ATL, s - np, r);
        if (np == 2) swap_el(ATL.d + (nr - 1) + (intptr_t)nr * ATL.ld, ATL.d + r + (intptr_t)nr * ATL.ld);
      }
      if (np == 1) {
        const int k = s - 1;
        const double a11 = A.d[k + (intptr_t)k * A.ld];
        fm a01 = sub(A, 0, k, k, 1), A00 = sub(A, 0, 0, k, k);
        MVUpdateTrm(A00, a01, a01, -1.0 / a11, MTX_UPPER);
        InvScale(a01, a11);
        ipiv[k] = r == -1 ? s : r + 1;
      } else {
        const int k = s - 2;
        const double a = A.d[k + (intptr_t)k * A.ld], b = A.d[k + (intptr_t)(k + 1) * A.ld];
        const double d = A.d[(k + 1) + (intptr_t)(k + 1) * A.ld];
        const double i00 = d / b, i11 = a / b;
        double scale = 1.0 / ((a / b) * (d / b) - 1.0);
        scale /= b;
        const int m = k;
        fm a01 = sub(A, 0, k, m, 2), A00 = sub(A, 0, 0, m, m);
        bk_two_by_two(a01, A00, cw, m, i00, i11, scale, MTX_UPPER);
        ipiv[k] = -(r + 1);
        ipiv[k + 1] = ipiv[k];
      }
    }
    done += np;
  }
  free(cw);
}

/* ldlnp.go:211-235 (DecomposeLDLnoPiv): the unblocked path (the blocked one computes the
 * same factor; nb is accepted) */
int or_decompose_ldl_nopiv_fm(fm A, int flags) {
  if (A.c != A.r) return OR_ENOTSQUARE;
  unblkLDLnoPiv(A, (flags & MTX_LOWER) == 0);
  return OR_OK;
}

/* ldl.go:439-466 (DecomposeLDL), unblocked path; returns 1 on a zero pivot ("zero value on
 * diagonal") */
int or_decompose_ldl_fm(fm A, int64_t *ipiv, int npiv, int flags) {
  if (A.c != A.r) return OR_ENOTSQUARE;
  for (int k = 0; k < npiv; k++) ipiv[k] = 0;
  if (npiv < A.r) return OR_EPIVLEN;
  return unblkLDL(A, ipiv, (flags & MTX_LOWER) == 0);
}

/* ldlbk.go:1114-1140 (DecomposeBK), unblocked path (DSYTF2) */
int or_decompose_bk_fm(fm A, int64_t *ipiv, int npiv, int flags) {
  for (int k = 0; k < npiv; k++) ipiv[k] = 0;
  if (A.c != A.r) return OR_ENOTSQUARE;
  if (npiv < A.r) return OR_EPIVLEN;
  if (!(flags & (MTX_LOWER | MTX_UPPER))) return OR_OK;
  unblkDecompBK(A, ipiv, (flags & MTX_LOWER) == 0);
  return OR_OK;
}

/* diag.go:85-128 (SolveDiag, LEFT, D the diagonal of a square matrix): row k *= 1/d_k */
static void SolveDiagLeft(fm B, fm A) {
  for (int k = 0; k < B.r; k++) {
    const double f = 1.0 / A.d[k + (intptr_t)k * A.ld];
    for (int c = 0; c < B.c; c++) B.d[k + (intptr_t)c * B.ld] *= f;
  }
}

/* ldlnp.go:251-266 (SolveLDLnoPiv) */
void or_solve_ldl_nopiv_fm(fm B, fm A, int flags) {
  const int tri = (flags & MTX_UPPER) ? MTX_UPPER : ((flags & MTX_LOWER) ? MTX_LOWER : 0);
  if (!tri) return;
  or_solve_trm_fm(B, A, 1.0, tri | MTX_UNIT);
  SolveDiagLeft(B, A);
  or_solve_trm_fm(B, A, 1.0, tri | MTX_UNIT | MTX_TRANSA);
}

/* pivot.go:63-78 (applyRowPivots, offset 0): FORWARD k = 0.., BACKWARD k = ..0 */
static void applyRowPivotsLDL(fm B, const int64_t *ipiv, int n, int forward) {
  for (int t = 0; t < n; t++) {
    const int k = forward ? t : n - 1 - t;
    if (ipiv[k] > 0) swapRows(B, (int)ipiv[k] - 1, k);
  }
}

/* ldl.go:486-510 (SolveLDL) */
void or_solve_ldl_fm(fm B, fm A, const int64_t *ipiv, int flags) {
  const int n = A.r;
  if (flags & MTX_UPPER) {
    applyRowPivotsLDL(B, ipiv, n, 0);
    or_solve_trm_fm(B, A, 1.0, MTX_UPPER | MTX_UNIT);
    SolveDiagLeft(B, A);
    or_solve_trm_fm(B, A, 1.0, MTX_UPPER | MTX_UNIT | MTX_TRANSA);
    applyRowPivotsLDL(B, ipiv, n, 1);
  } else if (flags & MTX_LOWER) {
    applyRowPivotsLDL(B, ipiv, n, 1);
    or_solve_trm_fm(B, A, 1.0, MTX_LOWER | MTX_UNIT);
    SolveDiagLeft(B, A);
    or_solve_trm_fm(B, A, 1.0, MTX_LOWER | MTX_UNIT | MTX_TRANSA);
    applyRowPivotsLDL(B, ipiv, n, 0);
  }
}

/* ldlbks.go:15-156 (unblkSolveBKLower), both phases */
static void unblkSolveBKLower(fm B, fm A, const int64_t *ipiv) {
  const int n = A.r;
  for (int k = 0; k < n;) {
    const int np = ipiv[k] < 0 ? 2 : 1;
    if (np == 1) {
      if (ipiv[k] != k + 1) swapRows(B, k, (int)ipiv[k] - 1);
      fm b1 = sub(B, k, 0, 1, B.c);
      MVRankUpdate(sub(B, k + 1, 0, n - k - 1, B.c), sub(A, k + 1, k, n - k - 1, 1), b1, -1.0);
      InvScale(b1, A.d[k + (intptr_t)k * A.ld]);
    } else {
      if (ipiv[k] != -(k + 1)) swapRows(B, k + 1, (int)(-ipiv[k]) - 1);
      const double b = A.d[(k + 1) + (intptr_t)k * A.ld];
      const double apb = A.d[k + (intptr_t)k * A.ld] / b;
      const double dpb = A.d[(k + 1) + (intptr_t)(k + 1) * A.ld] / b;
      double scale = apb * dpb - 1.0;
      scale *= b;
      fm b1 = sub(B, k, 0, 2, B.c);
      or_mult_fm(sub(B, k + 2, 0, n - k - 2, B.c), sub(A, k + 2, k, n - k - 2, 2), b1, -1.0, 1.0,
                 MTX_NOTRANS);
      for (int c = 0; c < B.c; c++) {
        double *s = B.d + k + (intptr_t)c * B.ld;
        const double s0 = s[0], s1 = s[1];
        s[0] = (dpb * s0 - s1) / scale;
        s[1] = (apb * s1 - s0) / scale;
      }
    }
    k += np;
  }
  for (int nc = n; nc > 0;) {
    const int np = ipiv[nc - 1] < 0 ? 2 : 1;
    if (np == 1) {
      const int k = nc - 1;
      fm b1 = sub(B, k, 0, 1, B.c);
      MVMult(b1, sub(B, k + 1, 0, n - k - 1, B.c), sub(A, k + 1, k, n - k - 1, 1), -1.0, 1.0,
             MTX_TRANSA);
      if (ipiv[k] != nc) swapRows(B, k, (int)ipiv[k] - 1);
    } else {
      const int k = nc - 2;
      or_mult_fm(sub(B, k, 0, 2, B.c), sub(A, k + 2, k, n - k - 2, 2), sub(B, k + 2, 0, n - k - 2, B.c),
                 -1.0, 1.0, MTX_TRANSA);
      if (ipiv[k] != -nc) swapRows(B, k + 1, (int)(-ipiv[k]) - 1);
    }
    nc -= np;
  }
}

/* ldlbks.go:303-318 (SolveBK).  LOWER restates unblkSolveBKLower.  The reference's UPPER
 * branch (unblkSolveBKUpper, ldlbks.go:159-296) updates an empty block of B in its first
 * phase and mismatched ones in its second (its partitions run the wrong way for U); the
 * oracle solves A X = B with the UPPER factor through the same steps on the index-reversed
 * problem (row/column i <-> n-1-i turns U D U^T into L D L^T). */
void or_solve_bk_fm(fm B, fm A, const int64_t *ipiv, int flags) {
  const int n = A.r;
  if (flags & MTX_LOWER) {
    unblkSolveBKLower(B, A, ipiv);
  } else if (flags & MTX_UPPER) {
    double *ar = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1) * (n > 0 ? n : 1));
    double *br = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1) * (B.c > 0 ? B.c : 1));
    int64_t *pr = (int64_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(int64_t));
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) ar[i + (size_t)j * n] = A.d[(n - 1 - i) + (intptr_t)(n - 1 - j) * A.ld];
    for (int c = 0; c < B.c; c++)
      for (int i = 0; i < n; i++) br[i + (size_t)c * n] = B.d[(n - 1 - i) + (intptr_t)c * B.ld];
    for (int i = 0; i < n; i++) {
      const int64_t p = ipiv[n - 1 - i];
      pr[i] = p > 0 ? n + 1 - p : -(n + 1 + p);
    }
    unblkSolveBKLower((fm){br, n, B.c, n > 0 ? n : 1}, (fm){ar, n, n, n > 0 ? n : 1}, pr);
    for (int c = 0; c < B.c; c++)
      for (int i = 0; i < n; i++) B.d[(n - 1 - i) + (intptr_t)c * B.ld] = br[i + (size_t)c * n];
    free(ar);
    free(br);
    free(pr);
  }
}

/* house.go:152-183 (applyHHTo2x1, side RIGHT) with the caller's w1: [a1 A2] = [a1 A2] H,
 * w1 = tau (a1 + A2 v), a1 -= w1, A2 -= w1 v^T */
static void applyHHTo2x1Right(double tval, fm v, fm a1, fm A2, fm w1) {
  if (tval == 0.0) return;
  const int n = a1.r * a1.c;
  for (int k = 0; k < n; k++) *vel(w1, k) = *vel(a1, k);
  MVMult(w1, A2, v, 1.0, 1.0, MTX_NOTRANS);
  Scale(w1, tval);
  for (int k = 0; k < n; k++) *vel(a1, k) -= *vel(w1, k);
  MVRankUpdate(A2, w1, v, -1.0);
}

/* qrwym.go:28-106 (unblockedMultQLeft) and :114-190 (unblockedMultQRight): one reflector at a
 * time, forward for Q^T C and C Q, backward for Q C and C Q^T; tau(j) is the j-th entry */
static void unblockedMultQ(fm C, fm A, fm tau, int flags) {
  const int k = A.r < A.c ? A.r : A.c;
  const int right = (flags & MTX_RIGHT) != 0, trans = (flags & MTX_TRANS) != 0;
  const int forward = right ? !trans : trans;
  const int wl = right ? C.r : C.c;
  double *wb = (double *)calloc((size_t)(wl > 0 ? wl : 1), sizeof(double));
  for (int t = 0; t < k && t < tau.r * tau.c; t++) {
    const int j = forward ? t : k - 1 - t;
    const double tj = *vel(tau, j);
    fm v = sub(A, j + 1, j, A.r - j - 1, 1);
    if (!right) {
      double tv = tj;
      applyHouseholderLeft((fm){&tv, 1, 1, 1}, v, sub(C, j, 0, 1, C.c),
                           sub(C, j + 1, 0, C.r - j - 1, C.c));
    } else {
      fm w = {wb, C.r, 1, C.r > 0 ? C.r : 1};
      applyHHTo2x1Right(tj, v, sub(C, 0, j, C.r, 1), sub(C, 0, j + 1, C.r, C.c - j - 1), w);
    }
  }
  free(wb);
}

/* qrwym.go:573-630 (MultQ): the unblocked path for any nb (the blocked one builds its T
 * blocks with the per-68-row-block GEMV of BuildT); W is checked as the reference checks it */
int or_mult_q_fm(fm C, fm A, fm tau, fm W, int flags, int nb) {
  if (nb != 0 && W.d == NULL) return OR_ENOWORK;
  if (flags & MTX_RIGHT) {
    if (C.c != A.r) return OR_ECQSIZE;
    if (nb != 0 && (W.c < nb || W.r < C.r)) return OR_EWORKSMALL;
  } else if (nb != 0 && (W.c < nb || W.r < C.c)) {
    return OR_EWORKSMALL;
  }
  unblockedMultQ(C, A, tau, flags);
  return OR_OK;
}

/* qrwym.go:717-760 (SolveQR); with MTX_TRANS the minimum-norm solution as SolveQRT computes
 * it (the reference rebinds B to an empty view there, qrwym.go:735) */
int or_solve_qr_fm(fm B, fm A, fm tau, fm W, int flags, int nb) {
  fm R = sub(A, 0, 0, A.c, A.c), BT = sub(B, 0, 0, A.c, B.c);
  if (flags & MTX_TRANS) {
    or_solve_trm_fm(BT, R, 1.0, MTX_LEFT | MTX_UPPER | MTX_TRANSA);
    fm BB = sub(B, A.c, 0, B.r - A.c, B.c);
    for (int j = 0; j < BB.c; j++)
      for (int i = 0; i < BB.r; i++) BB.d[i + (intptr_t)j * BB.ld] = 0.0;
    return or_mult_q_fm(B, A, tau, W, MTX_LEFT, nb);
  }
  int rc = or_mult_q_fm(B, A, tau, W, MTX_LEFT | MTX_TRANS, nb);
  if (rc) return rc;
  return or_solve_trm_fm(BT, R, 1.0, MTX_LEFT | MTX_UPPER);
}

/* ---------------- flat C entry points for the ctypes harness ---------------- */

#define FM(p, r, c, ld) ((fm){(p), (r), (c), (ld)})

int or_mult(double *C, int cr, int cc, int ldc, double *A, int ar, int ac, int lda, double *B,
            int br, int bc, int ldb, double alpha, double beta, int flags) {
  return or_mult_fm(FM(C, cr, cc, ldc), FM(A, ar, ac, lda), FM(B, br, bc, ldb), alpha, beta, flags);
}
int or_rank_update_sym(double *C, int cr, int cc, int ldc, double *A, int ar, int ac, int lda,
                       double alpha, double beta, int flags) {
  return or_rank_update_sym_fm(FM(C, cr, cc, ldc), FM(A, ar, ac, lda), alpha, beta, flags);
}
int or_solve_trm(double *B, int br, int bc, int ldb, double *A, int ar, int ac, int lda,
                 double alpha, int flags) {
  return or_solve_trm_fm(FM(B, br, bc, ldb), FM(A, ar, ac, lda), alpha, flags);
}
int or_decompose_chol(double *A, int ar, int ac, int lda, int flags, int nb) {
  return or_decompose_chol_fm(FM(A, ar, ac, lda), flags, nb);
}
int or_decompose_lu(double *A, int ar, int ac, int lda, int64_t *piv, int npiv, int nb) {
  pv p = {piv, npiv};
  return or_decompose_lu_fm(FM(A, ar, ac, lda), p, nb);
}
/* blockedCHOL's steps k0 <= k < k1 (k0 a multiple of nb): a long factorization timed in
 * slices; running the slices [0, k1), [k1, k2), ... in order equals one DecomposeCHOL call
 * with nb > 0 and nb <= order (chol.go:123-126) */
int or_decompose_chol_steps(double *A, int ar, int ac, int lda, int flags, int nb, int k0, int k1) {
  fm a = FM(A, ar, ac, lda);
  if (a.c != a.r) return OR_ENOTSQUARE;
  if (nb <= 0 || a.c < nb || k0 % nb) return OR_ESIZE;
  return blockedCHOL_steps(a, flags, nb, k0, k1);
}
void or_solve_chol(double *B, int br, int bc, int ldb, double *A, int ar, int ac, int lda, int flags) {
  or_solve_chol_fm(FM(B, br, bc, ldb), FM(A, ar, ac, lda), flags);
}
int or_solve_lu(double *B, int br, int bc, int ldb, double *A, int ar, int ac, int lda, int64_t *piv,
                int npiv, int flags) {
  pv p = {piv, npiv};
  return or_solve_lu_fm(FM(B, br, bc, ldb), FM(A, ar, ac, lda), p, flags);
}
int or_mult_sym(double *C, int cr, int cc, int ldc, double *A, int ar, int ac, int lda,
                double *B, int br, int bc, int ldb, double alpha, double beta, int flags) {
  return or_mult_sym_fm(FM(C, cr, cc, ldc), FM(A, ar, ac, lda), FM(B, br, bc, ldb), alpha, beta,
                        flags);
}
int or_mult_trm(double *B, int br, int bc, int ldb, double *A, int ar, int ac, int lda,
                double alpha, int flags) {
  return or_mult_trm_fm(FM(B, br, bc, ldb), FM(A, ar, ac, lda), alpha, flags);
}
int or_rank_update2_sym(double *C, int cr, int cc, int ldc, double *A, int ar, int ac, int lda,
                        double *B, int br, int bc, int ldb, double alpha, double beta,
                        int flags) {
  return or_rank_update2_sym_fm(FM(C, cr, cc, ldc), FM(A, ar, ac, lda), FM(B, br, bc, ldb),
                                alpha, beta, flags);
}
int or_update_trm(double *C, int cr, int cc, int ldc, double *A, int ar, int ac, int lda,
                  double *B, int br, int bc, int ldb, double alpha, double beta, int flags) {
  return or_update_trm_fm(FM(C, cr, cc, ldc), FM(A, ar, ac, lda), FM(B, br, bc, ldb), alpha, beta,
                          flags);
}
int or_inverse_trm(double *A, int ar, int ac, int lda, int flags, int nb) {
  return or_inverse_trm_fm(FM(A, ar, ac, lda), flags, nb);
}
/* mmult.go:69-73 */
int or_num_workers(int n) {
  int old = nWorker;
  nWorker = n;
  return old;
}
/* mmult.go:63-67 */
void or_blocking_params(int mb, int nb, int kb) {
  vpLen = kb;
  nB = nb;
  mB = mb;
}
/* QR entry points; a NULL W stands for the reference's nil workspace */
int or_decompose_qrt(double *A, int ar, int ac, int lda, double *T, int tr, int tc, int ldt,
                     double *W, int wr, int wc, int ldw, int nb) {
  return or_decompose_qrt_fm(FM(A, ar, ac, lda), FM(T, tr, tc, ldt), FM(W, wr, wc, ldw), nb);
}
int or_decompose_qr(double *A, int ar, int ac, int lda, double *tau, int taur, double *W, int wr,
                    int wc, int ldw, int nb) {
  return or_decompose_qr_fm(FM(A, ar, ac, lda), FM(tau, taur, 1, taur > 0 ? taur : 1),
                            FM(W, wr, wc, ldw), nb);
}
int or_build_t(double *T, int tr, int tc, int ldt, double *A, int ar, int ac, int lda, double *tau,
               int taur) {
  return or_build_t_fm(FM(T, tr, tc, ldt), FM(A, ar, ac, lda), FM(tau, taur, 1, taur > 0 ? taur : 1));
}
int or_mult_qt(double *C, int cr, int cc, int ldc, double *A, int ar, int ac, int lda, double *T,
               int tr, int tc, int ldt, double *W, int wr, int wc, int ldw, int flags, int nb) {
  return or_mult_qt_fm(FM(C, cr, cc, ldc), FM(A, ar, ac, lda), FM(T, tr, tc, ldt),
                       FM(W, wr, wc, ldw), flags, nb);
}
int or_solve_qrt(double *B, int br, int bc, int ldb, double *A, int ar, int ac, int lda, double *T,
                 int tr, int tc, int ldt, double *W, int wr, int wc, int ldw, int flags, int nb) {
  return or_solve_qrt_fm(FM(B, br, bc, ldb), FM(A, ar, ac, lda), FM(T, tr, tc, ldt),
                         FM(W, wr, wc, ldw), flags, nb);
}
int or_build_q(double *A, int ar, int ac, int lda, double *tau, int taur, double *W, int wr, int wc,
               int ldw, int nb) {
  return or_build_q_fm(FM(A, ar, ac, lda), FM(tau, taur, 1, taur > 0 ? taur : 1),
                       FM(W, wr, wc, ldw), nb);
}
int or_build_qt(double *A, int ar, int ac, int lda, double *T, int tr, int tc, int ldt, double *W,
                int wr, int wc, int ldw, int nb) {
  return or_build_qt_fm(FM(A, ar, ac, lda), FM(T, tr, tc, ldt), FM(W, wr, wc, ldw), nb);
}
/* LDL^T entry points (ldlnp.go, ldl.go, ldlbk.go, ldlbks.go) */
int or_decompose_ldl_nopiv(double *A, int ar, int ac, int lda, int flags) {
  return or_decompose_ldl_nopiv_fm(FM(A, ar, ac, lda), flags);
}
void or_solve_ldl_nopiv(double *B, int br, int bc, int ldb, double *A, int ar, int ac, int lda,
                        int flags) {
  or_solve_ldl_nopiv_fm(FM(B, br, bc, ldb), FM(A, ar, ac, lda), flags);
}
int or_decompose_ldl(double *A, int ar, int ac, int lda, int64_t *piv, int npiv, int flags) {
  return or_decompose_ldl_fm(FM(A, ar, ac, lda), piv, npiv, flags);
}
void or_solve_ldl(double *B, int br, int bc, int ldb, double *A, int ar, int ac, int lda,
                  const int64_t *piv, int flags) {
  or_solve_ldl_fm(FM(B, br, bc, ldb), FM(A, ar, ac, lda), piv, flags);
}
int or_decompose_bk(double *A, int ar, int ac, int lda, int64_t *piv, int npiv, int flags) {
  return or_decompose_bk_fm(FM(A, ar, ac, lda), piv, npiv, flags);
}
void or_solve_bk(double *B, int br, int bc, int ldb, double *A, int ar, int ac, int lda,
                 const int64_t *piv, int flags) {
  or_solve_bk_fm(FM(B, br, bc, ldb), FM(A, ar, ac, lda), piv, flags);
}
int or_mult_q(double *C, int cr, int cc, int ldc, double *A, int ar, int ac, int lda, double *tau,
              int taur, double *W, int wr, int wc, int ldw, int flags, int nb) {
  return or_mult_q_fm(FM(C, cr, cc, ldc), FM(A, ar, ac, lda), FM(tau, taur, 1, taur > 0 ? taur : 1),
                      FM(W, wr, wc, ldw), flags, nb);
}
int or_solve_qr(double *B, int br, int bc, int ldb, double *A, int ar, int ac, int lda, double *tau,
                int taur, double *W, int wr, int wc, int ldw, int flags, int nb) {
  return or_solve_qr_fm(FM(B, br, bc, ldb), FM(A, ar, ac, lda), FM(tau, taur, 1, taur > 0 ? taur : 1),
                        FM(W, wr, wc, ldw), flags, nb);
}
