/*
 * matops_b200.h -- C ABI of the B200 (sm_100a) implementation of hrautila/matops's
 * level-3 hot path: GEMM, SYRK and TRSM, the rest of the level-3 surface, and the Cholesky /
 * LU / QR (compact WY) / symmetric indefinite LDL^T factorizations and solves built on
 * them, all in IEEE double precision on device-resident column-major matrices; plus a
 * mixed-precision Cholesky solve, batched small systems and the Cholesky adjoints.
 *
 * Every operation entry point mirrors one exported Go function of the reference package
 * (file:line in its source tree) with the same argument meaning, flag bits and error
 * conditions; a cgo shim keeps the Go signatures and forwards FloatMatrix views as
 * mo_matrix values.  All calls are asynchronous on the context's stream unless noted;
 * results that the Go function returns synchronously (the Cholesky panic index) make
 * that entry point synchronize.
 *
 * Plain C: pointers, sizes and ints only.  Thread-safety: one context per host thread.
 */
#ifndef MATOPS_B200_H
#define MATOPS_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MO_API __attribute__((visibility("default")))
#else
#define MO_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Flag bits: identical values to matops.Flags (mmult.go:18-30, calgo/cmops.go:19-31). */
#define MO_NOTRANS 0x0
#define MO_TRANSA 0x1
#define MO_TRANSB 0x2
#define MO_LOWER 0x4
#define MO_UPPER 0x8
#define MO_LEFT 0x10
#define MO_RIGHT 0x20
#define MO_UNIT 0x40
#define MO_TRANS 0x80

/* Status codes.  0 = nil error.  Negative values name the Go error of the reference
 * (message in comment) or a device-side failure.  Positive values are LAPACK-style info:
 * for mo_decompose_chol, k+1 when column k's pivot square root is NaN (the reference
 * panics with "illegal value at k", chol.go:33-36). */
#define MO_OK 0
#define MO_ESIZE (-1)        /* "Mult: size mismatch"                    mmult.go:224 */
#define MO_ENOTSQUARE (-2)   /* "A not a square matrix"                  chol.go:119 */
#define MO_EPIVLEN (-3)      /* "pivot array < min(A.Rows(),A.Cols())"    lu.go:260-262 */
#define MO_ECNOTSQUARE (-4)  /* "C not a square matrix"                  mmult.go:428 */
#define MO_EABSIZE (-5)      /* "A, B size mismatch"                     mmult.go:406 */
#define MO_ESYMSIZE (-7)     /* "MultSym: size mismatch"                 mmult.go:290 */
#define MO_EINVAL (-10)      /* NULL context/pointer, negative size, ld < rows        */
#define MO_ECUDA (-20)       /* CUDA runtime error                                    */
#define MO_EDEVTIMEOUT (-21) /* a bounded device-side wait gave up                    */
#define MO_ENOMEM (-22)      /* device allocation failed                              */
#define MO_ENOKERNEL (-23)   /* no sm_100a kernel image for this device               */
#define MO_ESTATICLIMIT (-11) /* larger than the fixed scratch of mo_solve_trm_static   */
#define MO_EBATCHN (-12)     /* a batched matrix order outside 1..MO_BATCH_MAX_N      */
#define MO_EWORKSMALL (-13)  /* "work space too small"  qrwy.go:526 ("workspace too small",
                                qrwym.go:667)                                         */
#define MO_ENOWORK (-14)     /* "workspace not defined"                  qrwym.go:652 */
#define MO_ECQSIZE (-15)     /* "C*Q: C.Cols != A.Rows"                  qrwym.go:656 */
#define MO_ETSMALL (-16)     /* "reflector matrix T too small"           qrwy.go:550 */
#define MO_ELDLWORK (-17)    /* "No workspace for blocking invocation"   ldlnp.go:224 */
#define MO_EZERODIAG (-18)   /* "zero value on diagonal"                 ldl.go:62 ("zero on
                                diagonal." for UPPER, ldl.go:334)                     */
#define MO_EBKWORK (-19)     /* "Workspace too small"                    ldlbk.go:1121 */

typedef struct mo_ctx mo_ctx;

/* A device-resident column-major matrix view: element (i,j) is data[i + j*ld].  This is
 * a FloatMatrix view (FloatArray() from the view's (0,0), LeadingIndex() = ld) with its
 * backing array mirrored in device memory. */
typedef struct mo_matrix {
  double *data;
  int64_t rows;
  int64_t cols;
  int64_t ld;
} mo_matrix;

/* ---- context: device, stream, workspace, package-global settings ---- */
MO_API int mo_ctx_create(int device, mo_ctx **ctx);
MO_API int mo_ctx_destroy(mo_ctx *ctx);
/* stream is a cudaStream_t passed as void*; NULL selects the legacy default stream */
MO_API int mo_set_stream(mo_ctx *ctx, void *stream);
/* wait for all work on the context's stream; returns the first error recorded */
MO_API int mo_sync(mo_ctx *ctx);
MO_API const char *mo_strerror(int status);
/* BlockingParams(mb, nb, kb), mmult.go:63-67.  Only nb changes results here: it is the
 * diagonal block size of RankUpdateSym's beta (see mo_rank_update_sym). Returns 0. */
MO_API int mo_blocking_params(mo_ctx *ctx, int mb, int nb, int kb);
/* NumWorkers(n), mmult.go:69-73: kept for the shim; the GPU ignores it. Returns the old value. */
MO_API int mo_num_workers(mo_ctx *ctx, int n);
/* 1 = RankUpdateSym applies beta to the whole triangle (BLAS SYRK); 0 (default) = the
 * reference's behaviour, beta only inside the nb x nb diagonal blocks (calgo/dmmat_rank.c:
 * 28-56 vs 96-121).  Returns the old value. */
MO_API int mo_set_syrk_blas_beta(mo_ctx *ctx, int on);
/* No counterpart in the reference (its calls cannot wait on another thread of work): the
 * number of polls a device-side wait on another CTA's step flag makes before it gives up
 * and records MO_EDEVTIMEOUT (the triangular solves with at most 64 right-hand sides, i.e.
 * SolveCHOL / SolveTrm with few columns and the refinement of mo_dsposv_ir).  Default
 * MO_SPIN_LIMIT_DEFAULT; a failing wait ends its kernel early, leaves no copy in flight and
 * the context stays usable (mo_sync returns MO_EDEVTIMEOUT once, the next call runs
 * normally).  *old (optional) receives the previous value. */
#define MO_SPIN_LIMIT_DEFAULT (1u << 26)
MO_API int mo_set_spin_limit(mo_ctx *ctx, uint32_t polls, uint32_t *old);

/* ---- tracing: per-kernel-class device time (CUDA events on the context's stream) ---- */
#define MO_PROF_GEMM 0     /* DMMA GEMM / SYRK engine (trailing updates, TRSM sweeps)  */
#define MO_PROF_DIAG 1     /* diagonal-block Cholesky factor + inverse                  */
#define MO_PROF_TRTRI 2    /* diagonal-block triangular inverses for TRSM               */
#define MO_PROF_PANEL 3    /* LU panel (pivot search, interchanges, rank-1 updates)      */
#define MO_PROF_LASWP 4    /* row interchanges outside the panel                        */
#define MO_PROF_OTHER 5    /* everything else, incl. operand splits and FP32 conversions */
#define MO_PROF_LPGEMM 6   /* split-product (BF16x3 / TF32x3) tcgen05 GEMMs              */
#define MO_PROF_IR 7       /* refinement: FP64 residuals, norms, GMRES vector kernels   */
#define MO_PROF_BATCH 8    /* batched factor + solve launches (whole graph)              */
#define MO_PROF_CLASSES 9
typedef struct mo_profile {
  int64_t launches[MO_PROF_CLASSES]; /* kernel launches since the last reset            */
  double ms[MO_PROF_CLASSES];        /* summed device time (only while enabled)         */
  double flops[MO_PROF_CLASSES];     /* algorithmic flops of those launches             */
  double bytes[MO_PROF_CLASSES];     /* algorithmic DRAM bytes of those launches        */
} mo_profile;
/* on != 0: bracket every launch with CUDA events (adds ~2 events per launch) */
MO_API int mo_profile_enable(mo_ctx *ctx, int on);
/* synchronizes, fills *out with the totals since the last reset, then resets them */
MO_API int mo_profile_read(mo_ctx *ctx, mo_profile *out);
/* FP64 tensor-pipe throughput of this device: a register-resident mma.sync.f64 loop on
 * every SM for about `ms` milliseconds; *tflops receives the measured rate. */
MO_API int mo_measure_fp64_peak(mo_ctx *ctx, double ms, double *tflops);

/* ---- device memory helpers for shims that hold host-side matrices ---- */
MO_API int mo_malloc(mo_ctx *ctx, void **ptr, size_t bytes);
MO_API int mo_free(mo_ctx *ctx, void *ptr);
/* copy a host column-major matrix (leading dim ld_src) into the device view dst */
MO_API int mo_upload(mo_ctx *ctx, mo_matrix dst, const double *src, int64_t ld_src);
/* No counterpart in the reference (a host -> device helper for shims that hold host
 * matrices, like mo_upload): copy only the triangle that flags selects (MO_LOWER
 * default, MO_UPPER) of a square host matrix into the square device view dst, in
 * 128-column blocks that also carry the rest
 * of each 128 x 128 diagonal block: about n (n + 128) / 2 elements instead of n^2, for
 * the symmetric entry points that read one triangle.  The other triangle of dst is left
 * as it was.  Asynchronous on the context's stream. */
MO_API int mo_upload_tri(mo_ctx *ctx, mo_matrix dst, const double *src, int64_t ld_src, int flags);
/* copy the device view src into host memory with leading dim ld_dst */
MO_API int mo_download(mo_ctx *ctx, double *dst, int64_t ld_dst, mo_matrix src);
MO_API int mo_upload_bytes(mo_ctx *ctx, void *dst_dev, const void *src_host, size_t bytes);
MO_API int mo_download_bytes(mo_ctx *ctx, void *dst_host, const void *src_dev, size_t bytes);

/* ---- level 3 ---- */

/* Mult(C, A, B, alpha, beta, flags), mmult.go:198-256:
 *   C = beta*C + alpha*op(A)*op(B), op per MO_TRANSA / MO_TRANSB.
 * Empty product (per the flag-dependent rule of mmult.go:205-222) -> MO_OK, no work.
 * beta == 0 does not read C (calgo/vec_scale.c:118-133). */
MO_API int mo_mult(mo_ctx *ctx, mo_matrix C, mo_matrix A, mo_matrix B, double alpha, double beta,
            int flags);

/* RankUpdateSym(C, A, alpha, beta, flags), mmult.go:426-445 (SYRK):
 *   triangle(C) = beta*C + alpha*A*A^T   (MO_LOWER or MO_UPPER selects the triangle)
 *   triangle(C) = beta*C + alpha*A^T*A   with MO_TRANSA.
 * Non-square C -> MO_ECNOTSQUARE.  Rows of op(A) != rows of C -> MO_EABSIZE (the reference
 * does not check and reads out of range). */
MO_API int mo_rank_update_sym(mo_ctx *ctx, mo_matrix C, mo_matrix A, double alpha, double beta,
                       int flags);

/* SolveTrm(B, A, alpha, flags), mmult.go:388-422 (TRSM):
 *   B = alpha * op(A)^-1 * B   (MO_LEFT, or neither side bit)
 *   B = alpha * B * op(A)^-1   (MO_RIGHT)
 * A triangular: MO_UPPER selects upper, otherwise lower; MO_UNIT = unit diagonal;
 * MO_TRANSA = op(A) = A^T.  Size checks as mmult.go:394-407. */
MO_API int mo_solve_trm(mo_ctx *ctx, mo_matrix B, mo_matrix A, double alpha, int flags);

/* MultSym(C, A, B, alpha, beta, flags), mmult.go:266-330 (SYMM, calgo/dmmat_symm.c:253):
 *   C = beta*C + alpha*S*op(B)   without MO_RIGHT (MO_LEFT or no side bit: mmult.go:260's
 *                                default, which the reference's kernel computes for orders up
 *                                to its block size 68)
 *   C = beta*C + alpha*op(B)*S   with MO_RIGHT
 * S is the symmetric matrix whose upper (MO_UPPER) or lower triangle A stores; op(B) = B^T
 * with MO_TRANSB.  Size check and empty rule as mmult.go:273-291 (MO_ESYMSIZE); shapes
 * that pass it but do not fit the product -> MO_EABSIZE (the reference reads out of
 * range).  Asynchronous; uses n^2 doubles of context workspace. */
MO_API int mo_mult_sym(mo_ctx *ctx, mo_matrix C, mo_matrix A, mo_matrix B, double alpha,
                       double beta, int flags);

/* MultTrm(B, A, alpha, flags), mmult.go:338-375 (TRMM, calgo/dmmat_trid.c:780):
 *   B = alpha*op(T)*B   (MO_LEFT, or neither side bit)
 *   B = alpha*B*op(T)   (MO_RIGHT)
 * T triangular: MO_UPPER selects upper, otherwise lower; MO_UNIT = unit diagonal (not
 * read); op(T) = T^T with MO_TRANSA.  Size checks as mmult.go:343-355.  Asynchronous; uses
 * n^2 + size(B) doubles of context workspace. */
MO_API int mo_mult_trm(mo_ctx *ctx, mo_matrix B, mo_matrix A, double alpha, int flags);

/* RankUpdate2Sym(C, A, B, alpha, beta, flags), mmult.go:453-475 (SYR2K,
 * calgo/dmmat_rank.c:132):
 *   triangle(C) = beta*C + alpha*(A*B^T + B*A^T)     (A^T*B + B^T*A with MO_TRANSA)
 * MO_LOWER or MO_UPPER (exactly one) selects the triangle.  Like mo_rank_update_sym, beta
 * is applied inside the nb x nb diagonal blocks only (and there twice without MO_TRANSA,
 * as calgo/dmmat_rank.c:167, 228 do) unless mo_set_syrk_blas_beta(ctx, 1).  Non-square C
 * -> MO_ECNOTSQUARE; A and B of different shapes or op(A) rows != order of C ->
 * MO_EABSIZE (the reference does not check).  Asynchronous. */
MO_API int mo_rank_update2_sym(mo_ctx *ctx, mo_matrix C, mo_matrix A, mo_matrix B, double alpha,
                               double beta, int flags);

/* UpdateTrm(C, A, B, alpha, beta, flags), mmult.go:501-523 (calgo/dmmat_rank.c:292):
 *   triangle(C) = beta*C + alpha*op(A)*op(B)    (MO_UPPER selects upper, else lower)
 * beta inside the nb x nb diagonal blocks only unless mo_set_syrk_blas_beta(ctx, 1).  Non-
 * square C -> MO_ECNOTSQUARE; op(A) n x P and op(B) P x n not matching -> MO_EABSIZE.
 * Asynchronous. */
MO_API int mo_update_trm(mo_ctx *ctx, mo_matrix C, mo_matrix A, mo_matrix B, double alpha,
                         double beta, int flags);

/* InverseTrm(A, flags, nb), trinv.go:219-243: A := the inverse of its lower (MO_LOWER) or
 * upper (otherwise) triangle, in place; MO_UNIT: unit diagonal, not read or written.  The
 * opposite strict triangle is not touched.  Non-square A -> MO_ENOTSQUARE (the reference
 * does not check).  nb is accepted; the device blocks by 128 and doubles.  No singularity
 * check (a zero diagonal gives inf, as the reference's 1/a11).  Asynchronous; uses about
 * 1.25 n^2 doubles of context workspace. */
MO_API int mo_inverse_trm(mo_ctx *ctx, mo_matrix A, int flags, int nb);

/* ---- factorizations and solves ---- */

/* ---- QR with the compact WY form (qrwy.go, qrwym.go, house.go) ----
 *
 * A (m x n) = Q R, k = min(m, n) reflectors H(j) = I - tau_j v_j v_j^T (LAPACK dlarfg,
 * house.go:55-78), Q = H(0)...H(k-1) = I - Y T Y^T with Y the unit lower trapezoid stored
 * below A's diagonal and T the k x k upper triangular block reflector (LAPACK dlarft).
 * These compute the LAPACK quantities the reference's documentation names at every size.
 * The reference's own transposed GEMV (calgo/dmvec_gemv.c:368-395) rescales its output by
 * beta once per 68 rows, so its DecomposeQRT / BuildT / blocked DecomposeQR / MultQ give the
 * same T only while at most 68 rows lie below each reflector (m <= 69), and a different,
 * non-orthogonal Q beyond that.  W: the reference's workspace argument; data == NULL stands
 * for nil.  W is checked as the reference checks it; the device works in context workspace
 * (about (m + k) k + 2 max(m, n) 128 doubles).  m <= 148 * 895 rows, k <= 65535. */

/* DecomposeQRT(A, T, W, nb), qrwy.go:517-538: A = Q R in place, T's upper k x k triangle
 * set (its strict lower part untouched).  nb > 0 and A.cols > nb with a non-NULL W smaller
 * than A.cols x nb -> MO_EWORKSMALL; T smaller than k x k -> MO_ETSMALL.  The device
 * blocks by 32 / 128 whatever nb is (results agree to rounding).  Asynchronous. */
MO_API int mo_decompose_qrt(mo_ctx *ctx, mo_matrix A, mo_matrix T, mo_matrix W, int nb);

/* DecomposeQR(A, tau, W, nb), qrwy.go:474-497: as mo_decompose_qrt with the scalar factors
 * in tau (a vector view of at least k entries) instead of T (LAPACK DGEQRF). */
MO_API int mo_decompose_qr(mo_ctx *ctx, mo_matrix A, mo_matrix tau, mo_matrix W, int nb);

/* BuildT(T, A, tau), qrwy.go:546-556: T's upper triangle <- the block reflector of A's
 * reflectors and tau; columns whose tau is zero are not written (as the reference).  T
 * smaller than A.cols x A.cols -> MO_ETSMALL. */
MO_API int mo_build_t(mo_ctx *ctx, mo_matrix T, mo_matrix A, mo_matrix tau);

/* MultQT(C, A, T, W, flags, nb), qrwym.go:646-688: C = Q C (MO_LEFT or no side bit),
 * Q^T C (with MO_TRANS), C Q (MO_RIGHT), C Q^T (MO_RIGHT|MO_TRANS); Q from mo_decompose_qrt's
 * A and T, in the reference's order of reflectors.  nb (0: T.cols) sizes the W check as in
 * the reference; the device applies 256 reflectors at a time whatever nb is (results agree
 * to rounding).
 * W NULL -> MO_ENOWORK; MO_RIGHT with C.cols != A.rows -> MO_ECQSIZE; W smaller than
 * C.rows (MO_RIGHT) or C.cols (left) x nb -> MO_EWORKSMALL; left with C.rows != A.rows ->
 * MO_EABSIZE (unchecked by the reference).  Asynchronous. */
MO_API int mo_mult_qt(mo_ctx *ctx, mo_matrix C, mo_matrix A, mo_matrix T, mo_matrix W, int flags,
                      int nb);

/* MultQ(C, A, tau, W, flags, nb), qrwym.go:573-630: mo_mult_qt with Q from A and tau
 * (DORMQR); nb == 0 needs no W. */
MO_API int mo_mult_q(mo_ctx *ctx, mo_matrix C, mo_matrix A, mo_matrix tau, mo_matrix W, int flags,
                     int nb);

/* BuildQ(A, tau, W, nb), qrwyk.go:232-267 (DORGQR): A (m x n, m >= n, the reflectors of
 * mo_decompose_qr) := the first n columns of Q, columns of the identity taking the
 * reflectors in reverse order.  nb != 0 with W NULL -> MO_ENOWORK, W smaller than A.cols x nb
 * -> MO_EWORKSMALL; m < n -> MO_EABSIZE.  tau's first n entries are used (the reference
 * counts them from tau's end).  The reference's "zero the upper part" (qrwyk.go:75, :143) is
 * taken to clear the entries above the diagonal, as DORGQR does. */
MO_API int mo_build_q(mo_ctx *ctx, mo_matrix A, mo_matrix tau, mo_matrix W, int nb);

/* BuildQT(A, T, W, nb), qrwyk.go:278-293: mo_build_q with Q from mo_decompose_qrt's T
 * (nb == 0: A.cols; W NULL -> MO_ENOWORK). */
MO_API int mo_build_qt(mo_ctx *ctx, mo_matrix A, mo_matrix T, mo_matrix W, int nb);

/* SolveQRT(B, A, T, W, flags, nb), qrwym.go:784-819, A m x n with m >= n: least squares
 * X = argmin ||A X - B|| into B's first n rows (B = Q^T B, then R^-1); with MO_TRANS the
 * minimum-norm solution of A^T X = B (B's first n rows = R^-T B, the rows below cleared,
 * then B = Q B).  m < n or B.rows < n -> MO_EABSIZE. */
MO_API int mo_solve_qrt(mo_ctx *ctx, mo_matrix B, mo_matrix A, mo_matrix T, mo_matrix W,
                        int flags, int nb);

/* SolveQR(B, A, tau, W, flags, nb), qrwym.go:717-760: mo_solve_qrt with Q from tau.  With
 * MO_TRANS the reference rebinds B to an empty view before applying Q (qrwym.go:735); this
 * applies Q as mo_solve_qrt does. */
MO_API int mo_solve_qr(mo_ctx *ctx, mo_matrix B, mo_matrix A, mo_matrix tau, mo_matrix W,
                       int flags, int nb);

/* ---- symmetric indefinite LDL^T (ldlnp.go, ldl.go, ldlbk.go, ldlbks.go) ----
 *
 * MO_LOWER selects the lower triangle (A = L D L^T, unit L below the diagonal, D on it),
 * otherwise the upper (A = U D U^T).  ipiv: device int64 array of npiv >= n entries in the
 * reference's encoding (1-based partner rows; see each function).  The device runs the
 * reference's unblocked sweep (nb is checked as the reference checks it, then ignored): the
 * pivots are the reference's unblocked path's, values agree to rounding.  Orders up to
 * a few thousand; one cooperative launch with a grid barrier per pivot decision. */

/* DecomposeLDLnoPiv(A, W, flags, nb), ldlnp.go:211-235: no interchanges.  Non-square ->
 * MO_ENOTSQUARE; nb > 0 and n >= nb with W NULL -> MO_ELDLWORK.  Asynchronous. */
MO_API int mo_decompose_ldl_nopiv(mo_ctx *ctx, mo_matrix A, mo_matrix W, int flags, int nb);

/* SolveLDLnoPiv(B, A, flags), ldlnp.go:251-266: B = A^-1 B (unit solve, D, transposed unit
 * solve); neither MO_LOWER nor MO_UPPER -> no-op. */
MO_API int mo_solve_ldl_nopiv(mo_ctx *ctx, mo_matrix B, mo_matrix A, int flags);

/* DecomposeLDL(A, W, ipiv, flags, nb), ldl.go:439-466: 1 x 1 pivots, at each step the
 * largest |diagonal entry| of the part left (first one on ties) is brought to the front
 * with whole-row interchanges; ipiv[k] = 1-based partner or 0.  ipiv is zeroed first; npiv
 * < n -> MO_EPIVLEN; a zero pivot -> MO_EZERODIAG (A then partly factored).  Synchronizes. */
MO_API int mo_decompose_ldl(mo_ctx *ctx, mo_matrix A, mo_matrix W, int64_t *ipiv, int64_t npiv,
                            int flags, int nb);

/* SolveLDL(B, A, ipiv, flags), ldl.go:486-510: the interchanges, the two unit-triangular
 * solves and D, in the reference's order. */
MO_API int mo_solve_ldl(mo_ctx *ctx, mo_matrix B, mo_matrix A, const int64_t *ipiv,
                        int64_t npiv, int flags);

/* DecomposeBK(A, W, ipiv, flags, nb), ldlbk.go:1114-1140: Bunch-Kaufman (DSYTF2), 1 x 1 and
 * 2 x 2 pivots, interchanges inside the part not yet factored; ipiv[k] = 1-based partner
 * (k + 1 itself when none), both rows of a 2 x 2 block hold -(partner + 1).  W NULL or
 * smaller than n x 2 (n x (nb + 1) when nb > 0 and n >= nb) -> MO_EBKWORK; non-square ->
 * MO_ENOTSQUARE (the reference does not check); neither MO_LOWER nor MO_UPPER -> no-op.
 * Asynchronous. */
MO_API int mo_decompose_bk(mo_ctx *ctx, mo_matrix A, mo_matrix W, int64_t *ipiv, int64_t npiv,
                           int flags, int nb);

/* SolveBK(B, A, ipiv, flags), ldlbks.go:303-318 (DSYTRS): B = A^-1 B with DecomposeBK's
 * factor.  LOWER follows unblkSolveBKLower's two sweeps; for UPPER the reference's sweeps
 * run over empty and mismatched blocks of B (ldlbks.go:159-296), and this solves with the
 * UPPER factor through the same steps on the index-reversed problem. */
MO_API int mo_solve_bk(mo_ctx *ctx, mo_matrix B, mo_matrix A, const int64_t *ipiv, int64_t npiv,
                       int flags);

/* DecomposeCHOL(A, flags, nb), chol.go:116-127: A = L*L^T (MO_LOWER) or U^T*U (otherwise)
 * in place; the opposite strict triangle is not referenced.  Non-square -> MO_ENOTSQUARE.
 * nb is the reference's block size; the device picks its own blocking (results agree to
 * rounding).  Synchronizes; returns k+1 > 0 when column k's pivot is not positive
 * (sqrt gives NaN), with that pivot's value in *bad_value if non-NULL; A's contents are
 * then unspecified. */
MO_API int mo_decompose_chol(mo_ctx *ctx, mo_matrix A, int flags, int nb, double *bad_value);

/* SolveCHOL(B, A, flags), chol.go:147-158: B = (A A^T)^-1 B with the factor from
 * mo_decompose_chol (MO_UPPER checked first, then MO_LOWER; neither -> no-op). */
MO_API int mo_solve_chol(mo_ctx *ctx, mo_matrix B, mo_matrix A, int flags);

/* DecomposeLU(A, pivots, nb), lu.go:257-272: P*A = L*U with partial pivoting, L unit lower
 * (diagonal not stored), in place.  pivots: device int64 array of npiv entries; on return
 * pivots[k] is the 0-based absolute row swapped with row k (pivots[k] == k: no swap),
 * entries >= min(rows,cols) are set to 0.  npiv < min(rows,cols) -> MO_EPIVLEN.  The pivot
 * at each column is the first row holding the largest |value| (pivot.go:98-107). */
MO_API int mo_decompose_lu(mo_ctx *ctx, mo_matrix A, int64_t *pivots, int64_t npiv, int nb);

/* SolveLU(B, A, pivots, flags), lu.go:320-334: apply the row swaps to B in forward order
 * (pivot.go:55-61), then B = U^-1 L^-1 B; with MO_TRANSA the same swaps followed by
 * L^-T then U^-T, exactly the reference's sequence. */
MO_API int mo_solve_lu(mo_ctx *ctx, mo_matrix B, mo_matrix A, const int64_t *pivots, int64_t npiv,
                int flags);

/* ---- mixed-precision Cholesky solve with FP64 refinement (no counterpart in the
 * reference; LAPACK's dsposv is the model) ---- */

/* low-precision factor arithmetic: every O(n^3) product is formed from three tensor-core
 * products of split operands with FP32 accumulation, on an FP32 copy of A */
#define MO_PREC_BF16X3 1 /* x = bf16 hi + bf16 lo (about 16 significant bits)     */
#define MO_PREC_TF32X3 2 /* x = tf32 hi + tf32 lo (FP32 accuracy: "FP32" factor)   */
/* refinement method (low byte) and option bits */
#define MO_IR_AUTO 0          /* classic refinement, GMRES-IR once it converges slowly  */
#define MO_IR_CLASSIC 1       /* x += (L L^T)^-1 (b - A x)                              */
#define MO_IR_GMRES 2         /* x += GMRES(A, b - A x) preconditioned by (L L^T)^-1    */
#define MO_IR_NO_FALLBACK 0x100 /* do not re-solve in FP64 when refinement fails      */
#define MO_IR_HISTORY 32
typedef struct mo_ir_info {
  int iters;        /* refinement steps taken (corrections applied)                    */
  int gmres_iters;  /* inner GMRES iterations, summed over the steps                   */
  int converged;    /* 1 if berr <= tol                                                */
  int fallback;     /* 1 if X came from the FP64 factorization (DecomposeCHOL path)    */
  int shifts;       /* low-precision factorizations retried with a diagonal shift      */
  int method;       /* MO_IR_CLASSIC or MO_IR_GMRES: the method of the last step       */
  int abandoned;    /* 1 if MO_IR_AUTO stopped refining because the steps it projected
                       from the last reduction would cost more than the FP64 path, or a
                       classic step reduced berr less than 3x (a GMRES step is also cut
                       off once it has run as long as the FP64 path would)             */
  int prec;         /* split format of the factor used: MO_PREC_BF16X3, or MO_PREC_TF32X3
                       also when MO_IR_AUTO moved from a BF16x3 factor that broke down   */
  double berr;      /* max over columns of |b - A x|_inf / (|A|_inf |x|_inf + |b|_inf) */
  double shift;     /* relative diagonal shift of the factored matrix (0 = none)       */
  double history[MO_IR_HISTORY]; /* berr before each step (history[0]: x = 0)          */
} mo_ir_info;
/* X = A^-1 B for symmetric positive definite A (n x n, float64; only the triangle that
 * flags selects, MO_LOWER (default) or MO_UPPER, is read; A is not modified).  A is
 * factored as L L^T in the low precision `prec` and X is refined in FP64 until the
 * normwise backward error is <= tol, for at most maxit steps (method as above).  If the
 * low-precision factorization breaks down, it is retried on A + s*diag(A) with a growing
 * relative shift s (with MO_IR_AUTO, a BF16x3 factor that breaks down is first redone with
 * the TF32x3 split, unshifted).  MO_IR_AUTO also stops refining when the GMRES-IR steps it
 * projects from the last reduction would cost more than the FP64 path, and falls back.
 * Unless MO_IR_NO_FALLBACK is set, a solve that does not converge is
 * redone with the FP64 factorization.  B and X are n x nrhs (X may be B).  Returns 0, a
 * size/argument error, or i > 0 if the FP64 fallback found A not positive definite at
 * column i - 1.  `info` may be NULL.  Synchronous. */
MO_API int mo_dsposv_ir(mo_ctx *ctx, mo_matrix X, mo_matrix A, mo_matrix B, int flags, int prec,
                        int method, double tol, int maxit, mo_ir_info *info);

/* The split-product GEMM of the factorization as a plain operation on FP32 data:
 * C = alpha*op(A)*op(B) + beta*C, C M x N, op(A) M x K, op(B) K x N, column-major float
 * device arrays; flags: MO_TRANSA, MO_TRANSB, and MO_LOWER to update only C(i, j) with
 * i >= j (N <= M).  Asynchronous on the context's stream. */
MO_API int mo_lp_gemm(mo_ctx *ctx, int prec, int64_t M, int64_t N, int64_t K, float alpha,
                      const float *A, int64_t lda, const float *B, int64_t ldb, float beta,
                      float *C, int64_t ldc, int flags);

/* ---- reverse mode (no counterpart in the reference: the adjoints of DecomposeCHOL,
 * chol.go:116, and SolveCHOL, chol.go:147, for LOWER factors) ---- */

/* Given the factor L of A = L L^T (as mo_decompose_chol leaves it with MO_LOWER; only
 * its lower triangle is read) and Lbar, the adjoint of L (lower triangle read), overwrite
 * Lbar with the symmetric gradient Abar (both triangles): for every symmetric
 * perturbation dA, d(loss) = sum_ij Abar_ij dA_ij.  Blocked right to left on the FP64
 * GEMM engine, about 2 n^3 / 3 flops; it reads no stored forward panel and needs only a
 * few 128 x 128 blocks of scratch.  flags: MO_LOWER (MO_UPPER -> MO_EINVAL).
 * Asynchronous on the context's stream. */
MO_API int mo_decompose_chol_adjoint(mo_ctx *ctx, mo_matrix L, mo_matrix Lbar, int flags);
/* The same for `count` independent matrices (host arrays of views), spread over a pool of
 * streams forked from and joined back into the context's stream. */
MO_API int mo_decompose_chol_adjoint_batched(mo_ctx *ctx, int count, const mo_matrix *L,
                                             const mo_matrix *Lbar, int flags);
/* Adjoint of X = A^-1 B solved with the factor L (SolveCHOL LOWER): Xbar (n x nrhs) is
 * overwritten with Bbar = A^-1 Xbar, and Abar (n x n) receives Abar -= (Bbar X^T +
 * X Bbar^T) / 2, the symmetric gradient of the solve with respect to A.  Asynchronous. */
MO_API int mo_solve_chol_adjoint(mo_ctx *ctx, mo_matrix L, mo_matrix X, mo_matrix Xbar,
                                 mo_matrix Abar, int flags);

/* ---- batched factor + solve of many small systems (no counterpart in the reference,
 * which factors one matrix per call: DecomposeCHOL chol.go:116 / SolveCHOL chol.go:147,
 * DecomposeLU lu.go:257 / SolveLU lu.go:320; each matrix gets the same results those
 * calls give, to rounding, and the same pivots) ---- */
#define MO_BATCH_CHOL 1     /* A_i = L_i L_i^T (lower; the strict upper part is not read) */
#define MO_BATCH_LU 2       /* P_i A_i = L_i U_i with partial pivoting                    */
#define MO_BATCH_MAX_N 512  /* largest order in a batch                                   */
#define MO_BATCH_BUCKETS 4  /* schedule buckets: n <= 64, <= 128, <= 256, <= 512         */
typedef struct mo_batch mo_batch;
/* A plan for `count` square matrices of orders n[0..count) (host array, 1..MO_BATCH_MAX_N,
 * else MO_EBATCHN), each with nrhs right-hand sides (0: factor only).  The plan orders the
 * matrices longest first, groups them by the kernel configuration chosen for their size
 * bucket and records one CUDA graph (queue reset + one persistent kernel per group, the
 * group with the largest matrices first) on its first run. */
MO_API int mo_batch_create(mo_ctx *ctx, int kind, int count, const int32_t *n, int nrhs,
                           mo_batch **plan);
MO_API int mo_batch_destroy(mo_batch *plan);
/* Factor every A_i in place and, when B is non-NULL, solve A_i X_i = B_i in place (B_i is
 * n_i x nrhs).  All arrays are DEVICE arrays of `count` entries: A / B / piv hold device
 * pointers, lda / ldb leading dimensions (>= n_i).  piv (LU only) receives n_i 0-based
 * row indices per matrix (piv[k] = row exchanged with row k).  info[i] = 0, or for
 * Cholesky the column + 1 whose pivot is not positive (that matrix is left partially
 * factored and not solved), for LU the first column + 1 with an exactly zero pivot.
 * Asynchronous on the context's stream: one graph launch; a call with other pointer
 * arrays updates the graph's kernel parameters instead of re-recording it. */
MO_API int mo_batch_run(mo_batch *plan, double *const *A, const int64_t *lda, double *const *B,
                        const int64_t *ldb, int64_t *const *piv, int *info);
/* Autotuner: for each size bucket in the plan, times every kernel configuration (panel
 * width 32 or 16, CTAs per SM) on synthetic matrices of the plan's own orders (`reps`
 * timed runs each, best kept) and keeps the fastest.  ms (optional, MO_BATCH_BUCKETS x 2
 * doubles) receives the times (-1 where a bucket is empty).  Synchronous. */
MO_API int mo_batch_tune(mo_batch *plan, int reps, double *ms);
/* Read (set = 0) or replace (set = 1) the per-bucket configuration table (MO_BATCH_BUCKETS
 * ints, each 0 or 1), e.g. to persist a tuned schedule and restore it in a later run. */
MO_API int mo_batch_schedule(mo_batch *plan, int *cfg, int set);

/* ---- device mirrors of host arrays: residency for a shim that holds FloatMatrix data
 * in host slices (no counterpart in the reference, whose calls work in place on host
 * views, FloatArray() + LeadingIndex(), mmult.go:228-233; views of one array overlap,
 * partition.go:210-340) ---- */
typedef struct mo_mirror mo_mirror;
/* Register the host array [host, host + count) (a FloatMatrix's whole backing slice) with
 * the context: device memory of the same size is allocated on the first device view.  A
 * range overlapping a registered one -> MO_EINVAL. */
MO_API int mo_mirror_create(mo_ctx *ctx, double *host, int64_t count, mo_mirror **mirror);
/* Unregister and free the device copy (the host array is untouched). */
MO_API int mo_mirror_destroy(mo_mirror *mirror);
/* The registered array that contains host address p, and p's element offset in it; a
 * view of any sub-matrix maps to its root array this way.  Not registered -> MO_EINVAL. */
MO_API int mo_mirror_find(const double *p, mo_mirror **mirror, int64_t *offset);
/* Device view of the host view (p, rows, cols, ld) inside the mirror: uploads the whole
 * array first if the host copy is newer; write != 0 marks the device copy newer.  The view
 * must lie inside the array, else MO_EINVAL. */
MO_API int mo_mirror_view(mo_mirror *mirror, const double *p, int64_t rows, int64_t cols,
                          int64_t ld, int write, mo_matrix *out);
/* Bring the host array up to date (download if the device copy is newer); synchronous. */
MO_API int mo_mirror_to_host(mo_mirror *mirror);
/* The caller changed the host array: the next device view uploads it.  MO_EINVAL if the
 * device copy also has changes not yet brought back (mo_mirror_to_host first). */
MO_API int mo_mirror_host_modified(mo_mirror *mirror);
/* 0 = copies equal, 1 = host newer, 2 = device newer */
MO_API int mo_mirror_state(const mo_mirror *mirror);

/* ---- allocation-free variant (no counterpart in the reference) ---- */

/* Largest order of A accepted by mo_solve_trm_static. */
#define MO_SOLVE_TRM_STATIC_MAX_N 1024

/* mo_solve_trm_static: the triangular solve of mo_solve_trm (same arguments, flags, size
 * checks and results) for callers that must not have a library allocate device memory --
 * e.g. an application whose GPU memory is all handed out by its own pool allocator, a
 * service held to a fixed footprint on a shared GPU, or a latency-critical loop that cannot
 * pay for cudaMalloc's implicit synchronization.  It needs no context and calls no
 * allocation routine: its only scratch is a 1 MiB block compiled into this library, which
 * every GPU that loads the library keeps until the process exits.
 *   - order of A (A's column count) > MO_SOLVE_TRM_STATIC_MAX_N -> MO_ESTATICLIMIT.
 *   - runs on `stream` (a cudaStream_t, NULL = legacy default stream) of the current device
 *     and waits for it; returns 0, a size error, or a device-side failure code.
 *   - every call on a device uses the same block, which keeps the previous call's data:
 *     calls that overlap on the GPU race; serialize them.
 *   - every call looks the block's device address up with the caller's device current
 *     (allocating nothing); the first call on a device also loads this library's kernels
 *     there, so make it before any stream capture begins. */
MO_API int mo_solve_trm_static(mo_matrix B, mo_matrix A, double alpha, int flags, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MATOPS_B200_H */
