/*
 * oracle/calgo_iface.h -- TEST INFRASTRUCTURE ONLY (the oracle), never product code.
 *
 * The kernel-level interface that the restated Go drivers (oracle/drivers.c) call.
 * Names, argument order and the two view structs are kept identical to the C kernels
 * of hrautila/matops (calgo/cmops.h:50-58 for mdata_t/mvec_t, cmops.h:14-25 for the
 * flag values, and the prototypes at cmops.h:135-213) so that the SAME driver source
 * links either against this repository's restatement (oracle/calgo_port.c) or against
 * the reference's own calgo C files compiled from its sources (oracle/_ref).
 */
#ifndef MATOPS_ORACLE_CALGO_IFACE_H
#define MATOPS_ORACLE_CALGO_IFACE_H

enum {
  MTX_NOTRANS = 0,
  MTX_TRANSA  = 0x1,
  MTX_TRANSB  = 0x2,
  MTX_LOWER   = 0x4,
  MTX_UPPER   = 0x8,
  MTX_LEFT    = 0x10,
  MTX_RIGHT   = 0x20,
  MTX_UNIT    = 0x40,
  MTX_TRANS   = 0x80
};

/* column-major block: md -> element (0,0), step = column stride */
typedef struct mdata { double *md; int step; } mdata_t;
/* strided vector: md -> element 0, inc = element stride */
typedef struct mvec { double *md; int inc; } mvec_t;

void dmult_mm_blocked3(mdata_t *C, const mdata_t *A, const mdata_t *B,
                       double alpha, double beta, int flags,
                       int P, int S, int L, int R, int E, int vlen, int NB, int MB);
void dmmat_rank_blk(mdata_t *C, const mdata_t *A, double alpha, double beta,
                    int flags, int P, int S, int E, int vlen, int NB);
void dmmat_solve_blk(mdata_t *B, const mdata_t *A, double alpha, int flags,
                     int N, int S, int E, int NB);
void dmvec_symv_rank(mdata_t *A, const mvec_t *X, double alpha, int flags,
                     int S, int L, int NB);
void dmult_gemv_blocked(mvec_t *Y, const mdata_t *A, const mvec_t *X,
                        double alpha, double beta, int flags,
                        int S, int L, int R, int E, int vlen, int MB);
void dmvec_solve_blocked(mvec_t *X, const mdata_t *A, int flags, int N, int NB);
double dvec_dot(const mvec_t *X, const mvec_t *Y, double alpha, int N);
void dvec_invscal(mvec_t *X, double alpha, int N);
void dvec_swap(mvec_t *X, mvec_t *Y, int N);
void dmvec_rank(mdata_t *A, const mvec_t *X, const mvec_t *Y, double alpha, int S, int L, int R,
                int E, int NB, int MB);
void dvec_scal(mvec_t *X, double alpha, int N);
/* the rest of the level-3 surface (calgo/cmops.h:149-152, 200-201, 218-226) */
void dmult_symm_blocked2(mdata_t *C, const mdata_t *A, const mdata_t *B,
                         double alpha, double beta, int flags,
                         int P, int S, int L, int R, int E, int vlen, int NB, int MB);
void dmmat_trmm_blk(mdata_t *B, const mdata_t *A, double alpha, int flags,
                    int N, int S, int E, int NB);
void dmmat_rank2_blk(mdata_t *C, const mdata_t *A, const mdata_t *B,
                     double alpha, double beta, int flags, int P, int S, int E, int vlen, int NB);
void dmmat_trmupd_blk(mdata_t *C, const mdata_t *A, const mdata_t *B, double alpha, double beta,
                      int flags, int P, int S, int E, int vlen, int NB);

/* the QR path's level-1/2 kernels (calgo/cmops.h:107, 117-119, 193) */
double dvec_nrm2(const mvec_t *X, int N);
void dmmat_scale_plus(mdata_t *A, const mdata_t *B, double alpha, double beta, int flags,
                      int S, int L, int R, int E);
void dmvec_trid_unb(mvec_t *X, const mdata_t *A, int flags, int N);
/* the LDL^T path's triangular rank-1 update (calgo/cmops.h:181) */
void dmvec_trmv_upd(mdata_t *A, const mvec_t *X, const mvec_t *Y, double alpha, int flags, int S,
                    int L, int NB);

#endif
