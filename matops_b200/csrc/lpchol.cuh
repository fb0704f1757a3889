// Mixed-precision Cholesky factor (lpchol.cu): workspace layout and entry points.
#pragma once
#include "lp.cuh"

namespace mo {

struct LpChol {
  int n = 0, NP = 0, prec = 0;
  float *W = nullptr;  // NP x NP FP32 working matrix; its lower triangle becomes L
  int64_t ldw = 0;
  double *inv = nullptr;  // NP/128 FP64 inverses of L's 128 x 128 diagonal blocks
  LpSplit Linv{};         // split inverse of the current diagonal block
  LpSplit PA{};           // split A21 of the next panel (256 wide: two block columns)
  LpSplit P[2]{};         // split L21 of a pair of panels side by side (K-major, 256
                          // wide), by pair parity
};

// device bytes for the workspace of an order-n factorization
size_t lp_chol_bytes(int n, int prec);
// carve the workspace out of `mem` (lp_chol_bytes(n, prec) bytes)
int lp_chol_setup(int n, int prec, void *mem, LpChol &f);
// W = FP32(lower triangle of A) (upper: transpose of its upper triangle), diagonal scaled
// by (1 + shift), identity padding
int lp_chol_convert(mo_ctx *ctx, const LpChol &f, View A, bool upper, double shift);
// factor W in place; a failing pivot sets *d_info = column + 1 (device word)
int lp_chol_factor(mo_ctx *ctx, LpChol &f, int *d_info, double *d_bad);

// Triangular solves with the factor (lpsolve.cu): the FP64 inverses of its
// kLpSolveBlock x kLpSolveBlock diagonal blocks and the scratch of the solve steps
constexpr int kLpSolveBlock = 1024;
struct LpSolve {
  int n = 0, NP = 0, nblk = 0, nrhs = 0, sms = 0;
  const float *W = nullptr;  // the factor (lp_chol_factor's W), read in place
  int64_t ldw = 0;
  double *Dinv = nullptr;    // nblk blocks, each kLpSolveBlock^2 column-major (ld kLpSolveBlock)
  double *T = nullptr;       // scratch of the block-inverse merges
  double *Y = nullptr;       // n x min(nrhs, 64): the forward solve's result
  double *part[2] = {};      // partial sums of the K-split products, per stream
  unsigned *cnt[2] = {};     // per 64-row tile: K chunks finished (zero between launches)
};
size_t lp_solve_bytes(int n, int nrhs, int sms);
int lp_solve_setup(int n, int nrhs, int sms, void *mem, LpSolve &s);
// after lp_chol_factor: the diagonal-block inverses (and the factor's address)
int lp_solve_prepare(mo_ctx *ctx, const LpChol &f, LpSolve &s);
// D (n x nr, ld n) <- (L L^T)^-1 D; every launch returns at once while *skip != 0
int lp_solve_apply(mo_ctx *ctx, const LpSolve &s, double *D, int nr, const int *skip);

}  // namespace mo
