// Low-precision building blocks of the mixed-precision Cholesky solve: FP32 storage,
// split-product GEMMs on the tensor cores (mma.sync) with FP32 accumulation.
//
// An FP32 value x is split into a high and a low part, x ~ hi + lo, and a product is
// formed from three tensor-core products, a*b ~ hi_a*hi_b + hi_a*lo_b + lo_a*hi_b:
//   kLpBf16x3 : hi = bf16(x), lo = bf16(x - hi)      (about 16 significant bits)
//   kLpTf32x3 : hi = tf32(x), lo = tf32(x - hi)      (about FP32 accuracy)
// Operands are stored pre-split and K-major ("rows x k", element (r, k) at r * ldk + k),
// so the GEMM's inner loop does no conversion: the split happens once per panel.
#pragma once
#include "context.cuh"

namespace mo {

enum LpPrec { kLpBf16x3 = 1, kLpTf32x3 = 2 };

inline int lp_esize(int prec) { return prec == kLpBf16x3 ? 2 : 4; }

// a pre-split operand: `rows` x k elements, K-major, hi and lo parts (each rows * ldk
// elements of 2 (bf16) or 4 (tf32, FP32 bit pattern) bytes)
struct LpSplit {
  void *hi;
  void *lo;
  int64_t ldk;  // elements between consecutive rows (multiple of 32)
};

inline LpSplit lp_rows(const LpSplit &s, int prec, int64_t r0) {
  const int64_t off = r0 * s.ldk * lp_esize(prec);
  return LpSplit{(char *)s.hi + off, (char *)s.lo + off, s.ldk};
}

// C (FP32, column-major, M x N) = beta*C + alpha * A * B^T, where A is an M-row split
// operand and B an N-row split operand, both with K columns.  M and N are multiples of
// 128, K a multiple of 32.  mode kGemmLower updates only C(i, j) with i >= j (tiles
// wholly above the diagonal are skipped).  max_ctas > 0 caps the persistent grid.
struct LpGemmArgs {
  int M = 0, N = 0, K = 0;
  float alpha = 1.f, beta = 0.f;
  LpSplit A{}, B{};
  float *C = nullptr;
  int64_t ldc = 0;
  int mode = kGemm;
  int max_ctas = 0;
  // optional: also write rows out_row0 .. M - 1 of the result, split, to `out` (K-major:
  // out row r - out_row0 holds C's row r, columns 0 .. N - 1); needs a TMA-compatible C
  LpSplit out{};
  int out_row0 = 0;
};
int lp_gemm(mo_ctx *ctx, int prec, const LpGemmArgs &a);

// split X (rows x cols FP32, column-major, ld) into out (K-major: out row r = row r of X)
int lp_split(mo_ctx *ctx, int prec, const float *X, int64_t ld, int rows, int cols, LpSplit out);

}  // namespace mo
