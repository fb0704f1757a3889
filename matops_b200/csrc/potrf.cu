// Blocked Cholesky factorization (DecomposeCHOL) and solve (SolveCHOL) on the device.
//
// Reference: chol.go:58-94 (blockedCHOL, right-looking FLAME variant 3) with the panel
// chol.go:17-56 (unblockedCHOL: sqrt, true division, SYR), SolveCHOL chol.go:147-158.
// Here the nb x nb diagonal block (nb = 128) is factored AND inverted by one CTA in
// shared memory (potrf_diag_kernel); the panel below becomes one in-place GEMM with the
// inverse (A21 <- A21 * L11^-T) and the trailing update one SYRK, both on the FP64
// tensor pipe.  A failing pivot (sqrt -> NaN, chol.go:34-36) is recorded in a device
// info word; every later diagonal kernel sees it and does nothing.
#include "context.cuh"
#include "tri.cuh"

namespace mo {
namespace {

constexpr int NB = 128;

__global__ void __launch_bounds__(TRI_THREADS)
    potrf_diag_kernel(double *A, int64_t lda, int n, bool upper, double *inv, int *info,
                      double *bad_value, int col0) {
  if (*(volatile int *)info != 0) return;  // an earlier block failed
  extern __shared__ double sm[];
  double *S = sm;
  double *W = sm + TRI_MAX * LDS;
  __shared__ int s_bad;
  __shared__ double s_badv;
  const int NP = round_up32(n);
  // upper storage: A = U^T U with U^T lower, so load/store the transpose
  tri_load_lower(S, A, lda, n, upper, false);
  __syncthreads();
  tri_potrf_lower(S, NP, &s_bad, &s_badv);
  if (s_bad >= 0) {
    if (threadIdx.x == 0) {
      *info = col0 + s_bad + 1;
      *bad_value = s_badv;
    }
    return;
  }
  tri_store_lower(S, A, lda, n, upper, false);
  __syncthreads();
  tri_inverse_lower(S, NP, W);
  __syncthreads();
  tri_store_lower(S, inv, NB, n, false, true);
}

}  // namespace

namespace {

int set_diag_smem() {
  return mo_smem_attr((const void *)potrf_diag_kernel, TRI_SMEM_BYTES);
}

// Panel step at column k (block order b) on ctx->stream: factor + invert the diagonal
// block, then L21 = A21 * L11^-T (lower) or U12 = U11^-T * A12 (upper) in place.
int panel(mo_ctx *ctx, View A, bool upper, int k, int b, int *d_info, double *d_bad, double *inv,
          bool stream_k) {
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_DIAG);
  potrf_diag_kernel<<<1, TRI_THREADS, TRI_SMEM_BYTES, ctx->stream>>>(A.at(k, k), A.ld, b, upper,
                                                                     inv, d_info, d_bad, k);
  // factor b^3/3 + inverse b^3/3; reads the triangle, writes it and the inverse
  prof_end(ctx, ps, 2.0 * b * b * b / 3.0, 8.0 * 2.0 * b * b);
  MO_CUDA_TRY(cudaGetLastError());
  const int rest = A.rows - k - b;
  if (rest <= 0) return MO_OK;
  const View Linv{inv, b, b, NB};
  GemmOpts o;
  o.stream_k = stream_k;
  if (!upper) {
    const View A21 = A.sub(k + b, k, rest, b);
    return gemm_ex(ctx, A21, A21, false, Linv, true, 1.0, 0.0, o);  // A21 * L11^-T
  }
  const View A12 = A.sub(k, k + b, b, rest);
  return gemm_ex(ctx, A12, Linv, false, A12, false, 1.0, 0.0, o);  // U11^-T * A12
}

}  // namespace

// Right-looking blocked Cholesky, two 128-column steps per trailing update (K = 256: the
// trailing matrix is read and written once per pair), with look-ahead: pair p covers
// block columns a and b = a + 1.
//   S1 (aux):  [panel a] [column b -= L_b,a L_b,a^T] [panel b] -> record E1
//   S0 (main): wait E1 -> [the next pair's two columns, K = 256] -> record E0 -> [the rest
//              of the trailing matrix, K = 256, leaving a few SMs to S1]
//   S1 waits E0 before the next pair.  (Upper storage: the same on U = L^T.)
int potrf(mo_ctx *ctx, View A, bool upper, int *d_info, double *d_bad, double *inv) {
  int rc = set_diag_smem();
  if (rc) return rc;
  const int n = A.rows;
  if (n <= NB) return panel(ctx, A, upper, 0, n, d_info, d_bad, inv, true);
  cudaStream_t s0 = ctx->stream, s1 = nullptr;
  if ((rc = aux_stream(ctx, &s1))) return rc;
  if ((rc = stream_wait(ctx, s1, s0, ctx->ev_fork))) return rc;
  const int free_sms = 8;  // SMs the trailing update leaves to the look-ahead stream
  // C (rows r0.., columns c0.., r x c) -= op(P) op(Q) over the panel columns [k0, k0 + K)
  auto update = [&](int r0, int c0, int r, int c, int k0, int K, int mode, int max_ctas) {
    GemmOpts o;
    o.mode = mode;
    o.stream_k = false;
    o.max_ctas = max_ctas;
    if (!upper)
      return gemm_ex(ctx, A.sub(r0, c0, r, c), A.sub(r0, k0, r, K), false, A.sub(c0, k0, c, K), true,
                     -1.0, 1.0, o);
    return gemm_ex(ctx, A.sub(r0, c0, r, c), A.sub(k0, r0, K, r), true, A.sub(k0, c0, K, c), false,
                   -1.0, 1.0, o);
  };
  for (int ka = 0; ka < n; ka += 2 * NB) {
    const int ba = min(NB, n - ka), kb = ka + ba;
    const int bb = kb < n ? min(NB, n - kb) : 0;
    {
      StreamSwap sw(ctx, s1);
      if ((rc = panel(ctx, A, upper, ka, ba, d_info, d_bad, inv, false))) return rc;
      if (bb > 0) {
        // column (row) block b, rows (columns) kb..n: the triangle of its diagonal block only
        const int rest = n - kb;
        if (!upper) rc = update(kb, kb, rest, bb, ka, ba, kGemmLower, 0);
        else rc = update(kb, kb, bb, rest, ka, ba, kGemmUpper, 0);
        if (rc) return rc;
        if ((rc = panel(ctx, A, upper, kb, bb, d_info, d_bad, inv, false))) return rc;
      }
    }
    if ((rc = stream_wait(ctx, s0, s1, ctx->ev_join))) return rc;  // the pair's panels done
    const int kc = kb + bb, rest = n - kc;
    if (bb == 0 || rest <= 0) break;
    const int K = ba + bb;
    // 1. the next pair's block columns (rows for upper storage), K = 256
    const int nn = min(2 * NB, rest);
    if (!upper) rc = update(kc, kc, rest, nn, ka, K, kGemmLower, 0);
    else rc = update(kc, kc, nn, rest, ka, K, kGemmUpper, 0);
    if (rc) return rc;
    if ((rc = stream_wait(ctx, s1, s0, ctx->ev_fork))) return rc;
    // 2. the rest of the trailing matrix, K = 256
    const int r2 = rest - nn;
    if (r2 > 0 &&
        (rc = update(kc + nn, kc + nn, r2, r2, ka, K, upper ? kSyrkUpper : kSyrkLower,
                     ctx->sms - free_sms)))
      return rc;
  }
  return MO_OK;
}

}  // namespace mo
