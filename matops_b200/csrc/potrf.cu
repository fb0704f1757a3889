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

// Right-looking blocked Cholesky with one step of look-ahead: the panel of step k+1
// (diagonal factor + TRSM) runs on a second, high-priority stream while the trailing
// SYRK of step k runs on the caller's stream with a few SMs left free for it.
//   S0 (caller):  [update next panel column k+1 | record E0] [SYRK rest of step k]
//   S1 (aux):     wait E0 -> panel(k+1) -> record E1            (S0 waits E1 at k+1)
int potrf(mo_ctx *ctx, View A, bool upper, int *d_info, double *d_bad, double *inv) {
  int rc = set_diag_smem();
  if (rc) return rc;
  const int n = A.rows;
  if (n <= NB) return panel(ctx, A, upper, 0, n, d_info, d_bad, inv, true);
  cudaStream_t s0 = ctx->stream, s1 = nullptr;
  if ((rc = aux_stream(ctx, &s1))) return rc;
  if ((rc = stream_wait(ctx, s1, s0, ctx->ev_fork))) return rc;
  const int free_sms = 8;  // SMs the trailing update leaves to the look-ahead panel
  {
    StreamSwap sw(ctx, s1);
    if ((rc = panel(ctx, A, upper, 0, NB, d_info, d_bad, inv, false))) return rc;
  }
  for (int k = 0; k < n; k += NB) {
    const int b = min(NB, n - k);
    const int rest = n - k - b;
    if ((rc = stream_wait(ctx, s0, s1, ctx->ev_join))) return rc;  // panel k done
    if (rest <= 0) break;
    const int b2 = min(NB, rest);
    // 1. next panel column: rows k+b.., columns k+b..k+b+b2, one triangle only
    GemmOpts onext;
    onext.mode = upper ? kGemmUpper : kGemmLower;
    onext.stream_k = false;
    if (!upper) {
      const View A21 = A.sub(k + b, k, rest, b);
      rc = gemm_ex(ctx, A.sub(k + b, k + b, rest, b2), A21, false, A.sub(k + b, k, b2, b), true,
                   -1.0, 1.0, onext);
    } else {
      const View A12 = A.sub(k, k + b, b, rest);
      rc = gemm_ex(ctx, A.sub(k + b, k + b, b2, rest), A.sub(k, k + b, b, b2), true, A12, false,
                   -1.0, 1.0, onext);
    }
    if (rc) return rc;
    if ((rc = stream_wait(ctx, s1, s0, ctx->ev_fork))) return rc;
    // 2. panel k+b on the look-ahead stream
    {
      StreamSwap sw(ctx, s1);
      if ((rc = panel(ctx, A, upper, k + b, b2, d_info, d_bad, inv, false))) return rc;
    }
    // 3. the rest of the trailing update on the caller's stream
    const int r2 = rest - b2;
    if (r2 > 0) {
      GemmOpts ot;
      ot.mode = upper ? kSyrkUpper : kSyrkLower;
      ot.max_ctas = ctx->sms - free_sms;
      const View C = A.sub(k + b + b2, k + b + b2, r2, r2);
      if (!upper)
        rc = gemm_ex(ctx, C, A.sub(k + b + b2, k, r2, b), false, A.sub(k + b + b2, k, r2, b),
                     true, -1.0, 1.0, ot);
      else
        rc = gemm_ex(ctx, C, A.sub(k, k + b + b2, b, r2), true, A.sub(k, k + b + b2, b, r2),
                     false, -1.0, 1.0, ot);
      if (rc) return rc;
    }
  }
  return MO_OK;
}

}  // namespace mo
