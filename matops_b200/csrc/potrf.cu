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

int potrf(mo_ctx *ctx, View A, bool upper, int *d_info, double *d_bad, double *inv) {
  static int attr_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(attr_mask & (1 << (dev & 31)))) {
    MO_CUDA_TRY(cudaFuncSetAttribute(potrf_diag_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, TRI_SMEM_BYTES));
    attr_mask |= 1 << (dev & 31);
  }
  const int n = A.rows;
  for (int k = 0; k < n; k += NB) {
    const int b = min(NB, n - k);
    ProfScope ps;
    prof_begin(ctx, ps, MO_PROF_DIAG);
    potrf_diag_kernel<<<1, TRI_THREADS, TRI_SMEM_BYTES, ctx->stream>>>(A.at(k, k), A.ld, b, upper,
                                                                       inv, d_info, d_bad, k);
    // factor b^3/3 + inverse b^3/3; reads the triangle, writes it and the inverse
    prof_end(ctx, ps, 2.0 * b * b * b / 3.0, 8.0 * 2.0 * b * b);
    MO_CUDA_TRY(cudaGetLastError());
    const int rest = n - k - b;
    if (rest <= 0) break;
    const View Linv{inv, b, b, NB};
    int rc;
    if (!upper) {
      const View A21 = A.sub(k + b, k, rest, b);
      rc = gemm(ctx, A21, A21, false, Linv, true, 1.0, 0.0);  // A21 * L11^-T (in place)
      if (!rc) rc = syrk(ctx, A.sub(k + b, k + b, rest, rest), A21, false, false, -1.0, 1.0, 0);
    } else {
      const View A12 = A.sub(k, k + b, b, rest);
      rc = gemm(ctx, A12, Linv, false, A12, false, 1.0, 0.0);  // U11^-T * A12 (in place)
      if (!rc) rc = syrk(ctx, A.sub(k + b, k + b, rest, rest), A12, true, true, -1.0, 1.0, 0);
    }
    if (rc) return rc;
  }
  return MO_OK;
}

}  // namespace mo
