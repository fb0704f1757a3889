// Triangular solve (TRSM, all 8 side/uplo/trans variants, unit or not) on the device.
//
// Reference semantics: calgo/dmmat_solve.c:864-908 (dispatch), blocked variants :464-862
// (solve with alpha = 1, scale by alpha).  Here: every 128 x 128 diagonal block of op(A)
// is inverted once in shared memory (one CTA per block, tri_inverse_lower), then the
// sweep runs as in-place GEMMs on the FP64 tensor pipe:
//   left,  op(A) lower:  X_i = inv(A_ii) B_i ;  B_{>i} -= op(A)_{>i,i} X_i
//   left,  op(A) upper:  same, bottom-up
//   right, op(A) upper:  X_j = B_j inv(A_jj) ;  B_{>j} -= X_j op(A)_{j,>j}
//   right, op(A) lower:  same, right-to-left
// alpha is folded into the first block step (the first update uses beta = alpha).
#include "context.cuh"
#include "tri.cuh"

namespace mo {
namespace {

constexpr int NBT = 128;

__global__ void __launch_bounds__(TRI_THREADS)
    trtri_blocks_kernel(const double *A, int64_t lda, int N, bool load_transposed,
                        bool store_transposed, bool unit, double *inv) {
  extern __shared__ double sm[];
  double *S = sm;
  double *W = sm + TRI_MAX * LDS;
  const int r0 = blockIdx.x * NBT;
  const int n = min(NBT, N - r0);
  const int NP = round_up32(n);
  tri_load_lower(S, A + r0 + (int64_t)r0 * lda, lda, n, load_transposed, unit);
  __syncthreads();
  tri_inverse_lower(S, NP, W);
  __syncthreads();
  tri_store_lower(S, inv + (size_t)blockIdx.x * NBT * NBT, NBT, n, store_transposed, true);
}

int set_tri_smem(const void *fn) {
  return mo_smem_attr(fn, TRI_SMEM_BYTES);
}

}  // namespace

// Inverts every NBT x NBT diagonal block of op(A) (order N) into inv (nblk x NBT x NBT,
// column-major, ld = NBT, zeros in the opposite triangle).
int trtri_blocks(mo_ctx *ctx, View A, int N, bool trans, bool lower_eff, bool unit, double *inv) {
  const int nblk = (N + NBT - 1) / NBT;
  // the lower triangle loaded into shared memory is op(A)'s block if op(A) is lower,
  // else its transpose; load_transposed iff (trans == lower_eff)
  const bool load_t = (trans == lower_eff);
  int rc = set_tri_smem((const void *)trtri_blocks_kernel);
  if (rc) return rc;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_TRTRI);
  trtri_blocks_kernel<<<nblk, TRI_THREADS, TRI_SMEM_BYTES, ctx->stream>>>(
      A.d, A.ld, N, load_t, !lower_eff, unit, inv);
  prof_end(ctx, ps, nblk * (double)NBT * NBT * NBT / 3.0, 8.0 * nblk * 1.5 * NBT * NBT);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

int trsm_few(mo_ctx *ctx, View B, View A, int flags, double alpha, double *inv, int *flag_buf);

int trsm(mo_ctx *ctx, View B, View A, int flags, double alpha) {
  const int N = A.cols;
  const int nrhs = (flags & MO_RIGHT) ? B.rows : B.cols;
  if (N == 0 || nrhs == 0) return MO_OK;
  const int nblk = (N + NBT - 1) / NBT;
  const size_t inv_bytes = (size_t)nblk * NBT * NBT * sizeof(double);
  double *inv = nullptr;
  // step flags of the few-column solve: up to 4 column groups x 64-row blocks, 32 ints apart
  const size_t flag_ints = (size_t)4 * 32 * ((N + 63) / 64) + 64;
  int rc = workspace(ctx, inv_bytes + sizeof(int) * flag_ints, (void **)&inv);
  if (rc) return rc;
  // few right-hand sides: one cooperative launch instead of a sweep of 2*nblk GEMMs
  if (nblk > 1 && nrhs <= 64)
    return trsm_few(ctx, B, A, flags, alpha, inv,
                    reinterpret_cast<int *>(reinterpret_cast<char *>(inv) + inv_bytes));
  return trsm_with_scratch(ctx, B, A, flags, alpha, inv);
}

// The sweep of trsm() with the caller's scratch for the inverted diagonal blocks
// (ceil(N/128) blocks of 128 x 128 doubles).
int trsm_with_scratch(mo_ctx *ctx, View B, View A, int flags, double alpha, double *inv) {
  const int N = A.cols;
  const bool right = (flags & MO_RIGHT) != 0;
  const bool upper = (flags & MO_UPPER) != 0;
  const bool tr = (flags & MO_TRANSA) != 0;
  const bool unit = (flags & MO_UNIT) != 0;
  const bool lower_eff = upper ? tr : !tr;
  const int nrhs = right ? B.rows : B.cols;
  if (N == 0 || nrhs == 0) return MO_OK;
  const int nblk = (N + NBT - 1) / NBT;
  int rc = trtri_blocks(ctx, A, N, tr, lower_eff, unit, inv);
  if (rc) return rc;
  // op(A)[r:r+nr, c:c+nc] as a stored view, transposed iff tr
  auto opA = [&](int r, int c, int nr, int nc) -> View {
    return tr ? A.sub(c, r, nc, nr) : A.sub(r, c, nr, nc);
  };
  auto invb = [&](int i, int bi) { return View{inv + (size_t)i * NBT * NBT, bi, bi, NBT}; };
  bool first = true;
  if (!right) {
    for (int step = 0; step < nblk; ++step) {
      const int i = lower_eff ? step : nblk - 1 - step;
      const int r0 = i * NBT, bi = min(NBT, N - r0);
      const View Bi = B.sub(r0, 0, bi, nrhs);
      rc = gemm(ctx, Bi, invb(i, bi), false, Bi, false, first ? alpha : 1.0, 0.0);
      if (rc) return rc;
      if (lower_eff && r0 + bi < N) {
        const int rest = N - r0 - bi;
        const View Ab = opA(r0 + bi, r0, rest, bi);
        rc = gemm(ctx, B.sub(r0 + bi, 0, rest, nrhs), Ab, tr, Bi, false, -1.0, first ? alpha : 1.0);
      } else if (!lower_eff && r0 > 0) {
        const View Ab = opA(0, r0, r0, bi);
        rc = gemm(ctx, B.sub(0, 0, r0, nrhs), Ab, tr, Bi, false, -1.0, first ? alpha : 1.0);
      }
      if (rc) return rc;
      first = false;
    }
  } else {
    for (int step = 0; step < nblk; ++step) {
      const int j = lower_eff ? nblk - 1 - step : step;
      const int c0 = j * NBT, bj = min(NBT, N - c0);
      const View Bj = B.sub(0, c0, nrhs, bj);
      rc = gemm(ctx, Bj, Bj, false, invb(j, bj), false, first ? alpha : 1.0, 0.0);
      if (rc) return rc;
      if (!lower_eff && c0 + bj < N) {
        const int rest = N - c0 - bj;
        const View Ab = opA(c0, c0 + bj, bj, rest);
        rc = gemm(ctx, B.sub(0, c0 + bj, nrhs, rest), Bj, false, Ab, tr, -1.0, first ? alpha : 1.0);
      } else if (lower_eff && c0 > 0) {
        const View Ab = opA(c0, 0, bj, c0);
        rc = gemm(ctx, B.sub(0, 0, nrhs, c0), Bj, false, Ab, tr, -1.0, first ? alpha : 1.0);
      }
      if (rc) return rc;
      first = false;
    }
  }
  return MO_OK;
}

}  // namespace mo
