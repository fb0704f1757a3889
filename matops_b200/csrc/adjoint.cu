// Reverse mode (adjoint) of the Cholesky factorization and of the Cholesky solve, FP64.
// The reference has no derivatives; these are the adjoints of DecomposeCHOL (chol.go:116)
// and SolveCHOL (chol.go:147) for LOWER factors.
//
// Cholesky adjoint, blocked right to left (block size 128), in place on Lbar.  With the
// factor partitioned at block column j as
//       [ .  .      ]        R = L(j, 0:j)      D = L(j, j)
//       [ R  D      ]        C = L(j+1:, 0:j)   B = L(j+1:, j)
//       [ C  B  .   ]
// and Rbar, Dbar, Cbar, Bbar the matching blocks of the adjoint storage, each step undoes
// the forward step of the left-looking algorithm (B = (A_B - C R^T) D^-T, D = chol(A_D -
// R R^T)) and leaves the adjoint of the lower-triangle entries of A in place of Dbar, Bbar:
//   Bbar <- Bbar D^-1                      (GEMM with the 128 x 128 inverse of D)
//   Dbar <- Dbar - tril(Bbar^T B)          (GEMM, lower mode)
//   Cbar <- Cbar - Bbar R                  (GEMM)
//   Rbar <- Rbar - Bbar^T C                (GEMM)
//   Dbar <- Phi(S + S^T), S = D^-T Phi(D^T Dbar) D^-1   (unblocked adjoint of chol(D))
//   Rbar <- Rbar - (S + S^T) R             (GEMM)
// Phi(X) = lower triangle of X with the diagonal halved.  The result is the adjoint with
// respect to the lower-triangle entries of A; a last pass turns it into the symmetric
// gradient (both triangles, off-diagonal entries halved).  Only L is read besides Lbar:
// no forward panel is stored, and the extra device memory is five 128 x 128 blocks per
// stream whatever n is.  The flops are about 2 n^3 / 3 (twice the factorization).
//
// Solve adjoint: X = A^-1 B with A = L L^T.  Bbar = A^-1 Xbar (two triangular solves with
// L, as SolveCHOL), and the symmetric gradient Abar -= (Bbar X^T + X Bbar^T) / 2.
#include <algorithm>
#include <vector>

#include "context.cuh"

namespace mo {
int trtri_blocks(mo_ctx *ctx, View A, int N, bool trans, bool lower_eff, bool unit, double *inv);

namespace {

constexpr int NBA = 128;
constexpr int NSTREAMS = 8;

// Dz = tril(D), Gz = tril(G) (both jb x jb, ld NBA), zero elsewhere in the NBA x NBA blocks
__global__ void adj_tril_copy_kernel(const double *D, int64_t ldd, const double *G, int64_t ldg,
                                     int jb, double *Dz, double *Gz) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NBA * NBA; e += gridDim.x * blockDim.x) {
    const int i = e % NBA, j = e / NBA;
    const bool in = i < jb && j < jb && i >= j;
    Dz[e] = in ? D[i + (int64_t)j * ldd] : 0.0;
    Gz[e] = in ? G[i + (int64_t)j * ldg] : 0.0;
  }
}

// X <- Phi(X): lower triangle with the diagonal halved, upper triangle zeroed
__global__ void adj_phi_kernel(double *X) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NBA * NBA; e += gridDim.x * blockDim.x) {
    const int i = e % NBA, j = e / NBA;
    X[e] = i > j ? X[e] : (i == j ? 0.5 * X[e] : 0.0);
  }
}

// E = S + S^T (NBA x NBA scratch); Gblk (jb x jb, lower entries) = Phi(S + S^T)
__global__ void adj_sym_kernel(const double *S, double *E, double *G, int64_t ldg, int jb) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NBA * NBA; e += gridDim.x * blockDim.x) {
    const int i = e % NBA, j = e / NBA;
    const double v = S[e] + S[j + i * NBA];
    E[e] = v;
    if (i < jb && j < jb && i >= j) G[i + (int64_t)j * ldg] = i == j ? 0.5 * v : v;
  }
}

// lower-entry adjoint -> symmetric gradient: G(i, j) = G(j, i) = G(i, j) / 2 for i > j
__global__ void adj_symmetrize_kernel(double *G, int64_t ld, int n) {
  const int64_t tot = (int64_t)n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    if (i > j) {
      const double v = 0.5 * G[i + (int64_t)j * ld];
      G[i + (int64_t)j * ld] = v;
      G[j + (int64_t)i * ld] = v;
    }
  }
}

struct AdjScratch {
  double *inv, *Dz, *X1, *X2;  // NBA x NBA each
};

// one matrix, on ctx->stream; stream_k must be off when several streams share the context
int chol_adjoint_one(mo_ctx *ctx, View L, View G, const AdjScratch &w, bool stream_k) {
  const int n = L.rows;
  cudaStream_t st = ctx->stream;
  GemmOpts plain;
  plain.stream_k = stream_k;
  GemmOpts lower = plain;
  lower.mode = kGemmLower;
  const int last = ((n - 1) / NBA) * NBA;
  int rc;
  for (int j0 = last; j0 >= 0; j0 -= NBA) {
    const int jb = std::min(NBA, n - j0), below = n - j0 - jb;
    const View D = L.sub(j0, j0, jb, jb), Dbar = G.sub(j0, j0, jb, jb);
    const View R = L.sub(j0, 0, jb, j0), Rbar = G.sub(j0, 0, jb, j0);
    const View Dinv{w.inv, jb, jb, NBA};
    if ((rc = trtri_blocks(ctx, D, jb, false, true, false, w.inv))) return rc;
    if (below > 0) {
      const View B = L.sub(j0 + jb, j0, below, jb), Bbar = G.sub(j0 + jb, j0, below, jb);
      if ((rc = gemm_ex(ctx, Bbar, Bbar, false, Dinv, false, 1.0, 0.0, plain))) return rc;
      if ((rc = gemm_ex(ctx, Dbar, Bbar, true, B, false, -1.0, 1.0, lower))) return rc;
      if (j0 > 0) {
        const View C = L.sub(j0 + jb, 0, below, j0), Cbar = G.sub(j0 + jb, 0, below, j0);
        if ((rc = gemm_ex(ctx, Cbar, Bbar, false, R, false, -1.0, 1.0, plain))) return rc;
        if ((rc = gemm_ex(ctx, Rbar, Bbar, true, C, false, -1.0, 1.0, plain))) return rc;
      }
    }
    // adjoint of chol(D): S = D^-T Phi(D^T Dbar) D^-1
    const View Dz{w.Dz, jb, jb, NBA}, X1{w.X1, jb, jb, NBA}, X2{w.X2, jb, jb, NBA};
    adj_tril_copy_kernel<<<64, 256, 0, st>>>(D.d, D.ld, Dbar.d, Dbar.ld, jb, w.Dz, w.X1);
    MO_CUDA_TRY(cudaGetLastError());
    if ((rc = gemm_ex(ctx, X2, Dz, true, X1, false, 1.0, 0.0, plain))) return rc;
    adj_phi_kernel<<<64, 256, 0, st>>>(w.X2);
    MO_CUDA_TRY(cudaGetLastError());
    if ((rc = gemm_ex(ctx, X1, X2, false, Dinv, false, 1.0, 0.0, plain))) return rc;
    if ((rc = gemm_ex(ctx, X2, Dinv, true, X1, false, 1.0, 0.0, plain))) return rc;
    // (entries of the scratch blocks outside jb x jb are never read as part of a view)
    adj_sym_kernel<<<64, 256, 0, st>>>(w.X2, w.X1, Dbar.d, Dbar.ld, jb);  // X1 = S + S^T
    MO_CUDA_TRY(cudaGetLastError());
    if (j0 > 0) {
      const View E{w.X1, jb, jb, NBA};
      if ((rc = gemm_ex(ctx, Rbar, E, false, R, false, -1.0, 1.0, plain))) return rc;
    }
  }
  const int64_t tot = (int64_t)n * n;
  adj_symmetrize_kernel<<<(int)std::min<int64_t>((tot + 255) / 256, 4096), 256, 0, st>>>(G.d, G.ld, n);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

size_t scratch_doubles() { return 4 * (size_t)NBA * NBA; }

AdjScratch carve(double *base) {
  const size_t blk = (size_t)NBA * NBA;
  return AdjScratch{base, base + blk, base + 2 * blk, base + 3 * blk};
}

int adj_workspace(mo_ctx *ctx, size_t bytes, double **out) {
  if (bytes > ctx->ws_adj_bytes) {
    MO_CUDA_TRY(cudaDeviceSynchronize());
    if (ctx->ws_adj) cudaFree(ctx->ws_adj);
    ctx->ws_adj = nullptr;
    ctx->ws_adj_bytes = 0;
    MO_CUDA_TRY(cudaMalloc(&ctx->ws_adj, bytes));
    ctx->ws_adj_bytes = bytes;
  }
  *out = (double *)ctx->ws_adj;
  return MO_OK;
}

}  // namespace
}  // namespace mo

using namespace mo;

extern "C" int mo_decompose_chol_adjoint(mo_ctx *ctx, mo_matrix Lm, mo_matrix Gm, int flags) {
  int rc = enter(ctx);
  if (rc) return rc;
  View L, G;
  if ((rc = to_view(Lm, L)) || (rc = to_view(Gm, G))) return rc;
  if (L.rows != L.cols || G.rows != G.cols) return MO_ENOTSQUARE;
  if (G.rows != L.rows) return MO_ESIZE;
  if (flags & MO_UPPER) return MO_EINVAL;
  if (L.rows == 0) return MO_OK;
  double *ws = nullptr;
  if ((rc = adj_workspace(ctx, scratch_doubles() * sizeof(double), &ws))) return rc;
  return chol_adjoint_one(ctx, L, G, carve(ws), true);
}

extern "C" int mo_decompose_chol_adjoint_batched(mo_ctx *ctx, int count, const mo_matrix *Lm,
                                                 const mo_matrix *Gm, int flags) {
  int rc = enter(ctx);
  if (rc) return rc;
  if (count < 0 || (count > 0 && (!Lm || !Gm))) return MO_EINVAL;
  if (flags & MO_UPPER) return MO_EINVAL;
  std::vector<View> L(count), G(count);
  for (int i = 0; i < count; ++i) {
    if ((rc = to_view(Lm[i], L[i])) || (rc = to_view(Gm[i], G[i]))) return rc;
    if (L[i].rows != L[i].cols || G[i].rows != G[i].cols) return MO_ENOTSQUARE;
    if (G[i].rows != L[i].rows) return MO_ESIZE;
  }
  if (count == 0) return MO_OK;
  double *ws = nullptr;
  if ((rc = adj_workspace(ctx, NSTREAMS * scratch_doubles() * sizeof(double), &ws))) return rc;
  // the matrices are independent: spread them over a pool of streams forked from and
  // joined back into the context's stream
  if (ctx->pool.empty()) {
    for (int s = 0; s < NSTREAMS; ++s) {
      cudaStream_t st;
      MO_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      ctx->pool.push_back(st);
      cudaEvent_t ev;
      MO_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      ctx->pool_ev.push_back(ev);
    }
  }
  const cudaStream_t main = ctx->stream;
  MO_CUDA_TRY(cudaEventRecord(ctx->ev_fork, main));
  for (int s = 0; s < NSTREAMS; ++s) MO_CUDA_TRY(cudaStreamWaitEvent(ctx->pool[s], ctx->ev_fork, 0));
  for (int i = 0; i < count && !rc; ++i) {
    const int s = i % NSTREAMS;
    StreamSwap sw(ctx, ctx->pool[s]);
    rc = chol_adjoint_one(ctx, L[i], G[i], carve(ws + s * scratch_doubles()), false);
  }
  for (int s = 0; s < NSTREAMS; ++s) {
    cudaEventRecord(ctx->pool_ev[s], ctx->pool[s]);
    cudaStreamWaitEvent(main, ctx->pool_ev[s], 0);
  }
  return rc;
}

extern "C" int mo_solve_chol_adjoint(mo_ctx *ctx, mo_matrix Lm, mo_matrix Xm, mo_matrix XBm,
                                     mo_matrix Gm, int flags) {
  int rc = enter(ctx);
  if (rc) return rc;
  View L, X, XB, G;
  if ((rc = to_view(Lm, L)) || (rc = to_view(Xm, X)) || (rc = to_view(XBm, XB)) ||
      (rc = to_view(Gm, G)))
    return rc;
  if (L.rows != L.cols || G.rows != G.cols) return MO_ENOTSQUARE;
  if (X.rows != L.rows || XB.rows != L.rows || X.cols != XB.cols || G.rows != L.rows)
    return MO_ESIZE;
  if (flags & MO_UPPER) return MO_EINVAL;
  if (L.rows == 0 || X.cols == 0) return MO_OK;
  // Bbar = (L L^T)^-1 Xbar, as SolveCHOL LOWER (chol.go:151-153)
  if ((rc = trsm(ctx, XB, L, MO_LOWER, 1.0))) return rc;
  if ((rc = trsm(ctx, XB, L, MO_LOWER | MO_TRANSA, 1.0))) return rc;
  // Abar -= (Bbar X^T + X Bbar^T) / 2
  if ((rc = gemm(ctx, G, XB, false, X, true, -0.5, 1.0))) return rc;
  return gemm(ctx, G, X, false, XB, true, -0.5, 1.0);
}
