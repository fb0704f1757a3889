// Reverse mode (adjoint) of the Cholesky factorization and of the Cholesky solve, FP64.
// The reference has no derivatives; these are the adjoints of DecomposeCHOL (chol.go:116)
// and SolveCHOL (chol.go:147) for LOWER factors.
//
// Cholesky adjoint, blocked right to left (block size 256), in place on Lbar.  With the
// factor partitioned at block column j as
//       [ .  .      ]        R = L(j, 0:j)      D = L(j, j)
//       [ R  D      ]        C = L(j+1:, 0:j)   B = L(j+1:, j)
//       [ C  B  .   ]
// and Rbar, Dbar, Cbar, Bbar the matching blocks of the adjoint storage, each step undoes
// the forward step of the left-looking algorithm (B = (A_B - C R^T) D^-T, D = chol(A_D -
// R R^T)) and leaves the adjoint of the lower-triangle entries of A in place of Dbar, Bbar:
//   Bbar <- Bbar D^-1                      (GEMM with the inverse of D)
//   Dbar <- Dbar - tril(Bbar^T B)          (GEMM, lower mode)
//   Cbar <- Cbar - Bbar R                  (GEMM)
//   Rbar <- Rbar - Bbar^T C                (GEMM)
//   Dbar <- Phi(S + S^T), S = D^-T Phi(D^T Dbar) D^-1   (unblocked adjoint of chol(D))
//   Rbar <- Rbar - (S + S^T) R             (GEMM)
// Phi(X) = lower triangle of X with the diagonal halved.  The result is the adjoint with
// respect to the lower-triangle entries of A; a last pass turns it into the symmetric
// gradient (both triangles, off-diagonal entries halved).  Only L is read besides Lbar:
// no forward panel is stored, and the extra device memory is five 256 x 256 blocks per
// stream whatever n is.  The flops are about 2 n^3 / 3 (twice the factorization).
//
// Batched form: orders up to 512 run in one persistent kernel (each CTA takes whole matrices,
// longest first, and runs the same sweep with 32-column blocks inside the CTA); larger
// orders use the single-matrix sweep above, spread over a pool of streams.
//
// Solve adjoint: X = A^-1 B with A = L L^T.  Bbar = A^-1 Xbar (two triangular solves with
// L, as SolveCHOL), and the symmetric gradient Abar -= (Bbar X^T + X Bbar^T) / 2.
#include <algorithm>
#include <vector>

#include "context.cuh"

namespace mo {
int trtri_blocks(mo_ctx *ctx, View A, int N, bool trans, bool lower_eff, bool unit, double *inv);

namespace {

constexpr int NBA = 256;   // block columns per step of the single-matrix sweep
constexpr int NBI = 128;   // order of the diagonal inverses trtri_blocks forms
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

// Di (NBA x NBA) = the 128 x 128 diagonal-block inverses of a jb x jb triangle (inv:
// trtri_blocks' layout, NBI x NBI blocks back to back), zeros elsewhere
__global__ void adj_place_kernel(const double *inv, double *Di, int jb) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NBA * NBA; e += gridDim.x * blockDim.x) {
    const int i = e % NBA, j = e / NBA, b = i / NBI;
    Di[e] = (b == j / NBI && i < jb && j < jb)
                ? inv[(size_t)b * NBI * NBI + (i - b * NBI) + (size_t)(j - b * NBI) * NBI]
                : 0.0;
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
  double *inv, *Dz, *X1, *X2, *Di;  // NBA x NBA each (inv: trtri_blocks' 128-blocks)
};

// one matrix, on ctx->stream; stream_k must be off when several streams share the context
int chol_adjoint_one(mo_ctx *ctx, View L, View G, const AdjScratch &w, bool stream_k) {
  const int n = L.rows;
  cudaStream_t st = ctx->stream;
  GemmOpts plain;
  plain.stream_k = stream_k;
  const int last = ((n - 1) / NBA) * NBA;
  int rc;
  for (int j0 = last; j0 >= 0; j0 -= NBA) {
    const int jb = std::min(NBA, n - j0), below = n - j0 - jb;
    const View D = L.sub(j0, j0, jb, jb), Dbar = G.sub(j0, j0, jb, jb);
    const View R = L.sub(j0, 0, jb, j0), Rbar = G.sub(j0, 0, jb, j0);
    // D^-1: the 128 x 128 diagonal blocks' inverses, then X21 = -X22 (D21 X11)
    if ((rc = trtri_blocks(ctx, D, jb, false, true, false, w.inv))) return rc;
    adj_place_kernel<<<64, 256, 0, st>>>(w.inv, w.Di, jb);
    MO_CUDA_TRY(cudaGetLastError());
    if (jb > NBI) {
      const int mc = jb - NBI;
      const View X11{w.Di, NBI, NBI, NBA}, X22{w.Di + NBI + (size_t)NBI * NBA, mc, mc, NBA};
      const View T{w.X2, mc, NBI, NBA}, X21{w.Di + NBI, mc, NBI, NBA};
      if ((rc = gemm_ex(ctx, T, L.sub(j0 + NBI, j0, mc, NBI), false, X11, false, 1.0, 0.0, plain)))
        return rc;
      if ((rc = gemm_ex(ctx, X21, X22, false, T, false, -1.0, 0.0, plain))) return rc;
    }
    const View Dinv{w.Di, jb, jb, NBA};
    if (below > 0) {
      const View B = L.sub(j0 + jb, j0, below, jb), Bbar = G.sub(j0 + jb, j0, below, jb);
      if ((rc = gemm_ex(ctx, Bbar, Bbar, false, Dinv, false, 1.0, 0.0, plain))) return rc;
      // one 128 x 128 tile with K = rows below: as a plain product it is spread over the
      // device by stream-K (a triangle-mode launch would run on one SM); the strict upper
      // part of Dbar it also writes is never read and is overwritten at the end
      if ((rc = gemm_ex(ctx, Dbar, Bbar, true, B, false, -1.0, 1.0, plain))) return rc;
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

// ---------------------------------------------------------------------------------------
// Batched form for orders up to kAdjBatchMaxN: one persistent kernel, each CTA takes whole
// matrices from a longest-first queue and runs the same reverse sweep with 32-column
// blocks inside the CTA: every product is a small GEMM over shared-memory tiles (FP64 FMA,
// 4 outputs per thread), the 32 x 32 diagonal work (D^-1 and the adjoint of chol(D)) stays
// in shared memory, and L and Lbar are read and written in place (they stay in L2 at these
// orders).  One launch replaces the per-matrix chain of about 25 launches per block.
// ---------------------------------------------------------------------------------------
constexpr int AB = 32;     // block columns per step
constexpr int ABT = 256;   // threads per CTA
constexpr int ALD = AB + 1;
constexpr int kAdjBatchMaxN = 512;

struct AdjBatchArgs {
  int count;
  const int *order;           // queue: matrix indices, longest first
  int *counter;               // next queue position (zeroed before the launch)
  const int *n;
  double *const *L;
  const int64_t *ldl;
  double *const *G;
  const int64_t *ldg;
};

struct AdjSmem {
  double As[AB][ALD], Bs[AB][ALD];    // GEMM staging
  double Dm[AB][ALD], Di[AB][ALD];    // D (lower, identity padded) and D^-1
  double X1[AB][ALD], X2[AB][ALD];    // the adjoint of chol(D)
  int idx;
};

// C (M x N, ldc) += alpha op(A) op(B), op(A) M x K, op(B) K x N; `lower`: only i >= j.
// op(A)(i, k) = ta ? A[k + i lda] : A[i + k lda]; op(B)(k, j) = tb ? B[j + k ldb] : B[k + j ldb].
// C must not overlap A or B.  Ends with a barrier.
__device__ void adj_gemm(AdjSmem &s, int M, int N, int K, double alpha, const double *A, int64_t lda,
                         bool ta, const double *B, int64_t ldb, bool tb, double *C, int64_t ldc,
                         bool lower) {
  const int tid = threadIdx.x, r = tid & 31, cg = tid >> 5;  // row r, columns 4 cg .. + 3
  for (int i0 = 0; i0 < M; i0 += AB)
    for (int j0 = 0; j0 < N; j0 += AB) {
      if (lower && j0 > i0 + AB - 1) continue;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int k0 = 0; k0 < K; k0 += AB) {
        __syncthreads();
        for (int e = tid; e < AB * AB; e += ABT) {
          const int a = e & 31, b = e >> 5;
          const int ii = ta ? b : a, ka = ta ? a : b;  // consecutive threads: consecutive addresses
          const int gi = i0 + ii, gk = k0 + ka;
          s.As[ii][ka] = (gi < M && gk < K) ? (ta ? A[gk + (int64_t)gi * lda] : A[gi + (int64_t)gk * lda]) : 0.0;
          const int kb = tb ? b : a, jj = tb ? a : b;
          const int gk2 = k0 + kb, gj = j0 + jj;
          s.Bs[kb][jj] = (gk2 < K && gj < N) ? (tb ? B[gj + (int64_t)gk2 * ldb] : B[gk2 + (int64_t)gj * ldb]) : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < AB; ++k) {
          const double av = s.As[r][k];
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[c] = fma(av, s.Bs[k][4 * cg + c], acc[c]);
        }
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int gi = i0 + r, gj = j0 + 4 * cg + c;
        if (gi < M && gj < N && (!lower || gi >= gj)) C[gi + (int64_t)gj * ldc] += alpha * acc[c];
      }
    }
  __syncthreads();
}

// Z = op(X) op(Y) for 32 x 32 shared-memory blocks (Z distinct from X and Y); ends with a barrier
__device__ void adj_mm32(double (*Z)[ALD], const double (*X)[ALD], bool tx, const double (*Y)[ALD],
                         bool ty) {
  const int tid = threadIdx.x, r = tid & 31, cg = tid >> 5;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
  for (int k = 0; k < AB; ++k) {
    const double xv = tx ? X[k][r] : X[r][k];
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] = fma(xv, ty ? Y[4 * cg + c][k] : Y[k][4 * cg + c], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) Z[r][4 * cg + c] = acc[c];
  __syncthreads();
}

// the reverse sweep of one matrix (order n <= kAdjBatchMaxN) by the whole CTA
__device__ void adj_matrix(AdjSmem &s, const double *L, int64_t ldl, double *G, int64_t ldg, int n) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int last = ((n - 1) / AB) * AB;
  for (int j0 = last; j0 >= 0; j0 -= AB) {
    const int jb = min(AB, n - j0), below = n - j0 - jb;
    const double *D = L + j0 + (int64_t)j0 * ldl;
    double *Dbar = G + j0 + (int64_t)j0 * ldg;
    for (int e = tid; e < AB * AB; e += ABT) {
      const int i = e & 31, j = e >> 5;
      s.Dm[i][j] = (i < jb && j < jb) ? (i >= j ? D[i + (int64_t)j * ldl] : 0.0) : (i == j ? 1.0 : 0.0);
    }
    __syncthreads();
    // D^-1 (lower): lane c of warp 0 solves D x = e_c
    if (warp == 0) {
      const double rdi = 1.0 / s.Dm[lane][lane];
      double x[AB];
#pragma unroll
      for (int i = 0; i < AB; ++i) {
        double s0 = (i == lane) ? 1.0 : 0.0, s1 = 0.0;
#pragma unroll
        for (int m = 0; m + 1 < i; m += 2) {
          s0 = fma(-s.Dm[i][m], x[m], s0);
          s1 = fma(-s.Dm[i][m + 1], x[m + 1], s1);
        }
        if (i & 1) s0 = fma(-s.Dm[i][i - 1], x[i - 1], s0);
        const double rd = __shfl_sync(0xffffffffu, rdi, i);
        x[i] = (i < lane) ? 0.0 : (s0 + s1) * rd;
      }
#pragma unroll
      for (int i = 0; i < AB; ++i) s.Di[i][lane] = x[i];
    }
    __syncthreads();
    if (below > 0) {
      double *Bbar = G + (j0 + jb) + (int64_t)j0 * ldg;
      const double *B = L + (j0 + jb) + (int64_t)j0 * ldl;
      // Bbar <- Bbar D^-1 in 32-row chunks through the staging tiles
      for (int r0 = 0; r0 < below; r0 += AB) {
        for (int e = tid; e < AB * AB; e += ABT) {
          const int i = e & 31, k = e >> 5;
          s.As[i][k] = (r0 + i < below && k < jb) ? Bbar[(r0 + i) + (int64_t)k * ldg] : 0.0;
        }
        __syncthreads();
        adj_mm32(s.Bs, s.As, false, s.Di, false);
        for (int e = tid; e < AB * AB; e += ABT) {
          const int i = e & 31, j = e >> 5;
          if (r0 + i < below && j < jb) Bbar[(r0 + i) + (int64_t)j * ldg] = s.Bs[i][j];
        }
        __syncthreads();
      }
      adj_gemm(s, jb, jb, below, -1.0, Bbar, ldg, true, B, ldl, false, Dbar, ldg, true);
      if (j0 > 0) {
        adj_gemm(s, below, j0, jb, -1.0, Bbar, ldg, false, L + j0, ldl, false, G + (j0 + jb), ldg,
                 false);  // Cbar -= Bbar R
        adj_gemm(s, jb, j0, below, -1.0, Bbar, ldg, true, L + (j0 + jb), ldl, false, G + j0, ldg,
                 false);  // Rbar -= Bbar^T C
      }
    }
    // adjoint of chol(D): S = D^-T Phi(D^T tril(Dbar)) D^-1
    for (int e = tid; e < AB * AB; e += ABT) {
      const int i = e & 31, j = e >> 5;
      s.X1[i][j] = (i < jb && j < jb && i >= j) ? Dbar[i + (int64_t)j * ldg] : 0.0;
    }
    __syncthreads();
    adj_mm32(s.X2, s.Dm, true, s.X1, false);
    for (int e = tid; e < AB * AB; e += ABT) {
      const int i = e & 31, j = e >> 5;
      s.X2[i][j] = i > j ? s.X2[i][j] : (i == j ? 0.5 * s.X2[i][j] : 0.0);
    }
    __syncthreads();
    adj_mm32(s.X1, s.X2, false, s.Di, false);
    adj_mm32(s.X2, s.Di, true, s.X1, false);
    // E = S + S^T; Dbar (lower) = Phi-like copy of E
    for (int e = tid; e < AB * AB; e += ABT) {
      const int i = e & 31, j = e >> 5;
      const double v = s.X2[i][j] + s.X2[j][i];
      s.X1[i][j] = v;
      if (i < jb && j < jb && i >= j) Dbar[i + (int64_t)j * ldg] = i == j ? 0.5 * v : v;
    }
    __syncthreads();
    if (j0 > 0)  // Rbar -= E R
      adj_gemm(s, jb, j0, jb, -1.0, &s.X1[0][0], ALD, true, L + j0, ldl, false, G + j0, ldg, false);
  }
  // lower-entry adjoint -> symmetric gradient
  for (int64_t e = tid; e < (int64_t)n * n; e += ABT) {
    const int i = (int)(e % n), j = (int)(e / n);
    if (i > j) {
      const double v = 0.5 * G[i + (int64_t)j * ldg];
      G[i + (int64_t)j * ldg] = v;
      G[j + (int64_t)i * ldg] = v;
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(ABT) adj_batch_kernel(AdjBatchArgs p) {
  extern __shared__ __align__(16) unsigned char adj_smem_raw[];
  AdjSmem &s = *reinterpret_cast<AdjSmem *>(adj_smem_raw);
  for (;;) {
    if (threadIdx.x == 0) s.idx = atomicAdd(p.counter, 1);
    __syncthreads();
    const int q = s.idx;
    __syncthreads();
    if (q >= p.count) break;
    const int m = p.order[q];
    adj_matrix(s, p.L[m], p.ldl[m], p.G[m], p.ldg[m], p.n[m]);
  }
}

size_t scratch_doubles() { return 5 * (size_t)NBA * NBA; }

AdjScratch carve(double *base) {
  const size_t blk = (size_t)NBA * NBA;
  return AdjScratch{base, base + blk, base + 2 * blk, base + 3 * blk, base + 4 * blk};
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
  // orders up to kAdjBatchMaxN: one persistent kernel over a longest-first queue; larger
  // ones: the single-matrix sweep, spread over a pool of streams
  std::vector<int> small, big;
  for (int i = 0; i < count; ++i) {
    if (L[i].rows == 0) continue;
    (L[i].rows <= kAdjBatchMaxN ? small : big).push_back(i);
  }
  std::stable_sort(small.begin(), small.end(), [&](int a, int b) { return L[a].rows > L[b].rows; });
  const int ns = (int)small.size();
  const size_t arr_bytes = (size_t)ns * (2 * sizeof(int) + 4 * sizeof(int64_t)) + 64;
  const size_t scr_bytes = big.empty() ? 0 : NSTREAMS * scratch_doubles() * sizeof(double);
  double *ws = nullptr;
  if ((rc = adj_workspace(ctx, scr_bytes + arr_bytes, &ws))) return rc;
  const cudaStream_t main = ctx->stream;
  if (!big.empty() && ctx->pool.empty()) {
    for (int s = 0; s < NSTREAMS; ++s) {
      cudaStream_t st;
      MO_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      ctx->pool.push_back(st);
      cudaEvent_t ev;
      MO_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      ctx->pool_ev.push_back(ev);
    }
  }
  if (!big.empty()) {
    cudaStream_t unused;
    if ((rc = aux_stream(ctx, &unused))) return rc;  // creates ev_fork
    MO_CUDA_TRY(cudaEventRecord(ctx->ev_fork, main));
    for (int s = 0; s < NSTREAMS; ++s) MO_CUDA_TRY(cudaStreamWaitEvent(ctx->pool[s], ctx->ev_fork, 0));
  }
  if (ns > 0) {
    // queue and views (packed: order, n | L, ldl, G, ldg), one upload
    char *base = reinterpret_cast<char *>(ws) + scr_bytes;
    std::vector<int64_t> h64(4 * (size_t)ns);
    std::vector<int> h32(2 * (size_t)ns);
    for (int q = 0; q < ns; ++q) {
      const int i = small[q];
      h32[q] = q;  // the arrays below are already in queue order
      h32[ns + q] = L[i].rows;
      h64[q] = (int64_t)reinterpret_cast<uintptr_t>(L[i].d);
      h64[ns + q] = L[i].ld;
      h64[2 * ns + q] = (int64_t)reinterpret_cast<uintptr_t>(G[i].d);
      h64[3 * ns + q] = G[i].ld;
    }
    int64_t *d64 = reinterpret_cast<int64_t *>(base);
    int *d32 = reinterpret_cast<int *>(base + 4 * (size_t)ns * sizeof(int64_t));
    int *dcnt = d32 + 2 * ns;
    MO_CUDA_TRY(cudaMemcpyAsync(d64, h64.data(), h64.size() * sizeof(int64_t), cudaMemcpyHostToDevice, main));
    MO_CUDA_TRY(cudaMemcpyAsync(d32, h32.data(), h32.size() * sizeof(int), cudaMemcpyHostToDevice, main));
    MO_CUDA_TRY(cudaMemsetAsync(dcnt, 0, sizeof(int), main));
    AdjBatchArgs a;
    a.count = ns;
    a.order = d32;
    a.counter = dcnt;
    a.n = d32 + ns;
    a.L = reinterpret_cast<double *const *>(d64);
    a.ldl = d64 + ns;
    a.G = reinterpret_cast<double *const *>(d64 + 2 * ns);
    a.ldg = d64 + 3 * ns;
    if ((rc = mo_smem_attr((const void *)adj_batch_kernel, (int)sizeof(AdjSmem)))) return rc;
    int occ = 0;
    MO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, adj_batch_kernel, ABT, sizeof(AdjSmem)));
    const int grid = std::max(1, std::min(ns, ctx->sms * std::max(1, occ)));
    ProfScope ps;
    prof_begin(ctx, ps, MO_PROF_BATCH);
    adj_batch_kernel<<<grid, ABT, sizeof(AdjSmem), main>>>(a);
    double fl = 0.0;
    for (int i : small) fl += 2.0 * L[i].rows * (double)L[i].rows * L[i].rows / 3.0;
    prof_end(ctx, ps, fl, 0.0);
    MO_CUDA_TRY(cudaGetLastError());
  }
  if (!big.empty()) {
    for (size_t q = 0; q < big.size() && !rc; ++q) {
      const int s = (int)(q % NSTREAMS), i = big[q];
      StreamSwap sw(ctx, ctx->pool[s]);
      rc = chol_adjoint_one(ctx, L[i], G[i], carve(ws + s * scratch_doubles()), false);
    }
    for (int s = 0; s < NSTREAMS; ++s) {
      cudaEventRecord(ctx->pool_ev[s], ctx->pool[s]);
      cudaStreamWaitEvent(main, ctx->pool_ev[s], 0);
    }
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
