// Triangular solves with the factor of the mixed-precision Cholesky (the preconditioner of
// the FP64 refinement in ir.cu), as a short chain of block steps on the FP64 GEMM engine.
//
// The factor L (FP32, in the working matrix W of lpchol.cu) is copied once to FP64 (its
// lower triangle), and the inverses of its BS x BS diagonal blocks (BS = 1024) are formed in
// FP64 from the 128 x 128 diagonal-block inverses that the factorization already computed,
// by recursive doubling:
//     inv([A 0; B C]) = [inv(A) 0; -inv(C) B inv(A)  inv(C)]
// (levels 128 -> 256 -> 512 -> 1024; each level is two batched DMMA products over all
// blocks: T = B inv(A), then -inv(C) T, with the triangular zeros of inv(A) and inv(C)
// skipped).  A solve with nrhs columns is then nblk = n / BS steps of two GEMMs each:
//     L x = r  :  X_i = inv(L_ii) R_i ;  R_{>i} -= L_{>i,i} X_i           (top-down)
//     L^T x = r:  X_i = inv(L_ii)^T R_i ;  R_{<i} -= L_{i,<i}^T X_i       (bottom-up)
// so the dependency chain is 16 steps at n = 16384 instead of 256 row blocks of 64.  All
// arithmetic is FP64 (the FP32 entries of L are exact in FP64), so the correction has the
// accuracy of the FP64 substitution up to the conditioning of the diagonal blocks of L.
#include "lpchol.cuh"

namespace mo {
namespace {

constexpr int BS = kLpSolveBlock;  // diagonal block order of the solve
constexpr int MT = 64;             // output tile of the merge products
constexpr int KC = 32;             // depth of one staged chunk
constexpr int LDT = MT + 4;

// W (FP32 lower, ld ldw) -> L64 (FP64 lower, ld ldl), 32 x 32 tiles on or below the diagonal
__global__ void __launch_bounds__(256) lp_to_f64_kernel(const float *W, int64_t ldw, double *L64,
                                                        int64_t ldl, int NP) {
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  if (i0 + 31 < j0) return;
  for (int e = threadIdx.x; e < 32 * 32; e += 256) {
    const int i = i0 + (e & 31), j = j0 + (e >> 5);
    if (i < NP && j < NP && i >= j) L64[i + (int64_t)j * ldl] = (double)W[i + (int64_t)j * ldw];
  }
}

// Dinv block b, 128 x 128 diagonal sub-blocks <- the factorization's FP64 inverses (inv:
// NP / 128 column-major 128 x 128 blocks, zeros above the diagonal)
__global__ void __launch_bounds__(256) place_inv128_kernel(const double *inv, double *Dinv, int NP) {
  const int q = blockIdx.x;  // global 128-block index
  const int b = q * 128 / BS, lo = q * 128 - b * BS;
  double *dst = Dinv + (size_t)b * BS * BS + lo + (size_t)lo * BS;
  const double *src = inv + (size_t)q * 128 * 128;
  for (int e = threadIdx.x; e < 128 * 128; e += 256) dst[(e & 127) + (size_t)(e >> 7) * BS] = src[e];
  (void)NP;
}

// One merge level m of the block inverses (see the file comment).  blockIdx.y = merge z =
// b * (BS / (2m)) + q, covering rows/cols [o, o + 2m) of block b (o = q * 2m, local); the
// lower-left part (mc x m, mc = the second half's order) is computed in 64 x 64 tiles:
//   PHASE 1:  T_z = L64[B part] * inv(A)           (k from the tile's first column: inv(A)
//                                                    is lower triangular)
//   PHASE 2:  Dinv[lower-left] = -inv(C) * T_z      (k up to the tile's last row)
template <int PHASE>
__global__ void __launch_bounds__(128) inv_merge_kernel(const double *L64, int64_t ldl,
                                                        double *Dinv, double *T, int NP, int m) {
  __shared__ double As[KC][LDT];  // As[k][i]
  __shared__ double Bs[KC][LDT];  // Bs[k][j]
  const int per_blk = BS / (2 * m);
  const int z = blockIdx.y, b = z / per_blk, q = z % per_blk;
  const int bend = min(BS, NP - b * BS);  // local order of block b
  const int o = q * 2 * m;
  const int mc = min(m, bend - o - m);
  if (mc <= 0) return;
  const int tiles_j = m / MT;
  const int ti = blockIdx.x / tiles_j, tj = blockIdx.x % tiles_j;
  const int i0 = ti * MT, j0 = tj * MT;
  if (i0 >= mc) return;
  double *Db = Dinv + (size_t)b * BS * BS;
  double *Tz = T + (size_t)z * m * m;  // mc x m, ld m
  // operands: element (i, k) of the left factor, (k, j) of the right one
  const double *Ab, *Bb;
  int64_t lda, ldb;
  int klo, khi;
  if (PHASE == 1) {
    Ab = L64 + (int64_t)(b * BS + o + m) + (int64_t)(b * BS + o) * ldl;  // B part of L
    lda = ldl;
    Bb = Db + o + (size_t)o * BS;  // inv(A)
    ldb = BS;
    klo = j0;
    khi = m;
  } else {
    Ab = Db + (o + m) + (size_t)(o + m) * BS;  // inv(C)
    lda = BS;
    Bb = Tz;
    ldb = m;
    klo = 0;
    khi = min(mc, i0 + MT);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double acc[8][4];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[a][c] = 0.0;
  const int kA = PHASE == 1 ? m : mc;  // extent of k in the left operand
  for (int k0 = klo; k0 < khi; k0 += KC) {
    __syncthreads();
    for (int e = threadIdx.x; e < KC * MT; e += 128) {
      const int i = e % MT, k = e / MT;  // left: column-major, i fastest
      const int gi = i0 + i, gk = k0 + k;
      As[k][i] = (gi < mc && gk < khi && gk < kA) ? Ab[gi + (int64_t)gk * lda] : 0.0;
      const int kk = e % KC, j = e / KC;  // right: column-major, k fastest
      const int gk2 = k0 + kk, gj = j0 + j;
      Bs[kk][j] = (gk2 < khi && gj < m) ? Bb[gk2 + (int64_t)gj * ldb] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KC; k += 4) {
      const double a0 = As[k + t][16 * warp + g], a1 = As[k + t][16 * warp + g + 8];
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) dmma_16x8x4(acc[nt], a0, a1, Bs[k + t][8 * nt + g]);
    }
  }
  // write: (row, col) of acc[nt][c] = (16 warp + g + 8 (c >> 1), 8 nt + 2 t + (c & 1))
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int i = i0 + 16 * warp + g + 8 * (c >> 1), j = j0 + 8 * nt + 2 * t + (c & 1);
      if (i < mc && j < m) {
        if (PHASE == 1) Tz[i + (size_t)j * m] = acc[nt][c];
        else Db[(o + m + i) + (size_t)(o + j) * BS] = -acc[nt][c];
      }
    }
}

}  // namespace

size_t lp_solve_bytes(int NP, int nrhs) {
  const size_t nb = (size_t)(NP + BS - 1) / BS;
  return (size_t)NP * NP * 8            // L64
         + nb * BS * BS * 8             // Dinv
         + nb * BS * (BS / 2) * 8       // merge scratch T
         + (size_t)BS * nrhs * 8        // X block
         + 4 * 256;
}

int lp_solve_setup(int NP, int nrhs, void *mem, LpSolve &s) {
  s.NP = NP;
  s.nblk = (NP + BS - 1) / BS;
  s.nrhs = nrhs;
  char *p = (char *)(((uintptr_t)mem + 255) & ~(uintptr_t)255);
  auto take = [&](size_t bytes) {
    char *r = p;
    p += (bytes + 255) & ~(size_t)255;
    return r;
  };
  s.L64 = (double *)take((size_t)NP * NP * 8);
  s.ldl = NP;
  s.Dinv = (double *)take((size_t)s.nblk * BS * BS * 8);
  s.T = (double *)take((size_t)s.nblk * BS * (BS / 2) * 8);
  s.Xb = (double *)take((size_t)BS * nrhs * 8);
  return MO_OK;
}

int lp_solve_prepare(mo_ctx *ctx, const LpChol &f, LpSolve &s) {
  cudaStream_t st = ctx->stream;
  const int NP = f.NP;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_OTHER);
  lp_to_f64_kernel<<<dim3(NP / 32, NP / 32), 256, 0, st>>>(f.W, f.ldw, s.L64, s.ldl, NP);
  MO_CUDA_TRY(cudaMemsetAsync(s.Dinv, 0, (size_t)s.nblk * BS * BS * 8, st));
  place_inv128_kernel<<<NP / 128, 256, 0, st>>>(f.inv, s.Dinv, NP);
  prof_end(ctx, ps, 0.0, 6.0 * NP * (double)NP + 8.0 * s.nblk * BS * (double)BS);
  MO_CUDA_TRY(cudaGetLastError());
  ProfScope pm;
  prof_begin(ctx, pm, MO_PROF_TRTRI);
  double flops = 0.0;
  for (int m = 128; m < BS; m *= 2) {
    const int merges = s.nblk * (BS / (2 * m));
    const dim3 grid((m / MT) * (m / MT), merges);
    inv_merge_kernel<1><<<grid, 128, 0, st>>>(s.L64, s.ldl, s.Dinv, s.T, NP, m);
    inv_merge_kernel<2><<<grid, 128, 0, st>>>(s.L64, s.ldl, s.Dinv, s.T, NP, m);
    flops += 2.0 * merges * (double)m * m * m;
  }
  prof_end(ctx, pm, flops, 0.0);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// D (n x nr, ld ldd) <- L^-1 D (trans == false) or L^-T D (trans == true)
int lp_solve_apply(mo_ctx *ctx, const LpSolve &s, int n, double *D, int64_t ldd, int nr,
                   bool trans, const int *skip) {
  if (nr > s.nrhs) return MO_EINVAL;
  cudaStream_t st = ctx->stream;
  const int nb = (n + BS - 1) / BS;
  const View L{s.L64, n, n, s.ldl};
  const View R{D, n, nr, ldd};
  GemmOpts o;
  o.stream_k = true;
  o.skip = skip;
  for (int step = 0; step < nb; ++step) {
    const int i = trans ? nb - 1 - step : step;
    const int r0 = i * BS, h = std::min(BS, n - r0);
    const View Di{s.Dinv + (size_t)i * BS * BS, h, h, BS};
    const View Xb{s.Xb, h, nr, BS};
    int rc = gemm_ex(ctx, Xb, Di, trans, R.sub(r0, 0, h, nr), false, 1.0, 0.0, o);
    if (rc) return rc;
    if (!trans && r0 + h < n) {
      rc = gemm_ex(ctx, R.sub(r0 + h, 0, n - r0 - h, nr), L.sub(r0 + h, r0, n - r0 - h, h), false,
                   Xb, false, -1.0, 1.0, o);
    } else if (trans && r0 > 0) {
      rc = gemm_ex(ctx, R.sub(0, 0, r0, nr), L.sub(r0, 0, h, r0), true, Xb, false, -1.0, 1.0, o);
    }
    if (rc) return rc;
    MO_CUDA_TRY(cudaMemcpy2DAsync(D + r0, (size_t)ldd * 8, s.Xb, (size_t)BS * 8, (size_t)h * 8, nr,
                                  cudaMemcpyDeviceToDevice, st));
  }
  return MO_OK;
}

}  // namespace mo
