// Mixed-precision blocked Cholesky: the trailing updates and panel products run as
// split-product GEMMs (lpgemm.cu) on an FP32 working copy, the 128 x 128 diagonal blocks
// are factored and inverted in FP32 (inverses kept in FP64 for the refinement).
//
// The working matrix W is NP x NP FP32 (NP = n rounded up to 128) holding the lower
// triangle of A (or the transpose of its upper triangle), padded with the identity so
// the padded factor is diag(L, I).  Block column k (128 columns), right-looking as in the
// FP64 driver (potrf.cu):
//   diag   : W11 Cholesky + inverse in shared memory (FP32); L11 back to W, the inverse
//            kept in FP64 for the refinement solves and split for (panel)
//   panel  : L21 = A21 * L11^-T   (split-product GEMM, written over A21; its epilogue also
//            writes the K-major hi/lo panel)
//   update : W22 -= P P^T (lower), applied for two block columns at once (K = 256) so that
//            the trailing matrix is read and written half as often; the next pair's two
//            columns are updated first, and that launch's epilogue writes the split A21 of
//            the next panel, so no separate split pass sits on the step-to-step chain
// The diagonal blocks and panels of a pair run on a look-ahead stream while the previous
// pair's trailing update runs on the caller's.  A NaN pivot stops the factorization; its
// global column is reported like DecomposeCHOL's (info = column + 1).
#include <cuda_bf16.h>

#include "lp.cuh"
#include "lpchol.cuh"
#include "tri.cuh"

namespace mo {
namespace {

constexpr int NB = 128;

// shared memory of lp_diag_kernel: the FP32 block plus the inverse's scratch sub-blocks
constexpr int LP_DIAG_SMEM = (TRI_MAX * LDS + 4 * SUB * (SUB + 1)) * (int)sizeof(float);

// W block (FP32, column-major) -> S (FP32 lower, row-major, LDS)
__device__ inline void lp_load_block(float *S, const float *G, int64_t ld) {
  for (int base = threadIdx.x; base < NB * NB; base += 8 * blockDim.x) {
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = base + u * blockDim.x;
      const int i = e % NB, j = e / NB;
      v[u] = (e < NB * NB && i >= j) ? G[i + (int64_t)j * ld] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = base + u * blockDim.x;
      if (e < NB * NB) S[(e % NB) * LDS + e / NB] = v[u];
    }
  }
}

// The diagonal block is factored and inverted in FP32, the precision of the working
// matrix it comes from and goes back to: its rounding is below that of the split-product
// updates that formed it (BF16x3) or equal to it (TF32x3), and the FP32 column chain
// (single-instruction reciprocal square root, 4-cycle FMA, one shuffle per value) is much
// shorter than the FP64 one.  The inverse goes out as FP64 (for the refinement solves)
// and split (for the panel product).
template <int PREC>
__global__ void __launch_bounds__(TRI_THREADS)
    lp_diag_kernel(float *W, int64_t ldw, double *inv, char *ihi, char *ilo, int *info,
                   double *bad_value, int col0, int n_true) {
  if (*(volatile int *)info != 0) return;
  extern __shared__ float smf[];
  float *S = smf;
  float *Wk = smf + TRI_MAX * LDS;
  __shared__ int s_bad;
  __shared__ double s_badv;
  lp_load_block(S, W, ldw);
  __syncthreads();
  tri_potrf_lower(S, NB, &s_bad, &s_badv);
  if (s_bad >= 0) {
    // a failure inside the identity padding cannot happen; report the true column
    if (threadIdx.x == 0 && col0 + s_bad < n_true) {
      *info = col0 + s_bad + 1;
      *bad_value = s_badv;
    }
    return;
  }
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int i = e % NB, j = e / NB;
    if (i >= j) W[i + (int64_t)j * ldw] = S[i * LDS + j];
  }
  __syncthreads();
  tri_inverse_lower(S, NB, Wk);
  __syncthreads();
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int i = e % NB, j = e / NB;
    inv[i + j * NB] = (i >= j) ? (double)S[i * LDS + j] : 0.0;
  }
  // split inverse, K-major: row r = row r of L11^-1 (the B operand of A21 * L11^-T)
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int r = e / NB, k = e % NB;
    const float x = (r >= k) ? S[r * LDS + k] : 0.f;
    if (PREC == kLpBf16x3) {
      const __nv_bfloat16 h = __float2bfloat16_rn(x);
      const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
      reinterpret_cast<__nv_bfloat16 *>(ihi)[e] = h;
      reinterpret_cast<__nv_bfloat16 *>(ilo)[e] = l;
    } else {
      uint32_t h, l;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - __uint_as_float(h)));
      reinterpret_cast<uint32_t *>(ihi)[e] = h;
      reinterpret_cast<uint32_t *>(ilo)[e] = l;
    }
  }
}

// A (FP64, n x n, lower or upper triangle referenced) -> W (FP32 lower, NP x NP, identity
// padding; the strict upper part of W is zeroed)
__global__ void __launch_bounds__(256) lp_convert_kernel(const double *A, int64_t lda, int n,
                                                         bool upper, float *W, int64_t ldw,
                                                         int NP, double shift) {
  __shared__ double T[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  if (i0 + 31 < j0) {
    for (int e = threadIdx.x; e < 32 * 32; e += 256)
      W[(i0 + e % 32) + (int64_t)(j0 + e / 32) * ldw] = 0.f;
    return;
  }
  // T[r][c] = lower(A)(i0 + r, j0 + c)
  for (int e = threadIdx.x; e < 32 * 32; e += 256) {
    const int a = e % 32, b = e / 32;
    if (!upper) {
      const int i = i0 + a, j = j0 + b;
      T[a][b] = (i < n && j < n && i >= j) ? A[i + (int64_t)j * lda] : 0.0;
    } else {
      // upper storage: lower(A)(i, j) = A(j, i); read A(j0 + a, i0 + b) coalesced in a
      const int i = i0 + b, j = j0 + a;
      T[b][a] = (i < n && j < n && i >= j) ? A[j + (int64_t)i * lda] : 0.0;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 32 * 32; e += 256) {
    const int r = e % 32, c = e / 32;
    const int i = i0 + r, j = j0 + c;
    double v = (i >= j) ? T[r][c] : 0.0;
    if (i == j) v = (i < n) ? v * (1.0 + shift) : 1.0;
    W[i + (int64_t)j * ldw] = (float)v;
  }
  (void)NP;
}

template <int PREC>
int set_lp_diag_smem() {
  return mo_smem_attr((const void *)lp_diag_kernel<PREC>, LP_DIAG_SMEM);
}

// diagonal block + panel of step k on ctx->stream; P receives the split L21.  The split
// A21 (f.PA) is made here for the first panel only: later ones come out of the previous
// step's next-block-column update (see lp_chol_factor).
int lp_panel(mo_ctx *ctx, LpChol &f, int k, int *d_info, double *d_bad, const LpSplit &P) {
  float *Wkk = f.W + k + (int64_t)k * f.ldw;
  double *inv = f.inv + (size_t)(k / NB) * NB * NB;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_DIAG);
  if (f.prec == kLpBf16x3)
    lp_diag_kernel<kLpBf16x3><<<1, TRI_THREADS, LP_DIAG_SMEM, ctx->stream>>>(
        Wkk, f.ldw, inv, (char *)f.Linv.hi, (char *)f.Linv.lo, d_info, d_bad, k, f.n);
  else
    lp_diag_kernel<kLpTf32x3><<<1, TRI_THREADS, LP_DIAG_SMEM, ctx->stream>>>(
        Wkk, f.ldw, inv, (char *)f.Linv.hi, (char *)f.Linv.lo, d_info, d_bad, k, f.n);
  prof_end(ctx, ps, 2.0 * NB * NB * NB / 3.0, 4.0 * 2.0 * NB * NB + 8.0 * NB * NB);
  MO_CUDA_TRY(cudaGetLastError());
  const int rest = f.NP - k - NB;
  if (rest <= 0) return MO_OK;
  float *A21 = Wkk + NB;
  int rc;
  if (k == 0 && (rc = lp_split(ctx, f.prec, A21, f.ldw, rest, NB, f.PA))) return rc;
  // L21 = A21 L11^-T, written to W and, split, to P by the GEMM's epilogue
  LpGemmArgs g;
  g.M = rest;
  g.N = NB;
  g.K = NB;
  g.alpha = 1.f;
  g.beta = 0.f;
  g.A = f.PA;
  g.B = f.Linv;
  g.C = A21;
  g.ldc = f.ldw;
  g.out = P;
  g.out_row0 = 0;
  return lp_gemm(ctx, f.prec, g);
}

}  // namespace

size_t lp_chol_bytes(int n, int prec) {
  const size_t NP = (size_t)((n + NB - 1) / NB) * NB;
  const size_t es = lp_esize(prec);
  return NP * NP * 4                 // W
         + (NP / NB) * NB * NB * 8   // FP64 inverses
         + 2 * NB * NB * es          // split inverse
         + 3 * 2 * NP * 2 * NB * es  // PA, P[0], P[1] (two panels wide)
         + 4096;
}

int lp_chol_setup(int n, int prec, void *mem, LpChol &f) {
  f.n = n;
  f.prec = prec;
  f.NP = ((n + NB - 1) / NB) * NB;
  const size_t NP = f.NP, es = lp_esize(prec);
  char *p = (char *)(((uintptr_t)mem + 255) & ~(uintptr_t)255);
  auto take = [&](size_t bytes) {
    char *r = p;
    p += (bytes + 255) & ~(size_t)255;
    return r;
  };
  f.W = (float *)take(NP * NP * 4);
  f.ldw = NP;
  f.inv = (double *)take((NP / NB) * NB * NB * 8);
  f.Linv.hi = take(NB * NB * es);
  f.Linv.lo = take(NB * NB * es);
  f.Linv.ldk = NB;
  LpSplit *bufs[3] = {&f.PA, &f.P[0], &f.P[1]};
  for (LpSplit *b : bufs) {
    b->hi = take(NP * 2 * NB * es);
    b->lo = take(NP * 2 * NB * es);
    b->ldk = 2 * NB;
  }
  return MO_OK;
}

int lp_chol_convert(mo_ctx *ctx, const LpChol &f, View A, bool upper, double shift) {
  const dim3 grid(f.NP / 32, f.NP / 32);
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_OTHER);
  lp_convert_kernel<<<grid, 256, 0, ctx->stream>>>(A.d, A.ld, f.n, upper, f.W, f.ldw, f.NP,
                                                   shift);
  prof_end(ctx, ps, 0.0, 8.0 * f.n * (double)f.n / 2 + 4.0 * (double)f.NP * f.NP);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// Right-looking factorization of W, two 128-column steps per trailing update (K = 256),
// with look-ahead.  Pair p covers block columns a = 2p and b = a + 1; Q = f.P[p & 1]
// holds their split panels side by side (K-major, 256 wide; row 0 = row 128 (a + 1) of
// W): L21 of a in k 0..127 from row 0, L21 of b in k 128..255 from row 128.
//   S1 (aux):  [diag a, panel a -> Q] [column b -= L21_a (rows of b) ^T] [diag b,
//              panel b -> Q] -> record E1
//   S0 (main): wait E1 -> [columns a + 2, a + 3 -= Q Q^T (K = 256), split A21 of a + 2
//              -> PA] -> record E0 -> [the rest of the trailing matrix (K = 256)]
//   S1 waits E0 before the next pair.
int lp_chol_factor(mo_ctx *ctx, LpChol &f, int *d_info, double *d_bad) {
  int rc = f.prec == kLpBf16x3 ? set_lp_diag_smem<kLpBf16x3>() : set_lp_diag_smem<kLpTf32x3>();
  if (rc) return rc;
  const int NP = f.NP;
  const int es = lp_esize(f.prec);
  cudaStream_t s0 = ctx->stream, s1 = nullptr;
  if ((rc = aux_stream(ctx, &s1))) return rc;
  if ((rc = stream_wait(ctx, s1, s0, ctx->ev_fork))) return rc;
  const int free_sms = 2;
  for (int ka = 0, pair = 0; ka < NP; ka += 2 * NB, ++pair) {
    const int kb = ka + NB;
    LpSplit &Q = f.P[pair & 1];
    // Q shifted to (row 128, k 128): where panel b's split goes
    const LpSplit Qb{(char *)Q.hi + (size_t)(NB * Q.ldk + NB) * es,
                     (char *)Q.lo + (size_t)(NB * Q.ldk + NB) * es, Q.ldk};
    {
      StreamSwap sw(ctx, s1);
      if ((rc = lp_panel(ctx, f, ka, d_info, d_bad, Q))) return rc;
      if (kb < NP) {
        // column b -= L21_a L21_a(rows of b)^T; its rows below b's diagonal block are
        // panel b's A21: split into PA by the epilogue
        LpGemmArgs g;
        g.M = NP - kb;
        g.N = NB;
        g.K = NB;
        g.alpha = -1.f;
        g.beta = 1.f;
        g.A = Q;
        g.B = Q;
        g.C = f.W + kb + (int64_t)kb * f.ldw;
        g.ldc = f.ldw;
        g.mode = kGemmLower;
        g.out = f.PA;
        g.out_row0 = NB;
        if ((rc = lp_gemm(ctx, f.prec, g))) return rc;
        if ((rc = lp_panel(ctx, f, kb, d_info, d_bad, Qb))) return rc;
      }
    }
    if ((rc = stream_wait(ctx, s0, s1, ctx->ev_join))) return rc;  // pair's panels done
    const int kc = ka + 2 * NB;  // first column of the next pair
    const int rest = NP - kc;
    if (rest <= 0) break;
    float *W22 = f.W + kc + (int64_t)kc * f.ldw;
    const LpSplit Qr = lp_rows(Q, f.prec, NB);  // rows from kc
    // 1. the next pair's two columns (one if only one is left), K = 256
    const int nn = std::min(2 * NB, rest);
    LpGemmArgs g;
    g.M = rest;
    g.N = nn;
    g.K = 2 * NB;
    g.alpha = -1.f;
    g.beta = 1.f;
    g.A = Qr;
    g.B = Qr;
    g.C = W22;
    g.ldc = f.ldw;
    g.mode = kGemmLower;
    g.out = f.PA;  // rows below the next pair's first diagonal block: its A21, split
    g.out_row0 = NB;
    if ((rc = lp_gemm(ctx, f.prec, g))) return rc;
    if ((rc = stream_wait(ctx, s1, s0, ctx->ev_fork))) return rc;
    // 2. the rest of the trailing matrix, K = 256
    const int r2 = rest - nn;
    if (r2 > 0) {
      LpGemmArgs t;
      t.M = r2;
      t.N = r2;
      t.K = 2 * NB;
      t.alpha = -1.f;
      t.beta = 1.f;
      t.A = lp_rows(Qr, f.prec, nn);
      t.B = t.A;
      t.C = W22 + nn + (int64_t)nn * f.ldw;
      t.ldc = f.ldw;
      t.mode = kGemmLower;
      t.max_ctas = ctx->sms - free_sms;
      if ((rc = lp_gemm(ctx, f.prec, t))) return rc;
    }
  }
  return MO_OK;
}

}  // namespace mo
