// Mixed-precision blocked Cholesky: the trailing updates and panel products run as
// split-product GEMMs (lpgemm.cu) on an FP32 working copy, the 128 x 128 diagonal blocks
// are factored and inverted in FP64.
//
// The working matrix W is NP x NP FP32 (NP = n rounded up to 128) holding the lower
// triangle of A (or the transpose of its upper triangle), padded with the identity so
// the padded factor is diag(L, I).  Step k (128 columns), right-looking as in the FP64
// driver (potrf.cu) with the same one-step look-ahead:
//   diag   : W11 -> FP64, Cholesky + inverse in shared memory; L11 back to W (FP32), the
//            FP64 inverse kept for the refinement solves, the split inverse for (panel)
//   panel  : L21 = A21 * L11^-T   (split-product GEMM, written over A21; its epilogue also
//            writes the K-major hi/lo panel P)
//   update : W22 -= P P^T (lower), the next block column first on the look-ahead path; that
//            launch's epilogue writes the next step's split A21, so no separate split pass
//            sits on the step-to-step chain
// A NaN pivot stops the factorization; its global column is reported like
// DecomposeCHOL's (info = column + 1).
#include <cuda_bf16.h>

#include "lp.cuh"
#include "lpchol.cuh"
#include "tri.cuh"

namespace mo {
namespace {

constexpr int NB = 128;

// W block (FP32, column-major) -> S (FP64 lower, row-major, LDS)
__device__ inline void lp_load_block(double *S, const float *G, int64_t ld) {
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
      if (e < NB * NB) S[(e % NB) * LDS + e / NB] = (double)v[u];
    }
  }
}

template <int PREC>
__global__ void __launch_bounds__(TRI_THREADS)
    lp_diag_kernel(float *W, int64_t ldw, double *inv, char *ihi, char *ilo, int *info,
                   double *bad_value, int col0, int n_true) {
  if (*(volatile int *)info != 0) return;
  extern __shared__ double sm[];
  double *S = sm;
  double *Wk = sm + TRI_MAX * LDS;
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
    if (i >= j) W[i + (int64_t)j * ldw] = (float)S[i * LDS + j];
  }
  __syncthreads();
  tri_inverse_lower(S, NB, Wk);
  __syncthreads();
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int i = e % NB, j = e / NB;
    inv[i + j * NB] = (i >= j) ? S[i * LDS + j] : 0.0;
  }
  // split inverse, K-major: row r = row r of L11^-1 (the B operand of A21 * L11^-T)
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int r = e / NB, k = e % NB;
    const float x = (r >= k) ? (float)S[r * LDS + k] : 0.f;
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
  return mo_smem_attr((const void *)lp_diag_kernel<PREC>, TRI_SMEM_BYTES);
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
    lp_diag_kernel<kLpBf16x3><<<1, TRI_THREADS, TRI_SMEM_BYTES, ctx->stream>>>(
        Wkk, f.ldw, inv, (char *)f.Linv.hi, (char *)f.Linv.lo, d_info, d_bad, k, f.n);
  else
    lp_diag_kernel<kLpTf32x3><<<1, TRI_THREADS, TRI_SMEM_BYTES, ctx->stream>>>(
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
         + 3 * 2 * NP * NB * es      // PA, P[0], P[1]
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
    b->hi = take(NP * NB * es);
    b->lo = take(NP * NB * es);
    b->ldk = NB;
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

// Right-looking factorization of W with one step of look-ahead (the structure of potrf):
//   S0 (caller):  [update next block column | record E0] [update the rest of the trailing
//                  matrix, leaving free_sms SMs]
//   S1 (aux):     wait E0 -> diag + panel + split of the next step -> record E1
int lp_chol_factor(mo_ctx *ctx, LpChol &f, int *d_info, double *d_bad) {
  int rc = f.prec == kLpBf16x3 ? set_lp_diag_smem<kLpBf16x3>() : set_lp_diag_smem<kLpTf32x3>();
  if (rc) return rc;
  const int NP = f.NP;
  cudaStream_t s0 = ctx->stream, s1 = nullptr;
  if ((rc = aux_stream(ctx, &s1))) return rc;
  if ((rc = stream_wait(ctx, s1, s0, ctx->ev_fork))) return rc;
  // SMs the trailing update leaves to the look-ahead stream (diagonal block + panel);
  // measured at n = 16384: 2 -> 34.26 ms, 8 -> 34.4 ms, 16 -> 34.82 ms per solve
  const int free_sms = 2;
  {
    StreamSwap sw(ctx, s1);
    if ((rc = lp_panel(ctx, f, 0, d_info, d_bad, f.P[0]))) return rc;
  }
  for (int k = 0, step = 0; k < NP; k += NB, ++step) {
    const int rest = NP - k - NB;
    if ((rc = stream_wait(ctx, s0, s1, ctx->ev_join))) return rc;  // panel k done
    if (rest <= 0) break;
    const LpSplit &P = f.P[step & 1];
    float *W22 = f.W + (k + NB) + (int64_t)(k + NB) * f.ldw;
    // 1. next block column (rest x 128, its top 128 x 128 block is diagonal)
    LpGemmArgs g;
    g.M = rest;
    g.N = NB;
    g.K = NB;
    g.alpha = -1.f;
    g.beta = 1.f;
    g.A = P;
    g.B = P;
    g.C = W22;
    g.ldc = f.ldw;
    g.mode = kGemmLower;
    // rows below its top 128 x 128 block are the next step's A21: the epilogue splits them
    // into f.PA for the next panel (which runs after this launch, on the look-ahead stream)
    g.out = f.PA;
    g.out_row0 = NB;
    if ((rc = lp_gemm(ctx, f.prec, g))) return rc;
    if ((rc = stream_wait(ctx, s1, s0, ctx->ev_fork))) return rc;
    // 2. the next step's diagonal block and panel on the look-ahead stream
    {
      StreamSwap sw(ctx, s1);
      if ((rc = lp_panel(ctx, f, k + NB, d_info, d_bad, f.P[(step + 1) & 1]))) return rc;
    }
    // 3. the rest of the trailing matrix
    const int r2 = rest - NB;
    if (r2 > 0) {
      LpGemmArgs t;
      t.M = r2;
      t.N = r2;
      t.K = NB;
      t.alpha = -1.f;
      t.beta = 1.f;
      t.A = lp_rows(P, f.prec, NB);
      t.B = t.A;
      t.C = W22 + NB + (int64_t)NB * f.ldw;
      t.ldc = f.ldw;
      t.mode = kGemmLower;
      t.max_ctas = ctx->sms - free_sms;
      if ((rc = lp_gemm(ctx, f.prec, t))) return rc;
    }
  }
  return MO_OK;
}

}  // namespace mo
