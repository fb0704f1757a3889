// The rest of the reference's level-3 surface on the FP64 GEMM engine: MultSym (SYMM),
// MultTrm (TRMM), RankUpdate2Sym (SYR2K) and UpdateTrm (triangular update).
//
// Reference semantics (mmult.go:266-523 over calgo/dmmat_symm.c:253, dmmat_trid.c:780,
// dmmat_rank.c:132 and :292):
//   MultSym        C = beta*C + alpha*S*op(B) (no MO_RIGHT) or beta*C + alpha*op(B)*S (MO_RIGHT),
//                  S symmetric stored in the triangle MO_UPPER (else lower) selects
//   MultTrm        B = alpha*op(T)*B (MO_LEFT or no side) / alpha*B*op(T) (MO_RIGHT), T
//                  triangular (MO_UPPER / lower, MO_UNIT)
//   RankUpdate2Sym triangle(C) = beta*C + alpha*(A*B^T + B*A^T)   (A^T*B + B^T*A, MO_TRANSA)
//   UpdateTrm      triangle(C) = beta*C + alpha*op(A)*op(B)
// The two triangle updates apply beta inside the nb x nb diagonal blocks only, as the
// reference's kernels do (and RankUpdate2Sym without MO_TRANSA applies it there twice,
// calgo/dmmat_rank.c:228); mo_set_syrk_blas_beta(ctx, 1) selects BLAS semantics.
//
// Device form: SYMM and TRMM expand the symmetric / triangular operand into a dense
// square (one pass of n^2 elements) and run one engine GEMM, writing TRMM's product to a
// scratch copy that is then moved into B; the triangle updates are the engine's triangle
// modes (tiles on one side of the diagonal and an element mask) with two distinct operands.
#include "context.cuh"

namespace mo {
namespace {

enum ExpandMode : int { kSymLower = 0, kSymUpper = 1, kTriLower = 2, kTriUpper = 3 };

// D (n x n, ld n) = the dense matrix that A's selected triangle defines: symmetric
// (mirrored) or triangular (zeros elsewhere, ones on the diagonal with unit)
__global__ void __launch_bounds__(256) expand_kernel(const double *A, int64_t lda, int n, int mode,
                                                     int unit, double *D) {
  __shared__ double T[32][33];
  const int bi = blockIdx.x, bj = blockIdx.y;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const bool upper = mode == kSymUpper || mode == kTriUpper;
  const bool sym = mode == kSymLower || mode == kSymUpper;
  // this tile of D, read directly when its elements are stored, else through the
  // transposed tile (staged in shared memory so that both reads are coalesced)
  const bool stored_tile = upper ? bi <= bj : bi >= bj;
  if (!sym && !stored_tile) {
    for (int r = ty; r < 32; r += 8) {
      const int i = bi * 32 + tx, j = bj * 32 + r;
      if (i < n && j < n) D[i + (int64_t)j * n] = 0.0;
    }
    return;
  }
  for (int r = ty; r < 32; r += 8) {
    // element (i, j) of D for stored tiles, (j, i) of the stored transpose otherwise
    const int i = (stored_tile ? bi : bj) * 32 + tx, j = (stored_tile ? bj : bi) * 32 + r;
    double v = 0.0;
    if (i < n && j < n) {
      const bool stored = upper ? i <= j : i >= j;
      v = stored ? A[i + (int64_t)j * lda] : (sym ? A[j + (int64_t)i * lda] : 0.0);
      if (i == j && unit) v = 1.0;
    }
    T[r][tx] = v;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int i = bi * 32 + tx, j = bj * 32 + r;
    if (i < n && j < n) D[i + (int64_t)j * n] = stored_tile ? T[r][tx] : T[tx][r];
  }
}

int expand(mo_ctx *ctx, View A, int n, int mode, bool unit, double *D) {
  const dim3 grid((n + 31) / 32, (n + 31) / 32);
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_OTHER);
  expand_kernel<<<grid, 256, 0, ctx->stream>>>(A.d, A.ld, n, mode, unit ? 1 : 0, D);
  prof_end(ctx, ps, 0.0, 12.0 * n * (double)n);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// T's 128 x 128 diagonal blocks <- the block inverses (nblk x 128 x 128, ld 128)
__global__ void __launch_bounds__(256) place_diag_kernel(const double *inv, double *T, int64_t ldt,
                                                         int n) {
  const int q = blockIdx.x, r0 = q * 128, h = min(128, n - r0);
  const double *src = inv + (size_t)q * 128 * 128;
  for (int e = threadIdx.x; e < 128 * 128; e += 256) {
    const int i = e & 127, j = e >> 7;
    if (i < h && j < h) T[(r0 + i) + (int64_t)(r0 + j) * ldt] = src[e];
  }
}

// A's triangle (lower or upper; strict with unit) <- T's
__global__ void __launch_bounds__(256) tri_back_kernel(const double *T, int64_t ldt, double *A,
                                                       int64_t lda, int n, int lower, int unit) {
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  if (lower ? i0 + 31 < j0 : j0 + 31 < i0) return;
  for (int e = threadIdx.x; e < 32 * 32; e += 256) {
    const int i = i0 + (e & 31), j = j0 + (e >> 5);
    if (i >= n || j >= n) continue;
    if (lower ? i < j : i > j) continue;
    if (unit && i == j) continue;
    A[i + (int64_t)j * lda] = T[i + (int64_t)j * ldt];
  }
}

// the diagonal-block size of the reference's beta (calgo/dmmat_rank.c:146-154), or 0 for
// BLAS semantics / beta == 1
int beta_block_of(mo_ctx *ctx, double beta, int n) {
  if (ctx->syrk_blas_beta || beta == 1.0) return 0;
  int nb = ctx->nb;
  if (nb > 68 || nb <= 0) nb = 68;
  if (nb > n) nb = n;
  return nb;
}

}  // namespace

int trtri_blocks(mo_ctx *ctx, View A, int N, bool trans, bool lower_eff, bool unit, double *inv);

}  // namespace mo

using mo::View;

extern "C" {

// mmult.go:266-330
int mo_mult_sym(mo_ctx *ctx, mo_matrix Cm, mo_matrix Am, mo_matrix Bm, double alpha, double beta,
                int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View C, A, B;
  if ((rc = mo::to_view(Cm, C)) || (rc = mo::to_view(Am, A)) || (rc = mo::to_view(Bm, B)))
    return rc;
  const int ar = A.rows, ac = A.cols, br = B.rows, bc = B.cols, cr = C.rows, cc = C.cols;
  bool ok, empty;
  switch (flags & (MO_TRANSA | MO_TRANSB)) {
    case MO_TRANSA | MO_TRANSB:
      empty = ac == 0 || br == 0;
      ok = ar == ac && cr == ac && cc == br && ar == bc;
      break;
    case MO_TRANSA:
      empty = ac == 0 || bc == 0;
      ok = ar == ac && cr == ac && cc == bc && ar == br;
      break;
    case MO_TRANSB:
      empty = ar == 0 || br == 0;
      ok = ar == ac && cr == ar && cc == br && ac == bc;
      break;
    default:
      empty = ar == 0 || bc == 0;
      ok = ar == ac && cr == ar && cc == bc && ac == br;
  }
  if (empty) return MO_OK;
  if (!ok) return MO_ESYMSIZE;
  const int n = ar;
  // S*op(B) unless MO_RIGHT (mmult.go:260's default; the reference's kernel gives S*B for
  // no side bit where its diagonal-block helper decides, calgo/dmmat_symm.c:239-244)
  const bool left = (flags & MO_RIGHT) == 0, tb = (flags & MO_TRANSB) != 0;
  // the products the shapes allow: S*op(B) (left) or op(B)*S; shapes the size check lets
  // through but that do not fit (the reference reads out of range) are refused
  const int orow = left ? n : (tb ? bc : br), ocol = left ? (tb ? br : bc) : n;
  if ((left && (tb ? bc : br) != n) || (!left && (tb ? br : bc) != n) || orow != cr || ocol != cc)
    return MO_EABSIZE;
  double *S = nullptr;
  if ((rc = mo::workspace(ctx, (size_t)n * n * sizeof(double), (void **)&S))) return rc;
  if ((rc = mo::expand(ctx, A, n, (flags & MO_UPPER) ? mo::kSymUpper : mo::kSymLower, false, S)))
    return rc;
  const View Sv{S, n, n, n};
  return left ? mo::gemm(ctx, C, Sv, false, B, tb, alpha, beta)
              : mo::gemm(ctx, C, B, tb, Sv, false, alpha, beta);
}

// mmult.go:338-375
int mo_mult_trm(mo_ctx *ctx, mo_matrix Bm, mo_matrix Am, double alpha, int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View B, A;
  if ((rc = mo::to_view(Bm, B)) || (rc = mo::to_view(Am, A))) return rc;
  bool ok = true, empty = false;
  switch (flags & (MO_LEFT | MO_RIGHT)) {
    case MO_LEFT:
      empty = B.rows == 0 || B.cols == 0;
      ok = B.rows == A.cols && A.cols == A.rows;
      break;
    case MO_RIGHT:
      empty = B.cols == 0 || B.rows == 0;
      ok = B.cols == A.rows && A.cols == A.rows;
      break;
    default:
      break;
  }
  if (empty) return MO_OK;
  if (!ok) return MO_EABSIZE;
  const bool right = (flags & MO_RIGHT) != 0;
  const int n = A.cols;
  if (n == 0 || B.rows == 0 || B.cols == 0) return MO_OK;
  if (A.rows < n || (right ? B.cols : B.rows) != n) return MO_EABSIZE;
  const size_t tbytes = (size_t)n * n * sizeof(double);
  const size_t xbytes = (size_t)B.rows * B.cols * sizeof(double);
  char *ws = nullptr;
  if ((rc = mo::workspace(ctx, tbytes + xbytes + 256, (void **)&ws))) return rc;
  double *T = (double *)ws, *X = (double *)(ws + ((tbytes + 255) & ~(size_t)255));
  if ((rc = mo::expand(ctx, A, n, (flags & MO_UPPER) ? mo::kTriUpper : mo::kTriLower,
                       (flags & MO_UNIT) != 0, T)))
    return rc;
  const View Tv{T, n, n, n}, Xv{X, B.rows, B.cols, B.rows};
  const bool ta = (flags & MO_TRANSA) != 0;
  rc = right ? mo::gemm(ctx, Xv, B, false, Tv, ta, alpha, 0.0)
             : mo::gemm(ctx, Xv, Tv, ta, B, false, alpha, 0.0);
  if (rc) return rc;
  MO_CUDA_TRY(cudaMemcpy2DAsync(B.d, (size_t)B.ld * 8, X, (size_t)B.rows * 8, (size_t)B.rows * 8,
                                B.cols, cudaMemcpyDeviceToDevice, ctx->stream));
  return MO_OK;
}

// mmult.go:453-475 (calgo/dmmat_rank.c:132-235)
int mo_rank_update2_sym(mo_ctx *ctx, mo_matrix Cm, mo_matrix Am, mo_matrix Bm, double alpha,
                        double beta, int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View C, A, B;
  if ((rc = mo::to_view(Cm, C)) || (rc = mo::to_view(Am, A)) || (rc = mo::to_view(Bm, B)))
    return rc;
  if (C.rows != C.cols) return MO_ECNOTSQUARE;
  const bool ta = (flags & MO_TRANSA) != 0;
  const int P = ta ? A.rows : A.cols, n = C.rows;
  if (P == 0 || n == 0) return MO_OK;
  if ((ta ? A.cols : A.rows) != n || B.rows != A.rows || B.cols != A.cols) return MO_EABSIZE;
  const bool up = (flags & MO_UPPER) != 0, lo = (flags & MO_LOWER) != 0;
  if (up == lo) return MO_EINVAL;
  mo::GemmOpts o;
  o.mode = up ? mo::kSyrkUpper : mo::kSyrkLower;
  o.beta_block = mo::beta_block_of(ctx, beta, n);
  // first A op(B)^T-like product with beta, then the mirrored one: beta again inside the
  // diagonal blocks without MO_TRANSA (the reference's second diagonal pass), else 1
  if ((rc = mo::gemm_ex(ctx, C, A, ta, B, !ta, alpha, beta, o))) return rc;
  const double beta2 = (o.beta_block > 0 && !ta) ? beta : 1.0;
  return mo::gemm_ex(ctx, C, B, ta, A, !ta, alpha, beta2, o);
}

// mmult.go:501-523 (calgo/dmmat_rank.c:292-355)
int mo_update_trm(mo_ctx *ctx, mo_matrix Cm, mo_matrix Am, mo_matrix Bm, double alpha,
                  double beta, int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View C, A, B;
  if ((rc = mo::to_view(Cm, C)) || (rc = mo::to_view(Am, A)) || (rc = mo::to_view(Bm, B)))
    return rc;
  if (C.rows != C.cols) return MO_ECNOTSQUARE;
  const bool ta = (flags & MO_TRANSA) != 0, tb = (flags & MO_TRANSB) != 0;
  const int P = ta ? A.rows : A.cols, n = C.rows;
  if (P == 0 || n == 0) return MO_OK;
  if ((ta ? A.cols : A.rows) != n || (tb ? B.rows : B.cols) != n || (tb ? B.cols : B.rows) != P)
    return MO_EABSIZE;
  mo::GemmOpts o;
  o.mode = (flags & MO_UPPER) ? mo::kSyrkUpper : mo::kSyrkLower;
  o.beta_block = mo::beta_block_of(ctx, beta, n);
  return mo::gemm_ex(ctx, C, A, ta, B, tb, alpha, beta, o);
}

// trinv.go:219-243 (InverseTrm).  The triangle is expanded into a dense square T (zeros
// outside it, ones on the diagonal with MO_UNIT), its 128 x 128 diagonal blocks are
// inverted in shared memory, and the inverse is assembled bottom-up by recursive doubling
// on the FP64 engine:
//   lower:  inv([A 0; B C]) = [inv(A) 0; -inv(C) B inv(A)  inv(C)]
//   upper:  inv([A B; 0 C]) = [inv(A) -inv(A) B inv(C); 0 inv(C)]
// before the triangle is written back into A (the other triangle and, with MO_UNIT, the
// diagonal are not written).
int mo_inverse_trm(mo_ctx *ctx, mo_matrix Am, int flags, int nb) {
  (void)nb;
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A;
  if ((rc = mo::to_view(Am, A))) return rc;
  if (A.rows != A.cols) return MO_ENOTSQUARE;
  const int n = A.rows;
  if (n == 0) return MO_OK;
  const bool lower = (flags & MO_LOWER) != 0, unit = (flags & MO_UNIT) != 0;
  const int nblk = (n + 127) / 128;
  int mtop = 128;  // largest merge half: the biggest power-of-two multiple of 128 below n
  while (2 * mtop < n) mtop *= 2;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t tb = al((size_t)n * n * 8), ib = al((size_t)nblk * 128 * 128 * 8),
               wb = al((size_t)mtop * mtop * 8);
  char *ws = nullptr;
  if ((rc = mo::workspace(ctx, tb + ib + wb, (void **)&ws))) return rc;
  double *T = (double *)ws, *inv = (double *)(ws + tb), *W = (double *)(ws + tb + ib);
  const View Tv{T, n, n, n};
  if ((rc = mo::expand(ctx, A, n, lower ? mo::kTriLower : mo::kTriUpper, unit, T))) return rc;
  if ((rc = mo::trtri_blocks(ctx, Tv, n, false, lower, false, inv))) return rc;
  {
    mo::ProfScope ps;
    mo::prof_begin(ctx, ps, MO_PROF_OTHER);
    mo::place_diag_kernel<<<nblk, 256, 0, ctx->stream>>>(inv, T, n, n);
    mo::prof_end(ctx, ps, 0.0, 16.0 * nblk * 128 * 128);
    MO_CUDA_TRY(cudaGetLastError());
  }
  for (int m = 128; m < n; m *= 2) {
    for (int o = 0; o + m < n; o += 2 * m) {
      const int mc = std::min(m, n - o - m);
      const View Ai = Tv.sub(o, o, m, m), Ci = Tv.sub(o + m, o + m, mc, mc);
      if (lower) {
        const View B = Tv.sub(o + m, o, mc, m), Wv{W, mc, m, mc};
        if ((rc = mo::gemm(ctx, Wv, B, false, Ai, false, 1.0, 0.0))) return rc;
        if ((rc = mo::gemm(ctx, B, Ci, false, Wv, false, -1.0, 0.0))) return rc;
      } else {
        const View B = Tv.sub(o, o + m, m, mc), Wv{W, m, mc, m};
        if ((rc = mo::gemm(ctx, Wv, B, false, Ci, false, 1.0, 0.0))) return rc;
        if ((rc = mo::gemm(ctx, B, Ai, false, Wv, false, -1.0, 0.0))) return rc;
      }
    }
  }
  mo::ProfScope pb;
  mo::prof_begin(ctx, pb, MO_PROF_OTHER);
  mo::tri_back_kernel<<<dim3((n + 31) / 32, (n + 31) / 32), 256, 0, ctx->stream>>>(
      T, n, A.d, A.ld, n, lower ? 1 : 0, unit ? 1 : 0);
  mo::prof_end(ctx, pb, 0.0, 8.0 * n * (double)n);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

}  // extern "C"
