// Triangular solves with the factor of the mixed-precision Cholesky (the preconditioner of
// the FP64 refinement in ir.cu), in steps of BS = 1024 rows on the FP64 GEMM engine.
//
// Once per factorization, the FP64 inverses of L's BS x BS diagonal blocks are formed from
// the 128 x 128 inverses the factorization already computed, by recursive doubling
//     inv([A 0; B C]) = [inv(A) 0; -inv(C) B inv(A)  inv(C)]
// (levels 128 -> 256 -> 512 -> 1024; each level is two batched DMMA products over all
// blocks: T = B inv(A), then -inv(C) T, skipping the triangular zeros of inv(A) and
// inv(C); B is read from the FP32 factor, whose values are exact in FP64).  A solve of the
// n x nr right-hand sides D then takes n / BS steps of two products (step_kernel):
//     L y = d  :  Y_i = inv(L_ii) D_i ;  D_{>i} -= L_{>i,i} Y_i          (top-down)
//     L^T x = y:  X_i = inv(L_ii)^T Y_i ;  Y_{<i} -= L_{i,<i}^T X_i      (bottom-up, X -> D)
// so the dependency chain is 2 n / BS launches per solve, each spread over the whole
// device, instead of n / 64 dependent 64-row steps.  The factor is read in place (FP32)
// and the arithmetic is FP64: the correction has the accuracy of FP64 substitution up to
// the conditioning of the diagonal blocks of L.
#include <type_traits>

#include "lpchol.cuh"

namespace mo {
namespace {

constexpr int BS = kLpSolveBlock;  // diagonal block order of the solve
constexpr int MT = 64;             // output tile of the merge products
constexpr int KC = 32;             // depth of one staged chunk
constexpr int LDT = MT + 4;

// Dinv block b, 128 x 128 diagonal sub-blocks <- the factorization's FP64 inverses (inv:
// NP / 128 column-major 128 x 128 blocks, zeros above the diagonal)
__global__ void __launch_bounds__(256) place_inv128_kernel(const double *inv, double *Dinv) {
  const int q = blockIdx.x;  // global 128-block index
  const int b = q * 128 / BS, lo = q * 128 - b * BS;
  double *dst = Dinv + (size_t)b * BS * BS + lo + (size_t)lo * BS;
  const double *src = inv + (size_t)q * 128 * 128;
  for (int e = threadIdx.x; e < 128 * 128; e += 256) dst[(e & 127) + (size_t)(e >> 7) * BS] = src[e];
}

// One merge level m of the block inverses.  blockIdx.y = merge z = b * (BS / (2m)) + q,
// covering rows/cols [o, o + 2m) of block b (o = q * 2m, local); the lower-left part
// (mc x m, mc = the second half's order) is computed in 64 x 64 tiles:
//   PHASE 1:  T_z = L[B part] * inv(A)           (k from the tile's first column: inv(A)
//                                                  is lower triangular)
//   PHASE 2:  Dinv[lower-left] = -inv(C) * T_z    (k up to the tile's last row)
template <int PHASE>
__global__ void __launch_bounds__(128) inv_merge_kernel(const float *W, int64_t ldw,
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
  const double *Ab = nullptr, *Bb;
  const float *Af = nullptr;
  int64_t lda, ldb;
  int klo, khi;
  if (PHASE == 1) {
    Af = W + (int64_t)(b * BS + o + m) + (int64_t)(b * BS + o) * ldw;  // B part of L (FP32)
    lda = ldw;
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
      const bool ok = gi < mc && gk < khi && gk < kA;
      As[k][i] = !ok ? 0.0 : (PHASE == 1 ? (double)Af[gi + (int64_t)gk * lda] : Ab[gi + (int64_t)gk * lda]);
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

// ---------------------------------------------------------------------------------------
// One solve step: C (M x nr) = beta * C + alpha * op(A) * B, with op(A) M x K (FP32 factor
// or FP64 block inverse, plain or transposed), B K x nr FP64 (nr <= NRT <= 64).  A CTA
// takes 64 rows and one K chunk; 32-deep chunks of op(A) and B pass through shared memory
// by 16-byte (A) and 8-byte (B) cp.async, double-buffered, and eight warps (4 x 2, each 16
// rows x NRT / 2 columns) multiply them on the FP64 tensor pipe (mma.sync m16n8k4, FP32
// values converted exactly when the fragments are read).  With several K chunks per row
// tile the partial products go to scratch, and the CTA that finishes a tile last adds them
// in chunk order (a fixed order: the result does not depend on timing) and writes C.
// ---------------------------------------------------------------------------------------
constexpr int ST_THREADS = 256;
constexpr int SR = 64;   // rows per tile
constexpr int SK = 32;   // k per staged chunk

struct StepArgs {
  const void *A;
  int64_t lda;
  int tri;  // 0 full, 1: op(A) lower triangular (k <= i), 2: upper (k >= i)
  const double *B;
  int64_t ldb;
  double *C;
  int64_t ldc;
  int M, K, nr;
  double alpha, beta;
  int kc, kchunks;  // K per chunk (multiple of SK) and chunks per row tile
  double *part;     // kchunks x tiles x SR x NRT partial sums
  unsigned *cnt;    // per row tile: chunks finished (zero between launches)
  const int *skip;
};

template <bool F64, bool TRANS>
struct AStage {
  // element (i, k) of the staged op(A) chunk; stride chosen so fragment reads (lane 4g + t:
  // i = g (+8), k = t) hit distinct banks
  using T = typename std::conditional<F64, double, float>::type;
  static constexpr int LD = TRANS ? 36 : (F64 ? 68 : 72);
  static constexpr int ELEMS = TRANS ? SR * LD : SK * LD;
  __device__ static T &at(T *s, int i, int k) { return TRANS ? s[i * LD + k] : s[k * LD + i]; }
};

__device__ __forceinline__ void cp16(void *dst, const void *src, bool ok) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(ok ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit_grp() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_grp1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_grp0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <bool F64, bool TRANS, int NRT>
__global__ void __launch_bounds__(ST_THREADS) step_kernel(const StepArgs p) {
  using AS = AStage<F64, TRANS>;
  using T = typename AS::T;
  constexpr int LDB = 36;  // Bs[c][k]
  constexpr int NF = NRT / 16;  // n fragments per warp (warp columns: NRT / 2)
  if (p.skip && *(volatile const int *)p.skip) return;
  extern __shared__ __align__(16) double st_smem[];
  T *const As = reinterpret_cast<T *>(st_smem);           // [2][AS::ELEMS]
  double *const Bs = reinterpret_cast<double *>(As + 2 * AS::ELEMS);  // [2][NRT * LDB]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int wr = warp & 3, cw = (warp >> 2) * (NRT / 2);
  const int mt = blockIdx.x, kq = blockIdx.y;
  const int i0 = mt * SR;
  int k_lo = kq * p.kc, k_hi = min(p.K, k_lo + p.kc);
  if (p.tri == 1) k_hi = min(k_hi, i0 + SR);
  if (p.tri == 2) k_lo = max(k_lo, i0);
  const int nchunk = k_hi > k_lo ? (k_hi - k_lo + SK - 1) / SK : 0;
  auto stage = [&](int c, int buf) {
    const int k0 = k_lo + c * SK;
    T *a = As + buf * AS::ELEMS;
    if (!F64 && !TRANS) {  // A[i + k lda]: per k, 64 floats in 16 pieces
      for (int e = tid; e < SK * 16; e += ST_THREADS) {
        const int k = e >> 4, i = (e & 15) * 4;
        const bool ok = k0 + k < k_hi && i0 + i < p.M;
        const float *src = static_cast<const float *>(p.A) + (i0 + i) + (int64_t)(k0 + k) * p.lda;
        cp16(&AS::at(a, i, k), ok ? src : p.A, ok);
      }
    } else if (!F64 && TRANS) {  // A[k + i lda]: per i, 32 floats in 8 pieces
      for (int e = tid; e < SR * 8; e += ST_THREADS) {
        const int i = e >> 3, k = (e & 7) * 4;
        const bool ok = k0 + k < k_hi && i0 + i < p.M;
        const float *src = static_cast<const float *>(p.A) + (k0 + k) + (int64_t)(i0 + i) * p.lda;
        cp16(&AS::at(a, i, k), ok ? src : p.A, ok);
      }
    } else if (F64 && !TRANS) {  // per k, 64 doubles in 32 pieces
      for (int e = tid; e < SK * 32; e += ST_THREADS) {
        const int k = e >> 5, i = (e & 31) * 2;
        const bool ok = k0 + k < k_hi && i0 + i < p.M;
        const double *src = static_cast<const double *>(p.A) + (i0 + i) + (int64_t)(k0 + k) * p.lda;
        cp16(&AS::at(a, i, k), ok ? src : p.A, ok);
      }
    } else {  // per i, 32 doubles in 16 pieces
      for (int e = tid; e < SR * 16; e += ST_THREADS) {
        const int i = e >> 4, k = (e & 15) * 2;
        const bool ok = k0 + k < k_hi && i0 + i < p.M;
        const double *src = static_cast<const double *>(p.A) + (k0 + k) + (int64_t)(i0 + i) * p.lda;
        cp16(&AS::at(a, i, k), ok ? src : p.A, ok);
      }
    }
    double *b = Bs + buf * NRT * LDB;
    for (int e = tid; e < NRT * SK; e += ST_THREADS) {
      const int c2 = e >> 5, k = e & 31;
      const bool ok = c2 < p.nr && k0 + k < k_hi;
      const double *src = p.B + (k0 + k) + (int64_t)c2 * p.ldb;
      cp_async_8(&b[c2 * LDB + k], ok ? src : p.B, ok ? 8 : 0);
    }
  };
  double d[NF][4];
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int q = 0; q < 4; ++q) d[f][q] = 0.0;
  if (nchunk > 0) {
    stage(0, 0);
    cp_commit_grp();
    for (int c = 0; c < nchunk; ++c) {
      const int buf = c & 1;
      if (c + 1 < nchunk) stage(c + 1, buf ^ 1);
      cp_commit_grp();
      cp_wait_grp1();
      __syncthreads();
      T *a = As + buf * AS::ELEMS;
      const double *b = Bs + buf * NRT * LDB;
#pragma unroll
      for (int kk = 0; kk < SK; kk += 4) {
        const double a0 = (double)AS::at(a, 16 * wr + g, kk + t);
        const double a1 = (double)AS::at(a, 16 * wr + g + 8, kk + t);
#pragma unroll
        for (int f = 0; f < NF; ++f) dmma_16x8x4(d[f], a0, a1, b[(cw + 8 * f + g) * LDB + kk + t]);
      }
      __syncthreads();
    }
    cp_wait_grp0();
  }
  // this thread's outputs: row i0 + 16 wr + g + 8 h, column cw + 8 f + 2 t + e <- d[f][2h + e]
  auto apply = [&](int f, int q, double v) {
    const int r = i0 + 16 * wr + g + 8 * (q >> 1), c2 = cw + 8 * f + 2 * t + (q & 1);
    if (r < p.M && c2 < p.nr) {
      double *cp = p.C + r + (int64_t)c2 * p.ldc;
      *cp = p.beta == 0.0 ? p.alpha * v : fma(p.alpha, v, p.beta * *cp);
    }
  };
  if (p.kchunks == 1) {
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int q = 0; q < 4; ++q) apply(f, q, d[f][q]);
    return;
  }
  // partial products of this chunk; the last chunk of the tile to finish adds them all
  const int ntiles = gridDim.x;
  auto slot = [&](int chunk, int f, int q) -> double * {
    const int r = 16 * wr + g + 8 * (q >> 1), c2 = cw + 8 * f + 2 * t + (q & 1);
    return p.part + (((size_t)chunk * ntiles + mt) * SR + r) * NRT + c2;
  };
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int q = 0; q < 4; ++q) *slot(kq, f, q) = d[f][q];
  __threadfence();
  __syncthreads();
  __shared__ int s_last;
  if (tid == 0) s_last = atomicAdd(&p.cnt[mt], 1u) == (unsigned)(p.kchunks - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double v = 0.0;
      for (int ch = 0; ch < p.kchunks; ++ch) v += __ldcg(slot(ch, f, q));
      apply(f, q, v);
    }
  if (tid == 0) p.cnt[mt] = 0u;
}

}  // namespace

// scratch of the K-split: at most this many (row tile, chunk) pairs per launch
static size_t step_pairs(int NP, int sms) { return (size_t)2 * sms + NP / SR + 8; }

size_t lp_solve_bytes(int n, int nrhs, int sms) {
  const size_t NP = (size_t)((n + 127) / 128) * 128;
  const size_t nb = (NP + BS - 1) / BS;
  return nb * BS * BS * 8                         // Dinv
         + nb * BS * (BS / 2) * 8                 // merge scratch T
         + (size_t)n * std::min(nrhs, 64) * 8     // Y (one group of <= 64 columns)
         + 2 * step_pairs((int)NP, sms) * SR * 64 * 8 // K-split partial sums, per stream
         + 2 * (NP / SR + 64) * 4                     // per-tile counters, per stream
         + 6 * 256;
}

int lp_solve_setup(int n, int nrhs, int sms, void *mem, LpSolve &s) {
  s.n = n;
  s.NP = ((n + 127) / 128) * 128;
  s.nblk = (s.NP + BS - 1) / BS;
  s.nrhs = nrhs;
  s.sms = sms;
  char *p = (char *)(((uintptr_t)mem + 255) & ~(uintptr_t)255);
  auto take = [&](size_t bytes) {
    char *r = p;
    p += (bytes + 255) & ~(size_t)255;
    return r;
  };
  s.Dinv = (double *)take((size_t)s.nblk * BS * BS * 8);
  s.T = (double *)take((size_t)s.nblk * BS * (BS / 2) * 8);
  s.Y = (double *)take((size_t)n * std::min(nrhs, 64) * 8);
  for (int q = 0; q < 2; ++q) {
    s.part[q] = (double *)take(step_pairs(s.NP, sms) * SR * 64 * 8);
    s.cnt[q] = (unsigned *)take((size_t)(s.NP / SR + 64) * 4);
  }
  return MO_OK;
}

int lp_solve_prepare(mo_ctx *ctx, const LpChol &f, LpSolve &s) {
  cudaStream_t st = ctx->stream;
  const int NP = f.NP;
  if (NP != s.NP) return MO_EINVAL;
  s.W = f.W;
  s.ldw = f.ldw;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_OTHER);
  for (int q = 0; q < 2; ++q)
    MO_CUDA_TRY(cudaMemsetAsync(s.cnt[q], 0, (size_t)(s.NP / SR + 64) * 4, st));
  MO_CUDA_TRY(cudaMemsetAsync(s.Dinv, 0, (size_t)s.nblk * BS * BS * 8, st));
  place_inv128_kernel<<<NP / 128, 256, 0, st>>>(f.inv, s.Dinv);
  prof_end(ctx, ps, 0.0, 8.0 * s.nblk * BS * (double)BS);
  MO_CUDA_TRY(cudaGetLastError());
  ProfScope pm;
  prof_begin(ctx, pm, MO_PROF_TRTRI);
  double flops = 0.0;
  for (int m = 128; m < BS; m *= 2) {
    const int merges = s.nblk * (BS / (2 * m));
    const dim3 grid((m / MT) * (m / MT), merges);
    inv_merge_kernel<1><<<grid, 128, 0, st>>>(f.W, f.ldw, s.Dinv, s.T, NP, m);
    inv_merge_kernel<2><<<grid, 128, 0, st>>>(f.W, f.ldw, s.Dinv, s.T, NP, m);
    flops += 2.0 * merges * (double)m * m * m;
  }
  prof_end(ctx, pm, flops, 0.0);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

namespace {

template <bool F64, bool TRANS, int NRT>
int launch_step_t(mo_ctx *ctx, const StepArgs &a, dim3 grid) {
  using AS = AStage<F64, TRANS>;
  const int smem = (int)(2 * (AS::ELEMS * sizeof(typename AS::T) + NRT * 36 * sizeof(double)));
  if (int rc = mo_smem_attr((const void *)step_kernel<F64, TRANS, NRT>, smem)) return rc;
  step_kernel<F64, TRANS, NRT><<<grid, ST_THREADS, smem, ctx->stream>>>(a);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// C (M x nr, ldc) = beta C + alpha op(A) B, op(A) M x K
int step(mo_ctx *ctx, const LpSolve &s, int q, const void *A, int64_t lda, bool f64, bool trans,
         int tri, const double *B, int64_t ldb, double *C, int64_t ldc, int M, int K, int nr,
         double alpha, double beta, const int *skip) {
  if (M <= 0 || nr <= 0) return MO_OK;
  StepArgs a;
  a.A = A;
  a.lda = lda;
  a.tri = tri;
  a.B = B;
  a.ldb = ldb;
  a.C = C;
  a.ldc = ldc;
  a.M = M;
  a.K = K;
  a.nr = nr;
  a.alpha = alpha;
  a.beta = beta;
  a.skip = skip;
  a.part = s.part[q];
  a.cnt = s.cnt[q];
  // enough (tile, chunk) pairs for two CTAs per SM, chunks of at least 128
  const int tiles = (M + SR - 1) / SR;
  int kch = std::max(1, std::min((2 * s.sms + tiles - 1) / tiles, (K + 127) / 128));
  int kc = ((K + kch - 1) / kch + SK - 1) / SK * SK;
  kch = (K + kc - 1) / kc;
  if ((size_t)tiles * kch > step_pairs(s.NP, s.sms) || tiles > s.NP / SR + 64) return MO_EINVAL;
  a.kc = kc;
  a.kchunks = kch;
  const dim3 grid(tiles, kch);
  const int nrt = nr <= 16 ? 16 : (nr <= 32 ? 32 : 64);
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_IR);
  int rc;
#define MO_STEP(F, TR)                                                   \
  rc = nrt == 16 ? launch_step_t<F, TR, 16>(ctx, a, grid)                \
                 : (nrt == 32 ? launch_step_t<F, TR, 32>(ctx, a, grid)   \
                              : launch_step_t<F, TR, 64>(ctx, a, grid))
  if (f64) {
    if (trans) MO_STEP(true, true);
    else MO_STEP(true, false);
  } else {
    if (trans) MO_STEP(false, true);
    else MO_STEP(false, false);
  }
#undef MO_STEP
  prof_end(ctx, ps, 2.0 * M * (double)K * nr,
           (f64 ? 8.0 : 4.0) * M * (double)K + 8.0 * (K + 2.0 * M) * nr);
  return rc;
}

// the forward and the backward block solve of the columns [c0, c0 + w) of D, with the
// scratch set q, on the context's current stream
int solve_group(mo_ctx *ctx, const LpSolve &s, int q, double *D, int c0, int w, const int *skip) {
  const int n = s.n;
  double *Dc = D + (int64_t)c0 * n, *Y = s.Y + (int64_t)c0 * n;
  int rc;
  for (int b = 0; b < s.nblk; ++b) {
    const int o0 = b * BS, h = std::min(BS, n - o0);
    if (h <= 0) break;
    const double *Di = s.Dinv + (size_t)b * BS * BS;
    // Y_b = inv(L_bb) D_b
    if ((rc = step(ctx, s, q, Di, BS, true, false, 1, Dc + o0, n, Y + o0, n, h, h, w, 1.0, 0.0, skip)))
      return rc;
    // D_{>b} -= L_{>b,b} Y_b
    const int rest = n - o0 - h;
    if (rest > 0 &&
        (rc = step(ctx, s, q, s.W + (o0 + h) + (int64_t)o0 * s.ldw, s.ldw, false, false, 0, Y + o0, n,
                   Dc + o0 + h, n, rest, h, w, -1.0, 1.0, skip)))
      return rc;
  }
  for (int b = s.nblk - 1; b >= 0; --b) {
    const int o0 = b * BS, h = std::min(BS, n - o0);
    if (h <= 0) continue;
    const double *Di = s.Dinv + (size_t)b * BS * BS;
    // X_b = inv(L_bb)^T Y_b  (into D)
    if ((rc = step(ctx, s, q, Di, BS, true, true, 2, Y + o0, n, Dc + o0, n, h, h, w, 1.0, 0.0, skip)))
      return rc;
    // Y_{<b} -= L_{b,<b}^T X_b
    if (o0 > 0 && (rc = step(ctx, s, q, s.W + o0, s.ldw, false, true, 0, Dc + o0, n, Y, n, o0, h, w,
                             -1.0, 1.0, skip)))
      return rc;
  }
  return MO_OK;
}

}  // namespace

// D (n x nr, ld n) <- (L L^T)^-1 D, as the forward and the backward block solve.  More
// than 32 columns are split in two halves solved on two streams: each chain of launches
// is latency-bound in its small steps, and two independent chains fill each other's gaps.
int lp_solve_apply(mo_ctx *ctx, const LpSolve &s, double *D, int nr, const int *skip) {
  if (s.n == 0 || nr == 0) return MO_OK;
  if (nr > s.nrhs) return MO_EINVAL;
  int rc;
  for (int c0 = 0; c0 < nr; c0 += 64) {
    const int w = std::min(64, nr - c0);
    if (w <= 32) {
      if ((rc = solve_group(ctx, s, 0, D, c0, w, skip))) return rc;
      continue;
    }
    const int w0 = (w + 1) / 2;
    cudaStream_t s0 = ctx->stream, s1 = nullptr;
    if ((rc = aux_stream(ctx, &s1))) return rc;
    if ((rc = stream_wait(ctx, s1, s0, ctx->ev_fork))) return rc;
    {
      StreamSwap sw(ctx, s1);
      if ((rc = solve_group(ctx, s, 1, D, c0 + w0, w - w0, skip))) return rc;
    }
    if ((rc = solve_group(ctx, s, 0, D, c0, w0, skip))) return rc;
    if ((rc = stream_wait(ctx, s0, s1, ctx->ev_join))) return rc;
  }
  return MO_OK;
}

}  // namespace mo
