// Triangular solves with the factor of the mixed-precision Cholesky (the preconditioner of
// the FP64 refinement in ir.cu): one cooperative kernel over the whole device that walks
// the factor in steps of BS = 1024 rows.
//
// The inverses of the BS x BS diagonal blocks of L are formed once per factorization in
// FP64 from the 128 x 128 diagonal-block inverses that the factorization already computed,
// by recursive doubling:
//     inv([A 0; B C]) = [inv(A) 0; -inv(C) B inv(A)  inv(C)]
// (levels 128 -> 256 -> 512 -> 1024; each level is two batched DMMA products over all
// blocks: T = B inv(A), then -inv(C) T, with the triangular zeros of inv(A) and inv(C)
// skipped; B is read from the FP32 factor, whose values are exact in FP64).  A solve of the
// n x nr right-hand sides R then takes n / BS steps, each two phases separated by grid
// barriers:
//     L x = r  :  X_i = inv(L_ii) R_i ;  R_{>i} -= L_{>i,i} X_i           (top-down)
//     L^T x = r:  X_i = inv(L_ii)^T R_i ;  R_{<i} -= L_{i,<i}^T X_i       (bottom-up)
// so the dependency chain is 16 steps at n = 16384 instead of 256 row blocks of 64, with no
// launch between them.  Both phases are FP64 tensor-pipe products (mma.sync m16n8k4) on
// 16-row tiles: phase A gives each of the first h / 16 CTAs one tile of X_i, phase B deals
// the 16-row tiles of the rows to update round-robin over all CTAs, which keep all their
// tiles' accumulators in registers while 32-deep chunks of L (converted from FP32) and of
// X_i pass through shared memory.  The correction has the accuracy of FP64 substitution up
// to the conditioning of the diagonal blocks of L.
#include "lpchol.cuh"

namespace mo {
namespace {

constexpr int BS = kLpSolveBlock;  // diagonal block order of the solve
constexpr int MT = 64;             // output tile of the merge products
constexpr int KC = 32;             // depth of one staged chunk
constexpr int LDT = MT + 4;

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
// the cooperative solve
// ---------------------------------------------------------------------------------------
constexpr int ST = 256;      // threads per CTA
constexpr int KCH = 32;      // k per staged chunk
constexpr int MTMAX = 16;    // 16-row tiles per CTA and pass of phase B
constexpr int LDA_S = 16 + 2;   // As[k][r] row stride (doubles)

struct SolveArgs {
  const float *W;
  int64_t ldw;
  const double *Dinv;
  double *D;
  int64_t ldd;
  double *Xb;  // BS x nr (ld BS)
  int n, nr, nblk;
  int trans;
  unsigned *bar;  // arrival counter (zeroed before the launch) and abort word
  int *status;
  uint32_t spin;
  const int *skip;
};

// bounded grid barrier: returns false (after recording MO_EDEVTIMEOUT and raising the abort
// word) when the other CTAs do not arrive within `spin` polls, or when another CTA aborted
__device__ bool solve_barrier(const SolveArgs &p, unsigned target) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(p.bar, 1u);
    int ok = 1;
    uint32_t it = 0;
    while (*(volatile unsigned *)p.bar < target) {
      if (*(volatile unsigned *)(p.bar + 1)) {
        ok = 0;
        break;
      }
      if (++it > p.spin) {
        set_status(p.status, MO_EDEVTIMEOUT);
        atomicExch(p.bar + 1, 1u);
        ok = 0;
        break;
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// acc[t] (t < ntile) += A(rows of tile t, 0..K) * B(0..K, n-tile nt) for this warp, where the
// CTA's tiles are 16-row blocks with first rows row0[t]; the A chunk (16 x KCH per tile) and
// the B chunk (KCH x nr) pass through shared memory.
//   lda(i, k) -> value of A at (row i of the global row space, k), FP64
//   ldb(k, c) -> value of B at (k, c)
// Warps: warp w takes n-tile nt = w % NT and tiles t with t % G == w / NT (G = 8 / NT).
template <bool KFAST, class LA, class LB>
__device__ __forceinline__ void tile_products(double (&acc)[MTMAX][4], const int *row0, int ntile,
                                              int K, int nr, LA lda, LB ldb, double *As,
                                              double *Bs) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
  const int NT = (nr + 7) / 8, G = 8 / NT;
  const int nt = warp % NT, grp = warp / NT;
  const bool mma_warp = grp < G;
  const int ldbs = nr + 1;
  for (int k0 = 0; k0 < K; k0 += KCH) {
    __syncthreads();
    // A: tile t rows (16) x KCH, stored As[(t * KCH + k) * LDA_S + r]; consecutive threads
    // walk the direction in which A is contiguous (k with KFAST, else the rows)
    for (int e = threadIdx.x; e < ntile * 16 * KCH; e += ST) {
      const int tt = e / (16 * KCH), rem = e % (16 * KCH);
      const int r = KFAST ? rem / KCH : rem % 16, k = KFAST ? rem % KCH : rem / 16;
      As[(tt * KCH + k) * LDA_S + r] = (k0 + k < K) ? lda(row0[tt] + r, k0 + k) : 0.0;
    }
    for (int e = threadIdx.x; e < KCH * nr; e += ST) {
      const int k = e % KCH, c = e / KCH;
      Bs[k * ldbs + c] = (k0 + k < K) ? ldb(k0 + k, c) : 0.0;
    }
    __syncthreads();
    if (mma_warp) {
#pragma unroll
      for (int kk = 0; kk < KCH; kk += 4) {
        const int col = 8 * nt + g;
        const double b0 = col < nr ? Bs[(kk + t4) * ldbs + col] : 0.0;
#pragma unroll
        for (int tt = 0; tt < MTMAX; ++tt) {
          if (tt < ntile && tt % G == grp) {
            const double *a = As + (tt * KCH + kk + t4) * LDA_S;
            dmma_16x8x4(acc[tt], a[g], a[g + 8], b0);
          }
        }
      }
    }
  }
}

__global__ void __launch_bounds__(ST, 1) blk_solve_kernel(SolveArgs p) {
  if (p.skip && *(volatile const int *)p.skip) return;
  extern __shared__ double sm[];
  double *As = sm;                                   // MTMAX x KCH x LDA_S
  double *Bs = sm + MTMAX * KCH * LDA_S;             // KCH x (nr + 1)
  __shared__ int row0[MTMAX];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
  const int NT = (p.nr + 7) / 8, G = 8 / NT, nt = warp % NT, grp = warp / NT;
  const int C = gridDim.x, c = blockIdx.x;
  unsigned phase = 0;
  for (int step = 0; step < p.nblk; ++step) {
    const int i = p.trans ? p.nblk - 1 - step : step;
    const int r0 = i * BS, h = min(BS, p.n - r0);
    const double *Di = p.Dinv + (size_t)i * BS * BS;
    // ---- phase A: tile c of X_i = op(Dinv_i) R_i ----
    const int ta = (h + 15) / 16;
    for (int tile = c; tile < ta; tile += C) {
      if (threadIdx.x == 0) row0[0] = 16 * tile;
      double acc[MTMAX][4] = {};
      if (p.trans)
        tile_products<true>(acc, row0, 1, h, p.nr,
                      [&](int r, int k) { return r < h ? Di[k + (size_t)r * BS] : 0.0; },
                      [&](int k, int cc) { return p.D[(r0 + k) + (int64_t)cc * p.ldd]; }, As, Bs);
      else
        tile_products<false>(acc, row0, 1, h, p.nr,
                      [&](int r, int k) { return r < h ? Di[r + (size_t)k * BS] : 0.0; },
                      [&](int k, int cc) { return p.D[(r0 + k) + (int64_t)cc * p.ldd]; }, As, Bs);
      if (grp == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = 16 * tile + g + 8 * (q >> 1), cc = 8 * nt + 2 * t4 + (q & 1);
          if (r < h && cc < p.nr) p.Xb[r + (size_t)cc * BS] = acc[0][q];
        }
      }
    }
    if (!solve_barrier(p, (++phase) * C)) return;
    // ---- phase B: X_i into D, and the update of the rows not yet solved ----
    for (int e = threadIdx.x + c * ST; e < h * p.nr; e += C * ST) {
      const int r = e % h, cc = e / h;
      p.D[(r0 + r) + (int64_t)cc * p.ldd] = p.Xb[r + (size_t)cc * BS];
    }
    const int u0 = p.trans ? 0 : r0 + h, u1 = p.trans ? r0 : p.n;  // rows to update
    const int tu = (u1 - u0 + 15) / 16;
    for (int base = c; base < tu; base += C * MTMAX) {
      // this pass: tiles base, base + C, ... (up to MTMAX of them)
      int ntile = 0;
      for (int tile = base; tile < tu && ntile < MTMAX; tile += C) ++ntile;
      if (threadIdx.x < ntile) row0[threadIdx.x] = u0 + 16 * (base + threadIdx.x * C);
      __syncthreads();
      double acc[MTMAX][4] = {};
      if (p.trans)
        tile_products<true>(acc, row0, ntile, h, p.nr,
                      [&](int r, int k) { return r < u1 ? (double)p.W[(r0 + k) + (int64_t)r * p.ldw] : 0.0; },
                      [&](int k, int cc) { return p.Xb[k + (size_t)cc * BS]; }, As, Bs);
      else
        tile_products<false>(acc, row0, ntile, h, p.nr,
                      [&](int r, int k) { return r < u1 ? (double)p.W[r + (int64_t)(r0 + k) * p.ldw] : 0.0; },
                      [&](int k, int cc) { return p.Xb[k + (size_t)cc * BS]; }, As, Bs);
      if (grp < G) {
#pragma unroll
        for (int tt = 0; tt < MTMAX; ++tt) {
          if (tt < ntile && tt % G == grp) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int r = row0[tt] + g + 8 * (q >> 1), cc = 8 * nt + 2 * t4 + (q & 1);
              if (r < u1 && cc < p.nr) p.D[r + (int64_t)cc * p.ldd] -= acc[tt][q];
            }
          }
        }
      }
      __syncthreads();  // row0 is rewritten by the next pass
    }
    if (!solve_barrier(p, (++phase) * C)) return;
  }
}

}  // namespace

size_t lp_solve_bytes(int NP, int nrhs) {
  const size_t nb = (size_t)(NP + BS - 1) / BS;
  return nb * BS * BS * 8          // Dinv
         + nb * BS * (BS / 2) * 8  // merge scratch T
         + (size_t)BS * nrhs * 8   // X block
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
  s.Dinv = (double *)take((size_t)s.nblk * BS * BS * 8);
  s.T = (double *)take((size_t)s.nblk * BS * (BS / 2) * 8);
  s.Xb = (double *)take((size_t)BS * nrhs * 8);
  s.bar = (unsigned *)take(256);
  return MO_OK;
}

int lp_solve_prepare(mo_ctx *ctx, const LpChol &f, LpSolve &s) {
  cudaStream_t st = ctx->stream;
  const int NP = f.NP;
  s.W = f.W;
  s.ldw = f.ldw;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_OTHER);
  MO_CUDA_TRY(cudaMemsetAsync(s.Dinv, 0, (size_t)s.nblk * BS * BS * 8, st));
  place_inv128_kernel<<<NP / 128, 256, 0, st>>>(f.inv, s.Dinv, NP);
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

// D (n x nr, ld ldd) <- L^-1 D (trans == false) or L^-T D (trans == true): one cooperative
// launch over the whole device
int lp_solve_apply(mo_ctx *ctx, const LpSolve &s, int n, double *D, int64_t ldd, int nr,
                   bool trans, const int *skip) {
  if (nr > s.nrhs || nr > 64 || n > s.NP) return MO_EINVAL;
  if (n == 0 || nr == 0) return MO_OK;
  const size_t smem = (size_t)(MTMAX * KCH * LDA_S + KCH * (nr + 1)) * sizeof(double);
  if (int rc = mo_smem_attr((const void *)blk_solve_kernel, (int)smem)) return rc;
  int occ = 0;
  MO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, blk_solve_kernel, ST, smem));
  if (occ < 1) return MO_ENOKERNEL;
  const int grid = ctx->sms;  // one CTA per SM: every CTA is resident, as the barriers need
  SolveArgs a;
  a.W = s.W;
  a.ldw = s.ldw;
  a.Dinv = s.Dinv;
  a.D = D;
  a.ldd = ldd;
  a.Xb = s.Xb;
  a.n = n;
  a.nr = nr;
  a.nblk = (n + BS - 1) / BS;
  a.trans = trans ? 1 : 0;
  a.bar = s.bar;
  a.status = &control(ctx)->status;
  a.spin = ctx->spin_limit;
  a.skip = skip;
  MO_CUDA_TRY(cudaMemsetAsync(s.bar, 0, 2 * sizeof(unsigned), ctx->stream));
  void *args[] = {&a};
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_IR);
  MO_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)blk_solve_kernel, dim3(grid), dim3(ST),
                                          args, smem, ctx->stream));
  prof_end(ctx, ps, (double)n * n * nr, 4.0 * (double)n * n / 2 + 8.0 * (double)a.nblk * BS * BS +
                                            16.0 * n * nr);
  return MO_OK;
}

}  // namespace mo
