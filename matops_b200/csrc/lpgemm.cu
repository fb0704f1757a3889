// Split-product GEMM on the tensor cores (BF16x3 / TF32x3, FP32 accumulation) for the
// mixed-precision Cholesky; see lp.cuh for the number format.
//
// Tile 128 x 128, 256 threads (8 warps as 2 x 4, warp tile 64 x 32).  A stage holds 64
// bytes of K per row (32 bf16 or 16 tf32 elements) for the four parts A.hi, A.lo, B.hi,
// B.lo, loaded with 16-byte cp.async into a 4-deep ring; fragments come from ldmatrix
// (a 16-byte chunk of row r is stored at chunk c ^ ((r >> 1) & 3), so the 8 rows of an
// ldmatrix phase fall in distinct banks).  One k-step is 32 bytes of K: m16n8k16 for bf16,
// m16n8k8 for tf32 -- both read A as (rows 0-7 | 8-15) x (bytes 0-15 | 16-31) and B as
// rows 0-7 x (bytes 0-15 | 16-31), so one ldmatrix addressing serves both.  Each
// product issues lo*hi, hi*lo, hi*hi into one FP32 accumulator.  CTAs are persistent;
// the slab stream runs across tile boundaries, so the next tile's loads are in flight
// during a tile's epilogue.
#include <cuda_bf16.h>

#include <algorithm>

#include "lp.cuh"

namespace mo {
namespace {

constexpr int LBM = 128, LBN = 128;
constexpr int LTHREADS = 256;
constexpr int LSTAGES = 4;
constexpr int LROWB = 64;                  // bytes of K per row per stage
constexpr int LPART = LBM * LROWB;         // 8 KB
constexpr int LSTAGE = 4 * LPART;          // A.hi, A.lo, B.hi, B.lo
constexpr int LSMEM = LSTAGES * LSTAGE;    // 128 KB

struct LpParams {
  int M, N, K;
  float alpha, beta;
  const char *a_hi, *a_lo, *b_hi, *b_lo;
  int64_t a_ldb, b_ldb;  // bytes between rows
  float *C;
  int64_t ldc;
  int mode;
  int mt, nt;     // tiles per dimension
  int ntiles;     // tiles in the schedule
  int kslabs;     // K / (elements per 64 bytes)
};

__device__ __forceinline__ uint32_t swz(int r, int c) {
  return (uint32_t)(r * LROWB + ((c ^ ((r >> 1) & 3)) << 4));
}

__device__ __forceinline__ void cp_async_16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2,
                                        uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

template <int PREC>
__device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                    uint32_t b1) {
  if (PREC == kLpBf16x3)
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
  else
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// tile index -> (tm, tn); lower mode enumerates tiles with tm >= tn column by column
__device__ __forceinline__ void tile_coords(const LpParams &p, int t, int &tm, int &tn) {
  if (p.mode == kGemmLower) {
    int c = 0;
    while (t >= p.mt - c) {
      t -= p.mt - c;
      ++c;
    }
    tn = c;
    tm = c + t;
  } else {
    tm = t % p.mt;
    tn = t / p.mt;
  }
}

// issue the cp.async copies of slab `s` of tile (tm, tn) into stage buffer `st`
__device__ __forceinline__ void load_slab(const LpParams &p, uint32_t st, int tm, int tn, int s) {
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int idx = threadIdx.x + i * LTHREADS;
    const int part = idx >> 9, rem = idx & 511;
    const int r = rem >> 2, c = rem & 3;
    const char *base;
    int64_t ldb;
    int row;
    if (part < 2) {
      base = part == 0 ? p.a_hi : p.a_lo;
      ldb = p.a_ldb;
      row = tm * LBM + r;
    } else {
      base = part == 2 ? p.b_hi : p.b_lo;
      ldb = p.b_ldb;
      row = tn * LBN + r;
    }
    cp_async_16(st + part * LPART + swz(r, c), base + row * ldb + s * LROWB + c * 16);
  }
}

template <int PREC>
__global__ void __launch_bounds__(LTHREADS, 1) lp_gemm_kernel(LpParams p) {
  extern __shared__ __align__(128) char lsm[];
  const uint32_t sbase = smem_u32(lsm);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp & 1, wn = warp >> 1;
  const int g = lane >> 2, t4 = lane & 3;
  const int mine = (p.ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  if (mine <= 0) return;
  const int G = mine * p.kslabs;
  auto slab_tile = [&](int gi, int &tm, int &tn, int &s) {
    const int ti = gi / p.kslabs;
    s = gi - ti * p.kslabs;
    tile_coords(p, (int)blockIdx.x + ti * (int)gridDim.x, tm, tn);
  };
#pragma unroll
  for (int gi = 0; gi < LSTAGES - 1; ++gi) {
    if (gi < G) {
      int tm, tn, s;
      slab_tile(gi, tm, tn, s);
      load_slab(p, sbase + gi * LSTAGE, tm, tn, s);
    }
    cp_commit();
  }
  // ldmatrix row/chunk of this lane for the A (x4: rows +8 by q&1, chunk by q>>1) and
  // B (x4: rows +8 by q>>1, chunk by q&1) fragment loads
  const int q = lane >> 3, rr = lane & 7;
  const int a_row = wm * 64 + rr + 8 * (q & 1), a_ch = q >> 1;
  const int b_row = wn * 32 + rr + 8 * (q >> 1), b_ch = q & 1;
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

  for (int gi = 0; gi < G; ++gi) {
    cp_wait<LSTAGES - 2>();
    __syncthreads();
    if (gi + LSTAGES - 1 < G) {
      int tm, tn, s;
      slab_tile(gi + LSTAGES - 1, tm, tn, s);
      load_slab(p, sbase + ((gi + LSTAGES - 1) % LSTAGES) * LSTAGE, tm, tn, s);
    }
    cp_commit();
    const uint32_t st = sbase + (gi % LSTAGES) * LSTAGE;
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      uint32_t ah[4][4], al[4][4], bh[4][2], bl[4][2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const uint32_t off = swz(a_row + 16 * mt, 2 * ks + a_ch);
        ldsm_x4(st + off, ah[mt][0], ah[mt][1], ah[mt][2], ah[mt][3]);
        ldsm_x4(st + LPART + off, al[mt][0], al[mt][1], al[mt][2], al[mt][3]);
      }
#pragma unroll
      for (int np = 0; np < 2; ++np) {
        const uint32_t off = swz(b_row + 16 * np, 2 * ks + b_ch);
        ldsm_x4(st + 2 * LPART + off, bh[2 * np][0], bh[2 * np][1], bh[2 * np + 1][0],
                bh[2 * np + 1][1]);
        ldsm_x4(st + 3 * LPART + off, bl[2 * np][0], bl[2 * np][1], bl[2 * np + 1][0],
                bl[2 * np + 1][1]);
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          mma<PREC>(acc[mt][nt], al[mt], bh[nt][0], bh[nt][1]);
          mma<PREC>(acc[mt][nt], ah[mt], bl[nt][0], bl[nt][1]);
          mma<PREC>(acc[mt][nt], ah[mt], bh[nt][0], bh[nt][1]);
        }
    }
    if ((gi + 1) % p.kslabs == 0) {
      // epilogue of this tile: C = beta*C + alpha*acc (column-major), lower mask
      int tm, tn, s;
      slab_tile(gi, tm, tn, s);
      const int i0 = tm * LBM + wm * 64 + g, j0 = tn * LBN + wn * 32 + 2 * t4;
      const bool lower = p.mode == kGemmLower;
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        float cv[4][4];
        if (p.beta != 0.f) {
#pragma unroll
          for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int i = i0 + 16 * mt + 8 * (e >> 1), j = j0 + 8 * nt + (e & 1);
              cv[nt][e] = ((!lower || i >= j) && i < p.M && j < p.N) ? p.C[i + (int64_t)j * p.ldc]
                                                                      : 0.f;
            }
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int i = i0 + 16 * mt + 8 * (e >> 1), j = j0 + 8 * nt + (e & 1);
            float v = p.alpha * acc[mt][nt][e];
            if (p.beta != 0.f) v = fmaf(p.beta, cv[nt][e], v);
            if ((!lower || i >= j) && i < p.M && j < p.N) p.C[i + (int64_t)j * p.ldc] = v;
            acc[mt][nt][e] = 0.f;
          }
      }
    }
  }
  cp_wait<0>();
}

// ---------------------------------------------------------------------------------------
// split: X (FP32 column-major) -> K-major hi/lo.  A CTA takes 64 rows x 32 columns,
// stages them transposed in shared memory and writes 8 consecutive k per thread and part.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// by_col: out row r = column r of X (X is cols x rows, column-major): no transpose
template <int PREC>
__global__ void __launch_bounds__(256) lp_split_cols_kernel(const float *X, int64_t ld, int rows,
                                                            int cols, char *hi, char *lo,
                                                            int64_t ldk) {
  const int r = blockIdx.x, k = blockIdx.y * 256 + threadIdx.x;
  if (r >= rows || k >= cols) return;
  const float x = X[k + (int64_t)r * ld];
  const int64_t e = (int64_t)r * ldk + k;
  if (PREC == kLpBf16x3) {
    __nv_bfloat16 h, l;
    split_bf16(x, h, l);
    reinterpret_cast<__nv_bfloat16 *>(hi)[e] = h;
    reinterpret_cast<__nv_bfloat16 *>(lo)[e] = l;
  } else {
    const uint32_t h = to_tf32(x);
    reinterpret_cast<uint32_t *>(hi)[e] = h;
    reinterpret_cast<uint32_t *>(lo)[e] = to_tf32(x - __uint_as_float(h));
  }
}

template <int PREC>
__global__ void __launch_bounds__(256) lp_split_kernel(const float *X, int64_t ld, int rows,
                                                       int cols, char *hi, char *lo,
                                                       int64_t ldk) {
  __shared__ float T[32][65];
  const int r0 = blockIdx.x * 64, c0 = blockIdx.y * 32;
  for (int e = threadIdx.x; e < 64 * 32; e += 256) {
    const int r = e & 63, c = e >> 6;
    T[c][r] = (r0 + r < rows && c0 + c < cols) ? X[(r0 + r) + (int64_t)(c0 + c) * ld] : 0.f;
  }
  __syncthreads();
  const int r = threadIdx.x >> 2, kq = (threadIdx.x & 3) * 8;
  if (r0 + r >= rows || c0 + kq >= cols) return;
  constexpr int ES = PREC == kLpBf16x3 ? 2 : 4;
  const int64_t off = ((int64_t)(r0 + r) * ldk + c0 + kq) * ES;
  if (PREC == kLpBf16x3) {
    __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) split_bf16(T[kq + u][r], h[u], l[u]);
    *reinterpret_cast<uint4 *>(hi + off) = *reinterpret_cast<const uint4 *>(h);
    *reinterpret_cast<uint4 *>(lo + off) = *reinterpret_cast<const uint4 *>(l);
  } else {
    __align__(16) uint32_t h[8], l[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const float x = T[kq + u][r];
      h[u] = to_tf32(x);
      l[u] = to_tf32(x - __uint_as_float(h[u]));
    }
    *reinterpret_cast<uint4 *>(hi + off) = *reinterpret_cast<const uint4 *>(h);
    *reinterpret_cast<uint4 *>(hi + off + 16) = *reinterpret_cast<const uint4 *>(h + 4);
    *reinterpret_cast<uint4 *>(lo + off) = *reinterpret_cast<const uint4 *>(l);
    *reinterpret_cast<uint4 *>(lo + off + 16) = *reinterpret_cast<const uint4 *>(l + 4);
  }
}

template <int PREC>
int launch_lp(mo_ctx *ctx, LpParams &p, int grid) {
  static int attr_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(attr_mask & (1 << (dev & 31)))) {
    MO_CUDA_TRY(cudaFuncSetAttribute(lp_gemm_kernel<PREC>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, LSMEM));
    attr_mask |= 1 << (dev & 31);
  }
  lp_gemm_kernel<PREC><<<grid, LTHREADS, LSMEM, ctx->stream>>>(p);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

}  // namespace

int lp_gemm(mo_ctx *ctx, int prec, const LpGemmArgs &a) {
  if (a.M <= 0 || a.N <= 0 || a.K <= 0) return MO_OK;
  // the split operands must hold roundup(M or N, 128) rows and K % 32 == 0 columns
  // (zeros past the true extents); C is written only inside M x N
  if (a.K % 32) return MO_EINVAL;
  if (prec != kLpBf16x3 && prec != kLpTf32x3) return MO_EINVAL;
  const int es = lp_esize(prec);
  LpParams p;
  p.M = a.M;
  p.N = a.N;
  p.K = a.K;
  p.alpha = a.alpha;
  p.beta = a.beta;
  p.a_hi = (const char *)a.A.hi;
  p.a_lo = (const char *)a.A.lo;
  p.b_hi = (const char *)a.B.hi;
  p.b_lo = (const char *)a.B.lo;
  p.a_ldb = a.A.ldk * es;
  p.b_ldb = a.B.ldk * es;
  p.C = a.C;
  p.ldc = a.ldc;
  p.mode = a.mode == kGemmLower ? kGemmLower : kGemm;
  p.mt = (a.M + LBM - 1) / LBM;
  p.nt = (a.N + LBN - 1) / LBN;
  if (p.mode == kGemmLower && p.nt > p.mt) return MO_EINVAL;
  p.ntiles = p.mode == kGemmLower ? p.nt * p.mt - p.nt * (p.nt - 1) / 2 : p.mt * p.nt;
  p.kslabs = a.K * es / LROWB;
  int grid = std::min(p.ntiles, ctx->sms);
  if (a.max_ctas > 0) grid = std::min(grid, a.max_ctas);
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_LPGEMM);
  const int rc = prec == kLpBf16x3 ? launch_lp<kLpBf16x3>(ctx, p, grid)
                                   : launch_lp<kLpTf32x3>(ctx, p, grid);
  const double tiles_flops = (double)p.ntiles * LBM * LBN * a.K * 2.0;
  prof_end(ctx, ps, tiles_flops,
           (double)p.ntiles * LBM * LBN * 4.0 * (a.beta != 0.f ? 2.0 : 1.0) +
               (double)(a.M + a.N) * a.K * es * 2.0);
  return rc;
}

int lp_split(mo_ctx *ctx, int prec, const float *X, int64_t ld, int rows, int cols,
             LpSplit out) {
  if (rows <= 0 || cols <= 0) return MO_OK;
  // groups of 8 columns: a partial last group writes zeros up to the next multiple of 8
  if (out.ldk % 8 || out.ldk < ((cols + 7) & ~7)) return MO_EINVAL;
  const dim3 grid((rows + 63) / 64, (cols + 31) / 32);
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_LPGEMM);
  if (prec == kLpBf16x3)
    lp_split_kernel<kLpBf16x3><<<grid, 256, 0, ctx->stream>>>(X, ld, rows, cols, (char *)out.hi,
                                                               (char *)out.lo, out.ldk);
  else
    lp_split_kernel<kLpTf32x3><<<grid, 256, 0, ctx->stream>>>(X, ld, rows, cols, (char *)out.hi,
                                                               (char *)out.lo, out.ldk);
  prof_end(ctx, ps, 0.0, (double)rows * cols * (4.0 + 2.0 * lp_esize(prec)));
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

int lp_split_cols(mo_ctx *ctx, int prec, const float *X, int64_t ld, int rows, int cols,
                  LpSplit out) {
  if (rows <= 0 || cols <= 0) return MO_OK;
  const dim3 grid(rows, (cols + 255) / 256);
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_LPGEMM);
  if (prec == kLpBf16x3)
    lp_split_cols_kernel<kLpBf16x3><<<grid, 256, 0, ctx->stream>>>(X, ld, rows, cols,
                                                                    (char *)out.hi,
                                                                    (char *)out.lo, out.ldk);
  else
    lp_split_cols_kernel<kLpTf32x3><<<grid, 256, 0, ctx->stream>>>(X, ld, rows, cols,
                                                                    (char *)out.hi,
                                                                    (char *)out.lo, out.ldk);
  prof_end(ctx, ps, 0.0, (double)rows * cols * (4.0 + 2.0 * lp_esize(prec)));
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

}  // namespace mo

// C = alpha*op(A)*op(B) + beta*C in FP32 storage with split-product tensor-core
// arithmetic; the operands are split into the context's mixed-precision workspace
extern "C" int mo_lp_gemm(mo_ctx *ctx, int prec, int64_t M, int64_t N, int64_t K, float alpha,
                          const float *A, int64_t lda, const float *B, int64_t ldb, float beta,
                          float *C, int64_t ldc, int flags) {
  using namespace mo;
  int rc = enter(ctx);
  if (rc) return rc;
  if (M < 0 || N < 0 || K < 0 || M > (1 << 30) || N > (1 << 30) || K > (1 << 30))
    return MO_EINVAL;
  if (prec != MO_PREC_BF16X3 && prec != MO_PREC_TF32X3) return MO_EINVAL;
  const bool ta = flags & MO_TRANSA, tb = flags & MO_TRANSB;
  if (M == 0 || N == 0) return MO_OK;
  if (!A || !B || !C || ldc < M || lda < (ta ? K : M) || ldb < (tb ? N : K)) return MO_EINVAL;
  if ((flags & MO_LOWER) && N > M) return MO_EINVAL;
  const int lp = prec == MO_PREC_BF16X3 ? kLpBf16x3 : kLpTf32x3;
  const int es = lp_esize(lp);
  const int64_t Mp = (M + 127) / 128 * 128, Np = (N + 127) / 128 * 128, Kp = (K + 31) / 32 * 32;
  const size_t abytes = (size_t)Mp * Kp * es, bbytes = (size_t)Np * Kp * es;
  const size_t need = 2 * (abytes + bbytes) + 1024;
  if (need > ctx->ws_ir_bytes) {
    MO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (ctx->ws_ir) cudaFree(ctx->ws_ir);
    ctx->ws_ir = nullptr;
    ctx->ws_ir_bytes = 0;
    MO_CUDA_TRY(cudaMalloc(&ctx->ws_ir, need));
    ctx->ws_ir_bytes = need;
  }
  char *p = (char *)ctx->ws_ir;
  LpSplit sa{p, p + abytes, Kp}, sb{p + 2 * abytes, p + 2 * abytes + bbytes, Kp};
  MO_CUDA_TRY(cudaMemsetAsync(p, 0, 2 * (abytes + bbytes), ctx->stream));
  if (K > 0) {
    // A operand rows m: op(A)(m, :)  -- column m of A when transposed
    rc = ta ? lp_split_cols(ctx, lp, A, lda, (int)M, (int)K, sa)
            : lp_split(ctx, lp, A, lda, (int)M, (int)K, sa);
    if (rc) return rc;
    // B operand rows n: op(B)(:, n)  -- row n of B when transposed
    rc = tb ? lp_split(ctx, lp, B, ldb, (int)N, (int)K, sb)
            : lp_split_cols(ctx, lp, B, ldb, (int)N, (int)K, sb);
    if (rc) return rc;
  }
  LpGemmArgs g;
  g.M = (int)M;
  g.N = (int)N;
  g.K = (int)Kp;
  g.alpha = alpha;
  g.beta = beta;
  g.A = sa;
  g.B = sb;
  g.C = C;
  g.ldc = ldc;
  g.mode = (flags & MO_LOWER) ? kGemmLower : kGemm;
  return lp_gemm(ctx, lp, g);
}
