// Triangular solve with few right-hand sides (<= 64) in one cooperative launch.
//
// op(A) X = alpha*B with op(A) n x n triangular, split into 64-row blocks.  CTA c owns the
// blocks of steps c, c+P, ... (steps run top-down for a lower op(A), bottom-up for upper).
// For each owned step s it keeps its block of B in DMMA accumulator fragments, subtracts
// op(A)[s, s'] X_s' for every earlier step s' as soon as that step's flag is published,
// multiplies by the inverse of the diagonal block and publishes X_s (written over B) with
// its flag.  The critical path is one 64 x 64 x nrhs update plus one 64 x 64 x nrhs product
// per step on the FP64 tensor pipe (mma.sync m16n8k4); the next block of op(A) is prefetched
// with cp.async while the CTA waits.  Blocks of op(A) are staged with coalesced reads (also
// for op(A) = A^T).  Every wait is bounded and reports MO_EDEVTIMEOUT.
//
// B is addressed with a row and a column stride, so a right-side solve with few rows,
// X op(A) = alpha*B, runs as op(A)^T X^T = alpha*B^T on the transposed view.
#include <algorithm>

#include "context.cuh"

namespace mo {
int trtri_blocks(mo_ctx *ctx, View A, int N, bool trans, bool lower_eff, bool unit, double *inv);

namespace {

constexpr int TB = 64;    // block order of the sweep
constexpr int IB = 128;   // order of the precomputed inverse blocks (trtri_blocks)
constexpr int FEW_THREADS = 128;  // 4 warps x 16 rows
constexpr int MAX_RHS = 64;
constexpr int LDL = TB + 4;   // smem row stride (== 4 mod 16 doubles: 2-way at most)
constexpr int LDX = MAX_RHS + 4;
constexpr int FEW_SMEM = (3 * TB * LDL + TB * LDX) * 8;  // inverse, 2 x op(A) block, X

struct FewArgs {
  const void *A;  // double, or float for the mixed-precision factor (FP64 arithmetic)
  int64_t lda;
  bool trans;      // op(A) = A^T
  bool lower_eff;  // op(A) lower -> steps top-down
  int N, nblk;
  double *B;
  int64_t brs, bcs;  // element (i, c) of B at B[i*brs + c*bcs]
  int nrhs;
  double alpha;
  const double *inv;  // 128 x 128 inverses of op(A)'s diagonal blocks (ld 128)
  bool inv_t;         // inv holds the inverses of A's blocks: read them transposed
  int *flags;         // [nblk]
  int epoch;
  int *status;
};

__device__ __forceinline__ int step_block(const FewArgs &p, int s) {
  return p.lower_eff ? s : p.nblk - 1 - s;
}

__device__ __forceinline__ void cp_async_join() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

__device__ __forceinline__ void cp_async_el(double *dst, const double *src, uint32_t n) {
  cp_async_8(dst, src, n ? 8u : 0u);
}
__device__ __forceinline__ void cp_async_el(float *dst, const float *src, uint32_t n) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(n ? 4u : 0u)
               : "memory");
}

// issue cp.async copies of op(A)[rb*64 .., cb*64 ..] into L (row-major, ld LDL); zero past N
template <typename TA>
__device__ __forceinline__ void stage_block(const FewArgs &p, TA *L, int rb, int cb) {
  const int r0 = rb * TB, c0 = cb * TB;
  const TA *A = static_cast<const TA *>(p.A);
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
    const int i = e % TB, j = e / TB;  // consecutive threads -> consecutive A addresses
    if (!p.trans) {
      const bool ok = r0 + i < p.N && c0 + j < p.N;
      cp_async_el(L + i * LDL + j, ok ? A + (r0 + i) + (int64_t)(c0 + j) * p.lda : A, ok);
    } else {
      const bool ok = c0 + i < p.N && r0 + j < p.N;
      cp_async_el(L + j * LDL + i, ok ? A + (c0 + i) + (int64_t)(r0 + j) * p.lda : A, ok);
    }
  }
}

// issue cp.async copies of the inverse of diagonal block rb (64 x 64 sub-block of a 128
// inverse) into I (row-major, ld LDL), zero past the block's order
__device__ __forceinline__ void stage_inverse(const FewArgs &p, double *I, int rb) {
  const int nbh = min(TB, p.N - rb * TB);
  const double *iv = p.inv + (size_t)(rb / 2) * IB * IB + (rb % 2) * TB * (IB + 1);
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
    const int i = e % TB, j = e / TB;  // column-major source, ld 128
    const bool ok = i < nbh && j < nbh;
    const double *src = p.inv_t ? iv + j + i * IB : iv + i + j * IB;
    cp_async_8(I + i * LDL + j, ok ? src : iv, ok ? 8u : 0u);
  }
}

// acc[nt] (+)= sign * M(16 rows of this warp, 64) * X(64, 8 nt ..)
template <int NT, typename TM>
__device__ __forceinline__ void block_mma(double (&acc)[NT][4], const TM *M, const double *X,
                                          double sign) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const TM *m0 = M + (16 * warp + g) * LDL + t;
  const TM *m1 = m0 + 8 * LDL;
  const double *xb = X + t * LDX + g;
#pragma unroll 4
  for (int k = 0; k < TB; k += 4) {
    const double a0 = sign * (double)m0[k], a1 = sign * (double)m1[k];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) dmma_16x8x4(acc[nt], a0, a1, xb[k * LDX + 8 * nt]);
  }
}

template <typename TA, int NT>
__global__ void __launch_bounds__(FEW_THREADS, 1) trsm_few_kernel(FewArgs p) {
  extern __shared__ double sm[];
  double *I = sm;                                       // inverse of the owned diagonal block
  TA *Lb0 = reinterpret_cast<TA *>(sm + TB * LDL);      // op(A) blocks, double-buffered
  TA *Lb1 = reinterpret_cast<TA *>(sm + 2 * TB * LDL);
  double *Xs = sm + 3 * TB * LDL;    // X of a step (row-major, ld LDX)
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  if (threadIdx.x == 0) s_abort = 0;
  __syncthreads();
  for (int s = blockIdx.x; s < p.nblk; s += gridDim.x) {
    const int pb = step_block(p, s);
    stage_inverse(p, I, pb);
    if (s > 0) stage_block(p, Lb0, pb, step_block(p, 0));
    // B block in accumulator layout: rows 16w+g (+8), columns 8nt+2t (+1)
    double acc[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = pb * TB + 16 * warp + g + 8 * (q >> 1);
        const int col = 8 * nt + 2 * t + (q & 1);
        acc[nt][q] = (row < p.N && col < p.nrhs) ? p.alpha * p.B[row * p.brs + col * p.bcs] : 0.0;
      }
    for (int s2 = 0; s2 < s; ++s2) {
      const int qb = step_block(p, s2);
      cp_async_join();  // op(A) block of s2 (and, the first time, the inverse) have landed
      __syncthreads();  // ... for every thread; the other buffer is free again
      if (s2 + 1 < s) stage_block(p, (s2 & 1) ? Lb0 : Lb1, pb, step_block(p, s2 + 1));
      if (threadIdx.x == 0) {
        uint32_t it = 0;
        while (atomicAdd(&p.flags[s2], 0) != p.epoch) {
          if (++it > MO_SPIN_LIMIT) {
            set_status(p.status, MO_EDEVTIMEOUT);
            s_abort = 1;
            break;
          }
        }
        __threadfence();
      }
      __syncthreads();
      if (s_abort) {
        cp_async_join();
        return;
      }
      // X of step s2 (written by another CTA): L2 reads, 16 in flight per thread
      for (int e0 = threadIdx.x; e0 < TB * 8 * NT; e0 += 16 * FEW_THREADS) {
        double v[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int e = e0 + u * FEW_THREADS;
          const int k = e / (8 * NT), c = e % (8 * NT);
          const int xr = qb * TB + k;
          v[u] = (e < TB * 8 * NT && xr < p.N && c < p.nrhs)
                     ? __ldcg(p.B + xr * p.brs + c * p.bcs) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int e = e0 + u * FEW_THREADS;
          if (e < TB * 8 * NT) Xs[(e / (8 * NT)) * LDX + e % (8 * NT)] = v[u];
        }
      }
      __syncthreads();
      block_mma<NT>(acc, (s2 & 1) ? Lb1 : Lb0, Xs, -1.0);
      __syncthreads();
    }
    // X_s = inv(op(A)_ss) * acc
    cp_async_join();
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q)
        Xs[(16 * warp + g + 8 * (q >> 1)) * LDX + 8 * nt + 2 * t + (q & 1)] = acc[nt][q];
    __syncthreads();
    double x[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) x[nt][q] = 0.0;
    block_mma<NT>(x, I, Xs, 1.0);
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = pb * TB + 16 * warp + g + 8 * (q >> 1);
        const int col = 8 * nt + 2 * t + (q & 1);
        if (row < p.N && col < p.nrhs) p.B[row * p.brs + col * p.bcs] = x[nt][q];
      }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicExch(&p.flags[s], p.epoch);
  }
}

template <typename TA, int NT>
int launch_few(mo_ctx *ctx, FewArgs &p) {
  static int attr_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  const void *kern = (const void *)trsm_few_kernel<TA, NT>;
  if (!(attr_mask & (1 << (dev & 31)))) {
    MO_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, FEW_SMEM));
    attr_mask |= 1 << (dev & 31);
  }
  int occ = 0;
  MO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, FEW_THREADS, FEW_SMEM));
  if (occ < 1) return MO_EINVAL;
  const int grid = std::min(p.nblk, occ * ctx->sms);
  void *args[] = {&p};
  MO_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(FEW_THREADS), args, FEW_SMEM,
                                          ctx->stream));
  return MO_OK;
}

}  // namespace

namespace {

// flags -> (B strides, effective transposition and sweep direction) and the launch
int few_run(mo_ctx *ctx, View B, const void *A, bool a32, int64_t lda, int N, int flags,
            double alpha, const double *inv, bool inv_t, int *flag_buf) {
  const bool right = (flags & MO_RIGHT) != 0;
  const bool upper = (flags & MO_UPPER) != 0;
  bool tr = (flags & MO_TRANSA) != 0;
  bool lower_eff = upper ? tr : !tr;
  const int nrhs = right ? B.rows : B.cols;
  if (nrhs > MAX_RHS || N <= 0 || nrhs <= 0) return MO_EINVAL;
  FewArgs p;
  if (!right) {
    p.brs = 1;
    p.bcs = B.ld;
  } else {
    // X op(A) = alpha B  <=>  op(A)^T X^T = alpha B^T
    p.brs = B.ld;
    p.bcs = 1;
    tr = !tr;
    lower_eff = !lower_eff;
  }
  p.A = A;
  p.lda = lda;
  p.trans = tr;
  p.lower_eff = lower_eff;
  p.N = N;
  p.nblk = (N + TB - 1) / TB;
  p.B = B.d;
  p.nrhs = nrhs;
  p.alpha = alpha;
  p.inv = inv;
  p.inv_t = inv_t;
  p.flags = flag_buf;
  p.epoch = ++ctx->sk_epoch;
  p.status = reinterpret_cast<int *>(ctx->d_status);
  MO_CUDA_TRY(cudaMemsetAsync(flag_buf, 0, sizeof(int) * p.nblk, ctx->stream));
  ProfScope ps;
  prof_begin(ctx, ps, a32 ? MO_PROF_IR : MO_PROF_GEMM);
  const int nt = (nrhs + 7) / 8;
  int rc;
  if (a32) {
    if (nt <= 2) rc = launch_few<float, 2>(ctx, p);
    else if (nt <= 4) rc = launch_few<float, 4>(ctx, p);
    else rc = launch_few<float, 8>(ctx, p);
  } else {
    if (nt <= 2) rc = launch_few<double, 2>(ctx, p);
    else if (nt <= 4) rc = launch_few<double, 4>(ctx, p);
    else rc = launch_few<double, 8>(ctx, p);
  }
  prof_end(ctx, ps, (double)N * N * nrhs,
           (a32 ? 4.0 : 8.0) * (double)N * N / 2 + 8.0 * 2.0 * N * nrhs);
  return rc;
}

}  // namespace

// Left solve (right solves via the transposed view of B) with nrhs <= 64.  `inv` receives
// the 128 x 128 diagonal-block inverses; `flag_buf` holds one int per 64-row block.
int trsm_few(mo_ctx *ctx, View B, View A, int flags, double alpha, double *inv, int *flag_buf) {
  const bool right = (flags & MO_RIGHT) != 0;
  const bool upper = (flags & MO_UPPER) != 0;
  bool tr = (flags & MO_TRANSA) != 0;
  const bool unit = (flags & MO_UNIT) != 0;
  bool lower_eff = upper ? tr : !tr;
  if (right) {
    tr = !tr;
    lower_eff = !lower_eff;
  }
  const int N = A.cols;
  const int nrhs = right ? B.rows : B.cols;
  if (nrhs > MAX_RHS || N <= 0 || nrhs <= 0) return MO_EINVAL;
  int rc = trtri_blocks(ctx, A, N, tr, lower_eff, unit, inv);
  if (rc) return rc;
  return few_run(ctx, B, A.d, false, A.ld, N, flags, alpha, inv, false, flag_buf);
}

// Left solve with an FP32 lower-triangular L (order N, ld) in FP64 arithmetic, using the
// FP64 inverses of L's 128 x 128 diagonal blocks (ld 128): op(L) X = B in place, op = L
// (trans == false) or L^T.
int trsm_few_f32(mo_ctx *ctx, View B, const float *L, int64_t ldl, int N, bool trans,
                 const double *inv_L, int *flag_buf) {
  const int flags = MO_LOWER | (trans ? MO_TRANSA : 0);
  return few_run(ctx, B, L, true, ldl, N, flags, 1.0, inv_L, trans, flag_buf);
}

}  // namespace mo
