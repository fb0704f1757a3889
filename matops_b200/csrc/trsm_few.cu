// Triangular solve with few right-hand sides (<= 64) in one cooperative launch.
//
// op(A) X = alpha*B with op(A) n x n triangular, split into 64-row blocks.  The columns of
// B are cut into groups of at most MO_FEW_GROUP (32), each solved by its own set of CTAs
// with its own step flags, so the work on the dependency chain per step is that of one
// group.  Within a set, CTA c owns the blocks of steps c, c+P, ... (top-down for a lower
// op(A), bottom-up for upper).  For each owned step s it keeps its block of B in DMMA
// accumulator fragments and subtracts op(A)[s, s'] X_s' for the earlier steps s' in
// rounds: it waits for the oldest missing step's flag, takes every consecutive published
// step up to a chunk of 1-3 blocks (as deep as shared memory allows), and applies them as
// one K = 64 x chunk product while the next chunk of op(A) streams in by cp.async (and,
// once every earlier step is known published, the next chunk's X rows stream into
// registers).  Then X_s = inv(op(A)_ss) (B_s - ...) is published (written over B) with
// its flag.  The critical path per step is one 64 x 64 x group update plus one
// 64 x 64 x group product on the FP64 tensor pipe (mma.sync m16n8k4).  Blocks of op(A)
// are staged with coalesced reads (also for op(A) = A^T).  Every wait is bounded and
// reports MO_EDEVTIMEOUT.
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
#ifndef MO_FEW_GROUP
#define MO_FEW_GROUP 32  // columns per group (measured: 32 beats 16 and 64 at n = 16384, 64 RHS)
#endif
#ifndef MO_PAIR_GROUP
#define MO_PAIR_GROUP 32  // columns per group of the paired-step kernel (measured: 32 beats 64)
#endif
constexpr int LDL = TB + 4;   // smem row stride (== 4 mod 16 doubles: 2-way at most)

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
  int groups;         // independent column groups of B (gw columns each), one per CTA set
  int gw;
  const double *inv;  // 128 x 128 inverses of op(A)'s diagonal blocks (ld 128)
  bool inv_t;         // inv holds the inverses of A's blocks: read them transposed
  bool vec;           // A's base and leading dimension allow 16-byte copies
  int *flags;         // [groups * nblk]
  int epoch;
  int *status;
  uint32_t spin_limit;  // polls of a step flag before the wait gives up (MO_EDEVTIMEOUT)
  const int *skip;      // optional: when the word is set at launch the grid returns at once
};

// step flags sit one per 128-byte line, and pollers read them with acquire loads (not
// atomics), so polling CTAs do not queue at the L2 ahead of the publishing store
constexpr int FLAG_STRIDE = 32;
__device__ __forceinline__ int flag_load(const int *f) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(f) : "memory");
  return v;
}

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

// Blocks of op(A) sit in the chunk buffer in the orientation of their source, so that
// 16-byte copies fill them: for op(A) = A (column-major A, contiguous along op(A)'s rows)
// block element (i, k) is at [k * ldb + i]; for op(A) = A^T at [i * ldb + k].  ldb keeps
// the DMMA fragment reads free of bank conflicts (few_block_ld).
template <typename TA>
__host__ __device__ constexpr int few_block_ld(bool trans) {
  return sizeof(TA) == 4 ? (trans ? 68 : 72) : 68;
}

__device__ __forceinline__ void cp_async_16(void *dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(bytes)
               : "memory");
}

// issue cp.async copies of `cnt` blocks of op(A) -- block row rb, the block columns of
// steps s0 .. s0 + cnt - 1 -- into the chunk buffer L (block j at j * 64 * ldb); zero past N
template <typename TA>
__device__ __forceinline__ void stage_chunk(const FewArgs &p, TA *L, int rb, int s0, int cnt) {
  constexpr int V = 16 / sizeof(TA);  // elements per 16-byte copy
  const int ldb = few_block_ld<TA>(p.trans);
  const int r0 = rb * TB;
  const TA *A = static_cast<const TA *>(p.A);
  for (int j = 0; j < cnt; ++j) {
    const int c0 = step_block(p, s0 + j) * TB;
    TA *Lj = L + (size_t)j * TB * ldb;
    if (p.vec) {
      // chunk e: V consecutive source elements along the contiguous direction
      for (int e = threadIdx.x; e < TB * TB / V; e += blockDim.x) {
        const int u = (e % (TB / V)) * V, w = e / (TB / V);  // contiguous index, other index
        // non-trans: rows r0 + u.. of column c0 + w; trans: rows c0 + u.. of column r0 + w
        const int cr = p.trans ? c0 + u : r0 + u, cc = p.trans ? r0 + w : c0 + w;
        const int nv = (cc < p.N) ? max(0, min(V, p.N - cr)) : 0;
        const TA *src = nv ? A + cr + (int64_t)cc * p.lda : A;
        cp_async_16(Lj + w * ldb + u, src, (uint32_t)(nv * sizeof(TA)));
      }
    } else {
      for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
        const int u = e % TB, w = e / TB;
        const int cr = p.trans ? c0 + u : r0 + u, cc = p.trans ? r0 + w : c0 + w;
        const bool ok = cr < p.N && cc < p.N;
        cp_async_el(Lj + w * ldb + u, ok ? A + cr + (int64_t)cc * p.lda : A, ok);
      }
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

// acc[nt] (+)= sign * M(16 rows of this warp, nb blocks of 64 columns) * X(64 nb, 8 nt ..)
// M element (row, col) of block j at M[j * mbs + row * rs + col * cs]; X element (k, c) at
// X[c * ldx + k] (column-major).
template <int NT, typename TM>
__device__ __forceinline__ void block_mma(double (&acc)[NT][4], const TM *M, int rs, int cs,
                                          int mbs, int nb, const double *X, int ldx,
                                          double sign, int warp = -1) {
  if (warp < 0) warp = threadIdx.x >> 5;  // the 16-row group of the 64-row block
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  for (int j = 0; j < nb; ++j) {
    const TM *m0 = M + (size_t)j * mbs + (16 * warp + g) * rs + t * cs;
    const TM *m1 = m0 + 8 * rs;
    const double *xb = X + g * ldx + j * TB + t;
#pragma unroll 4
    for (int k = 0; k < TB; k += 4) {
      const double a0 = sign * (double)m0[k * cs], a1 = sign * (double)m1[k * cs];
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) dmma_16x8x4(acc[nt], a0, a1, xb[8 * nt * ldx + k]);
    }
  }
}

// Shared memory: the owned block's inverse, two chunk buffers of CH blocks of op(A), and
// two buffers for the X rows of a chunk (column-major, ld CH * 64 + 4).
template <typename TA, int NT>
constexpr int few_smem_ch(int ch) {
  return TB * LDL * 8 + 2 * ch * TB * few_block_ld<TA>(false) * (int)sizeof(TA) +
         2 * 8 * NT * (ch * TB + 4) * 8;
}
// the deepest chunk (up to 3 blocks) that fits in 225 KB of shared memory
template <typename TA, int NT>
constexpr int few_ch() {
  return few_smem_ch<TA, NT>(3) <= 225 * 1024 ? 3 : (few_smem_ch<TA, NT>(2) <= 225 * 1024 ? 2 : 1);
}
template <typename TA, int NT>
constexpr int few_smem() { return few_smem_ch<TA, NT>(few_ch<TA, NT>()); }

template <typename TA, int NT>
__global__ void __launch_bounds__(FEW_THREADS, 1) trsm_few_kernel(FewArgs p) {
  if (p.skip && *(volatile const int *)p.skip) return;
  constexpr int CH = few_ch<TA, NT>(), LDXK = CH * TB + 4;  // X chunk: column-major, ld LDXK
  constexpr int CBLK = TB * few_block_ld<TA>(false);        // chunk buffer elements per block
  constexpr int XPT = CH * TB * 8 * NT / FEW_THREADS;  // X values per thread per chunk
  extern __shared__ double sm[];
  double *I = sm;                                                   // owned block's inverse
  TA *const Lc0 = reinterpret_cast<TA *>(sm + TB * LDL);            // op(A) chunks
  TA *const Lc1 = Lc0 + CH * CBLK;
  double *const Xs0 = reinterpret_cast<double *>(Lc1 + CH * CBLK);  // X rows of a chunk
  double *const Xs1 = Xs0 + 8 * NT * LDXK;
  // orientation of the op(A) blocks in the chunk buffers (see stage_chunk)
  const int lb = few_block_ld<TA>(p.trans);
  const int mrs = p.trans ? lb : 1, mcs = p.trans ? 1 : lb, mbs = TB * lb;
  __shared__ int s_abort, s_ready, s_known;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  if (threadIdx.x == 0) s_abort = 0;
  __syncthreads();
  // column group of this CTA: B columns [gid * gw, gid * gw + nrhs), its own step flags
  const int gid = blockIdx.x % p.groups, gcta = gridDim.x / p.groups;
  double *B = p.B + (int64_t)gid * p.gw * p.bcs;
  const int nrhs = min(p.gw, p.nrhs - gid * p.gw);
  int *flags = p.flags + (size_t)gid * p.nblk * FLAG_STRIDE;
  // X rows of steps s0 .. s0 + cnt - 1 (published by other CTAs), read past L1
  auto x_load = [&](double (&v)[XPT], int s0, int cnt) {
    const int rows = cnt * TB;
#pragma unroll
    for (int u = 0; u < XPT; ++u) {
      const int e = threadIdx.x + u * FEW_THREADS;
      const int k = e % (CH * TB), c = e / (CH * TB);  // coalesced down each column of B
      const int xr = k < rows ? step_block(p, s0 + k / TB) * TB + k % TB : p.N;
      v[u] = (xr < p.N && c < nrhs) ? __ldcg(B + xr * p.brs + c * p.bcs) : 0.0;
    }
  };
  auto x_store = [&](const double (&v)[XPT], double *X) {
#pragma unroll
    for (int u = 0; u < XPT; ++u) {
      const int e = threadIdx.x + u * FEW_THREADS;
      X[(e / (CH * TB)) * LDXK + e % (CH * TB)] = v[u];
    }
  };
  for (int s = blockIdx.x / p.groups; s < p.nblk; s += gcta) {
    const int pb = step_block(p, s);
    stage_inverse(p, I, pb);
    // B block in accumulator layout: rows 16w+g (+8), columns 8nt+2t (+1)
    double acc[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = pb * TB + 16 * warp + g + 8 * (q >> 1);
        const int col = 8 * nt + 2 * t + (q & 1);
        acc[nt][q] = (row < p.N && col < nrhs) ? p.alpha * __ldcg(B + row * p.brs + col * p.bcs)
                                               : 0.0;
      }
    // Subtract op(A)[s, s2] X_s2 for every earlier step s2, up to CH steps per round.  Steps
    // publish their flags in order, so once the newest earlier step (s - 1) is published
    // every round proceeds without polling, and the X rows of the next round are loaded
    // into registers while the current round's product runs.
    if (threadIdx.x == 0)
      s_known = (s > 0 && flag_load(&flags[(s - 1) * FLAG_STRIDE]) == p.epoch) ? s - 1 : -1;
    int s2 = 0, cnt = min(CH, s), buf = 0;
    bool x_ok = false;
    if (s > 0) stage_chunk(p, Lc0, pb, 0, cnt);
    __syncthreads();
    int known = s_known;
    while (s2 < s) {
      int ready = cnt;
      if (!x_ok) {
        if (s2 + cnt - 1 > known) {
          if (threadIdx.x == 0) {
            uint32_t it = 0;
            while (flag_load(&flags[s2 * FLAG_STRIDE]) != p.epoch) {
              if (++it > p.spin_limit) {
                set_status(p.status, MO_EDEVTIMEOUT);
                s_abort = 1;
                break;
              }
            }
            int r = 1;
            while (r < cnt && flag_load(&flags[(s2 + r) * FLAG_STRIDE]) == p.epoch) ++r;
            s_ready = r;
            s_known = flag_load(&flags[(s - 1) * FLAG_STRIDE]) == p.epoch ? s - 1 : s2 + r - 1;
            __threadfence();
          }
          __syncthreads();
          if (s_abort) {
            cp_async_join();
            return;
          }
          ready = s_ready;
          known = s_known;
        }
        double v[XPT];
        x_load(v, s2, ready);
        x_store(v, buf ? Xs1 : Xs0);
      }
      cp_async_join();  // this round's blocks of op(A) (and the inverse) have landed
      __syncthreads();
      const int nxt = s2 + ready, ncnt = min(CH, s - nxt);
      const bool nx_ok = ncnt > 0 && nxt + ncnt - 1 <= known;
      double v[XPT];
      if (ncnt > 0) {
        stage_chunk(p, buf ? Lc0 : Lc1, pb, nxt, ncnt);
        if (nx_ok) x_load(v, nxt, ncnt);
      }
      block_mma<NT>(acc, buf ? Lc1 : Lc0, mrs, mcs, mbs, ready, buf ? Xs1 : Xs0, LDXK, -1.0);
      if (nx_ok) x_store(v, buf ? Xs0 : Xs1);
      __syncthreads();
      s2 = nxt;
      cnt = ncnt;
      buf ^= 1;
      x_ok = nx_ok;
    }
    // X_s = inv(op(A)_ss) * acc
    cp_async_join();
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q)
        Xs0[(8 * nt + 2 * t + (q & 1)) * LDXK + 16 * warp + g + 8 * (q >> 1)] = acc[nt][q];
    __syncthreads();
    double x[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) x[nt][q] = 0.0;
    block_mma<NT>(x, I, LDL, 1, 0, 1, Xs0, LDXK, 1.0);
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = pb * TB + 16 * warp + g + 8 * (q >> 1);
        const int col = 8 * nt + 2 * t + (q & 1);
        if (row < p.N && col < nrhs) B[row * p.brs + col * p.bcs] = x[nt][q];
      }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicExch(&flags[s * FLAG_STRIDE], p.epoch);
  }
}

template <typename TA, int NT>
int launch_few(mo_ctx *ctx, FewArgs &p) {
  const void *kern = (const void *)trsm_few_kernel<TA, NT>;
  constexpr int smem = few_smem<TA, NT>();
  if (int rc = mo_smem_attr(kern, smem)) return rc;
  int occ = 0;
  MO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, FEW_THREADS, smem));
  if (occ < 1) return MO_EINVAL;
  // every column group gets the same number of CTAs
  const int per = std::max(1, std::min(p.nblk, occ * ctx->sms / p.groups));
  const int grid = per * p.groups;
  void *args[] = {&p};
  MO_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(FEW_THREADS), args, smem,
                                          ctx->stream));
  return MO_OK;
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------------------
// Pairs of consecutive steps per CTA (FP32 op(A), the mixed-precision preconditioner).
// 8 warps: warps 0-3 hold step 2q's block, warps 4-7 step 2q + 1's.  The rounds over the
// earlier steps stage both block rows of a block column (one column per round) and share
// its X rows; then X_2q = inv * (B - ...) is published and, inside the CTA, step 2q + 1
// subtracts op(A)[2q + 1, 2q] X_2q straight from shared memory: every other hand-off on
// the dependency chain skips the flag, the L2 round trip and the fence.
// ---------------------------------------------------------------------------------------
constexpr int PAIR_THREADS = 256;
constexpr int PAIR_CBLK = TB * 72;  // floats per staged 64 x 64 block (largest orientation ld)

template <int NT>
constexpr int pair_smem() {
  // two inverses | op(A)[2q + 1, 2q] | two chunk buffers of two blocks | two X buffers
  return 2 * TB * LDL * 8 + PAIR_CBLK * 4 + 2 * 2 * PAIR_CBLK * 4 + 2 * 8 * NT * (TB + 4) * 8;
}

static_assert(pair_smem<8>() <= 227 * 1024 - 64, "pair kernel shared memory");

template <int NT>
__global__ void __launch_bounds__(PAIR_THREADS, 1) trsm_pair_kernel(FewArgs p) {
  if (p.skip && *(volatile const int *)p.skip) return;
  constexpr int LDXK = TB + 4;                        // X buffers: column-major 64 x 8NT
  constexpr int XPT = TB * 8 * NT / PAIR_THREADS;    // X values per thread per block
  extern __shared__ double sm[];
  double *const I0 = sm, *const I1 = sm + TB * LDL;
  float *const Ad = reinterpret_cast<float *>(sm + 2 * TB * LDL);
  float *const Lc0 = Ad + PAIR_CBLK;                  // block (pb0, col), then (pb1, col)
  float *const Lc1 = Lc0 + 2 * PAIR_CBLK;
  double *const Xs0 = reinterpret_cast<double *>(Lc1 + 2 * PAIR_CBLK);
  double *const Xs1 = Xs0 + 8 * NT * LDXK;
  __shared__ int s_abort, s_known;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int half = warp >> 2, wr = warp & 3;
  const int g = lane >> 2, t = lane & 3;
  if (threadIdx.x == 0) s_abort = 0;
  __syncthreads();
  const int gid = blockIdx.x % p.groups, gcta = gridDim.x / p.groups;
  double *B = p.B + (int64_t)gid * p.gw * p.bcs;
  const int nrhs = min(p.gw, p.nrhs - gid * p.gw);
  int *flags = p.flags + (size_t)gid * p.nblk * FLAG_STRIDE;
  const int lb = few_block_ld<float>(p.trans);
  const int mrs = p.trans ? lb : 1, mcs = p.trans ? 1 : lb;
  auto x_load = [&](double (&v)[XPT], int s0) {  // X rows of step s0, read past L1
#pragma unroll
    for (int u = 0; u < XPT; ++u) {
      const int e = threadIdx.x + u * PAIR_THREADS;
      const int k = e % TB, c = e / TB;
      const int xr = step_block(p, s0) * TB + k;
      v[u] = (xr < p.N && c < nrhs) ? __ldcg(B + xr * p.brs + c * p.bcs) : 0.0;
    }
  };
  auto x_store = [&](const double (&v)[XPT], double *X) {
#pragma unroll
    for (int u = 0; u < XPT; ++u) {
      const int e = threadIdx.x + u * PAIR_THREADS;
      X[(e / TB) * LDXK + e % TB] = v[u];
    }
  };
  auto stage_pair = [&](float *L, int pb0, int pb1, bool has1, int col_step) {
    stage_chunk(p, L, pb0, col_step, 1);
    if (has1) stage_chunk(p, L + PAIR_CBLK, pb1, col_step, 1);
  };
  const int npair = (p.nblk + 1) / 2;
  for (int q = blockIdx.x / p.groups; q < npair; q += gcta) {
    const int s0 = 2 * q, s1 = 2 * q + 1;
    const bool has1 = s1 < p.nblk;
    const int pb0 = step_block(p, s0), pb1 = has1 ? step_block(p, s1) : pb0;
    stage_inverse(p, I0, pb0);
    if (has1) {
      stage_inverse(p, I1, pb1);
      stage_chunk(p, Ad, pb1, s0, 1);  // op(A)[step 2q + 1, step 2q]
    }
    const int pbh = half ? pb1 : pb0;
    const bool live = half == 0 || has1;
    double acc[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int row = pbh * TB + 16 * wr + g + 8 * (r >> 1);
        const int col = 8 * nt + 2 * t + (r & 1);
        acc[nt][r] = (live && row < p.N && col < nrhs)
                         ? p.alpha * __ldcg(B + row * p.brs + col * p.bcs) : 0.0;
      }
    // subtract op(A)[step, s2] X_s2 for every earlier step s2, one block column per round
    if (threadIdx.x == 0)
      s_known = (s0 > 0 && flag_load(&flags[(s0 - 1) * FLAG_STRIDE]) == p.epoch) ? s0 - 1 : -1;
    int s2 = 0, buf = 0;
    bool x_ok = false;
    if (s0 > 0) stage_pair(Lc0, pb0, pb1, has1, 0);
    __syncthreads();
    int known = s_known;
    while (s2 < s0) {
      if (!x_ok) {
        if (s2 > known) {
          if (threadIdx.x == 0) {
            uint32_t it = 0;
            while (flag_load(&flags[s2 * FLAG_STRIDE]) != p.epoch) {
              if (++it > p.spin_limit) {
                set_status(p.status, MO_EDEVTIMEOUT);
                s_abort = 1;
                break;
              }
            }
            s_known = flag_load(&flags[(s0 - 1) * FLAG_STRIDE]) == p.epoch ? s0 - 1 : s2;
            __threadfence();
          }
          __syncthreads();
          if (s_abort) {
            cp_async_join();
            return;
          }
          known = s_known;
        }
        double v[XPT];
        x_load(v, s2);
        x_store(v, buf ? Xs1 : Xs0);
      }
      cp_async_join();
      __syncthreads();
      const int nxt = s2 + 1;
      const bool nx_ok = nxt < s0 && nxt <= known;
      double v[XPT];
      if (nxt < s0) {
        stage_pair(buf ? Lc0 : Lc1, pb0, pb1, has1, nxt);
        if (nx_ok) x_load(v, nxt);
      }
      if (live)
        block_mma<NT>(acc, (buf ? Lc1 : Lc0) + half * PAIR_CBLK, mrs, mcs, 0, 1,
                      buf ? Xs1 : Xs0, LDXK, -1.0, wr);
      if (nx_ok) x_store(v, buf ? Xs0 : Xs1);
      __syncthreads();
      s2 = nxt;
      buf ^= 1;
      x_ok = nx_ok;
    }
    cp_async_join();  // the inverses and op(A)[2q + 1, 2q]
    // step 2q: X_2q = inv(op(A)_2q) * acc (warps 0-3), kept in Xs1 for step 2q + 1
    if (half == 0) {
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int r = 0; r < 4; ++r)
          Xs0[(8 * nt + 2 * t + (r & 1)) * LDXK + 16 * wr + g + 8 * (r >> 1)] = acc[nt][r];
    }
    __syncthreads();
    if (half == 0) {
      double x[NT][4];
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int r = 0; r < 4; ++r) x[nt][r] = 0.0;
      block_mma<NT>(x, I0, LDL, 1, 0, 1, Xs0, LDXK, 1.0, wr);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int rr = 16 * wr + g + 8 * (r >> 1), col = 8 * nt + 2 * t + (r & 1);
          Xs1[col * LDXK + rr] = x[nt][r];
          if (pb0 * TB + rr < p.N && col < nrhs) B[(pb0 * TB + rr) * p.brs + col * p.bcs] = x[nt][r];
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicExch(&flags[s0 * FLAG_STRIDE], p.epoch);
    if (has1) {
      // step 2q + 1 (warps 4-7): acc -= op(A)[2q + 1, 2q] X_2q, then X = inv * acc
      if (half == 1) {
        block_mma<NT>(acc, Ad, mrs, mcs, 0, 1, Xs1, LDXK, -1.0, wr);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
          for (int r = 0; r < 4; ++r)
            Xs0[(8 * nt + 2 * t + (r & 1)) * LDXK + 16 * wr + g + 8 * (r >> 1)] = acc[nt][r];
      }
      __syncthreads();
      if (half == 1) {
        double x[NT][4];
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
          for (int r = 0; r < 4; ++r) x[nt][r] = 0.0;
        block_mma<NT>(x, I1, LDL, 1, 0, 1, Xs0, LDXK, 1.0, wr);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int rr = 16 * wr + g + 8 * (r >> 1), col = 8 * nt + 2 * t + (r & 1);
            if (pb1 * TB + rr < p.N && col < nrhs) B[(pb1 * TB + rr) * p.brs + col * p.bcs] = x[nt][r];
          }
      }
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) atomicExch(&flags[s1 * FLAG_STRIDE], p.epoch);
    }
  }
}

template <int NT>
int launch_pair(mo_ctx *ctx, FewArgs &p) {
  const void *kern = (const void *)trsm_pair_kernel<NT>;
  constexpr int smem = pair_smem<NT>();
  if (int rc = mo_smem_attr(kern, smem)) return rc;
  int occ = 0;
  MO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, PAIR_THREADS, smem));
  if (occ < 1) return MO_EINVAL;
  const int npair = (p.nblk + 1) / 2;
  const int per = std::max(1, std::min(npair, occ * ctx->sms / p.groups));
  const int grid = per * p.groups;
  void *args[] = {&p};
  MO_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(PAIR_THREADS), args, smem,
                                          ctx->stream));
  return MO_OK;
}

// flags -> (B strides, effective transposition and sweep direction) and the launch
int few_run(mo_ctx *ctx, View B, const void *A, bool a32, int64_t lda, int N, int flags,
            double alpha, const double *inv, bool inv_t, int *flag_buf,
            const int *skip = nullptr) {
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
  p.vec = ((uintptr_t)A % 16 == 0) && ((lda * (a32 ? 4 : 8)) % 16 == 0);
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
  p.spin_limit = ctx->spin_limit;
  p.skip = skip;
  // more than MO_FEW_GROUP columns: groups solved side by side by separate CTA sets, so
  // the per-step work on the dependency chain is that of one group
  const bool pair = a32 && p.nblk >= 4;
  const int gmax = pair ? MO_PAIR_GROUP : MO_FEW_GROUP;
  p.gw = nrhs > gmax ? gmax : nrhs;
  p.groups = (nrhs + p.gw - 1) / p.gw;
  MO_CUDA_TRY(cudaMemsetAsync(flag_buf, 0, sizeof(int) * p.nblk * p.groups * FLAG_STRIDE,
                              ctx->stream));
  ProfScope ps;
  prof_begin(ctx, ps, a32 ? MO_PROF_IR : MO_PROF_GEMM);
  const int nt = (p.gw + 7) / 8;
  int rc;
  if (pair) {
    // FP32 factor (the preconditioner of the mixed-precision solve): pairs of steps per CTA
    if (nt == 1) rc = launch_pair<1>(ctx, p);
    else if (nt == 2) rc = launch_pair<2>(ctx, p);
    else if (nt <= 4) rc = launch_pair<4>(ctx, p);
    else rc = launch_pair<8>(ctx, p);
  } else if (a32) {
    if (nt == 1) rc = launch_few<float, 1>(ctx, p);
    else if (nt == 2) rc = launch_few<float, 2>(ctx, p);
    else if (nt <= 4) rc = launch_few<float, 4>(ctx, p);
    else rc = launch_few<float, 8>(ctx, p);
  } else {
    if (nt == 1) rc = launch_few<double, 1>(ctx, p);
    else if (nt == 2) rc = launch_few<double, 2>(ctx, p);
    else if (nt <= 4) rc = launch_few<double, 4>(ctx, p);
    else rc = launch_few<double, 8>(ctx, p);
  }
  prof_end(ctx, ps, (double)N * N * nrhs,
           (a32 ? 4.0 : 8.0) * (double)N * N / 2 + 8.0 * 2.0 * N * nrhs);
  return rc;
}

}  // namespace

// Left solve (right solves via the transposed view of B) with nrhs <= 64.  `inv` receives
// the 128 x 128 diagonal-block inverses; `flag_buf` holds 4 x 32 ints per 64-row block.
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
                 const double *inv_L, int *flag_buf, const int *skip) {
  const int flags = MO_LOWER | (trans ? MO_TRANSA : 0);
  return few_run(ctx, B, L, true, ldl, N, flags, 1.0, inv_L, trans, flag_buf, skip);
}

}  // namespace mo
