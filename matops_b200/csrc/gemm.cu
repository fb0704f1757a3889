// FP64 GEMM / SYRK engine for sm_100a.
//
// One CTA computes a 128x128 tile of C.  A producer warp streams 128x16 slabs of op(A)
// and op(B) into a 6-stage shared-memory ring with 2-D TMA loads (128-byte swizzle, OOB
// zero fill); eight consumer warps (2 x 4, 64 x 32 each) run the FP64 tensor pipe through
// mma.sync.m16n8k4.f64 and hand stages back through mbarriers.  Operands whose base or
// leading dimension breaks TMA's 16-byte rules (arbitrary FloatMatrix views) use the
// same kernel with an 8-byte cp.async producer writing the identical swizzled layout.
// A C at most 64 columns wide and at least 2048 rows tall (the FP64 residual of a solve
// with few right-hand sides) takes 256x64 tiles in a 5-stage ring instead, with the
// consumer warps arranged 4 x 2, so that none of them idles on columns past N.
//
// Arithmetic (calgo/dmmat_gemm.c:364-415 semantics): C = beta*C + alpha*sum_k, with
// beta == 0 never reading C.  SYRK modes restrict tiles and elements to one triangle and
// can apply beta only on diagonal blocks (calgo/dmmat_rank.c:62-127).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "gemm.cuh"

namespace mo {
namespace {

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 6;
constexpr int CONSUMER_WARPS = 8;
// warpgroup 0 = producer (warp 0 issues the loads), warpgroups 1-2 = consumers.
// Register split via setmaxnreg: launch 384 x 168 = 64512 = 128 x 40 + 256 x 232.
constexpr int THREADS = 384;
constexpr int PRODUCER_REGS = 40, CONSUMER_REGS = 232;
static_assert(THREADS * 168 >= 128 * PRODUCER_REGS + 256 * CONSUMER_REGS, "register split");
// Tile geometry of one instantiation.  NARROW (C at most 64 columns wide, e.g. a residual
// B - A X with few right-hand sides): 256 x 64 tiles, warps in a 4 x 2 grid of the same
// 64 x 32 warp tiles, so all eight consumer warps issue MMAs where a 128 x 128 tile would
// leave half of them idle.
template <bool NARROW>
struct Geo {
  static constexpr int TBM = NARROW ? 256 : 128, TBN = NARROW ? 64 : 128;
  static constexpr int NSTAGES = NARROW ? 5 : STAGES;
  static constexpr int A_DBL = TBM * BK, B_DBL = TBN * BK, STAGE_DBL = A_DBL + B_DBL;
  static constexpr uint32_t SBYTES = STAGE_DBL * 8;
  static constexpr int SMEM = NSTAGES * SBYTES + 1024 + 2 * NSTAGES * 8;
  static constexpr int WN = TBN / 32;  // warp columns
};
static_assert(Geo<true>::SMEM <= 227 * 1024 && Geo<false>::SMEM <= 227 * 1024, "shared memory");

// Swizzled shared-memory layouts (TMA SWIZZLE_128B: 16-byte chunk ^= 128-byte row % 8).
// K-major slab: 128 rows (m or n) of 16 k-values (128 B per row).
__device__ __forceinline__ int kmaj_off(int mn, int k) {
  return mn * 16 + ((((k >> 1) ^ (mn & 7))) << 1) + (k & 1);
}
// MN-major slab: 8 boxes of [16 k-rows x 16 mn-values].
__device__ __forceinline__ int mnmaj_off(int mn, int k) {
  return (mn >> 4) * 256 + k * 16 + (((((mn & 15) >> 1) ^ (k & 7))) << 1) + (mn & 1);
}

struct KParams {
  int M, N, K;
  double alpha, beta;
  const double *A;
  int64_t lda;
  const double *B;
  int64_t ldb;
  double *C;
  int64_t ldc;
  int mode, beta_block;
  int *status;
  const int *skip;
  int tiles_m, tiles_n;
  int total_tiles;  // tiles of C (the triangle's tiles in SYRK modes)
  int kt;           // k-slabs per tile
  int dp_tiles;     // tiles [0, dp_tiles) are processed whole, round-robin over CTAs
  int sk_iters;     // stream-K iterations over the remaining tiles
  int sk_chunk;     // stream-K iterations per CTA
  double *partial;  // [gridDim.x][64 * 256] stream-K partial accumulators
  int *flags;       // [gridDim.x] epoch stamps of published partials
  int epoch;
};

// cp.async producer for one ROWS x 16 slab (ROWS = 64 or 128) of an operand whose element
// (mn, k) lives at src[k + mn*ld] (KMAJ) or src[mn + k*ld] (!KMAJ); out-of-range elements
// are zero-filled.
template <bool KMAJ, int ROWS = 128>
__device__ __forceinline__ void load_slab_cpasync(double *dst, const double *src, int64_t ld,
                                                  int mn0, int k0, int MN, int K, int lane) {
  if constexpr (KMAJ) {
#pragma unroll 8
    for (int i = 0; i < ROWS / 2; ++i) {
      int mn = 2 * i + (lane >> 4), k = lane & 15;
      int gm = mn0 + mn, gk = k0 + k;
      bool ok = gm < MN && gk < K;
      const double *s = ok ? src + gk + (int64_t)gm * ld : src;
      cp_async_8(dst + kmaj_off(mn, k), s, ok ? 8u : 0u);
    }
  } else {
#pragma unroll 4
    for (int k = 0; k < 16; ++k)
#pragma unroll
      for (int j = 0; j < ROWS / 32; ++j) {
        int mn = 32 * j + lane;
        int gm = mn0 + mn, gk = k0 + k;
        bool ok = gm < MN && gk < K;
        const double *s = ok ? src + gm + (int64_t)gk * ld : src;
        cp_async_8(dst + mnmaj_off(mn, k), s, ok ? 8u : 0u);
      }
  }
}

__device__ __forceinline__ void tile_coords(const KParams &p, int t, int &tm, int &tn) {
  if (p.mode == kGemm || p.mode == kGemmLower || p.mode == kGemmUpper) {
    // groups of GROUP_M tile rows, column-major inside a group: a wave of persistent CTAs
    // touches GROUP_M row panels of A and a narrow band of B, which stay in L2
    constexpr int GROUP_M = 8;
    const int per_group = GROUP_M * p.tiles_n;
    const int grp = t / per_group, r = t % per_group;
    const int m_first = grp * GROUP_M;
    const int gm = min(GROUP_M, p.tiles_m - m_first);
    tm = m_first + r % gm;
    tn = r / gm;
    return;
  }
  // t enumerates the triangle row by row: (r, c) with c <= r
  int r = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((r + 1) * (r + 2) / 2 <= t) ++r;
  while (r * (r + 1) / 2 > t) --r;
  const int c = t - r * (r + 1) / 2;
  if (p.mode == kSyrkLower) {
    tm = r;
    tn = c;
  } else {
    tm = c;
    tn = r;
  }
}

// One unit of work: k-slabs [k0, k1) of tile `tile`.  owner: this CTA finishes the tile
// (adds the partials of CTAs [first_contrib, blockIdx.x) and writes C); otherwise it
// publishes its partial sum.
struct Unit {
  int tile, k0, k1;
  bool owner;
  int first_contrib;
};

// Enumerates this CTA's units in processing order: whole tiles first, then its stream-K
// range from the highest tile down (so that a partial is published before this CTA waits
// for the partials of lower-numbered CTAs).  Returns the number of units; fills u[i] for
// i == idx.
__device__ __forceinline__ bool unit_at(const KParams &p, int idx, Unit &u) {
  const int P = gridDim.x, b = blockIdx.x;
  const int ndp = (p.dp_tiles > b) ? (p.dp_tiles - b + P - 1) / P : 0;
  if (idx < ndp) {
    u.tile = b + idx * P;
    u.k0 = 0;
    u.k1 = p.kt;
    u.owner = true;
    u.first_contrib = b;
    return true;
  }
  idx -= ndp;
  if (p.sk_iters <= 0) return false;
  const int s = b * p.sk_chunk, e = min(s + p.sk_chunk, p.sk_iters);
  if (s >= e) return false;
  const int first = s / p.kt, last = (e - 1) / p.kt;
  const int t = last - idx;
  if (t < first) return false;
  const int ts = t * p.kt, te = ts + p.kt;
  u.tile = p.dp_tiles + t;
  u.k0 = max(s, ts) - ts;
  u.k1 = min(e, te) - ts;
  u.owner = (e >= te);
  u.first_contrib = ts / p.sk_chunk;
  return true;
}

__device__ __forceinline__ void consumer_bar() {
  asm volatile("bar.sync 1, 256;" ::: "memory");
}

template <bool A_KMAJ, bool B_KMAJ, bool USE_TMA, bool NARROW>
__global__ void __launch_bounds__(THREADS, 1)
    dgemm_tile_kernel(const __grid_constant__ CUtensorMap tmA,
                      const __grid_constant__ CUtensorMap tmB, const KParams p) {
  using G = Geo<NARROW>;
  constexpr int STAGES = G::NSTAGES;
  extern __shared__ unsigned char smem_raw[];
  const uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023);
  double *tiles = reinterpret_cast<double *>(base);
  uint64_t *full = reinterpret_cast<uint64_t *>(base + STAGES * G::SBYTES);
  uint64_t *empty = full + STAGES;
  __shared__ int s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (p.skip && *(volatile const int *)p.skip) return;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], USE_TMA ? 1u : 32u);
      mbar_init(&empty[s], CONSUMER_WARPS);
    }
    s_abort = 0;
    fence_barrier_init();
  }
  __syncthreads();

  if (warp < 4) {
    // ------------------------------ producer warpgroup ------------------------------
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(PRODUCER_REGS));
    if (warp != 0) return;
    int it = 0;  // ring position, continues across units
    Unit u;
    for (int ui = 0; unit_at(p, ui, u); ++ui) {
      int tm, tn;
      tile_coords(p, u.tile, tm, tn);
      const int m0 = tm * G::TBM, n0 = tn * G::TBN;
      for (int kt = u.k0; kt < u.k1; ++kt, ++it) {
        const int s = it % STAGES;
        const uint32_t ph = (it / STAGES) & 1;
        if (!mbar_wait(&empty[s], ph ^ 1u, p.status)) {
          if constexpr (!USE_TMA) asm volatile("cp.async.wait_all;" ::: "memory");
          return;
        }
        double *As = tiles + s * G::STAGE_DBL;
        double *Bs = As + G::A_DBL;
        const int k0 = kt * BK;
        if constexpr (USE_TMA) {
          if (lane == 0) {
            mbar_arrive_expect_tx(&full[s], G::SBYTES);
            // K-major maps carry 128-row boxes (64 rows for a narrow B), MN-major maps
            // 16 x 16 boxes
            if (A_KMAJ) {
#pragma unroll
              for (int h = 0; h < G::TBM / 128; ++h)
                tma_load_2d(As + h * 128 * BK, &tmA, &full[s], k0, m0 + 128 * h);
            } else {
#pragma unroll
              for (int bb = 0; bb < G::TBM / 16; ++bb)
                tma_load_2d(As + bb * 256, &tmA, &full[s], m0 + 16 * bb, k0);
            }
            if (B_KMAJ) {
              tma_load_2d(Bs, &tmB, &full[s], k0, n0);
            } else {
#pragma unroll
              for (int bb = 0; bb < G::TBN / 16; ++bb)
                tma_load_2d(Bs + bb * 256, &tmB, &full[s], n0 + 16 * bb, k0);
            }
          }
          __syncwarp();
        } else {
#pragma unroll
          for (int h = 0; h < G::TBM / 128; ++h)
            load_slab_cpasync<A_KMAJ>(As + h * 128 * BK, p.A, p.lda, m0 + 128 * h, k0, p.M, p.K,
                                      lane);
          load_slab_cpasync<B_KMAJ, G::TBN>(Bs, p.B, p.ldb, n0, k0, p.N, p.K, lane);
          cp_async_arrive_noinc(&full[s]);
        }
      }
    }
    if constexpr (!USE_TMA) asm volatile("cp.async.wait_all;" ::: "memory");
    return;
  }

  // ------------------------------ consumer warpgroups ------------------------------
  asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(CONSUMER_REGS));
  const int ct = threadIdx.x - 128;  // consumer thread 0..255
  const int cw = warp - 4;
  // 2 x 4 (4 x 2 when narrow) grid of 64 x 32 warp tiles
  const int wm = cw >> (NARROW ? 1 : 2), wn = cw & (G::WN - 1);
  const int g = lane >> 2, t = lane & 3;
  // Fragment offsets into the swizzled slabs, split into a per-thread part computed once
  // and compile-time constants (mt, nt, kk).  K-major: element (mn, k) at
  // mn*16 + 2*((k>>1) ^ (mn&7)) + (k&1), with mn&7 == g and k = kk + t.
  // MN-major: (mn>>4)*256 + k*16 + 2*(((mn&15)>>1) ^ (k&7)) + (mn&1).
  int kv[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) kv[q] = 2 * ((2 * q) ^ (g & 6)) + 2 * ((t >> 1) ^ (g & 1)) + (t & 1);
  int xa[2][2], xb[2][2];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int q2 = 0; q2 < 2; ++q2) {
      xa[h][q2] = 2 * (((g >> 1) + 4 * h) ^ (4 * q2 + t));
      xb[h][q2] = 2 * (((g >> 1) + 4 * h) ^ (4 * q2 + t));
    }
  const int a_base = A_KMAJ ? (wm * 64 + g) * 16 : (wm * 4) * 256 + t * 16 + (g & 1);
  const int b_base = B_KMAJ ? (wn * 32 + g) * 16 : (wn * 2) * 256 + t * 16 + (g & 1);
  int it = 0;
  Unit u;
  for (int ui = 0; unit_at(p, ui, u); ++ui) {
    int tm, tn;
    tile_coords(p, u.tile, tm, tn);
    const int m0 = tm * G::TBM, n0 = tn * G::TBN;
    // warm L2 with this warp's C sub-tile (64 rows x 32 cols: 4 lines of 128 B per column)
    if (u.owner && (p.beta != 0.0 || p.beta_block > 0)) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int col = n0 + wn * 32 + lane;
        const int row = m0 + wm * 64 + 16 * q;
        if (col < p.N && row < p.M)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(p.C + row + (int64_t)col * p.ldc));
      }
    }
    double acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

    // a warp whose 32 columns all lie past N (narrow C, e.g. a residual with few
    // right-hand sides) keeps the stage hand-shake but issues no loads or MMAs
    const bool idle = n0 + wn * 32 >= p.N;
    for (int kt = u.k0; kt < u.k1; ++kt, ++it) {
      const int s = it % STAGES;
      const uint32_t ph = (it / STAGES) & 1;
      if (!mbar_wait(&full[s], ph, p.status)) return;
      const double *As = tiles + s * G::STAGE_DBL;
      const double *Bs = As + G::A_DBL;
#pragma unroll
      for (int kk = 0; kk < BK && !idle; kk += 4) {
        const int q = kk >> 2, q2 = q & 1;
        double a[4][2], b[4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
          if constexpr (A_KMAJ) {
            a[mt][0] = As[a_base + kv[q] + mt * 256];
            a[mt][1] = As[a_base + kv[q] + mt * 256 + 128];
          } else {
            a[mt][0] = As[a_base + xa[0][q2] + mt * 256 + kk * 16];
            a[mt][1] = As[a_base + xa[1][q2] + mt * 256 + kk * 16];
          }
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          if constexpr (B_KMAJ)
            b[nt] = Bs[b_base + kv[q] + nt * 128];
          else
            b[nt] = Bs[b_base + xb[nt & 1][q2] + (nt >> 1) * 256 + kk * 16];
        }
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma_16x8x4(acc[mt][nt], a[mt][0], a[mt][1], b[nt]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }

    if (!u.owner) {
      // publish the partial sum (fragment order: register r of consumer thread ct at
      // [r * 256 + ct], coalesced per warp), then stamp this CTA's flag
      double *slot = p.partial + (size_t)blockIdx.x * (64 * 256);
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int r = 0; r < 4; ++r) slot[((mt * 4 + nt) * 4 + r) * 256 + ct] = acc[mt][nt][r];
      __threadfence();
      consumer_bar();
      if (ct == 0) atomicExch(&p.flags[blockIdx.x], p.epoch);
      continue;
    }
    if (u.first_contrib < (int)blockIdx.x) {
      // add the partials of the lower-numbered CTAs that computed the tile's first slabs
      for (int c = u.first_contrib; c < (int)blockIdx.x; ++c) {
        if (ct == 0) {
          uint32_t i = 0;
          while (atomicAdd(&p.flags[c], 0) != p.epoch) {
            if (++i > MO_SPIN_LIMIT) {
              set_status(p.status, MO_EDEVTIMEOUT);
              s_abort = 1;
              break;
            }
          }
          __threadfence();
        }
        consumer_bar();
        if (s_abort) return;
        const double *slot = p.partial + (size_t)c * (64 * 256);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int r = 0; r < 4; ++r)
              acc[mt][nt][r] += __ldcg(slot + ((mt * 4 + nt) * 4 + r) * 256 + ct);
      }
    }

    // ------------------------------ epilogue ------------------------------
    // 16 elements at a time: all loads of C are issued before any store, so the L2 round
    // trips overlap (stores may alias later loads, which would otherwise serialize them)
    // C is read unless beta == 0 everywhere (with diagonal-block beta, off-block
    // elements use beta = 1)
    const bool need_c = p.beta != 0.0 || p.beta_block > 0;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      double cv[4][4];
      bool keep[4][4];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int row = m0 + wm * 64 + mt * 16 + g + ((r >> 1) << 3);
          const int col = n0 + wn * 32 + nt * 8 + 2 * t + (r & 1);
          bool k = row < p.M && col < p.N;
          if ((p.mode == kSyrkLower || p.mode == kGemmLower) && row < col) k = false;
          if ((p.mode == kSyrkUpper || p.mode == kGemmUpper) && row > col) k = false;
          keep[nt][r] = k;
          cv[nt][r] = (k && need_c) ? __ldcg(p.C + row + (int64_t)col * p.ldc) : 0.0;
        }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          if (!keep[nt][r]) continue;
          const int row = m0 + wm * 64 + mt * 16 + g + ((r >> 1) << 3);
          const int col = n0 + wn * 32 + nt * 8 + 2 * t + (r & 1);
          double bet = p.beta;
          if (p.beta_block > 0 && (row / p.beta_block) != (col / p.beta_block)) bet = 1.0;
          double v = p.alpha * acc[mt][nt][r];
          if (bet != 0.0) v = fma(bet, cv[nt][r], v);
          p.C[row + (int64_t)col * p.ldc] = v;
        }
    }
  }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2-D map over a column-major matrix whose contiguous dimension has `inner` elements.
bool make_tmap(CUtensorMap *tm, const double *ptr, uint64_t inner, uint64_t outer, int64_t ld,
               uint32_t box_inner, uint32_t box_outer) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {inner < 1 ? 1 : inner, outer < 1 ? 1 : outer};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(ptr), dims, strides,
                  box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <bool AK, bool BKM, bool TMA, bool NARROW>
int launch_inst(const KParams &kp, const CUtensorMap &ta, const CUtensorMap &tb, int grid,
                cudaStream_t st) {
  constexpr int SMEM_BYTES = Geo<NARROW>::SMEM;
  auto kern = dgemm_tile_kernel<AK, BKM, TMA, NARROW>;
  // setmaxnreg.inc only draws on the registers the CTA was launched with: refuse to launch
  // (instead of waiting forever) if the build did not keep the 168-register split (a
  // property of the binary, checked once)
  static std::atomic<int> regs_ok{0};
  if (!regs_ok.load()) {
    cudaFuncAttributes fa;
    MO_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (fa.numRegs * THREADS < 128 * PRODUCER_REGS + 256 * CONSUMER_REGS) return MO_ENOKERNEL;
    regs_ok.store(1);
  }
  // the shared-memory limit is set on every launch (a cheap host call), so that it holds
  // after a context reset
  if (int rc = mo_smem_attr((const void *)kern, SMEM_BYTES)) return rc;
  kern<<<grid, THREADS, SMEM_BYTES, st>>>(ta, tb, kp);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

template <bool TMA, bool NARROW>
int dispatch(bool ak, bool bk, const KParams &kp, const CUtensorMap &ta, const CUtensorMap &tb,
             int grid, cudaStream_t st) {
  if (ak) return bk ? launch_inst<true, true, TMA, NARROW>(kp, ta, tb, grid, st)
                    : launch_inst<true, false, TMA, NARROW>(kp, ta, tb, grid, st);
  return bk ? launch_inst<false, true, TMA, NARROW>(kp, ta, tb, grid, st)
            : launch_inst<false, false, TMA, NARROW>(kp, ta, tb, grid, st);
}

}  // namespace

bool gemm_tma_ok(const GemmArgs &a) {
  auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  return al(a.A) && al(a.B) && (a.lda % 2 == 0) && (a.ldb % 2 == 0) && encode_fn() != nullptr;
}

int gemm_partial_slots(int sms) { return sms; }
size_t gemm_partial_bytes(int sms) { return (size_t)sms * 64 * 256 * sizeof(double); }

int launch_gemm(const GemmArgs &a, cudaStream_t stream) {
  if (a.M <= 0 || a.N <= 0) return MO_OK;
  KParams kp;
  kp.M = a.M;
  kp.N = a.N;
  kp.K = a.K < 0 ? 0 : a.K;
  kp.alpha = a.alpha;
  kp.beta = a.beta;
  kp.A = a.A;
  kp.lda = a.lda;
  kp.B = a.B;
  kp.ldb = a.ldb;
  kp.C = a.C;
  kp.ldc = a.ldc;
  kp.mode = a.mode;
  kp.beta_block = a.beta_block;
  kp.status = a.status;
  kp.skip = a.skip;
  // narrow C (a residual with few right-hand sides): 256 x 64 tiles
  const bool narrow = a.mode == kGemm && a.N <= 64 && a.M >= 2048;
  const int tbm = narrow ? Geo<true>::TBM : BM, tbn = narrow ? Geo<true>::TBN : BN;
  const int tiles_m = (a.M + tbm - 1) / tbm, tiles_n = (a.N + tbn - 1) / tbn;
  kp.tiles_m = tiles_m;
  kp.tiles_n = tiles_n;
  long long T;
  if (a.mode == kGemm || a.mode == kGemmLower || a.mode == kGemmUpper) {
    T = (long long)tiles_m * tiles_n;
  } else {
    if (a.M != a.N) return MO_EINVAL;
    T = (long long)tiles_m * (tiles_m + 1) / 2;
  }
  if (T <= 0 || T > 0x7fffffffLL) return MO_EINVAL;
  kp.total_tiles = (int)T;
  kp.kt = (kp.K + BK - 1) / BK;
  int sms = a.sms > 0 ? a.sms : 148;
  if (a.max_ctas > 0 && a.max_ctas < sms) sms = a.max_ctas;
  // Schedule: whole tiles round-robin over persistent CTAs; when a GEMM has only a few,
  // unequal waves (e.g. 256 tiles on 148 SMs), the last one or two waves are split along
  // K evenly over all CTAs (stream-K) and finished by the CTA holding each tile's last slab.
  int grid = (int)std::min<long long>(T, sms);
  kp.dp_tiles = (int)T;
  kp.sk_iters = 0;
  kp.sk_chunk = 1;
  kp.partial = a.sk_partial;
  kp.flags = a.sk_flags;
  kp.epoch = a.sk_epoch;
  const long long waves = T / sms, rem = T % sms;
  if (a.mode == kGemm && a.sk_partial && a.sk_flags && rem != 0 && waves < 4 && kp.kt >= 8) {
    const long long dp = (waves >= 1 ? waves - 1 : 0) * sms;
    kp.dp_tiles = (int)dp;
    kp.sk_iters = (int)((T - dp) * kp.kt);
    grid = sms;
    kp.sk_chunk = (kp.sk_iters + grid - 1) / grid;
    if (kp.sk_chunk < 4) {
      // too little work for every CTA: fewer CTAs with 4 slabs each when that still uses
      // more SMs than whole tiles would (a few tiles with a long K, e.g. one 128 x 128
      // tile with K in the thousands), else data-parallel
      const long long g2 = kp.sk_iters / 4;
      if (kp.kt >= 32 && g2 > T) {
        grid = (int)std::min<long long>(g2, sms);
        kp.sk_chunk = (kp.sk_iters + grid - 1) / grid;
      } else {
        kp.dp_tiles = (int)T;
        kp.sk_iters = 0;
        kp.sk_chunk = 1;
        grid = (int)std::min<long long>(T, sms);
      }
    }
  }

  const bool ak = a.transA;   // op(A) stored K-major when A is transposed
  const bool bk = !a.transB;  // op(B) stored K-major when B is not transposed
  CUtensorMap ta, tb;
  const bool use_tma = !a.force_fallback && kp.K > 0 && gemm_tma_ok(a);
  if (use_tma) {
    bool okA = ak ? make_tmap(&ta, a.A, kp.K, a.M, a.lda, 16, 128)
                  : make_tmap(&ta, a.A, a.M, kp.K, a.lda, 16, 16);
    bool okB = bk ? make_tmap(&tb, a.B, kp.K, a.N, a.ldb, 16, (uint32_t)tbn)
                  : make_tmap(&tb, a.B, a.N, kp.K, a.ldb, 16, 16);
    if (okA && okB)
      return narrow ? dispatch<true, true>(ak, bk, kp, ta, tb, grid, stream)
                    : dispatch<true, false>(ak, bk, kp, ta, tb, grid, stream);
  }
  memset(&ta, 0, sizeof(ta));
  memset(&tb, 0, sizeof(tb));
  return narrow ? dispatch<false, true>(ak, bk, kp, ta, tb, grid, stream)
                : dispatch<false, false>(ak, bk, kp, ta, tb, grid, stream);
}

}  // namespace mo
