// FP64 GEMM / SYRK engine for sm_100a.
//
// One CTA computes a 128x128 tile of C.  A producer warp streams 128x16 slabs of op(A)
// and op(B) into a 6-stage shared-memory ring with 2-D TMA loads (128-byte swizzle, OOB
// zero fill); eight consumer warps (2 x 4, 64 x 32 each) run the FP64 tensor pipe through
// mma.sync.m16n8k4.f64 and hand stages back through mbarriers.  Operands whose base or
// leading dimension breaks TMA's 16-byte rules (arbitrary FloatMatrix views) use the
// same kernel with an 8-byte cp.async producer writing the identical swizzled layout.
//
// Arithmetic (calgo/dmmat_gemm.c:364-415 semantics): C = beta*C + alpha*sum_k, with
// beta == 0 never reading C.  SYRK modes restrict tiles and elements to one triangle and
// can apply beta only on diagonal blocks (calgo/dmmat_rank.c:62-127).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <cmath>
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
constexpr int TILE_DOUBLES = 128 * BK;                     // one operand slab: 16 KB
constexpr uint32_t STAGE_BYTES = 2 * TILE_DOUBLES * 8;     // A slab + B slab
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 2 * STAGES * 8;

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
  int tiles_m;
};

// cp.async producer for one 128 x 16 slab of an operand whose element (mn, k) lives at
// src[k + mn*ld] (KMAJ) or src[mn + k*ld] (!KMAJ); out-of-range elements are zero-filled.
template <bool KMAJ>
__device__ __forceinline__ void load_slab_cpasync(double *dst, const double *src, int64_t ld,
                                                  int mn0, int k0, int MN, int K, int lane) {
  if constexpr (KMAJ) {
#pragma unroll 8
    for (int i = 0; i < 64; ++i) {
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
      for (int j = 0; j < 4; ++j) {
        int mn = 32 * j + lane;
        int gm = mn0 + mn, gk = k0 + k;
        bool ok = gm < MN && gk < K;
        const double *s = ok ? src + gm + (int64_t)gk * ld : src;
        cp_async_8(dst + mnmaj_off(mn, k), s, ok ? 8u : 0u);
      }
  }
}

__device__ __forceinline__ void tile_of_block(const KParams &p, int bid, int &tm, int &tn) {
  if (p.mode == kGemm) {
    tm = bid % p.tiles_m;
    tn = bid / p.tiles_m;
    return;
  }
  // bid enumerates the triangle row by row: (r, c) with c <= r
  int r = (int)((sqrt(8.0 * (double)bid + 1.0) - 1.0) * 0.5);
  while ((r + 1) * (r + 2) / 2 <= bid) ++r;
  while (r * (r + 1) / 2 > bid) --r;
  int c = bid - r * (r + 1) / 2;
  if (p.mode == kSyrkLower) {
    tm = r;
    tn = c;
  } else {
    tm = c;
    tn = r;
  }
}

template <bool A_KMAJ, bool B_KMAJ, bool USE_TMA>
__global__ void __launch_bounds__(THREADS, 1)
    dgemm_tile_kernel(const __grid_constant__ CUtensorMap tmA,
                      const __grid_constant__ CUtensorMap tmB, const KParams p) {
  extern __shared__ unsigned char smem_raw[];
  const uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023);
  double *tiles = reinterpret_cast<double *>(base);
  uint64_t *full = reinterpret_cast<uint64_t *>(base + STAGES * STAGE_BYTES);
  uint64_t *empty = full + STAGES;

  int tm, tn;
  tile_of_block(p, blockIdx.x, tm, tn);
  const int m0 = tm * BM, n0 = tn * BN;
  const int num_kt = (p.K + BK - 1) / BK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], USE_TMA ? 1u : 32u);
      mbar_init(&empty[s], CONSUMER_WARPS);
    }
    fence_barrier_init();
  }
  __syncthreads();

  if (warp < 4) {
    // ------------------------------ producer warpgroup ------------------------------
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(PRODUCER_REGS));
    if (warp != 0) return;
    for (int kt = 0; kt < num_kt; ++kt) {
      const int s = kt % STAGES;
      const uint32_t ph = (kt / STAGES) & 1;
      if (!mbar_wait(&empty[s], ph ^ 1u, p.status)) break;
      double *As = tiles + s * 2 * TILE_DOUBLES;
      double *Bs = As + TILE_DOUBLES;
      const int k0 = kt * BK;
      if constexpr (USE_TMA) {
        if (lane == 0) {
          mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
          if (A_KMAJ) {
            tma_load_2d(As, &tmA, &full[s], k0, m0);
          } else {
#pragma unroll
            for (int b = 0; b < 8; ++b) tma_load_2d(As + b * 256, &tmA, &full[s], m0 + 16 * b, k0);
          }
          if (B_KMAJ) {
            tma_load_2d(Bs, &tmB, &full[s], k0, n0);
          } else {
#pragma unroll
            for (int b = 0; b < 8; ++b) tma_load_2d(Bs + b * 256, &tmB, &full[s], n0 + 16 * b, k0);
          }
        }
        __syncwarp();
      } else {
        load_slab_cpasync<A_KMAJ>(As, p.A, p.lda, m0, k0, p.M, p.K, lane);
        load_slab_cpasync<B_KMAJ>(Bs, p.B, p.ldb, n0, k0, p.N, p.K, lane);
        cp_async_arrive_noinc(&full[s]);
      }
    }
    if constexpr (!USE_TMA) asm volatile("cp.async.wait_all;" ::: "memory");
    return;
  }

  // ------------------------------ consumer warpgroups ------------------------------
  asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(CONSUMER_REGS));
  const int cw = warp - 4;
  const int wm = cw >> 2, wn = cw & 3;  // 2 x 4 grid of 64 x 32 warp tiles
  const int g = lane >> 2, t = lane & 3;
  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

  bool ok = true;
  for (int kt = 0; kt < num_kt; ++kt) {
    const int s = kt % STAGES;
    const uint32_t ph = (kt / STAGES) & 1;
    if (!mbar_wait(&full[s], ph, p.status)) {
      ok = false;
      break;
    }
    const double *As = tiles + s * 2 * TILE_DOUBLES;
    const double *Bs = As + TILE_DOUBLES;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      const int k = kk + t;
      double a[4][2], b[4];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int m = wm * 64 + mt * 16 + g;
        a[mt][0] = As[A_KMAJ ? kmaj_off(m, k) : mnmaj_off(m, k)];
        a[mt][1] = As[A_KMAJ ? kmaj_off(m + 8, k) : mnmaj_off(m + 8, k)];
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int n = wn * 32 + nt * 8 + g;
        b[nt] = Bs[B_KMAJ ? kmaj_off(n, k) : mnmaj_off(n, k)];
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma_16x8x4(acc[mt][nt], a[mt][0], a[mt][1], b[nt]);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (!ok) return;

  // ------------------------------ epilogue ------------------------------
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int row = m0 + wm * 64 + mt * 16 + g + ((r >> 1) << 3);
        const int col = n0 + wn * 32 + nt * 8 + 2 * t + (r & 1);
        if (row >= p.M || col >= p.N) continue;
        if (p.mode == kSyrkLower && row < col) continue;
        if (p.mode == kSyrkUpper && row > col) continue;
        double bet = p.beta;
        if (p.beta_block > 0 && (row / p.beta_block) != (col / p.beta_block)) bet = 1.0;
        double *cp = p.C + row + (int64_t)col * p.ldc;
        double v = p.alpha * acc[mt][nt][r];
        if (bet != 0.0) v = fma(bet, *cp, v);
        *cp = v;
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

template <bool AK, bool BKM, bool TMA>
int launch_inst(const KParams &kp, const CUtensorMap &ta, const CUtensorMap &tb, int grid,
                cudaStream_t st) {
  static std::atomic<uint64_t> attr_done{0};
  int dev = 0;
  cudaGetDevice(&dev);
  auto kern = dgemm_tile_kernel<AK, BKM, TMA>;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(attr_done.load() & bit)) {
    // setmaxnreg.inc only draws on the registers the CTA was launched with: refuse to
    // launch (instead of waiting forever) if the build did not keep the 168-register split
    cudaFuncAttributes fa;
    MO_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (fa.numRegs * THREADS < 128 * PRODUCER_REGS + 256 * CONSUMER_REGS) return MO_ENOKERNEL;
    MO_CUDA_TRY(
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    attr_done.fetch_or(bit);
  }
  kern<<<grid, THREADS, SMEM_BYTES, st>>>(ta, tb, kp);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

template <bool TMA>
int dispatch(bool ak, bool bk, const KParams &kp, const CUtensorMap &ta, const CUtensorMap &tb,
             int grid, cudaStream_t st) {
  if (ak) return bk ? launch_inst<true, true, TMA>(kp, ta, tb, grid, st)
                    : launch_inst<true, false, TMA>(kp, ta, tb, grid, st);
  return bk ? launch_inst<false, true, TMA>(kp, ta, tb, grid, st)
            : launch_inst<false, false, TMA>(kp, ta, tb, grid, st);
}

}  // namespace

bool gemm_tma_ok(const GemmArgs &a) {
  auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  return al(a.A) && al(a.B) && (a.lda % 2 == 0) && (a.ldb % 2 == 0) && encode_fn() != nullptr;
}

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
  const int tiles_m = (a.M + BM - 1) / BM, tiles_n = (a.N + BN - 1) / BN;
  kp.tiles_m = tiles_m;
  long long grid;
  if (a.mode == kGemm) {
    grid = (long long)tiles_m * tiles_n;
  } else {
    if (a.M != a.N) return MO_EINVAL;
    grid = (long long)tiles_m * (tiles_m + 1) / 2;
  }
  if (grid <= 0 || grid > 0x7fffffffLL) return MO_EINVAL;

  const bool ak = a.transA;   // op(A) stored K-major when A is transposed
  const bool bk = !a.transB;  // op(B) stored K-major when B is not transposed
  CUtensorMap ta, tb;
  const bool use_tma = !a.force_fallback && kp.K > 0 && gemm_tma_ok(a);
  if (use_tma) {
    bool okA = ak ? make_tmap(&ta, a.A, kp.K, a.M, a.lda, 16, 128)
                  : make_tmap(&ta, a.A, a.M, kp.K, a.lda, 16, 16);
    bool okB = bk ? make_tmap(&tb, a.B, kp.K, a.N, a.ldb, 16, 128)
                  : make_tmap(&tb, a.B, a.N, kp.K, a.ldb, 16, 16);
    if (okA && okB) return dispatch<true>(ak, bk, kp, ta, tb, (int)grid, stream);
  }
  memset(&ta, 0, sizeof(ta));
  memset(&tb, 0, sizeof(tb));
  return dispatch<false>(ak, bk, kp, ta, tb, (int)grid, stream);
}

}  // namespace mo
