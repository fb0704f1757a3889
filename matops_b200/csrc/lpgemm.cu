// Split-product GEMM on the 5th-generation tensor cores (tcgen05.mma with TMEM
// accumulators) for the mixed-precision Cholesky: C = beta*C + alpha * A * B^T with A, B
// stored pre-split (hi, lo) and K-major, each product formed as hi*hi + hi*lo + lo*hi
// with FP32 accumulation (BF16x3: kind::f16 with BF16 inputs; TF32x3: kind::tf32); see
// lp.cuh for the number format.
#include <cuda_bf16.h>

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "lp.cuh"

namespace mo {
namespace {

// Tile 128 x 128 of C per step of a persistent CTA; K consumed in stages of 128 bytes per
// operand row (64 bf16 or 32 tf32 elements), four 16 KB parts per stage (A.hi, A.lo,
// B.hi, B.lo) loaded by TMA with the 128-byte swizzle into a 2-deep ring.  Warp roles:
//   warp 0    TMA producer (one thread)
//   warp 1    TMEM owner (allocates 256 columns = two 128 x 128 FP32 accumulators) and
//             MMA issuer (one thread): per 32-byte K step three tcgen05.mma -- hi*hi,
//             hi*lo, lo*hi -- into the same accumulator; tcgen05.commit frees the smem
//             stage, and after the tile's last stage signals the epilogue
//   warps 2-9 epilogue: tcgen05.ld of their 32-lane quarter of the accumulator (TMEM lane
//             = tile row, quarter = warp % 4), C = alpha * acc + beta * C, coalesced along
//             the column; warps 2-5 take the tile's columns 0-63, warps 6-9 columns 64-127
// The accumulator is double-buffered, so the MMAs of tile t + 1 overlap the epilogue of
// tile t.  C (FP32, column-major) moves through shared memory in two 64-column halves,
// each with its own 32 KB buffer and its own four epilogue warps: the producer loads a
// half by TMA after the tile's operand stages, that half's warps combine it with the
// accumulator in place and one of their threads stores it back by TMA, so the two halves
// and their transfers proceed side by side (when C's base and leading dimension allow
// TMA; otherwise the epilogue reads and writes C directly).  Every wait is bounded
// (MO_SPIN_LIMIT) and reports MO_EDEVTIMEOUT.
constexpr int TB = 128;                  // tile rows = tile columns
constexpr int TSTAGES = 2;
constexpr int TPART = TB * 128;          // one operand part of a stage: 128 rows x 128 B
constexpr int TSTAGE = 4 * TPART;        // 64 KB
constexpr int TCTILE = TB * TB * 4;      // the C tile in shared memory (column-major FP32)
constexpr int TTHREADS = 320;
constexpr int TEPI_WARPS = 8;            // epilogue warps (2-9), four per 64-column half
constexpr int TSMEM = TSTAGES * TSTAGE + TCTILE + 1024 + 256;  // + alignment slack + barriers
constexpr int TMEM_COLS = 256;

struct TcParams {
  int M, N, K;
  float alpha, beta;
  float *C;
  int64_t ldc;
  int mode;
  int mt, nt;
  int ntiles;   // tiles in the schedule (lower mode: only those with tm >= tn)
  int kstages;  // ceil(K * esize / 128)
  int c_tma;    // C moves through shared memory by TMA (else plain loads and stores)
  int c_load;   // the C tile is read (beta != 0, or lower mode)
  char *shi, *slo;  // optional split copy of rows >= srow0 of the result (K-major)
  int64_t sldk;
  int srow0;
  int *status;
};

// tile index -> (tm, tn); lower mode enumerates tiles with tm >= tn column by column
__device__ __forceinline__ void tile_coords(const TcParams &p, int t, int &tm, int &tn) {
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

// UMMA shared-memory descriptor of a K-major operand with the 128-byte swizzle: start
// address >> 4, leading offset 1 (unused for swizzled K-major), stride between 8-row
// groups 1024 B, descriptor version 1, layout SWIZZLE_128B (2)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
         (2ull << 61);
}

// instruction descriptor: FP32 accumulator, A and B K-major, N = M = 128
template <int PREC>
__host__ __device__ constexpr uint32_t idesc() {
  return (1u << 4) | ((PREC == kLpBf16x3 ? 1u : 2u) << 7) | ((PREC == kLpBf16x3 ? 1u : 2u) << 10) |
         ((uint32_t)(TB >> 3) << 17) | ((uint32_t)(TB >> 4) << 24);
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

template <int PREC>
__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  if (PREC == kLpBf16x3)
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc<PREC>()), "r"(acc));
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc<PREC>()), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tma_store_2d(const void *tmap, const void *src, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(tmap),
      "r"(smem_u32(src)), "r"(x), "r"(y)
      : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

template <int PREC>
__global__ void __launch_bounds__(TTHREADS, 1)
    lp_gemm_tc_kernel(const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
                      const __grid_constant__ CUtensorMap tBh, const __grid_constant__ CUtensorMap tBl,
                      const __grid_constant__ CUtensorMap tC, const TcParams p) {
  extern __shared__ __align__(16) unsigned char tsm_raw[];
  // the swizzle pattern repeats every 1024 bytes: align the ring to it
  unsigned char *tsm = tsm_raw + ((1024 - (smem_u32(tsm_raw) & 1023)) & 1023);
  float *ctile = reinterpret_cast<float *>(tsm + TSTAGES * TSTAGE);
  uint64_t *full = reinterpret_cast<uint64_t *>(tsm + TSTAGES * TSTAGE + TCTILE);
  uint64_t *empty = full + TSTAGES;
  uint64_t *tfull = empty + TSTAGES;   // [2]
  uint64_t *tempty = tfull + 2;        // [2]
  // the C tile moves in two 64-column halves with their own buffers and barriers, so one
  // half's load or store overlaps the other half's epilogue
  uint64_t *cfull = tempty + 2;    // [2]
  uint64_t *cempty = cfull + 2;    // [2]
  uint64_t *cready = cempty + 2;   // [2] the four epilogue warps have written that half
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(cready + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < TSTAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], TEPI_WARPS);
    }
    for (int h = 0; h < 2; ++h) {
      mbar_init(&cfull[h], 1);
      mbar_init(&cempty[h], 1);
      mbar_init(&cready[h], 4);
    }
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  constexpr int ES = PREC == kLpBf16x3 ? 2 : 4;
  constexpr int KEL = 128 / ES;  // K elements per stage

  if (warp == 0 && lane == 0) {
    // producer: the operand stages of tile t, then (once the previous tile's C has been
    // stored) its C tile
    int g = 0, tc = 0, cu[2] = {0, 0};  // cu: uses of each C half buffer
    bool ok = true;
    for (int t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x, ++tc) {
      int tm, tn;
      tile_coords(p, t, tm, tn);
      for (int ks = 0; ks < p.kstages; ++ks, ++g) {
        const int slot = g % TSTAGES;
        const uint32_t ph = (g / TSTAGES) & 1;
        if (!mbar_wait(&empty[slot], ph ^ 1, p.status)) {
          ok = false;
          break;
        }
        unsigned char *st = tsm + slot * TSTAGE;
        mbar_arrive_expect_tx(&full[slot], TSTAGE);
        tma_load_2d(st, &tAh, &full[slot], ks * KEL, tm * TB);
        tma_load_2d(st + TPART, &tAl, &full[slot], ks * KEL, tm * TB);
        tma_load_2d(st + 2 * TPART, &tBh, &full[slot], ks * KEL, tn * TB);
        tma_load_2d(st + 3 * TPART, &tBl, &full[slot], ks * KEL, tn * TB);
      }
      if (!ok || !p.c_tma) continue;
      const int nh = tn * TB + TB / 2 < p.N ? 2 : 1;  // the second half only if it has columns
      for (int h = 0; h < nh; ++h) {
        if (!mbar_wait(&cempty[h], (cu[h] & 1) ^ 1, p.status)) {
          ok = false;
          break;
        }
        if (p.c_load) {
          mbar_arrive_expect_tx(&cfull[h], TCTILE / 2);
          tma_load_2d(ctile + h * TB * (TB / 2), &tC, &cfull[h], tm * TB, tn * TB + h * (TB / 2));
        } else {
          mbar_arrive(&cfull[h]);
        }
        ++cu[h];
      }
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    int g = 0, tc = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x, ++tc) {
      const int buf = tc & 1;
      if (!mbar_wait(&tempty[buf], ((tc >> 1) & 1) ^ 1, p.status)) break;
      tc_fence_after();
      const uint32_t d = tmem + buf * TB;
      for (int ks = 0; ks < p.kstages; ++ks, ++g) {
        const int slot = g % TSTAGES;
        if (!mbar_wait(&full[slot], (g / TSTAGES) & 1, p.status)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t base = smem_u32(tsm + slot * TSTAGE);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const uint64_t ah = sdesc(base + kk * 32), al = sdesc(base + TPART + kk * 32);
          const uint64_t bh = sdesc(base + 2 * TPART + kk * 32),
                         bl = sdesc(base + 3 * TPART + kk * 32);
          umma<PREC>(d, ah, bh, (ks | kk) != 0);
          umma<PREC>(d, ah, bl, 1);
          umma<PREC>(d, al, bh, 1);
        }
        umma_commit(&empty[slot]);
      }
      if (ok) umma_commit(&tfull[buf]);
    }
  } else if (warp >= 2) {
    // epilogue: warp w reads TMEM lanes 32 * (w % 4) .. + 31 (= tile rows) of the 64
    // columns of half h = (w - 2) / 4
    const int q = warp & 3;
    const int rl = q * 32 + lane;
    const int h = (warp - 2) >> 2;
    const bool storer = (warp - 2) % 4 == 0;  // warps 2 and 6: one thread stores the half
    float *const cb = ctile + h * TB * (TB / 2);  // this half: column-major 128 x 64
    int tc = 0, cu = 0;  // cu: uses of this half's buffer
    for (int t = blockIdx.x; t < p.ntiles; t += gridDim.x, ++tc) {
      int tm, tn;
      tile_coords(p, t, tm, tn);
      const int buf = tc & 1;
      if (!mbar_wait(&tfull[buf], (tc >> 1) & 1, p.status)) break;
      tc_fence_after();
      const int row = tm * TB + rl;
      // the second half exists only if the tile has columns there (the producer decides
      // the same way)
      const bool live = h == 0 || tn * TB + TB / 2 < p.N;
      if (p.c_tma) {
        bool fail = false;
        if (live) {
          if (!mbar_wait(&cfull[h], cu & 1, p.status)) break;
#pragma unroll 1
          for (int c0 = h * (TB / 2); c0 < (h + 1) * (TB / 2); c0 += 16) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + buf * TB + c0, v);
#pragma unroll
            for (int r = 0; r < 16; ++r) {
              const int col = tn * TB + c0 + r;
              float *cs = cb + (c0 - h * (TB / 2) + r) * TB + rl;
              const float a = p.alpha * __uint_as_float(v[r]);
              const float nv = p.beta == 0.f ? a : fmaf(p.beta, *cs, a);
              if (p.mode != kGemmLower || row >= col) *cs = nv;
            }
          }
        }
        // the accumulator has been read out (every epilogue warp arrives, live or not)
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty[buf]);
        if (!live) continue;
        // split copy of this thread's row (it wrote that row of the half itself)
        if (p.shi != nullptr && row < p.M && row >= p.srow0) {
          constexpr int ES = PREC == kLpBf16x3 ? 2 : 4;
          const int64_t obase = ((int64_t)(row - p.srow0) * p.sldk + tn * TB) * ES;
#pragma unroll 1
          for (int c0 = h * (TB / 2); c0 < (h + 1) * (TB / 2) && tn * TB + c0 < p.N; c0 += 8) {
            float x[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
              x[u] = tn * TB + c0 + u < p.N ? cb[(c0 - h * (TB / 2) + u) * TB + rl] : 0.f;
            if (PREC == kLpBf16x3) {
              __align__(16) __nv_bfloat16 hh[8], ll[8];
#pragma unroll
              for (int u = 0; u < 8; ++u) split_bf16(x[u], hh[u], ll[u]);
              *reinterpret_cast<uint4 *>(p.shi + obase + c0 * ES) = *reinterpret_cast<const uint4 *>(hh);
              *reinterpret_cast<uint4 *>(p.slo + obase + c0 * ES) = *reinterpret_cast<const uint4 *>(ll);
            } else {
              __align__(16) uint32_t hh[8], ll[8];
#pragma unroll
              for (int u = 0; u < 8; ++u) {
                hh[u] = to_tf32(x[u]);
                ll[u] = to_tf32(x[u] - __uint_as_float(hh[u]));
              }
#pragma unroll
              for (int v = 0; v < 2; ++v) {
                *reinterpret_cast<uint4 *>(p.shi + obase + (c0 + 4 * v) * ES) =
                    *reinterpret_cast<const uint4 *>(hh + 4 * v);
                *reinterpret_cast<uint4 *>(p.slo + obase + (c0 + 4 * v) * ES) =
                    *reinterpret_cast<const uint4 *>(ll + 4 * v);
              }
            }
          }
        }
        // this half's four warps' shared-memory writes, then one TMA store of the half
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&cready[h]);
        if (storer) {
          int ok = 1;
          if (lane == 0) {
            ok = mbar_wait(&cready[h], cu & 1, p.status) ? 1 : 0;
            if (ok) {
              tma_store_2d(&tC, cb, tm * TB, tn * TB + h * (TB / 2));
              mbar_arrive(&cempty[h]);
            }
          }
          if (!__shfl_sync(0xffffffffu, ok, 0)) fail = true;  // warp-uniform exit
        }
        ++cu;
        if (fail) break;
      } else {
        // C read and written in place: this warp's 64 columns
        const bool rok = row < p.M;
#pragma unroll 1
        for (int c0 = h * (TB / 2); c0 < (h + 1) * (TB / 2); c0 += 16) {
          float cv[16];
#pragma unroll
          for (int r = 0; r < 16; ++r) {
            const int col = tn * TB + c0 + r;
            cv[r] = (p.beta != 0.f && rok && col < p.N) ? p.C[row + (int64_t)col * p.ldc] : 0.f;
          }
          uint32_t v[16];
          tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + buf * TB + c0, v);
#pragma unroll
          for (int r = 0; r < 16; ++r) {
            const int col = tn * TB + c0 + r;
            if (rok && col < p.N && (p.mode != kGemmLower || row >= col))
              p.C[row + (int64_t)col * p.ldc] = fmaf(p.beta, cv[r], p.alpha * __uint_as_float(v[r]));
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty[buf]);
      }
    }
    // the last store of this half has been read out of shared memory; let it reach
    // global memory
    if (storer && lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------------------
// split: X (FP32 column-major) -> K-major hi/lo.  A CTA takes 64 rows x 32 columns,
// stages them transposed in shared memory and writes 8 consecutive k per thread and part.
// ---------------------------------------------------------------------------------------
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

PFN_cuTensorMapEncodeTiled_v12000 tc_encode_fn() {
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

// 2-D map over a K-major split operand: `rows` rows of K elements, `ldk` elements apart;
// box = 128 bytes of K x 128 rows, 128-byte swizzle; rows and K beyond the extents read 0
bool split_tmap(CUtensorMap *tm, const void *ptr, int prec, int64_t K, int64_t rows, int64_t ldk) {
  auto fn = tc_encode_fn();
  if (!fn) return false;
  const int es = lp_esize(prec);
  if (((uintptr_t)ptr & 15) || (ldk * es) % 16) return false;
  cuuint64_t dims[2] = {(cuuint64_t)std::max<int64_t>(K, 1), (cuuint64_t)std::max<int64_t>(rows, 1)};
  cuuint64_t strides[1] = {(cuuint64_t)(ldk * es)};
  cuuint32_t box[2] = {(cuuint32_t)(128 / es), (cuuint32_t)TB};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt =
      prec == kLpBf16x3 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(tm, dt, 2, const_cast<void *>(ptr), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// map over the FP32 column-major C: box 128 rows x 64 columns (half a tile), no swizzle
bool c_tmap(CUtensorMap *tm, float *C, int64_t M, int64_t N, int64_t ldc) {
  auto fn = tc_encode_fn();
  if (!fn) return false;
  if (((uintptr_t)C & 15) || (ldc * 4) % 16) return false;
  cuuint64_t dims[2] = {(cuuint64_t)std::max<int64_t>(M, 1), (cuuint64_t)std::max<int64_t>(N, 1)};
  cuuint64_t strides[1] = {(cuuint64_t)(ldc * 4)};
  cuuint32_t box[2] = {(cuuint32_t)TB, (cuuint32_t)(TB / 2)};  // one 64-column half
  cuuint32_t estr[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int PREC>
int launch_tc(mo_ctx *ctx, const CUtensorMap (&m)[5], const TcParams &p, int grid) {
  // set on every launch (a cheap host call), so that it holds after a context reset
  if (int rc = mo_smem_attr((const void *)lp_gemm_tc_kernel<PREC>, TSMEM)) return rc;
  lp_gemm_tc_kernel<PREC><<<grid, TTHREADS, TSMEM, ctx->stream>>>(m[0], m[1], m[2], m[3], m[4], p);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

}  // namespace

int lp_gemm(mo_ctx *ctx, int prec, const LpGemmArgs &a) {
  if (a.M <= 0 || a.N <= 0 || a.K <= 0) return MO_OK;
  // the split operands hold at least M (A) and N (B) rows of K elements, ldk apart,
  // K % 32 == 0; C is written only inside M x N
  if (a.K % 32) return MO_EINVAL;
  if (prec != kLpBf16x3 && prec != kLpTf32x3) return MO_EINVAL;
  const int es = lp_esize(prec);
  TcParams p;
  p.M = a.M;
  p.N = a.N;
  p.K = a.K;
  p.alpha = a.alpha;
  p.beta = a.beta;
  p.C = a.C;
  p.ldc = a.ldc;
  p.mode = a.mode == kGemmLower ? kGemmLower : kGemm;
  p.mt = (a.M + TB - 1) / TB;
  p.nt = (a.N + TB - 1) / TB;
  if (p.mode == kGemmLower && p.nt > p.mt) return MO_EINVAL;
  p.ntiles = p.mode == kGemmLower ? p.nt * p.mt - p.nt * (p.nt - 1) / 2 : p.mt * p.nt;
  p.kstages = (a.K * es + 127) / 128;
  p.status = &control(ctx)->status;
  CUtensorMap m[5];
  p.c_tma = c_tmap(&m[4], a.C, a.M, a.N, a.ldc) ? 1 : 0;
  if (!p.c_tma) m[4] = CUtensorMap{};
  p.c_load = (a.beta != 0.f || p.mode == kGemmLower) ? 1 : 0;
  p.shi = (char *)a.out.hi;
  p.slo = (char *)a.out.lo;
  p.sldk = a.out.ldk;
  p.srow0 = a.out_row0;
  if (p.shi && (!p.c_tma || a.out.ldk % 8 || a.N > a.out.ldk)) return MO_EINVAL;
  if (!split_tmap(&m[0], a.A.hi, prec, a.K, a.M, a.A.ldk) ||
      !split_tmap(&m[1], a.A.lo, prec, a.K, a.M, a.A.ldk) ||
      !split_tmap(&m[2], a.B.hi, prec, a.K, a.N, a.B.ldk) ||
      !split_tmap(&m[3], a.B.lo, prec, a.K, a.N, a.B.ldk))
    return MO_EINVAL;
  int grid = std::min(p.ntiles, ctx->sms);
  if (a.max_ctas > 0) grid = std::min(grid, a.max_ctas);
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_LPGEMM);
  const int rc = prec == kLpBf16x3 ? launch_tc<kLpBf16x3>(ctx, m, p, grid)
                                   : launch_tc<kLpTf32x3>(ctx, m, p, grid);
  // flops of the three products; bytes of C (read if beta != 0, written) and the operands
  const double tiles_flops = 3.0 * (double)p.ntiles * TB * TB * a.K * 2.0;
  prof_end(ctx, ps, tiles_flops,
           (double)p.ntiles * TB * TB * 4.0 * (a.beta != 0.f ? 2.0 : 1.0) +
               (double)(a.M + a.N) * a.K * es * 2.0 +
               (p.shi ? (double)std::max(0, a.M - a.out_row0) * a.N * es * 2.0 : 0.0));
  return rc;
}

int lp_split(mo_ctx *ctx, int prec, const float *X, int64_t ld, int rows, int cols,
             LpSplit out) {
  if (rows <= 0 || cols <= 0) return MO_OK;
  // groups of 8 columns: a partial last group writes zeros up to the next multiple of 8
  if (out.ldk % 8 || out.ldk < ((cols + 7) & ~7)) return MO_EINVAL;
  const dim3 grid((rows + 63) / 64, (cols + 31) / 32);
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_OTHER);
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
  prof_begin(ctx, ps, MO_PROF_OTHER);
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
