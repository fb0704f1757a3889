// QR factorization in the compact WY form and its applications (qrwy.go, qrwym.go,
// house.go): DecomposeQRT, BuildT, MultQT and SolveQRT on the device.
//
// Reference semantics: A (m x n) = Q R with Q = H(0) H(1) ... H(k-1), k = min(m, n),
// H(j) = I - tau_j v_j v_j^T (LAPACK dlarfg: v_j(j) = 1, beta = -sign(alpha) ||(alpha, x)||,
// tau = (beta - alpha) / beta, house.go:55-78), and Q = I - Y T Y^T with Y the unit lower
// trapezoid of the reflectors and T the k x k upper triangular block reflector built by
// the dlarft recurrence T(0:j, j) = -tau_j T(0:j, 0:j) Y(:, 0:j)^T v_j (qrwy.go:61-70,
// 121-129, 433-453).  A holds R on and above its diagonal and the reflectors below it.
//
// Device form, per 128-column block of A:
//   * four 32-column panels, each factored by ONE cooperative kernel: every CTA keeps a
//     slice of the panel's rows in shared memory; per column the CTAs publish their
//     partial products of the column with all panel columns (which give the norm below
//     the diagonal and, after the scaling, both the reflector's effect on the columns to
//     its right and the dlarft vector for the columns to its left), one grid barrier, and
//     every CTA reduces the partials in the same fixed order, so all of them hold the same
//     tau, beta and update row.  CTA 0 builds the panel's 32 x 32 T block.  The kernel also
//     writes the reflectors as an explicit unit lower trapezoid Y (zeros above) and the T
//     block with zeros below its diagonal, so that every later product is a plain GEMM;
//   * after each panel: the rest of the 128-column block takes the panel's reflectors
//     (W = C^T Y_p by a split-K kernel pair, W = W T_p, C -= Y_p W^T);
//   * after each block: its T (the four panel T blocks joined through Y_b^T Y_b by one CTA),
//     T's rows above it, -T(0:kb,0:kb) (Y(:,0:kb)^T Y_b) T_b, and the columns to its right
//     take Q_b^T in three products with K = 128 (W = C^T Y_b, W = W T_b, C -= Y_b W^T).
// The products run on the FP64 DMMA engine.  T is kept dense (zeros below the diagonal)
// in workspace and copied to the caller's upper triangle at the end.
//
// One deliberate difference: the reference's transposed matrix-vector product
// (calgo/dmvec_gemv.c:368-395) scales y by beta once per 68-row block of A instead of
// once, and unblockedQRT / BuildT call it with beta = -tau (qrwy.go:66, :125), so the
// reference's T is the dlarft T only while at most 68 rows lie below each column; with
// more rows its T, and in the blocked factorization the trailing updates that use it,
// differ from the LAPACK definitions that its documentation names (DGEQRT, DLARFT).
// This implementation computes the LAPACK quantities at every size (bit-for-bit the same
// algorithm as the reference wherever that GEMV takes one block).
#include <algorithm>

#include "context.cuh"

namespace mo {
namespace {

constexpr int kQrPanel = 32;    // columns of a Householder panel (one warp lane each)
constexpr int kQrBlock = 128;   // columns per trailing update (the K of its products)
constexpr int kQrThreads = 256;
constexpr int kQrRowsPerCta = 256;  // panel rows per CTA aimed at
constexpr int kQrMaxSmem = 220 * 1024;
constexpr int kQrApply = 256;   // reflectors per block when Q is applied to a matrix

struct QrScratch {
  double *part;        // [2][grid][32]: per-CTA column products, double-buffered by column
  double *prow;        // [2][32]: the pivot row's current values, published by its owner
  unsigned *bar;       // arrival counter of the grid barrier (zeroed before each launch)
  int *abort_flag;     // set by a CTA whose barrier wait gave up
};

// Bounded grid barrier over the co-resident CTAs of a cooperative launch.  Returns false
// (after recording MO_EDEVTIMEOUT, or when another CTA did) instead of waiting forever.
__device__ bool qr_grid_barrier(unsigned *counter, unsigned target, int *status,
                                int *abort_flag) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
    int ok = 1;
    for (unsigned i = 0;; ++i) {
      if (*(volatile unsigned *)counter >= target) break;
      if (*(volatile int *)abort_flag) {
        ok = 0;
        break;
      }
      if (i > MO_SPIN_LIMIT) {
        set_status(status, MO_EDEVTIMEOUT);
        atomicExch(abort_flag, 1);
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

// sqrt(x^2 + y^2) without needless overflow (house.go:18-32, LAPACK dlapy2)
__device__ __forceinline__ double qr_hypot(double x, double y) {
  const double xa = fabs(x), ya = fabs(y);
  double w = xa, z = xa;
  if (ya > w) w = ya;
  if (ya < z) z = ya;
  if (z == 0.0) return w;
  const double q = z / w;
  return w * sqrt(1.0 + q * q);
}

// Dynamic shared memory of the panel kernel for `rpc` rows per CTA.
__host__ __device__ constexpr size_t qr_panel_smem(int rpc) {
  return (size_t)kQrPanel * (rpc | 1) * sizeof(double) + 8 * 32 * sizeof(double);
}

// Factor the R x w panel P (w <= 32, column-major, ld ldp) in place: kmax = min(R, w)
// reflectors.  Writes Y (R x w, explicit unit lower trapezoid, zeros above) and Tb (w x w,
// the panel's T with zeros below the diagonal).  Grid: cooperative, rpc rows per CTA.
__global__ void __launch_bounds__(kQrThreads, 1)
    qr_panel_kernel(double *P, int64_t ldp, int R, int w, int rpc, double *Y, int64_t ldy,
                    double *Tb, int64_t ldt, QrScratch sc, int *status) {
  extern __shared__ double smem[];
  const int S = rpc | 1;  // odd column stride: lanes that read one row of 32 columns hit
                          // 32 different banks
  double *slab = smem;    // [w][S]
  double *red = smem + (size_t)kQrPanel * S;  // [8][32] per-warp partial sums
  __shared__ double s_w[32], s_z[32], s_t[32 * 33], s_scal[4];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = gridDim.x, cta = blockIdx.x;
  const int r0 = cta * rpc, nr = max(0, min(rpc, R - r0));
  const int kmax = min(R, w);

  for (int e = tid; e < w * rpc; e += kQrThreads) {
    const int c = e / rpc, r = e - c * rpc;
    slab[c * S + r] = r < nr ? P[(r0 + r) + (int64_t)c * ldp] : 0.0;
  }
  if (cta == 0)
    for (int e = tid; e < 32 * 33; e += kQrThreads) s_t[e] = 0.0;
  __syncthreads();

  // column products of column j with every panel column over this CTA's rows below row j
  // (q_j is the squared norm below the diagonal), and the pivot row from its owner
  auto publish = [&](int j) {
    const int par = j & 1;
    double acc0 = 0.0, acc1 = 0.0;
    const int lo = max(0, j + 1 - r0);
    if (lane < w) {
      const double *x = slab + j * S, *pc = slab + lane * S;
      int r = lo + warp;
      for (; r + 8 < nr; r += 16) {
        acc0 = fma(x[r], pc[r], acc0);
        acc1 = fma(x[r + 8], pc[r + 8], acc1);
      }
      if (r < nr) acc0 = fma(x[r], pc[r], acc0);
    }
    red[warp * 32 + lane] = acc0 + acc1;
    __syncthreads();
    if (tid < 32) {
      double s = 0.0;
#pragma unroll
      for (int g = 0; g < 8; ++g) s += red[g * 32 + tid];
      sc.part[((size_t)par * G + cta) * 32 + tid] = s;
      if (j >= r0 && j < r0 + nr) sc.prow[par * 32 + tid] = tid < w ? slab[tid * S + (j - r0)] : 0.0;
    }
  };

  if (kmax > 0) publish(0);
  for (int j = 0; j < kmax; ++j) {
    const int par = j & 1;
    if (!qr_grid_barrier(sc.bar, (unsigned)(j + 1) * G, status, sc.abort_flag)) return;
    // sum the CTAs' partials in one fixed order (every CTA gets the same values); warp 0
    // fetches the pivot row in the same round trip
    {
      double acc = 0.0;
      for (int g = warp; g < G; g += 8) acc += __ldcg(&sc.part[((size_t)par * G + g) * 32 + lane]);
      red[warp * 32 + lane] = acc;
    }
    const double prc = warp == 0 ? __ldcg(&sc.prow[par * 32 + lane]) : 0.0;
    __syncthreads();
    if (warp == 0) {
      double q = 0.0;
#pragma unroll
      for (int g = 0; g < 8; ++g) q += red[g * 32 + lane];
      // computeHouseholder (house.go:55-78) on [alpha; x] with ||x||^2 = q_j, in every lane
      const double s = __shfl_sync(0xffffffffu, q, j), alpha = __shfl_sync(0xffffffffu, prc, j);
      double tau = 0.0, denom = 1.0, beta = alpha;
      if (s != 0.0) {
        const double sign = signbit(alpha) ? -1.0 : 1.0;
        beta = -sign * qr_hypot(alpha, sqrt(s));
        denom = alpha - beta;
        tau = (beta - alpha) / beta;
      }
      // p_c = row j + v^T (rows below j) of column c, with v = x / denom
      const double p = lane < w ? prc + q / denom : 0.0;
      s_w[lane] = tau * p;   // applyHouseholder's w1 (columns right of j)
      s_z[lane] = -tau * p;  // the dlarft vector (columns left of j)
      if (lane == 0) {
        s_scal[0] = tau;
        s_scal[1] = denom;
        s_scal[2] = beta;
      }
    }
    __syncthreads();
    const double tau = s_scal[0], denom = s_scal[1], beta = s_scal[2];
    if (tau != 0.0) {
      // H(j) applied to this CTA's rows: v = x / denom, rows below j lose v_i w, row j
      // loses w and takes beta on the diagonal
      for (int r = tid; r < nr; r += kQrThreads) {
        const int i = r0 + r;
        if (i < j) continue;
        if (i == j) {
          for (int c = j + 1; c < w; ++c) slab[c * S + r] -= s_w[c];
          slab[j * S + r] = beta;
        } else {
          const double v = slab[j * S + r] / denom;
          slab[j * S + r] = v;
          for (int c = j + 1; c < w; ++c) slab[c * S + r] = fma(-v, s_w[c], slab[c * S + r]);
        }
      }
    }
    if (cta == 0 && tid < 32) {
      // T(0:j, j) = T(0:j, 0:j) z, T(j, j) = tau (zero column when tau == 0)
      double t = 0.0;
      if (tau != 0.0 && tid < j)
        for (int c = tid; c < j; ++c) t = fma(s_t[c * 33 + tid], s_z[c], t);
      __syncwarp();
      if (tid < j) s_t[j * 33 + tid] = t;
      if (tid == j) s_t[j * 33 + j] = tau;
    }
    __syncthreads();
    if (j + 1 < kmax) publish(j + 1);
  }
  __syncthreads();
  // write back: R and the reflectors into P, the explicit Y, the T block
  for (int e = tid; e < w * rpc; e += kQrThreads) {
    const int c = e / rpc, r = e - c * rpc;
    if (r >= nr) continue;
    const int i = r0 + r;
    const double v = slab[c * S + r];
    P[i + (int64_t)c * ldp] = v;
    Y[i + (int64_t)c * ldy] = i > c ? v : (i == c ? 1.0 : 0.0);
  }
  if (cta == 0)
    for (int e = tid; e < w * w; e += kQrThreads) {
      const int c = e / w, r = e - c * w;
      Tb[r + (int64_t)c * ldt] = r <= c ? s_t[c * 33 + r] : 0.0;
    }
}

// The 128-column block's T from its four 32 x 32 panel blocks (on the diagonal of Tb, ld
// ldt, zeros below) and the Gram matrix Zin = Y_b^T Y_b (ld ldz): for panel p the rows above
// it are T(0:32p, p) = -T(0:32p, 0:32p) Zin(0:32p, p) T_pp (qrwy.go:433-453 at panel
// granularity).  One CTA; the block lives in shared memory.
constexpr int kQrTBlockSmem = (128 * 129 + 96 * 33) * 8;
__global__ void __launch_bounds__(256) qr_t_block_kernel(double *Tb, int64_t ldt,
                                                         const double *Zin, int64_t ldz, int bo) {
  extern __shared__ double sm[];
  double *T = sm;               // [128][129], T(r, c) at c * 129 + r
  double *M1 = sm + 128 * 129;  // [32][33] x rows: M1(r, c) at c * 97 + r (r < 96)
  const int tid = threadIdx.x;
  for (int e = tid; e < bo * bo; e += 256) {
    const int c = e / bo, r = e - c * bo;
    T[c * 129 + r] = Tb[r + (int64_t)c * ldt];
  }
  __syncthreads();
  for (int p0 = kQrPanel; p0 < bo; p0 += kQrPanel) {
    const int w = min(kQrPanel, bo - p0), R = p0;
    // M1 = Zin(0:R, p0:p0+w) T(p0:p0+w, p0:p0+w)
    for (int e = tid; e < R * w; e += 256) {
      const int c = e / R, r = e - c * R;
      double acc = 0.0;
      for (int l = 0; l <= c; ++l)
        acc = fma(Zin[r + (int64_t)(p0 + l) * ldz], T[(p0 + c) * 129 + p0 + l], acc);
      M1[c * 97 + r] = acc;
    }
    __syncthreads();
    // T(0:R, p0:p0+w) = -T(0:R, 0:R) M1  (T upper triangular)
    for (int e = tid; e < R * w; e += 256) {
      const int c = e / R, r = e - c * R;
      double acc = 0.0;
      for (int l = r; l < R; ++l) acc = fma(T[l * 129 + r], M1[c * 97 + l], acc);
      T[(p0 + c) * 129 + r] = -acc;
    }
    __syncthreads();
  }
  for (int e = tid; e < bo * bo; e += 256) {
    const int c = e / bo, r = e - c * bo;
    if (r < (c / kQrPanel) * kQrPanel) Tb[r + (int64_t)c * ldt] = T[c * 129 + r];
  }
}

// Split-K product for a small C with a long K: C (M x N) = A^T B, A (K x M) and B (K x N)
// column-major.  Grid (chunks, tiles): each CTA multiplies one chunk of K rows for one
// 64 x 64 tile of C (16 x 16 threads, 4 x 4 outputs each, 32-row slabs staged in shared
// memory) and stores its partial tile; tn_reduce_kernel sums the chunks in order.  The
// engine would run such a product as one 128 x 128 tile whose K is split over ~100 CTAs
// and summed by one of them.
constexpr int kTnTile = 64, kTnSlab = 32;
__global__ void __launch_bounds__(256) tn_partial_kernel(const double *A, int64_t lda,
                                                         const double *B, int64_t ldb, int M,
                                                         int N, int K, int kc, double *part) {
  __shared__ double As[kTnSlab][kTnTile + 1], Bs[kTnSlab][kTnTile + 1];
  const int tiles_m = (M + kTnTile - 1) / kTnTile;
  const int tile = blockIdx.y, tm = tile % tiles_m, tn = tile / tiles_m;
  const int m0 = tm * kTnTile, n0 = tn * kTnTile;
  const int k_begin = blockIdx.x * kc, k_end = min(K, k_begin + kc);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[4][4] = {};
  for (int k0 = k_begin; k0 < k_end; k0 += kTnSlab) {
    // slab rows k0..k0+31 of A's columns m0.. and B's columns n0.. (zeros past the edges)
    for (int e = tid; e < kTnSlab * kTnTile; e += 256) {
      const int kk = e & (kTnSlab - 1), c = e / kTnSlab;
      const int k = k0 + kk;
      As[kk][c] = (k < k_end && m0 + c < M) ? A[k + (int64_t)(m0 + c) * lda] : 0.0;
      Bs[kk][c] = (k < k_end && n0 + c < N) ? B[k + (int64_t)(n0 + c) * ldb] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kTnSlab; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  double *out = part + ((size_t)blockIdx.x * gridDim.y + tile) * (kTnTile * kTnTile);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) out[(ty + 16 * i) + (tx + 16 * j) * kTnTile] = acc[i][j];
}

// C = alpha * (sum of the chunks' partial tiles, in chunk order) + beta * C (beta == 0: C
// not read)
__global__ void __launch_bounds__(256) tn_reduce_kernel(const double *part, int chunks, int tiles,
                                                        int M, int N, double *C, int64_t ldc,
                                                        double alpha, double beta) {
  const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (e >= (int64_t)M * N) return;
  const int i = (int)(e % M), j = (int)(e / M);
  const int tiles_m = (M + kTnTile - 1) / kTnTile;
  const int tile = (i / kTnTile) + (j / kTnTile) * tiles_m;
  const int off = (i % kTnTile) + (j % kTnTile) * kTnTile;
  double s = 0.0;
  for (int c = 0; c < chunks; ++c) s += part[((size_t)c * tiles + tile) * (kTnTile * kTnTile) + off];
  double *cp = C + i + (int64_t)j * ldc;
  *cp = beta == 0.0 ? alpha * s : fma(alpha, s, beta * *cp);
}

// Y (m x k) = the explicit unit lower trapezoid of A's reflectors (zeros above)
__global__ void __launch_bounds__(256) qr_expand_y_kernel(const double *A, int64_t lda, int m,
                                                          int k, double *Y, int64_t ldy) {
  const int i = blockIdx.x * 256 + threadIdx.x, c = blockIdx.y;
  if (i >= m || c >= k) return;
  Y[i + (int64_t)c * ldy] = i > c ? A[i + (int64_t)c * lda] : (i == c ? 1.0 : 0.0);
}

// Tw (k x k) = T's upper triangle with zeros below
__global__ void __launch_bounds__(256) qr_expand_t_kernel(const double *T, int64_t ldt, int k,
                                                          double *Tw, int64_t ldw) {
  const int i = blockIdx.x * 256 + threadIdx.x, c = blockIdx.y;
  if (i >= k || c >= k) return;
  Tw[i + (int64_t)c * ldw] = i <= c ? T[i + (int64_t)c * ldt] : 0.0;
}

// T's upper triangle (k x k) <- Tw; with tau, columns whose tau is zero are left as they
// are (qrwy.go:60 writes nothing for them)
__global__ void __launch_bounds__(256) qr_t_out_kernel(const double *Tw, int64_t ldw, int k,
                                                       double *T, int64_t ldt, const double *tau) {
  const int i = blockIdx.x * 256 + threadIdx.x, c = blockIdx.y;
  if (i >= k || c >= k || i > c) return;
  if (tau && tau[c] == 0.0) return;
  T[i + (int64_t)c * ldt] = Tw[i + (int64_t)c * ldw];
}

// BuildT's diagonal blocks: for each 32-column panel p (one CTA), T_p from the panel's Gram
// matrix Gm = Y_p^T Y_p (in Tw's block, overwritten) and tau: column j is
// T_p(0:j, j) = T_p(0:j, 0:j) (-tau_j Gm(0:j, j)), T_p(j, j) = tau_j (qrwy.go:29-84)
__global__ void __launch_bounds__(32) qr_buildt_diag_kernel(double *Tw, int64_t ldw, int k,
                                                            const double *tau) {
  __shared__ double s_t[32 * 33], s_z[32];
  const int p0 = blockIdx.x * kQrPanel, w = min(kQrPanel, k - p0), lane = threadIdx.x;
  double *B = Tw + p0 + (int64_t)p0 * ldw;
  for (int c = 0; c < 32; ++c) s_t[c * 33 + lane] = 0.0;
  __syncwarp();
  for (int j = 0; j < w; ++j) {
    const double tj = tau[p0 + j];
    if (lane < j) s_z[lane] = -tj * B[lane + (int64_t)j * ldw];
    __syncwarp();
    double t = 0.0;
    if (tj != 0.0 && lane < j)
      for (int c = lane; c < j; ++c) t = fma(s_t[c * 33 + lane], s_z[c], t);
    __syncwarp();
    if (lane < j) s_t[j * 33 + lane] = t;
    if (lane == j) s_t[j * 33 + j] = tj;
    __syncwarp();
  }
  for (int c = 0; c < w; ++c)
    if (lane < w) B[lane + (int64_t)c * ldw] = lane <= c ? s_t[c * 33 + lane] : 0.0;
}

// rows i >= r0 of the columns of B (rows x cols, ld) set to zero
__global__ void __launch_bounds__(256) qr_zero_rows_kernel(double *B, int64_t ld, int r0,
                                                           int rows) {
  const int i = r0 + blockIdx.x * 256 + threadIdx.x, c = blockIdx.y;
  if (i < rows) B[i + (int64_t)c * ld] = 0.0;
}

// one thread per element of an rows x cols grid (cols <= 65535)
template <typename F>
int launch_grid2(int rows, int cols, F &&launch) {
  if (rows <= 0 || cols <= 0) return MO_OK;
  launch(dim3((rows + 255) / 256, cols));
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

constexpr int kQrMaxCols = 65535;  // reflectors per call (one grid row of columns)

struct QrWork {
  double *Y = nullptr;   // m x k explicit reflectors (ld m)
  double *Tw = nullptr;  // k x k dense T, zeros below the diagonal (ld k)
  double *W = nullptr;   // products' scratch, wsize doubles each
  double *W2 = nullptr;
  double *Z = nullptr;   // k x 128
  double *X = nullptr;   // k x 128
  QrScratch sc{};
};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// bytes of the buffers below (panel scratch for `grid` CTAs)
size_t qr_workspace_bytes(int m, int k, int64_t wsize, int grid) {
  const size_t by = align256((size_t)m * k * 8), bt = align256((size_t)k * k * 8);
  const size_t bw = align256((size_t)wsize * 8), bz = align256((size_t)k * kQrBlock * 8);
  const size_t bp = align256((size_t)2 * grid * 32 * 8), br = align256(2 * 32 * 8);
  return by + bt + 2 * bw + 2 * bz + bp + br + 256;
}

// Carve the context workspace into the buffers above (panel scratch for `grid` CTAs).
int qr_workspace(mo_ctx *ctx, int m, int k, int64_t wsize, int grid, QrWork &q) {
  const size_t by = align256((size_t)m * k * 8), bt = align256((size_t)k * k * 8);
  const size_t bw = align256((size_t)wsize * 8), bz = align256((size_t)k * kQrBlock * 8);
  const size_t bp = align256((size_t)2 * grid * 32 * 8), br = align256(2 * 32 * 8);
  char *ws = nullptr;
  int rc = workspace(ctx, qr_workspace_bytes(m, k, wsize, grid), (void **)&ws);
  if (rc) return rc;
  q.Y = (double *)ws;
  ws += by;
  q.Tw = (double *)ws;
  ws += bt;
  q.W = (double *)ws;
  ws += bw;
  q.W2 = (double *)ws;
  ws += bw;
  q.Z = (double *)ws;
  ws += bz;
  q.X = (double *)ws;
  ws += bz;
  q.sc.part = (double *)ws;
  ws += bp;
  q.sc.prow = (double *)ws;
  ws += br;
  q.sc.bar = (unsigned *)ws;
  q.sc.abort_flag = (int *)(ws + 64);
  return MO_OK;
}

// CTAs and rows per CTA of the panel kernel for R rows
void panel_shape(mo_ctx *ctx, int R, int &grid, int &rpc) {
  grid = max(1, min(ctx->sms, (R + kQrRowsPerCta - 1) / kQrRowsPerCta));
  rpc = (R + grid - 1) / grid;
}

// the most rows a panel may have: every CTA's slice must fit in shared memory
int max_panel_rows(mo_ctx *ctx) {
  const int rpc = (int)((kQrMaxSmem - 8 * 32 * 8) / (kQrPanel * 8)) - 1;
  return rpc * ctx->sms;
}

// factor A[kp:m, kp:kp+bp]; its reflectors go to Y's and its T block to Tw's columns kp..
int panel(mo_ctx *ctx, View A, int kp, int bp, QrWork &q, int k) {
  const int m = A.rows, R = m - kp;
  int grid = 0, rpc = 0;
  panel_shape(ctx, R, grid, rpc);
  const size_t smem = qr_panel_smem(rpc);
  if (smem > (size_t)kQrMaxSmem) return MO_EINVAL;
  int rc = mo_smem_attr((const void *)qr_panel_kernel, (int)smem);
  if (rc) return rc;
  MO_CUDA_TRY(cudaMemsetAsync(q.sc.bar, 0, 128, ctx->stream));
  double *P = A.at(kp, kp);
  int64_t ldp = A.ld;
  int w = bp;
  double *Y = q.Y + kp + (int64_t)kp * m;
  int64_t ldy = m;
  double *Tb = q.Tw + kp + (int64_t)kp * k;
  int64_t ldt = k;
  QrScratch sc = q.sc;
  int *status = &control(ctx)->status;
  void *args[] = {&P, &ldp, (void *)&R, &w, &rpc, &Y, &ldy, &Tb, &ldt, &sc, &status};
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_PANEL);
  MO_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)qr_panel_kernel, dim3(grid),
                                          dim3(kQrThreads), args, smem, ctx->stream));
  prof_end(ctx, ps, 4.0 * R * (double)bp * bp, 8.0 * 3 * R * (double)bp);
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// T(0:kp, kp:kp+bp) = -T(0:kp, 0:kp) Z T(kp:kp+bp, kp:kp+bp) with Z = Y(:, 0:kp)^T
// Y(:, kp:kp+bp) (qrwy.go:433-453); Z is read from Zsrc (kp x bp, ld ldz), which may be T's
// own block (BuildT) because the result goes through X first
int t_columns(mo_ctx *ctx, int k, int kp, int bp, View Zsrc, QrWork &q) {
  if (kp == 0) return MO_OK;
  const View Tv{q.Tw, k, k, k}, Xv{q.X, kp, bp, kp};
  int rc = gemm(ctx, Xv, Zsrc, false, Tv.sub(kp, kp, bp, bp), false, 1.0, 0.0);
  if (!rc) rc = gemm(ctx, Tv.sub(0, kp, kp, bp), Tv.sub(0, 0, kp, kp), false, Xv, false, -1.0, 0.0);
  return rc;
}

// C = alpha * A^T B + beta * C: split-K kernels when C is small and K long, else the
// engine (its stream-K scratch doubles as the partial-tile buffer: same stream, in order)
int tn_product(mo_ctx *ctx, View C, View A, View B, double alpha, double beta) {
  const int M = C.rows, N = C.cols, K = A.rows;
  if (M <= 0 || N <= 0) return MO_OK;
  const int tiles = ((M + kTnTile - 1) / kTnTile) * ((N + kTnTile - 1) / kTnTile);
  const size_t cap = gemm_partial_bytes(ctx->sms) / sizeof(double) / (kTnTile * kTnTile);
  if (K < 1024 || tiles > 16 || K <= 0) return gemm(ctx, C, A, true, B, false, alpha, beta);
  double *part = ctx->sk_partial;
  // chunks of at least 128 rows, about two CTAs per SM, within the partial buffer
  int chunks = std::max(1, std::min<int>(K / 128, (2 * ctx->sms + tiles - 1) / tiles));
  chunks = std::min<int>(chunks, (int)(cap / tiles));
  const int kc = ((K + chunks - 1) / chunks + kTnSlab - 1) / kTnSlab * kTnSlab;
  chunks = (K + kc - 1) / kc;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_GEMM);
  tn_partial_kernel<<<dim3(chunks, tiles), 256, 0, ctx->stream>>>(A.d, A.ld, B.d, B.ld, M, N, K,
                                                                    kc, part);
  const int64_t mn = (int64_t)M * N;
  tn_reduce_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, ctx->stream>>>(
      part, chunks, tiles, M, N, C.d, C.ld, alpha, beta);
  prof_end(ctx, ps, 2.0 * M * N * (double)K, 8.0 * ((double)K * (M + N) + 2.0 * M * N));
  MO_CUDA_TRY(cudaGetLastError());
  return MO_OK;
}

// C (rows s.. of A's columns right of a block) = Q_b^T C for the block's reflectors:
// W = C^T Y_b, W = W T_b, C -= Y_b W^T (qrwy.go:266-303 with transpose)
int apply_left_t(mo_ctx *ctx, View C, const View &Yb, const View &Tb, QrWork &q) {
  const int nc = C.cols, b = Yb.cols;
  if (nc <= 0 || b <= 0) return MO_OK;
  const View W{q.W, nc, b, nc}, W2{q.W2, nc, b, nc};
  int rc = tn_product(ctx, W, C, Yb, 1.0, 0.0);
  if (!rc) rc = gemm(ctx, W2, W, false, Tb, false, 1.0, 0.0);
  if (!rc) rc = gemm(ctx, C, Yb, false, W2, true, -1.0, 1.0);
  return rc;
}

int t_out(mo_ctx *ctx, const QrWork &q, int k, View T, const double *tau_mask) {
  return launch_grid2(k, k, [&](dim3 g) {
    qr_t_out_kernel<<<g, 256, 0, ctx->stream>>>(q.Tw, k, k, T.d, T.ld, tau_mask);
  });
}

// tau (k entries, stride) <- T's diagonal
__global__ void qr_tau_out_kernel(const double *Tw, int64_t ldw, int k, double *tau,
                                  int64_t inc) {
  const int j = blockIdx.x * 256 + threadIdx.x;
  if (j < k) tau[j * inc] = Tw[j + (int64_t)j * ldw];
}

// tau (k entries, stride) -> a contiguous copy
__global__ void qr_tau_in_kernel(const double *tau, int64_t inc, int k, double *out) {
  const int j = blockIdx.x * 256 + threadIdx.x;
  if (j < k) out[j] = tau[j * inc];
}

}  // namespace

// One 128-column block [kb, kb + bo): its 32-column panels, the rest of the block after each
// panel, the block's T (the panels' T blocks joined through Y_b^T Y_b) and T's rows above
// it, all on the context's stream.
int factor_block(mo_ctx *ctx, View A, int kb, int bo, int k, QrWork &q) {
  const int m = A.rows;
  const View Yv{q.Y, m, k, m}, Tv{q.Tw, k, k, k};
  int rc;
  for (int kp = kb; kp < kb + bo; kp += kQrPanel) {
    const int bp = min(kQrPanel, kb + bo - kp);
    if ((rc = panel(ctx, A, kp, bp, q, k))) return rc;
    // the rest of the block takes the panel's reflectors
    const int c0 = kp + bp, rest = kb + bo - c0;
    if (rest > 0 &&
        (rc = apply_left_t(ctx, A.sub(kp, c0, m - kp, rest), Yv.sub(kp, kp, m - kp, bp),
                           Tv.sub(kp, kp, bp, bp), q)))
      return rc;
  }
  const View Yb = Yv.sub(kb, kb, m - kb, bo), Tb = Tv.sub(kb, kb, bo, bo);
  if (bo > kQrPanel) {
    const View Zin{q.W2, bo, bo, bo};
    if ((rc = tn_product(ctx, Zin, Yb, Yb, 1.0, 0.0))) return rc;
    if ((rc = mo_smem_attr((const void *)qr_t_block_kernel, kQrTBlockSmem))) return rc;
    qr_t_block_kernel<<<1, 256, kQrTBlockSmem, ctx->stream>>>(Tb.d, k, q.W2, bo, bo);
    MO_CUDA_TRY(cudaGetLastError());
  }
  if (kb > 0) {
    // T's rows above the block: -T(0:kb, 0:kb) (Y(kb:m, 0:kb)^T Y_b) T_b
    const View Z{q.Z, kb, bo, kb};
    if ((rc = tn_product(ctx, Z, Yv.sub(kb, 0, m - kb, kb), Yb, 1.0, 0.0))) return rc;
    if ((rc = t_columns(ctx, k, kb, bo, Z, q))) return rc;
  }
  return MO_OK;
}

// The device part of DecomposeQRT / DecomposeQR: A (m x n) factored in place; T's upper
// k x k triangle written when T.d, tau (k entries, stride tau_inc) when tau.  (Factoring
// the next block on a second stream beside the trailing update was measured slower: the
// update then runs without the panel's SMs and the T products without stream-K.)
int qr_factor(mo_ctx *ctx, View A, View T, double *tau, int64_t tau_inc) {
  const int m = A.rows, n = A.cols, k = min(m, n);
  if (k == 0) return MO_OK;
  if (m > max_panel_rows(ctx) || k > kQrMaxCols) return MO_EINVAL;
  int grid = 0, rpc = 0;
  panel_shape(ctx, m, grid, rpc);
  QrWork q;
  int rc = qr_workspace(ctx, m, k, (int64_t)max(n, 1) * kQrBlock, grid, q);
  if (rc) return rc;
  const View Yv{q.Y, m, k, m}, Tv{q.Tw, k, k, k};
  // the products read T's blocks below the diagonal and Y's rows above each panel inside
  // a 128-column block as zeros (the panels write only their own rows and T blocks)
  MO_CUDA_TRY(cudaMemsetAsync(q.Tw, 0, (size_t)k * k * sizeof(double), ctx->stream));
  MO_CUDA_TRY(cudaMemsetAsync(q.Y, 0, (size_t)m * k * sizeof(double), ctx->stream));
  for (int kb = 0; kb < k; kb += kQrBlock) {
    const int bo = min(kQrBlock, k - kb);
    if ((rc = factor_block(ctx, A, kb, bo, k, q))) return rc;
    const int c0 = kb + bo, nt = n - c0;
    if (nt > 0 && (rc = apply_left_t(ctx, A.sub(kb, c0, m - kb, nt), Yv.sub(kb, kb, m - kb, bo),
                                     Tv.sub(kb, kb, bo, bo), q)))
      return rc;
  }
  if (T.d && (rc = t_out(ctx, q, k, T, nullptr))) return rc;
  if (tau) {
    qr_tau_out_kernel<<<(k + 255) / 256, 256, 0, ctx->stream>>>(q.Tw, k, k, tau, tau_inc);
    MO_CUDA_TRY(cudaGetLastError());
  }
  return MO_OK;
}

// The dense block reflector of A's first k reflectors and tau into q.Tw (BuildT,
// qrwy.go:29-84): Tw = the upper triangle of Y^T Y, each 32 x 32 diagonal block replaced by
// its dlarft recurrence, then the blocks above the diagonal by t_columns in column order.
// q.Y must hold the expanded reflectors.
int qr_build_t(mo_ctx *ctx, int m, int k, const double *tau_c, QrWork &q) {
  const View Yv{q.Y, m, k, m}, Tv{q.Tw, k, k, k};
  MO_CUDA_TRY(cudaMemsetAsync(q.Tw, 0, (size_t)k * k * 8, ctx->stream));
  int rc = syrk(ctx, Tv, Yv, true, true, 1.0, 0.0, 0);
  if (rc) return rc;
  qr_buildt_diag_kernel<<<(k + kQrPanel - 1) / kQrPanel, 32, 0, ctx->stream>>>(q.Tw, k, k, tau_c);
  MO_CUDA_TRY(cudaGetLastError());
  for (int kp = kQrPanel; kp < k; kp += kQrPanel) {
    const int bp = min(kQrPanel, k - kp);
    if ((rc = t_columns(ctx, k, kp, bp, Tv.sub(0, kp, kp, bp), q))) return rc;
  }
  return MO_OK;
}

// C = Q C, Q^T C (MO_TRANS), C Q (MO_RIGHT), C Q^T (MO_RIGHT|MO_TRANS) with Q = I - Y T Y^T
// of k reflectors (q.Y, q.Tw), in blocks of nb reflectors in the order qrwym.go:382-566
// takes them: forward for Q^T C and C Q, backward (aligned at k) for Q C and C Q^T.  Each
// block reads only its reflectors' rows s..m, so blocks of a few hundred reflectors take
// about a third of the flops of one block of all k (which multiplies the zeros above Y's
// diagonal and the whole of T).
int qr_apply(mo_ctx *ctx, View C, int m, int k, int flags, int nb, QrWork &q) {
  const bool right = (flags & MO_RIGHT) != 0, trans = (flags & MO_TRANS) != 0;
  const bool forward = right ? !trans : trans;
  const View Yv{q.Y, m, k, m}, Tv{q.Tw, k, k, k};
  int rc = MO_OK;
  auto block = [&](int s, int b) -> int {
    const View Yb = Yv.sub(s, s, m - s, b), Tb = Tv.sub(s, s, b, b);
    if (!right) {
      const int nc = C.cols;
      const View Cs = C.sub(s, 0, m - s, nc), W{q.W, nc, b, nc}, W2{q.W2, nc, b, nc};
      int r = tn_product(ctx, W, Cs, Yb, 1.0, 0.0);
      if (!r) r = gemm(ctx, W2, W, false, Tb, !trans, 1.0, 0.0);
      if (!r) r = gemm(ctx, Cs, Yb, false, W2, true, -1.0, 1.0);
      return r;
    }
    const int nr = C.rows;
    const View Cs = C.sub(0, s, nr, m - s), W{q.W, nr, b, nr}, W2{q.W2, nr, b, nr};
    int r = gemm(ctx, W, Cs, false, Yb, false, 1.0, 0.0);
    if (!r) r = gemm(ctx, W2, W, false, Tb, trans, 1.0, 0.0);
    if (!r) r = gemm(ctx, Cs, W2, false, Yb, true, -1.0, 1.0);
    return r;
  };
  if (forward) {
    for (int s = 0; s < k && !rc; s += nb) rc = block(s, min(nb, k - s));
  } else {
    for (int e = k; e > 0 && !rc; e -= nb) {
      const int b = min(nb, e);
      rc = block(e - b, b);
    }
  }
  return rc;
}

// expand A's reflectors (and, when T.d, T's upper triangle) into q for k reflectors, with
// W buffers of wsize doubles
int qr_prepare(mo_ctx *ctx, View A, int k, View T, int64_t wsize, QrWork &q) {
  const int m = A.rows;
  int rc = qr_workspace(ctx, m, k, wsize, 1, q);
  if (rc) return rc;
  if ((rc = launch_grid2(m, k, [&](dim3 g) {
         qr_expand_y_kernel<<<g, 256, 0, ctx->stream>>>(A.d, A.ld, m, k, q.Y, m);
       })))
    return rc;
  if (T.d)
    rc = launch_grid2(k, k, [&](dim3 g) {
      qr_expand_t_kernel<<<g, 256, 0, ctx->stream>>>(T.d, T.ld, k, q.Tw, k);
    });
  return rc;
}

// contiguous copy of tau (k entries, stride inc)
void qr_tau_copy(mo_ctx *ctx, const double *tau, int64_t inc, int k, double *out) {
  qr_tau_in_kernel<<<(k + 255) / 256, 256, 0, ctx->stream>>>(tau, inc, k, out);
}

// T's upper triangle <- q.Tw, columns with tau == 0 left untouched
int qr_t_store(mo_ctx *ctx, const QrWork &q, int k, View T, const double *tau_c) {
  return t_out(ctx, q, k, T, tau_c);
}

// rows r0.. of B set to zero
void qr_zero_rows(mo_ctx *ctx, View B, int r0) {
  if (B.rows <= r0 || B.cols <= 0) return;
  for (int c0 = 0; c0 < B.cols; c0 += 65535) {
    const dim3 g((B.rows - r0 + 255) / 256, std::min(65535, B.cols - c0));
    qr_zero_rows_kernel<<<g, 256, 0, ctx->stream>>>(B.at(0, c0), B.ld, r0, B.rows);
  }
}

// A (m x n) := the first n columns of the identity
__global__ void __launch_bounds__(256) qr_eye_kernel(double *A, int64_t lda, int m) {
  const int i = blockIdx.x * 256 + threadIdx.x, c = blockIdx.y;
  if (i < m) A[i + (int64_t)c * lda] = i == c ? 1.0 : 0.0;
}

// BuildQ / BuildQT's device part: A (m x n, m >= n) := Q [I_n; 0] with Q from A's n
// reflectors and T (or tau)
int qr_build_q(mo_ctx *ctx, View A, View T, const double *tau, int64_t tau_inc) {
  const int m = A.rows, n = A.cols;
  if (n == 0 || m == 0) return MO_OK;
  if (n > kQrMaxCols) return MO_EINVAL;
  const int b = std::min(kQrApply, n);
  QrWork q;
  int rc = qr_prepare(ctx, A, n, T, std::max((int64_t)n * b, (int64_t)n), q);
  if (rc) return rc;
  if (!T.d) {
    qr_tau_copy(ctx, tau, tau_inc, n, q.W2);
    if ((rc = qr_build_t(ctx, m, n, q.W2, q))) return rc;
  }
  if ((rc = launch_grid2(m, n, [&](dim3 g) {
         qr_eye_kernel<<<g, 256, 0, ctx->stream>>>(A.d, A.ld, m);
       })))
    return rc;
  return qr_apply(ctx, A, m, n, MO_LEFT, b, q);
}

}  // namespace mo

using mo::View;

namespace {

// W as the reference's optional workspace: data == NULL stands for a nil matrix
bool is_nil(const mo_matrix &W) { return W.data == nullptr; }

// tau as a column vector view of at least k entries: pointer and stride
int tau_view(const mo_matrix &tau, int k, double **p, int64_t *inc) {
  if (tau.rows < 0 || tau.cols < 0) return MO_EINVAL;
  const int64_t len = tau.rows * tau.cols;
  if (len < k || (tau.rows != 1 && tau.cols != 1 && k > 0)) return MO_EINVAL;
  if (k > 0 && !tau.data) return MO_EINVAL;
  *p = tau.data;
  *inc = tau.cols == 1 ? 1 : tau.ld;  // a row vector steps by its leading index
  return MO_OK;
}

// the checks of MultQT / MultQ (qrwym.go:646-671, 573-600) shared by both
int mult_checks(const View &C, const View &A, const mo_matrix &Wm, int flags, int nb,
                bool need_w) {
  if (need_w && is_nil(Wm)) return MO_ENOWORK;
  if (flags & MO_RIGHT) {
    if (C.cols != A.rows) return MO_ECQSIZE;
    if (need_w && (Wm.cols < nb || Wm.rows < C.rows)) return MO_EWORKSMALL;
  } else {
    if (need_w && (Wm.cols < nb || Wm.rows < C.cols)) return MO_EWORKSMALL;
    // the reference leaves this unchecked and then updates with mismatched operands
    if (C.rows != A.rows && C.rows > 0 && C.cols > 0) return MO_EABSIZE;
  }
  return MO_OK;
}

int apply_q(mo_ctx *ctx, View C, View A, View T, const double *tau, int64_t tau_inc, int flags,
            int nb) {
  const int m = A.rows, k = std::min(A.rows, A.cols);
  if (k == 0 || C.rows == 0 || C.cols == 0) return MO_OK;
  if (k > 65535) return MO_EINVAL;
  // the device's own blocking (results agree with any nb to rounding)
  nb = std::min(mo::kQrApply, k);
  const int64_t wsize = std::max((int64_t)std::max(C.rows, C.cols) * nb, (int64_t)k);
  mo::QrWork q;
  int rc = mo::qr_prepare(ctx, A, k, T, wsize, q);
  if (rc) return rc;
  if (!T.d) {
    double *tc = q.W2;  // contiguous tau, consumed by qr_build_t before W2 is used
    mo::qr_tau_copy(ctx, tau, tau_inc, k, tc);
    if ((rc = mo::qr_build_t(ctx, m, k, tc, q))) return rc;
  }
  return mo::qr_apply(ctx, C, m, k, flags, nb, q);
}

// SolveQRT / SolveQR (qrwym.go:784-819, 717-760) on Q from (T) or (tau)
int solve_q(mo_ctx *ctx, View B, View A, View T, const double *tau, int64_t tau_inc,
            const mo_matrix &Wm, int flags, int nb, bool need_w) {
  const int n = A.cols;
  if (A.rows < n || B.rows < n) return MO_EABSIZE;
  const View R = A.sub(0, 0, n, n), BT = B.sub(0, 0, n, B.cols);
  int rc;
  if (flags & MO_TRANS) {
    // minimum-norm solution of A^T X = B: B' = R^-T B, rows below n cleared, X = Q B'
    if ((rc = mult_checks(B, A, Wm, MO_LEFT, nb, need_w))) return rc;
    if ((rc = mo::trsm(ctx, BT, R, MO_LEFT | MO_UPPER | MO_TRANSA, 1.0))) return rc;
    if (B.rows > n) {
      mo::qr_zero_rows(ctx, B, n);
    }
    return apply_q(ctx, B, A, T, tau, tau_inc, MO_LEFT, nb);
  }
  // least squares min ||A X - B||: B' = Q^T B, X = R^-1 B'(0:n)
  if ((rc = mult_checks(B, A, Wm, MO_LEFT | MO_TRANS, nb, need_w))) return rc;
  if ((rc = apply_q(ctx, B, A, T, tau, tau_inc, MO_LEFT | MO_TRANS, nb))) return rc;
  return mo::trsm(ctx, BT, R, MO_LEFT | MO_UPPER, 1.0);
}

}  // namespace

extern "C" {

// qrwy.go:517-538
int mo_decompose_qrt(mo_ctx *ctx, mo_matrix Am, mo_matrix Tm, mo_matrix Wm, int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A, T;
  if ((rc = mo::to_view(Am, A)) || (rc = mo::to_view(Tm, T))) return rc;
  if (!(nb == 0 || A.cols <= nb) && !is_nil(Wm) && (Wm.cols < nb || Wm.rows < A.cols))
    return MO_EWORKSMALL;
  const int k = std::min(A.rows, A.cols);
  if (T.rows < k || T.cols < k) return MO_ETSMALL;
  if (k > 0 && !T.d) return MO_EINVAL;
  return mo::qr_factor(ctx, A, T, nullptr, 0);
}

// qrwy.go:474-497
int mo_decompose_qr(mo_ctx *ctx, mo_matrix Am, mo_matrix taum, mo_matrix Wm, int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A;
  if ((rc = mo::to_view(Am, A))) return rc;
  const int k = std::min(A.rows, A.cols);
  double *tau = nullptr;
  int64_t inc = 1;
  if ((rc = tau_view(taum, k, &tau, &inc))) return rc;
  if (!(nb == 0 || A.cols <= nb) && !is_nil(Wm) && (Wm.cols < nb || Wm.rows < A.cols))
    return MO_EWORKSMALL;
  return mo::qr_factor(ctx, A, View{nullptr, 0, 0, 1}, tau, inc);
}

// qrwy.go:546-556
int mo_build_t(mo_ctx *ctx, mo_matrix Tm, mo_matrix Am, mo_matrix taum) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View T, A;
  if ((rc = mo::to_view(Tm, T)) || (rc = mo::to_view(Am, A))) return rc;
  if (T.cols < A.cols || T.rows < A.cols) return MO_ETSMALL;
  const int m = A.rows;
  int k = std::min(A.rows, A.cols);
  double *tau = nullptr;
  int64_t inc = 1;
  if (taum.rows * taum.cols < k) k = (int)(taum.rows * taum.cols);
  if ((rc = tau_view(taum, k, &tau, &inc))) return rc;
  if (k == 0) return MO_OK;
  if (k > 65535) return MO_EINVAL;
  mo::QrWork q;
  if ((rc = mo::qr_prepare(ctx, A, k, View{nullptr, 0, 0, 1}, k, q))) return rc;
  double *tc = q.W2;
  mo::qr_tau_copy(ctx, tau, inc, k, tc);
  if ((rc = mo::qr_build_t(ctx, m, k, tc, q))) return rc;
  return mo::qr_t_store(ctx, q, k, T, tc);
}

// qrwym.go:646-688
int mo_mult_qt(mo_ctx *ctx, mo_matrix Cm, mo_matrix Am, mo_matrix Tm, mo_matrix Wm, int flags,
               int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View C, A, T;
  if ((rc = mo::to_view(Cm, C)) || (rc = mo::to_view(Am, A)) || (rc = mo::to_view(Tm, T)))
    return rc;
  if (nb == 0) nb = T.cols;
  if ((rc = mult_checks(C, A, Wm, flags, nb, true))) return rc;
  const int k = std::min(A.rows, A.cols);
  if (T.rows < k || T.cols < k) return MO_ETSMALL;
  if (k > 0 && !T.d) return MO_EINVAL;
  return apply_q(ctx, C, A, T, nullptr, 0, flags, nb);
}

// qrwym.go:573-630
int mo_mult_q(mo_ctx *ctx, mo_matrix Cm, mo_matrix Am, mo_matrix taum, mo_matrix Wm, int flags,
              int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View C, A;
  if ((rc = mo::to_view(Cm, C)) || (rc = mo::to_view(Am, A))) return rc;
  if ((rc = mult_checks(C, A, Wm, flags, nb, nb != 0))) return rc;
  const int k = std::min(A.rows, A.cols);
  double *tau = nullptr;
  int64_t inc = 1;
  if ((rc = tau_view(taum, k, &tau, &inc))) return rc;
  return apply_q(ctx, C, A, View{nullptr, 0, 0, 1}, tau, inc, flags, nb);
}

// qrwym.go:784-819
int mo_solve_qrt(mo_ctx *ctx, mo_matrix Bm, mo_matrix Am, mo_matrix Tm, mo_matrix Wm, int flags,
                 int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View B, A, T;
  if ((rc = mo::to_view(Bm, B)) || (rc = mo::to_view(Am, A)) || (rc = mo::to_view(Tm, T)))
    return rc;
  if (nb == 0) nb = T.cols;
  const int k = std::min(A.rows, A.cols);
  if (T.rows < k || T.cols < k) return MO_ETSMALL;
  if (k > 0 && !T.d) return MO_EINVAL;
  return solve_q(ctx, B, A, T, nullptr, 0, Wm, flags, nb, true);
}

// qrwym.go:717-760
int mo_solve_qr(mo_ctx *ctx, mo_matrix Bm, mo_matrix Am, mo_matrix taum, mo_matrix Wm, int flags,
                int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View B, A;
  if ((rc = mo::to_view(Bm, B)) || (rc = mo::to_view(Am, A))) return rc;
  const int k = std::min(A.rows, A.cols);
  double *tau = nullptr;
  int64_t inc = 1;
  if ((rc = tau_view(taum, k, &tau, &inc))) return rc;
  return solve_q(ctx, B, A, View{nullptr, 0, 0, 1}, tau, inc, Wm, flags, nb, nb != 0);
}

// qrwyk.go:232-267
int mo_build_q(mo_ctx *ctx, mo_matrix Am, mo_matrix taum, mo_matrix Wm, int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A;
  if ((rc = mo::to_view(Am, A))) return rc;
  if (nb != 0 && is_nil(Wm)) return MO_ENOWORK;
  if (nb != 0 && (Wm.cols < nb || Wm.rows < A.cols)) return MO_EWORKSMALL;
  if (A.rows < A.cols) return MO_EABSIZE;
  double *tau = nullptr;
  int64_t inc = 1;
  if ((rc = tau_view(taum, A.cols, &tau, &inc))) return rc;
  return mo::qr_build_q(ctx, A, View{nullptr, 0, 0, 1}, tau, inc);
}

// qrwyk.go:278-293
int mo_build_qt(mo_ctx *ctx, mo_matrix Am, mo_matrix Tm, mo_matrix Wm, int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A, T;
  if ((rc = mo::to_view(Am, A)) || (rc = mo::to_view(Tm, T))) return rc;
  if (nb == 0) nb = A.cols;
  if (is_nil(Wm)) return MO_ENOWORK;
  if (Wm.cols < nb || Wm.rows < A.cols) return MO_EWORKSMALL;
  if (A.rows < A.cols) return MO_EABSIZE;
  if (T.rows < A.cols || T.cols < A.cols) return MO_ETSMALL;
  if (A.cols > 0 && !T.d) return MO_EINVAL;
  return mo::qr_build_q(ctx, A, T, nullptr, 0);
}

}  // extern "C"
