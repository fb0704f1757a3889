// extern "C" entry points (include/matops_b200.h): argument checking that mirrors the Go
// wrappers of the reference, then dispatch to the device drivers.
#include <climits>
#include <cstddef>
#include <cstring>

#include "context.cuh"

namespace mo {
int potrf(mo_ctx *ctx, View A, bool upper, int *d_info, double *d_bad, double *inv);
int getrf(mo_ctx *ctx, View A, int64_t *piv, int64_t npiv, int ref_nb);
int laswp_forward(mo_ctx *ctx, View B, const int64_t *piv, int64_t npiv);


int to_view(const mo_matrix &m, View &v) {
  if (m.rows < 0 || m.cols < 0 || m.rows > INT_MAX || m.cols > INT_MAX) return MO_EINVAL;
  if (m.rows > 0 && m.cols > 0) {
    if (!m.data) return MO_EINVAL;
    if (m.ld < m.rows || m.ld < 1) return MO_EINVAL;
  }
  v.d = m.data;
  v.rows = (int)m.rows;
  v.cols = (int)m.cols;
  v.ld = m.ld < 1 ? 1 : m.ld;
  return MO_OK;
}

int enter(mo_ctx *ctx) {
  if (!ctx) return MO_EINVAL;
  MO_CUDA_TRY(cudaSetDevice(ctx->device));
  return MO_OK;
}

int workspace(mo_ctx *ctx, size_t bytes, void **out) {
  if (bytes > ctx->ws_bytes) {
    MO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (ctx->ws) cudaFree(ctx->ws);
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
    size_t want = bytes < (size_t(1) << 22) ? (size_t(1) << 22) : bytes;
    MO_CUDA_TRY(cudaMalloc(&ctx->ws, want));
    ctx->ws_bytes = want;
  }
  *out = ctx->ws;
  return MO_OK;
}


int gemm_ex(mo_ctx *ctx, View C, View A, bool ta, View B, bool tb, double alpha, double beta,
            const GemmOpts &o) {
  GemmArgs g;
  g.M = C.rows;
  g.N = C.cols;
  g.K = ta ? A.rows : A.cols;
  g.alpha = alpha;
  g.beta = beta;
  g.A = A.d;
  g.lda = A.ld;
  g.transA = ta;
  g.B = B.d;
  g.ldb = B.ld;
  g.transB = tb;
  g.C = C.d;
  g.ldc = C.ld;
  g.mode = o.mode;
  g.beta_block = o.beta_block;
  g.status = &control(ctx)->status;
  g.skip = o.skip;
  g.sms = ctx->sms;
  g.max_ctas = o.max_ctas;
  if (o.stream_k && o.mode == kGemm) {
    g.sk_partial = ctx->sk_partial;
    g.sk_flags = ctx->sk_flags;
    g.sk_epoch = ++ctx->sk_epoch;
  }
  if (g.M <= 0 || g.N <= 0) return MO_OK;
  ProfScope ps;
  prof_begin(ctx, ps, MO_PROF_GEMM);
  const int rc = launch_gemm(g, ctx->stream);
  const double M = g.M, N = g.N, K = g.K;
  const bool tri = (o.mode == kSyrkLower || o.mode == kSyrkUpper);
  const double elems = tri ? N * (N + 1) / 2 : M * N;
  prof_end(ctx, ps, 2.0 * elems * K,
           8.0 * (M * K + (tri ? 0.0 : K * N) + elems * (beta != 0.0 ? 2 : 1)));
  return rc;
}

int gemm(mo_ctx *ctx, View C, View A, bool ta, View B, bool tb, double alpha, double beta) {
  return gemm_ex(ctx, C, A, ta, B, tb, alpha, beta, GemmOpts());
}

int syrk(mo_ctx *ctx, View C, View A, bool ta, bool upper, double alpha, double beta,
         int beta_block) {
  GemmOpts o;
  o.mode = upper ? kSyrkUpper : kSyrkLower;
  o.beta_block = beta_block;
  return gemm_ex(ctx, C, A, ta, A, !ta, alpha, beta, o);
}

int aux_stream(mo_ctx *ctx, cudaStream_t *out) {
  if (!ctx->aux) {
    int lo = 0, hi = 0;
    MO_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    MO_CUDA_TRY(cudaStreamCreateWithPriority(&ctx->aux, cudaStreamNonBlocking, hi));
    MO_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    MO_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  }
  *out = ctx->aux;
  return MO_OK;
}

int side_stream(mo_ctx *ctx, cudaStream_t *out) {
  if (!ctx->side) {
    MO_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    MO_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_side_fork, cudaEventDisableTiming));
    MO_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_side_join, cudaEventDisableTiming));
  }
  *out = ctx->side;
  return MO_OK;
}

int stream_wait(mo_ctx *ctx, cudaStream_t waiter, cudaStream_t producer, cudaEvent_t ev) {
  (void)ctx;
  MO_CUDA_TRY(cudaEventRecord(ev, producer));
  MO_CUDA_TRY(cudaStreamWaitEvent(waiter, ev, 0));
  return MO_OK;
}

}  // namespace mo

using mo::View;

extern "C" {

int mo_ctx_create(int device, mo_ctx **out) {
  if (!out) return MO_EINVAL;
  *out = nullptr;
  int ndev = 0;
  MO_CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return MO_EINVAL;
  MO_CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  MO_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) return MO_ENOKERNEL;  // sm_100a image only
  mo_ctx *ctx = new mo_ctx();
  ctx->device = device;
  ctx->sms = prop.multiProcessorCount;
  cudaError_t e = cudaMalloc(&ctx->d_status, sizeof(mo::Control));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_status, 0, sizeof(mo::Control));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->sk_partial, mo::gemm_partial_bytes(ctx->sms));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->sk_flags, sizeof(int) * ctx->sms);
  if (e == cudaSuccess) e = cudaMemset(ctx->sk_flags, 0, sizeof(int) * ctx->sms);
  if (e != cudaSuccess) {
    if (ctx->sk_partial) cudaFree(ctx->sk_partial);
    if (ctx->sk_flags) cudaFree(ctx->sk_flags);
    if (ctx->d_status) cudaFree(ctx->d_status);
    delete ctx;
    return mo_from_cuda_error(e);
  }
  *out = ctx;
  return MO_OK;
}

int mo_ctx_destroy(mo_ctx *ctx) {
  if (!ctx) return MO_EINVAL;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->ws_ir) cudaFree(ctx->ws_ir);
  if (ctx->ws_adj) cudaFree(ctx->ws_adj);
  for (auto s : ctx->pool) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  for (auto e : ctx->pool_ev) cudaEventDestroy(e);
  for (auto e : ctx->gmres_ev) cudaEventDestroy(e);
  if (ctx->h_gmres) cudaFreeHost(ctx->h_gmres);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->sk_partial) cudaFree(ctx->sk_partial);
  if (ctx->sk_flags) cudaFree(ctx->sk_flags);
  for (auto e : ctx->ev_pool) cudaEventDestroy(e);
  if (ctx->aux) {
    cudaStreamSynchronize(ctx->aux);
    cudaStreamDestroy(ctx->aux);
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  if (ctx->ev_side_fork) cudaEventDestroy(ctx->ev_side_fork);
  if (ctx->ev_side_join) cudaEventDestroy(ctx->ev_side_join);
  delete ctx;
  return MO_OK;
}

int mo_set_stream(mo_ctx *ctx, void *stream) {
  if (!ctx) return MO_EINVAL;
  ctx->stream = reinterpret_cast<cudaStream_t>(stream);
  return MO_OK;
}

int mo_sync(mo_ctx *ctx) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  MO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  int st = 0;
  MO_CUDA_TRY(cudaMemcpy(&st, &mo::control(ctx)->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st != 0) MO_CUDA_TRY(cudaMemset(&mo::control(ctx)->status, 0, sizeof(int)));
  return st;
}

const char *mo_strerror(int s) {
  switch (s) {
    case MO_OK: return "ok";
    case MO_ESIZE: return "Mult: size mismatch";
    case MO_ENOTSQUARE: return "A not a square matrix";
    case MO_EPIVLEN: return "pivot array < min(A.Rows(),A.Cols())";
    case MO_ECNOTSQUARE: return "C not a square matrix";
    case MO_EABSIZE: return "A, B size mismatch";
    case MO_ESYMSIZE: return "MultSym: size mismatch";
    case MO_EINVAL: return "invalid argument";
    case MO_ECUDA: return "CUDA runtime error";
    case MO_EDEVTIMEOUT: return "device-side wait timed out";
    case MO_ENOMEM: return "device out of memory";
    case MO_ENOKERNEL: return "no sm_100a kernel image for this device";
    case MO_ESTATICLIMIT: return "matrix order exceeds the fixed scratch of mo_solve_trm_static";
    case MO_EBATCHN: return "batched matrix order outside 1..MO_BATCH_MAX_N";
    case MO_EWORKSMALL: return "work space too small";
    case MO_ENOWORK: return "workspace not defined";
    case MO_ECQSIZE: return "C*Q: C.Cols != A.Rows";
    case MO_ETSMALL: return "reflector matrix T too small";
    case MO_ELDLWORK: return "No workspace for blocking invocation";
    case MO_EZERODIAG: return "zero value on diagonal";
    case MO_EBKWORK: return "Workspace too small";
    default: return s > 0 ? "illegal value (non-positive pivot)" : "unknown error";
  }
}

int mo_blocking_params(mo_ctx *ctx, int mb, int nb, int kb) {
  if (!ctx) return MO_EINVAL;
  ctx->mb = mb;
  ctx->nb = nb;
  ctx->kb = kb;
  return MO_OK;
}

int mo_num_workers(mo_ctx *ctx, int n) {
  if (!ctx) return MO_EINVAL;
  int old = ctx->workers;
  ctx->workers = n;
  return old;
}

int mo_set_syrk_blas_beta(mo_ctx *ctx, int on) {
  if (!ctx) return MO_EINVAL;
  int old = ctx->syrk_blas_beta;
  ctx->syrk_blas_beta = on ? 1 : 0;
  return old;
}

int mo_set_spin_limit(mo_ctx *ctx, uint32_t polls, uint32_t *old) {
  if (!ctx) return MO_EINVAL;
  if (old) *old = ctx->spin_limit;
  ctx->spin_limit = polls;
  return MO_OK;
}

int mo_malloc(mo_ctx *ctx, void **ptr, size_t bytes) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  if (!ptr) return MO_EINVAL;
  MO_CUDA_TRY(cudaMalloc(ptr, bytes ? bytes : 16));
  return MO_OK;
}

int mo_free(mo_ctx *ctx, void *ptr) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  MO_CUDA_TRY(cudaFree(ptr));
  return MO_OK;
}

int mo_upload(mo_ctx *ctx, mo_matrix dst, const double *src, int64_t ld_src) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View v;
  if ((rc = mo::to_view(dst, v))) return rc;
  if (v.rows == 0 || v.cols == 0) return MO_OK;
  if (!src || ld_src < v.rows) return MO_EINVAL;
  MO_CUDA_TRY(cudaMemcpy2DAsync(v.d, v.ld * 8, src, ld_src * 8, (size_t)v.rows * 8, v.cols,
                                cudaMemcpyHostToDevice, ctx->stream));
  return MO_OK;
}

int mo_upload_tri(mo_ctx *ctx, mo_matrix dst, const double *src, int64_t ld_src, int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View v;
  if ((rc = mo::to_view(dst, v))) return rc;
  if (v.rows != v.cols) return MO_ESIZE;
  if (v.rows == 0) return MO_OK;
  if (!src || ld_src < v.rows) return MO_EINVAL;
  const bool upper = (flags & MO_UPPER) != 0;
  const int64_t n = v.rows;
  // one 2-D copy per 128-column block: rows j0..n-1 (lower) or 0..j0+w-1 (upper), so the
  // bytes moved are n (n + 128) / 2 elements instead of n^2
  for (int64_t j0 = 0; j0 < n; j0 += 128) {
    const int64_t w = n - j0 < 128 ? n - j0 : 128;
    const int64_t r0 = upper ? 0 : j0, nr = upper ? j0 + w : n - j0;
    MO_CUDA_TRY(cudaMemcpy2DAsync(v.d + r0 + j0 * v.ld, v.ld * 8, src + r0 + j0 * ld_src,
                                  ld_src * 8, (size_t)nr * 8, w, cudaMemcpyHostToDevice,
                                  ctx->stream));
  }
  return MO_OK;
}

int mo_download(mo_ctx *ctx, double *dst, int64_t ld_dst, mo_matrix src) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View v;
  if ((rc = mo::to_view(src, v))) return rc;
  if (v.rows == 0 || v.cols == 0) return MO_OK;
  if (!dst || ld_dst < v.rows) return MO_EINVAL;
  MO_CUDA_TRY(cudaMemcpy2DAsync(dst, ld_dst * 8, v.d, v.ld * 8, (size_t)v.rows * 8, v.cols,
                                cudaMemcpyDeviceToHost, ctx->stream));
  return MO_OK;
}

int mo_upload_bytes(mo_ctx *ctx, void *dst, const void *src, size_t bytes) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  if (bytes == 0) return MO_OK;
  MO_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return MO_OK;
}

int mo_download_bytes(mo_ctx *ctx, void *dst, const void *src, size_t bytes) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  if (bytes == 0) return MO_OK;
  MO_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return MO_OK;
}

// mmult.go:198-256
int mo_mult(mo_ctx *ctx, mo_matrix Cm, mo_matrix Am, mo_matrix Bm, double alpha, double beta,
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
      ok = cr == ac && cc == br && ar == bc;
      break;
    case MO_TRANSA:
      empty = ac == 0 || bc == 0;
      ok = cr == ac && cc == bc && ar == br;
      break;
    case MO_TRANSB:
      empty = ar == 0 || br == 0;
      ok = cr == ar && cc == br && ac == bc;
      break;
    default:
      empty = ar == 0 || bc == 0;
      ok = cr == ar && cc == bc && ac == br;
  }
  if (empty) return MO_OK;
  if (!ok) return MO_ESIZE;
  return mo::gemm(ctx, C, A, (flags & MO_TRANSA) != 0, B, (flags & MO_TRANSB) != 0, alpha, beta);
}

// mmult.go:426-445 with calgo/cmops.go:219-240 and calgo/dmmat_rank.c:62-127
int mo_rank_update_sym(mo_ctx *ctx, mo_matrix Cm, mo_matrix Am, double alpha, double beta,
                       int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View C, A;
  if ((rc = mo::to_view(Cm, C)) || (rc = mo::to_view(Am, A))) return rc;
  if (C.rows != C.cols) return MO_ECNOTSQUARE;
  const bool ta = (flags & MO_TRANSA) != 0;
  const int P = ta ? A.rows : A.cols;
  const int n = C.rows;
  if (P == 0 || n == 0) return MO_OK;  // the reference returns before touching C
  if ((ta ? A.cols : A.rows) != n) return MO_EABSIZE;
  const bool up = (flags & MO_UPPER) != 0, lo = (flags & MO_LOWER) != 0;
  if (up == lo) return MO_EINVAL;  // exactly one triangle must be named
  int bb = 0;
  if (!ctx->syrk_blas_beta && beta != 1.0) {
    // calgo/dmmat_rank.c:75-83: NB clamped to (0, 68] and to the order of C
    int nb = ctx->nb;
    if (nb > 68 || nb <= 0) nb = 68;
    if (nb > n) nb = n;
    bb = nb;
  }
  return mo::syrk(ctx, C, A, ta, up, alpha, beta, bb);
}

// mmult.go:388-422
int mo_solve_trm(mo_ctx *ctx, mo_matrix Bm, mo_matrix Am, double alpha, int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View B, A;
  if ((rc = mo::to_view(Bm, B)) || (rc = mo::to_view(Am, A))) return rc;
  bool ok = true, empty = false;
  switch (flags & (MO_LEFT | MO_RIGHT)) {
    case MO_LEFT:
      empty = B.rows == 0;
      ok = B.rows == A.cols && A.cols == A.rows;
      break;
    case MO_RIGHT:
      empty = B.cols == 0;
      ok = B.cols == A.rows && A.cols == A.rows;
      break;
    default:
      break;
  }
  if (empty) return MO_OK;
  if (!ok) return MO_EABSIZE;
  // no side check in the reference when neither or both side bits are set; the triangle
  // order is A.Cols() (calgo/cmops.go:195-215); refuse shapes that would read out of range
  const int N = A.cols;
  const bool right = (flags & MO_RIGHT) != 0;
  if (N == 0 || (right ? B.rows : B.cols) == 0) return MO_OK;
  if (A.rows < N || (right ? B.cols : B.rows) < N) return MO_EABSIZE;
  View Bn = right ? B.sub(0, 0, B.rows, N) : B.sub(0, 0, N, B.cols);
  return mo::trsm(ctx, Bn, A.sub(0, 0, N, N), flags, alpha);
}

// chol.go:116-127
int mo_decompose_chol(mo_ctx *ctx, mo_matrix Am, int flags, int nb, double *bad_value) {
  (void)nb;
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A;
  if ((rc = mo::to_view(Am, A))) return rc;
  if (A.rows != A.cols) return MO_ENOTSQUARE;
  if (A.rows == 0) return MO_OK;
  mo::Control *cb = mo::control(ctx);
  MO_CUDA_TRY(cudaMemsetAsync(&cb->info, 0, sizeof(mo::Control) - offsetof(mo::Control, info), ctx->stream));
  double *inv = nullptr;
  if ((rc = mo::workspace(ctx, 128 * 128 * sizeof(double), (void **)&inv))) return rc;
  // LOWER selects L*L^T; any other flags factor the upper triangle (chol.go:39-49, 77-87)
  rc = mo::potrf(ctx, A, (flags & MO_LOWER) == 0, &cb->info, &cb->bad, inv);
  if (rc) return rc;
  MO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  mo::Control h;
  MO_CUDA_TRY(cudaMemcpy(&h, cb, sizeof(h), cudaMemcpyDeviceToHost));
  if (h.status) {
    cudaMemset(&cb->status, 0, sizeof(int));
    return h.status;
  }
  if (h.info > 0 && bad_value) *bad_value = h.bad;
  return h.info;
}

// chol.go:147-158
int mo_solve_chol(mo_ctx *ctx, mo_matrix Bm, mo_matrix Am, int flags) {
  int rc;
  if (flags & MO_UPPER) {
    rc = mo_solve_trm(ctx, Bm, Am, 1.0, MO_UPPER | MO_TRANSA);
    if (!rc) rc = mo_solve_trm(ctx, Bm, Am, 1.0, MO_UPPER);
    return rc;
  }
  if (flags & MO_LOWER) {
    rc = mo_solve_trm(ctx, Bm, Am, 1.0, MO_LOWER);
    if (!rc) rc = mo_solve_trm(ctx, Bm, Am, 1.0, MO_LOWER | MO_TRANSA);
    return rc;
  }
  return MO_OK;
}

// lu.go:257-272
int mo_decompose_lu(mo_ctx *ctx, mo_matrix Am, int64_t *piv, int64_t npiv, int nb) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View A;
  if ((rc = mo::to_view(Am, A))) return rc;
  const int mlen = A.rows < A.cols ? A.rows : A.cols;
  if (npiv < mlen) return MO_EPIVLEN;
  if (npiv > 0 && !piv) return MO_EINVAL;
  if (npiv > 0) MO_CUDA_TRY(cudaMemsetAsync(piv, 0, (size_t)npiv * sizeof(int64_t), ctx->stream));
  if (mlen == 0) return MO_OK;
  return mo::getrf(ctx, A, piv, npiv, nb);
}

// lu.go:320-334
int mo_solve_lu(mo_ctx *ctx, mo_matrix Bm, mo_matrix Am, const int64_t *piv, int64_t npiv,
                int flags) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  View B;
  if ((rc = mo::to_view(Bm, B))) return rc;
  if (npiv > 0 && !piv) return MO_EINVAL;
  if ((rc = mo::laswp_forward(ctx, B, piv, npiv))) return rc;
  if (flags & MO_TRANSA) {
    rc = mo_solve_trm(ctx, Bm, Am, 1.0, MO_LOWER | MO_UNIT | MO_TRANSA);
    if (!rc) rc = mo_solve_trm(ctx, Bm, Am, 1.0, MO_UPPER | MO_TRANSA);
  } else {
    rc = mo_solve_trm(ctx, Bm, Am, 1.0, MO_LOWER | MO_UNIT);
    if (!rc) rc = mo_solve_trm(ctx, Bm, Am, 1.0, MO_UPPER);
  }
  return rc;
}

}  // extern "C"
