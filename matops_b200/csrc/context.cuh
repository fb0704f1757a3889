// The mo_ctx object and internal entry points shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "gemm.cuh"

struct mo_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int *d_status = nullptr;  // device status word written by bounded waits
  int mb = 68, nb = 68, kb = 196;  // BlockingParams (mmult.go:33-35)
  int workers = 1;                 // NumWorkers (mmult.go:38)
  int syrk_blas_beta = 0;
  // polls of a flag that the few-right-hand-side triangular solve makes before it gives up
  // (mo_set_spin_limit); the mbarrier waits of the TMA pipelines keep MO_SPIN_LIMIT
  uint32_t spin_limit = MO_SPIN_LIMIT;
  // scratch owned by the context (grown on demand, freed in mo_ctx_destroy)
  void *ws = nullptr;
  size_t ws_bytes = 0;
  int sms = 148;
  // second, high-priority stream for look-ahead panels, and fork/join events
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // a third stream (default priority) for memory-bound work that overlaps a factorization
  cudaStream_t side = nullptr;
  cudaEvent_t ev_side_fork = nullptr, ev_side_join = nullptr;
  // stream-K scratch of the GEMM engine (allocated with the context)
  double *sk_partial = nullptr;
  int *sk_flags = nullptr;
  int sk_epoch = 0;
  // tracing (mo_profile_*)
  bool prof_on = false;
  mo_profile prof = {};
  struct Pending {
    int cls;
    cudaEvent_t ev0, ev1;
  };
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<Pending> pending;
  // workspace of the mixed-precision solver (separate from `ws`, which the FP64 routines
  // it may call for a fallback grow and reallocate)
  void *ws_ir = nullptr;
  size_t ws_ir_bytes = 0;
  // scratch of the Cholesky adjoint (a few 128 x 128 blocks per stream) and the stream
  // pool of its batched form
  void *ws_adj = nullptr;
  size_t ws_adj_bytes = 0;
  std::vector<cudaStream_t> pool;
  std::vector<cudaEvent_t> pool_ev;
  // GMRES convergence words read back without stopping the stream: pinned host slots and
  // one event per inner iteration
  int *h_gmres = nullptr;
  std::vector<cudaEvent_t> gmres_ev;
};

namespace mo {

// control block in device memory (ctx->d_status): status word, factorization info, value
// of the failing pivot
struct Control {
  int status;
  int info;
  double bad;
};
inline Control *control(mo_ctx *ctx) { return reinterpret_cast<Control *>(ctx->d_status); }

// brackets one kernel launch for tracing: counts it and, when tracing is on, records
// CUDA events around it on the context's stream
struct ProfScope {
  int cls;
  cudaEvent_t ev0, ev1;
};
void prof_begin(mo_ctx *ctx, ProfScope &s, int cls);
void prof_end(mo_ctx *ctx, ProfScope &s, double flops, double bytes);

struct View {
  double *d;
  int rows, cols;
  int64_t ld;
  double *at(int i, int j) const { return d + i + (int64_t)j * ld; }
  View sub(int i, int j, int r, int c) const { return View{at(i, j), r, c, ld}; }
};

// Validates a public mo_matrix: non-negative sizes that fit in int, ld >= rows, data
// non-NULL when non-empty.  Returns MO_OK or MO_EINVAL.
int to_view(const mo_matrix &m, View &v);

// make the context's device current for this call
int enter(mo_ctx *ctx);

// grow the context workspace to at least `bytes` (stream-ordered: synchronizes first)
int workspace(mo_ctx *ctx, size_t bytes, void **out);

// C = alpha*op(A)*op(B) + beta*C on device views (sizes already checked)
int gemm(mo_ctx *ctx, View C, View A, bool ta, View B, bool tb, double alpha, double beta);

// the same with engine options: masked modes, a cap on the persistent grid (to leave SMs
// to another stream), and whether the stream-K schedule may be used
struct GemmOpts {
  int mode = kGemm;
  int max_ctas = 0;
  bool stream_k = true;
  int beta_block = 0;
  const int *skip = nullptr;  // see GemmArgs::skip
};
int gemm_ex(mo_ctx *ctx, View C, View A, bool ta, View B, bool tb, double alpha, double beta,
            const GemmOpts &o);

// temporarily launch the context's work on another stream
struct StreamSwap {
  mo_ctx *c;
  cudaStream_t old;
  StreamSwap(mo_ctx *ctx, cudaStream_t s) : c(ctx), old(ctx->stream) { ctx->stream = s; }
  ~StreamSwap() { c->stream = old; }
};

// the context's auxiliary stream (created on first use, highest priority)
int aux_stream(mo_ctx *ctx, cudaStream_t *out);
int side_stream(mo_ctx *ctx, cudaStream_t *out);
// make `waiter` wait for all work enqueued so far on `producer`
int stream_wait(mo_ctx *ctx, cudaStream_t waiter, cudaStream_t producer, cudaEvent_t ev);

// triangle(C) = alpha*op(A)*op(A)^T + beta*C; beta_block as in GemmArgs
int syrk(mo_ctx *ctx, View C, View A, bool ta, bool upper, double alpha, double beta,
         int beta_block);

// B = alpha*op(A)^-1*B (left) or alpha*B*op(A)^-1 (right); A n x n triangle
int trsm(mo_ctx *ctx, View B, View A, int flags, double alpha);
// the same with caller-provided scratch for the ceil(n/128) inverted 128 x 128 blocks
int trsm_with_scratch(mo_ctx *ctx, View B, View A, int flags, double alpha, double *inv);

}  // namespace mo
