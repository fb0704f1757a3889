// mo_solve_trm_static: the triangular solve of mo_solve_trm without any device allocation.
//
// Some programs cannot let a library call cudaMalloc: a host application whose device
// memory is owned by its own pool allocator (memory handed out only by that pool), a
// service that must keep a fixed, declared footprint on a shared GPU, or a latency-bound
// loop that cannot afford cudaMalloc's implicit synchronization and unbounded cost.  This
// entry point serves them: the only device memory it uses beyond the caller's matrices is
// a fixed block compiled into the library (below), so every call runs with memory that
// already exists.
//
// Limits and rules (also stated in include/matops_b200.h):
//   * order of A <= MO_SOLVE_TRM_STATIC_MAX_N (1024): the scratch holds the inverses of
//     at most 8 diagonal blocks of 128 x 128 doubles (1 MiB).  Larger A -> MO_ESTATICLIMIT.
//   * the block is part of the library image: every GPU that loads the library keeps these
//     1 MiB (+ 32 bytes of status) until the process exits.
//   * all calls on a device share the block and it keeps the last call's contents; calls
//     that overlap on the GPU (other threads, other streams) race and must be serialized
//     by the caller.
//   * every call looks the block's device address up (cudaGetSymbolAddress) with the
//     caller's device current: the first call on a device loads this library's kernels
//     there, so make it before any stream capture begins.  Looking the address up on each
//     call (it allocates nothing once the module is loaded) keeps the address right after
//     a context reset, when the module and its block are loaded again elsewhere.
#include "context.cuh"

namespace {

constexpr int kMaxOrder = MO_SOLVE_TRM_STATIC_MAX_N;
constexpr int kBlock = 128;  // diagonal block order used by the triangular sweep
static_assert(kMaxOrder % kBlock == 0, "the scratch holds whole 128 x 128 blocks");
constexpr size_t kScratchDoubles = (size_t)((kMaxOrder + kBlock - 1) / kBlock) * kBlock * kBlock;

// Fixed device scratch: inverted diagonal blocks of the last call, and the context's
// control words (status first; the bounded device waits write into it).
static __device__ __align__(256) double g_static_trsm_scratch[kScratchDoubles];
static __device__ __align__(256) int g_static_trsm_status[8];

// The device addresses of the two blocks for the current device (the names themselves
// are host-side stand-ins and must not be passed to a kernel) and its SM count.
int device_slot(double **scratch, int **status, int *sms) {
  int dev = 0;
  MO_CUDA_TRY(cudaGetDevice(&dev));
  void *p = nullptr;
  MO_CUDA_TRY(cudaGetSymbolAddress(&p, g_static_trsm_scratch));
  *scratch = static_cast<double *>(p);
  MO_CUDA_TRY(cudaGetSymbolAddress(&p, g_static_trsm_status));
  *status = static_cast<int *>(p);
  MO_CUDA_TRY(cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev));
  return MO_OK;
}

}  // namespace

extern "C" int mo_solve_trm_static(mo_matrix Bm, mo_matrix Am, double alpha, int flags,
                                   void *stream) {
  int rc;
  mo::View B, A;
  if ((rc = mo::to_view(Bm, B)) || (rc = mo::to_view(Am, A))) return rc;
  // the size rules of SolveTrm (mmult.go:388-422), as in mo_solve_trm
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
  const int N = A.cols;
  const bool right = (flags & MO_RIGHT) != 0;
  if (N == 0 || (right ? B.rows : B.cols) == 0) return MO_OK;
  if (A.rows < N || (right ? B.cols : B.rows) < N) return MO_EABSIZE;
  if (N > kMaxOrder) return MO_ESTATICLIMIT;
  double *scratch = nullptr;
  int *status = nullptr, sms = 0, dev = 0;
  MO_CUDA_TRY(cudaGetDevice(&dev));
  if ((rc = device_slot(&scratch, &status, &sms))) return rc;

  // a context on the host stack: no scratch of its own, no stream-K (data-parallel GEMM
  // schedule only), status word in the fixed block
  mo_ctx ctx;
  ctx.device = dev;
  ctx.stream = static_cast<cudaStream_t>(stream);
  ctx.d_status = status;
  ctx.sms = sms;
  MO_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), ctx.stream));
  mo::View Bn = right ? B.sub(0, 0, B.rows, N) : B.sub(0, 0, N, B.cols);
  rc = mo::trsm_with_scratch(&ctx, Bn, A.sub(0, 0, N, N), flags, alpha, scratch);
  if (rc) return rc;
  // read the status word on the caller's stream (no device-wide synchronization)
  int st = 0;
  MO_CUDA_TRY(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  MO_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
  return st;
}
