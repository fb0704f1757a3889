// DGEMM / DSYRK engine: host-side interface.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mo {

enum GemmMode : int {
  kGemm = 0,       // C[M,N] = alpha*op(A)*op(B) + beta*C
  kSyrkLower = 1,  // only tiles / elements with row >= col are computed and written
  kSyrkUpper = 2,  // only row <= col
  kGemmLower = 3,  // rectangular tiles of C, elements with row < col left untouched
  kGemmUpper = 4,  // rectangular tiles of C, elements with row > col left untouched
};

struct GemmArgs {
  int M = 0, N = 0, K = 0;
  double alpha = 1.0, beta = 0.0;
  const double *A = nullptr;
  int64_t lda = 0;
  bool transA = false;  // op(A)(m,k) = A[k + m*lda] when true, A[m + k*lda] otherwise
  const double *B = nullptr;
  int64_t ldb = 0;
  bool transB = false;  // op(B)(k,n) = B[n + k*ldb] when true, B[k + n*ldb] otherwise
  double *C = nullptr;
  int64_t ldc = 0;
  int mode = kGemm;
  // > 0: beta applies only where row/beta_block == col/beta_block (elsewhere beta = 1)
  int beta_block = 0;
  int *status = nullptr;  // device status word (first error wins)
  // optional device word: when it is non-zero at launch the whole grid returns at once
  // (iterations enqueued ahead of a convergence test that has since ended them)
  const int *skip = nullptr;
  bool force_fallback = false;  // use the cp.async producer even when TMA is legal
  int sms = 148;                // persistent grid size
  int max_ctas = 0;             // > 0: cap the persistent grid (leave SMs to other streams)
  // stream-K scratch (nullptr: data-parallel schedule only): one 128 KB partial-sum slot
  // and one flag per CTA, and a value unique to this launch for the flags
  double *sk_partial = nullptr;
  int *sk_flags = nullptr;
  int sk_epoch = 0;
};

// Enqueue one launch on `stream`.  Returns MO_OK or a negative MO_E* code.
int launch_gemm(const GemmArgs &args, cudaStream_t stream);

// True when the TMA producer can be used for these operands (16-byte aligned bases,
// leading dimensions that are multiples of 2 doubles).
bool gemm_tma_ok(const GemmArgs &args);

// bytes of stream-K partial-sum scratch for a device with `sms` SMs
size_t gemm_partial_bytes(int sms);

}  // namespace mo
