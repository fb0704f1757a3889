// Tracing support: per-kernel-class event timing and launch counting, and the FP64
// tensor-pipe peak measurement used as the roofline denominator.
#include <cstring>

#include "context.cuh"

namespace mo {

void prof_begin(mo_ctx *ctx, ProfScope &s, int cls) {
  s.cls = cls;
  s.ev0 = s.ev1 = nullptr;
  ctx->prof.launches[cls] += 1;
  if (!ctx->prof_on) return;
  if (ctx->ev_used + 2 > ctx->ev_pool.size()) {
    for (int i = 0; i < 64; ++i) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return;
      ctx->ev_pool.push_back(e);
    }
  }
  s.ev0 = ctx->ev_pool[ctx->ev_used++];
  s.ev1 = ctx->ev_pool[ctx->ev_used++];
  cudaEventRecord(s.ev0, ctx->stream);
}

void prof_end(mo_ctx *ctx, ProfScope &s, double flops, double bytes) {
  ctx->prof.flops[s.cls] += flops;
  ctx->prof.bytes[s.cls] += bytes;
  if (!s.ev0) return;
  cudaEventRecord(s.ev1, ctx->stream);
  ctx->pending.push_back({s.cls, s.ev0, s.ev1});
}

namespace {

__global__ void __launch_bounds__(256) dmma_peak_kernel(double *out, int iters, double s) {
  double acc[4][4];
  double a0 = s * threadIdx.x, a1 = s * (threadIdx.x + 1), b = s * (threadIdx.x + 2);
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[c][j] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 4; ++c) dmma_16x8x4(acc[c], a0, a1, b);
  }
  double t = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int j = 0; j < 4; ++j) t += acc[c][j];
  out[blockIdx.x * blockDim.x + threadIdx.x] = t;
}

}  // namespace
}  // namespace mo

extern "C" {

int mo_profile_enable(mo_ctx *ctx, int on) {
  if (!ctx) return MO_EINVAL;
  ctx->prof_on = on != 0;
  return MO_OK;
}

int mo_profile_read(mo_ctx *ctx, mo_profile *out) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  if (!out) return MO_EINVAL;
  MO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (auto &p : ctx->pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.ev0, p.ev1) == cudaSuccess) ctx->prof.ms[p.cls] += ms;
  }
  ctx->pending.clear();
  ctx->ev_used = 0;
  *out = ctx->prof;
  memset(&ctx->prof, 0, sizeof(ctx->prof));
  return MO_OK;
}

int mo_measure_fp64_peak(mo_ctx *ctx, double ms, double *tflops) {
  int rc = mo::enter(ctx);
  if (rc) return rc;
  if (!tflops) return MO_EINVAL;
  const int blocks = ctx->sms * 2, threads = 256;
  double *out = nullptr;
  MO_CUDA_TRY(cudaMalloc(&out, sizeof(double) * blocks * threads));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int iters = 4096;
  float el = 0.f;
  for (int rep = 0; rep < 8; ++rep) {
    cudaEventRecord(e0, ctx->stream);
    mo::dmma_peak_kernel<<<blocks, threads, 0, ctx->stream>>>(out, iters, 1e-3);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&el, e0, e1);
    if (el >= ms * 0.9) break;
    iters = (int)(iters * (ms / (el > 0.01f ? el : 0.01f))) + 1;
    if (iters > (1 << 28)) iters = 1 << 28;
  }
  // 4 chains x 16*8*4 FMA x 2 flops per lane-group of 32 threads
  const double flops = 2.0 * 16 * 8 * 4 * 4 * (double)iters * blocks * (threads / 32);
  *tflops = flops / (el * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaError_t e = cudaGetLastError();
  cudaFree(out);
  if (e != cudaSuccess) return mo_from_cuda_error(e);
  return MO_OK;
}

}  // extern "C"
