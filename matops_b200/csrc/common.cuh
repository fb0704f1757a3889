// Shared device/host helpers for the matops_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/matops_b200.h"

#define MO_HOST_DEVICE __host__ __device__ __forceinline__

// Bounded spin: every wait in these kernels gives up after this many polls, records
// MO_EDEVTIMEOUT in the context's device status word and returns.
#ifndef MO_SPIN_LIMIT
#define MO_SPIN_LIMIT MO_SPIN_LIMIT_DEFAULT
#endif

namespace mo {

// ---------------------------------------------------------------------------------------
// device status word: first error wins (atomicCAS from 0)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void set_status(int *status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// ---------------------------------------------------------------------------------------
// mbarrier / TMA / cp.async wrappers (PTX ISA 8.x)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Returns false (after recording a timeout) if the phase never completed.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *status) {
  for (uint32_t i = 0; i < MO_SPIN_LIMIT; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  set_status(status, MO_EDEVTIMEOUT);
  return false;
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// 2-D tiled TMA load into this CTA's shared memory, completion on `bar` (no multicast).
__device__ __forceinline__ void tma_load_2d(void *dst, const void *tmap, uint64_t *bar, int x,
                                            int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// 8-byte cp.async with zero fill when src_bytes == 0
__device__ __forceinline__ void cp_async_8(void *dst, const void *src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}

__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// ---------------------------------------------------------------------------------------
// FP64 tensor-pipe MMA: D(16x8) += A(16x4) * B(4x8)
// fragment ownership (lane = 4*g + t): a0=(g,t) a1=(g+8,t); b0=(t,g);
// d0=(g,2t) d1=(g,2t+1) d2=(g+8,2t) d3=(g+8,2t+1)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

}  // namespace mo

// ---------------------------------------------------------------------------------------
// host-side helpers
// ---------------------------------------------------------------------------------------
#define MO_CUDA_TRY(expr)                                  \
  do {                                                     \
    cudaError_t _e = (expr);                               \
    if (_e != cudaSuccess) return mo_from_cuda_error(_e);  \
  } while (0)

// Sets the dynamic shared-memory limit of a kernel before its launch.  Called on every
// launch (a cheap host call) rather than cached per device, so that it holds after a
// context reset and needs no shared state between host threads.
static inline int mo_smem_attr(const void *fn, int bytes) {
  const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaErrorMemoryAllocation) return MO_ENOMEM;
  return e == cudaSuccess ? MO_OK : MO_ECUDA;
}

static inline int mo_from_cuda_error(cudaError_t e) {
  if (e == cudaErrorMemoryAllocation) return MO_ENOMEM;
  if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDeviceFunction)
    return MO_ENOKERNEL;
  return MO_ECUDA;
}
