// Device kernels of the direct-summation hot path (sm_100a).
//
//   scatter_kernel   staged j -> FP64 state + unpredicted record
//                    (role of dev_copy_particles, kernels.cu:245-301)
//   predict_kernel   FP64 Taylor predictor -> force records
//                    (role of dev_predictor, kernels.cu:307-411)
//   force_kernel     i-tile x j-slice Hermite 4th/6th force, nearest
//                    neighbour and neighbour list
//                    (role of dev_evaluate_gravity_*, kernels.cu:552-1041)
//   reduce_kernel    deterministic FP64 sum of the per-slice partials and
//                    nearest-neighbour min (replaces the FP64 atomics of
//                    kernels.cu:970-1003)
#pragma once
#include "sapb_internal.cuh"

namespace sapb {

// ------------------------------------------------------------------------
// PTX helpers: shared-memory mbarriers and 1-D bulk copies (TMA engine).
// ------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> shared, completion signalled on `bar`.  Both
// addresses must be 16-byte aligned and `bytes` a multiple of 16.  No
// cluster multicast is used anywhere in this library.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// One suspending probe of phase `parity`: the hardware may park the thread
// for a bounded time inside try_wait, so waiting warps do not burn issue
// slots of the warps that compute.
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
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
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for phase `parity` of `bar`, giving up after `limit_ns` of wall
// time (~2 s by default) or 2^22 rounds of 64 polls, whichever comes first.
// Returns false on timeout; the caller records the error and carries on
// without waiting again, so no thread can hang.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint64_t limit_ns = 2000000000ull) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
#pragma unroll 1
  for (uint32_t round = 0; round < (1u << 22); round++) {
#pragma unroll 1
    for (int k = 0; k < 64; k++)
      if (mbar_try(bar, parity)) return true;
    if (global_timer_ns() - t0 > limit_ns) return false;
  }
  return false;
}
// Barrier among the `nthreads` consumer threads only (id 1; id 0 is
// __syncthreads).
__device__ __forceinline__ void named_barrier(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ float rsqrt_mufu(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Nearest-neighbour key: (ds2 bits, id) ordered as one unsigned 64-bit word,
// so the minimum picks the smallest ds2 and, on exact ties, the smallest id
// taken as unsigned (the cross-block rule of kernels.cu:994-1003).
__device__ __forceinline__ unsigned long long nn_key(float ds2, int id) {
  return ((unsigned long long)__float_as_uint(ds2) << 32) | (unsigned int)id;
}

}  // namespace sapb
