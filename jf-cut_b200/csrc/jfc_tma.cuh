// jfc_tma.cuh — tensor-memory-access (TMA) staging helpers for sm_100a:
// shared-memory mbarriers, tiled bulk tensor loads from this GPU's own global
// memory into the issuing CTA's own shared memory, and the proxy fences they
// need.
#pragma once

#include <cstdint>

namespace jfc {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// One-arrival mbarrier (the issuing thread's arrive carries the byte count).
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Make initialised mbarriers visible to the async proxy (a CTA is a cluster of one).
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Non-blocking test of the phase with parity `parity` (acquire, CTA scope).
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for a phase: false after `cap` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned long long cap) {
  unsigned long long spins = 0;
  while (!mbar_test(bar, parity)) {
    if (++spins > cap) return false;
    if (spins > 8) __nanosleep(32);
  }
  return true;
}

// Tiled tensor loads (global -> this CTA's shared memory), completion counted
// in bytes on `bar`.  Coordinates are elements; the innermost one times the
// element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_4d(void* dst, const void* tmap, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

// A tensor map written to global memory by a host copy is read through the
// tensor-map proxy: acquire it before the first load that uses it.
__device__ __forceinline__ void fence_tmap_acquire(const void* tmap) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tmap) : "memory");
}

// Order generic-proxy global writes (observed through a barrier) before
// later async-proxy (tensor) reads of the same memory.
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// Order generic-proxy shared-memory accesses before a later tensor load into
// the same shared memory.
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace jfc
