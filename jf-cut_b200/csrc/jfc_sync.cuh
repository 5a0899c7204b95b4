// jfc_sync.cuh — device work queues and the grid barrier of the persistent
// (cooperative) phase kernels.
#pragma once

#include "jfc_internal.h"

namespace jfc {

constexpr unsigned FULL = 0xffffffffu;

// Polls a device-side wait makes before it gives up: ctr->spin_limit, or
// 2^26 (seconds) when it is 0.
__device__ __forceinline__ unsigned long long spin_cap(const DevCounters* ctr) {
  const unsigned long long v = *(const volatile unsigned long long*)&ctr->spin_limit;
  return v ? v : (1ull << 26);
}

// Grid-wide barrier of a cooperative launch.  Every wait is bounded: after
// spin_cap polls the barrier raises ctr->error and returns false, and every
// block leaves its loop on the next check, so a lost block can never hang
// the device.  `on_last` runs on the last block to arrive, before the
// release (queue / ticket resets between phases).
template <typename F>
__device__ __forceinline__ bool grid_sync(DevCounters* ctr, F on_last) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = &ctr->bar_gen;
    volatile int* verr = &ctr->error;
    const unsigned g = *vgen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(&ctr->bar_count, 1u) == gridDim.x - 1) {
      on_last();
      ctr->bar_count = 0;
      __threadfence();
      atomicAdd(&ctr->bar_gen, 1u);
    } else {
      unsigned long long spins = 0;
      const unsigned long long cap = spin_cap(ctr);
      while (*vgen == g) {
        if (*verr) { ok = 0; break; }
        if (++spins > cap) { atomicExch(&ctr->error, 1); ok = 0; break; }
        __nanosleep(100);
      }
    }
    __threadfence();
    s_ok = ok && (*verr == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ int vload(const int* p) { return *(const volatile int*)p; }

// Distance cap of the running global relabel: distances at or above it are
// stored as unreachable (JFC_INF); no cap when ctr->h_cap is 0.
// (set before the kernel that reads it runs, constant during it: an ordinary
// cached load, not a poll of L2 on every tile visit)
__device__ __forceinline__ int height_cap(const DevCounters* ctr) {
  const int v = ctr->h_cap;
  return v > 0 ? v : JFC_INF;
}
// The cap for grid g: its own when set, else the tile set's.
__device__ __forceinline__ int cap_of(const GridDev& g, const DevCounters* ctr) {
  return g.h_cap > 0 ? g.h_cap : height_cap(ctr);
}

// Device-wide nanosecond clock (phase timing of the persistent kernels).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Phase-clock instrumentation (builds with -DJFC_PHASE_CLOCK): thread 0 adds
// the SM cycles since `t` to counter k and restarts `t`.
#ifdef JFC_PHASE_CLOCK
#define JFC_PCLK_DECL long long _pclk = clock64();
#define JFC_PCLK(ctr, k)                                                            \
  do {                                                                              \
    if (threadIdx.x == 0) {                                                         \
      const long long _n = clock64();                                               \
      atomicAdd(&(ctr)->prof[k], (unsigned long long)(_n - _pclk));                 \
      _pclk = _n;                                                                   \
    }                                                                               \
  } while (0)
#else
#define JFC_PCLK_DECL
#define JFC_PCLK(ctr, k) do {} while (0)
#endif

// Warp-cooperative append of up to 32 candidate tiles: lane k offers `tile`
// when `want`; with `flags`, a tile is appended only by the lane that flips
// its flag 0 -> 1 (so a queue never holds a tile twice).
__device__ __forceinline__ void warp_append(bool want, int tile, int* flags, int* queue, int* qn) {
  bool won = false;
  if (want) won = flags ? (atomicExch(flags + tile, 1) == 0) : true;
  const unsigned m = __ballot_sync(FULL, won);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(qn, __popc(m));
  base = __shfl_sync(FULL, base, leader);
  if (won) queue[base + __popc(m & ((1u << lane) - 1u))] = tile;
}

// One warp-level ticket from a device counter.
__device__ __forceinline__ unsigned warp_ticket(unsigned* t) {
  unsigned v = 0;
  if ((threadIdx.x & 31) == 0) v = atomicAdd(t, 1u);
  return __shfl_sync(FULL, v, 0);
}

}  // namespace jfc
