// jfc_sync.cuh — device work queues and the grid barrier of the persistent
// (cooperative) phase kernels.
#pragma once

#include "jfc_internal.h"

namespace jfc {

constexpr unsigned FULL = 0xffffffffu;

// Grid-wide barrier of a cooperative launch.  Every wait is bounded: after
// ~2^26 polls (seconds) the barrier raises ctr->error and returns false, and
// every block leaves its loop on the next check, so a lost block can never
// hang the device.  `on_last` runs on the last block to arrive, before the
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
      while (*vgen == g) {
        if (*verr) { ok = 0; break; }
        if (++spins > (1ull << 26)) { atomicExch(&ctr->error, 1); ok = 0; break; }
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

// ---------------------------------------------------------------- work list
// Multi-producer / multi-consumer ring of tile ids for the BFS (chaotic
// relaxation: a tile may be visited as soon as it is queued).  Cell c holds
// (sequence << 32) | tile; a producer of position p waits until the cell's
// sequence is p (free for this lap), a consumer of position p until it is
// p + 1 (published), then frees it for lap p + cap.  A tile is queued at most
// once at a time (flag), so at most ntiles <= cap items are outstanding and
// every wait is on a thread that is already making progress.  `pending`
// counts items pushed and not yet finished (a push raises it before the item
// is visible, wl_done lowers it after the item's own pushes), so the list is
// finished exactly when pending == 0; pollers never touch it.  All waits are
// bounded and raise ctr->error when they run out.
constexpr unsigned long long kSpinLimit = 1ull << 26;

struct WorkList {
  unsigned long long* cells;
  unsigned cap;          // power of two
  int* flags;
  DevCounters* ctr;
};

// Called by one thread.  Returns false on a timed-out wait.
__device__ __forceinline__ bool wl_push(const WorkList& w, int tile) {
  if (atomicExch(w.flags + tile, 1) != 0) return true;
  atomicAdd(&w.ctr->wq_pending, 1);
  const unsigned p = atomicAdd(&w.ctr->wq_tail, 1u);
  unsigned long long* c = w.cells + (p & (w.cap - 1));
  unsigned long long spins = 0;
  while ((unsigned)(*(volatile unsigned long long*)c >> 32) != p) {
    if (++spins > kSpinLimit || *(volatile int*)&w.ctr->error) { atomicExch(&w.ctr->error, 1); return false; }
    __nanosleep(20);
  }
  atomicExch(c, ((unsigned long long)(p + 1u) << 32) | (unsigned)tile);
  return true;
}

// Called by one thread.  Returns a tile (to be released with wl_done), -1
// when the list is finished, -2 on error.
__device__ __forceinline__ int wl_pop(const WorkList& w) {
  DevCounters* ctr = w.ctr;
  volatile unsigned* vh = &ctr->wq_head;
  volatile unsigned* vt = &ctr->wq_tail;
  volatile int* vp = &ctr->wq_pending;
  unsigned long long spins = 0;
  for (;;) {
    const unsigned h = *vh;
    const unsigned t = *vt;
    if ((int)(t - h) > 0) {
      if (atomicCAS(&ctr->wq_head, h, h + 1u) == h) {
        unsigned long long* c = w.cells + (h & (w.cap - 1));
        unsigned long long v;
        while ((unsigned)((v = *(volatile unsigned long long*)c) >> 32) != h + 1u) {
          if (++spins > kSpinLimit || *(volatile int*)&ctr->error) { atomicExch(&ctr->error, 1); return -2; }
          __nanosleep(20);
        }
        const int tile = (int)(unsigned)(v & 0xffffffffull);
        atomicExch(c, (unsigned long long)(h + w.cap) << 32);
        atomicExch(w.flags + tile, 0);
        return tile;
      }
      continue;
    }
    if (*vp == 0) return -1;   // nothing queued and nothing being processed: finished
    if (++spins > kSpinLimit || *(volatile int*)&ctr->error) { atomicExch(&ctr->error, 1); return -2; }
    __nanosleep(64);
  }
}

// Release the item taken by wl_pop (after every push it caused).
__device__ __forceinline__ void wl_done(const WorkList& w) {
  __threadfence();
  atomicSub(&w.ctr->wq_pending, 1);
}

}  // namespace jfc
