// kernels_pr.cu — block-wise push-relabel sweep (the JF-Cut core).
//
// Reference: graphcut_relabel_push (src/QVisualizer/cl/GraphCut/graphcut_push_relabel.cl:25-203
// for 2D, :215-439 for 3D) driven by QGCWidget::relabelPush (QGCWidget.cpp:2136-2154).
// The reference runs one work-group per 16x16 / 8x8x4 tile with the tile + a
// one-cell halo in __local memory, loops {relabel even, relabel odd, push even,
// push odd} to a local fixpoint, and sends boundary flow out with global
// atomics; even tiles and odd tiles of the checkerboard run in separate
// launches so that adjacent tiles never run at once.
//
// B200 design: one WARP per tile of 32 columns x R rows.  Lane x keeps the
// whole column's excess, height and residual arcs in registers; horizontal
// neighbours are one __shfl away, vertical ones are in the same thread, so a
// push/relabel round needs no shared memory and no __syncthreads.  A tile visit
// runs up to `local_iters` rounds (early exit when nothing moves), writes back
// only rows that changed (full 128-byte rows), and flags the neighbour tiles it
// pushed into.  Warps take chunks of 32 list entries from a device work queue
// (one atomic per chunk) and ballot the flagged tiles, so inactive tiles cost
// one byte read.  Checkerboard tile parity is kept (the launch processes one
// parity), which makes boundary updates race-free exactly as in the reference.
//
// Push-relabel invariants: heights only grow between global relabels;
// relabel = 1 + min over residual arcs, applied only to active nodes with no
// admissible arc; pushes go along h(u) = h(v) + 1 with a fixed height vector,
// so two neighbours never push to each other in one round.
#include "jfc_internal.h"

namespace {

constexpr unsigned FULL = 0xffffffffu;

template <int DIMS, int TY_, int TZ_>
struct Shape {
  static constexpr int TY = TY_, TZ = TZ_;
  static constexpr int R = TY * TZ;
  static constexpr int XP = 0, YP = 1;
  static constexpr int ZP = DIMS == 2 ? 0 : 2;   // unused in 2D
  static constexpr int ZM = DIMS == 2 ? 0 : 3;   // unused in 2D
  static constexpr int YM = DIMS == 2 ? 2 : 4;
  static constexpr int XM = DIMS == 2 ? 3 : 5;
};

// All register state of one warp tile.
template <int DIMS, int TY, int TZ>
struct TileRegs {
  using S = Shape<DIMS, TY, TZ>;
  static constexpr int R = S::R;
  int e[R], h[R];
  int rxp[R], ryp[R], rym[R], rxm[R];
  int rzp[DIMS == 3 ? R : 1], rzm[DIMS == 3 ? R : 1];
  int hyT[TZ], hyB[TZ];               // halo rows above / below, per z
  int hzT[DIMS == 3 ? TY : 1], hzB[DIMS == 3 ? TY : 1];  // halo planes, per y
  unsigned de, dh, dxp, dyp, dym, dxm, dzp, dzm;          // dirty row masks
};

// Per-warp shared scratch: side-halo heights (read by lanes 0 / 31) and the
// flow pushed out of the tile, accumulated over the visit and sent to global
// memory once at the end (keeps the rare boundary addresses out of registers).
template <int DIMS, int TY, int TZ>
struct WarpSmem {
  static constexpr int R = TY * TZ;
  int side[2][R];                     // [0] left neighbour heights, [1] right
  int out_x[2][R];                    // [0] pushed to x-1, [1] pushed to x+1
  int out_y[2][TZ * 32];              // [0] pushed to y0-1, [1] to y0+TY (per z, lane)
  int out_z[2][DIMS == 3 ? TY * 32 : 1];  // [0] to z0-1, [1] to z0+TZ (per y, lane)
};

template <int DIMS, int TY, int TZ>
__device__ __forceinline__ int row_off(int pitch, int slab, int i) {
  const int y = i % TY, z = i / TY;
  return y * pitch + (DIMS == 3 ? z * slab : 0);
}

template <int DIMS, int TY, int TZ>
__device__ __forceinline__ void neighbour_heights(const TileRegs<DIMS, TY, TZ>& t,
                                                  const WarpSmem<DIMS, TY, TZ>& w, int i, int lane,
                                                  int& hxp, int& hxm, int& hyp, int& hym, int& hzp,
                                                  int& hzm) {
  const int y = i % TY, z = i / TY;
  hxm = __shfl_up_sync(FULL, t.h[i], 1);
  hxp = __shfl_down_sync(FULL, t.h[i], 1);
  if (lane == 0) hxm = w.side[0][i];
  if (lane == 31) hxp = w.side[1][i];
  hyp = (y < TY - 1) ? t.h[(i + 1 < t.R) ? i + 1 : i] : t.hyB[z];
  hym = (y > 0) ? t.h[(i > 0) ? i - 1 : 0] : t.hyT[z];
  if constexpr (DIMS == 3) {
    hzp = (z < TZ - 1) ? t.h[(i + TY < t.R) ? i + TY : i] : t.hzB[y];
    hzm = (z > 0) ? t.h[(i >= TY) ? i - TY : 0] : t.hzT[y];
  } else {
    hzp = JFC_INF; hzm = JFC_INF;
  }
}

// Relabel round: active nodes without an admissible arc move to 1 + min
// over residual arcs (graphcut_push_relabel.cl:80-99 recomputes the same
// minimum for every node with e >= 0; here only active, non-admissible ones
// move so heights stay monotone between global relabels).
template <int DIMS, int TY, int TZ>
__device__ __forceinline__ bool relabel_round(TileRegs<DIMS, TY, TZ>& t, const WarpSmem<DIMS, TY, TZ>& w,
                                              int lane) {
  bool any = false;
#pragma unroll
  for (int i = 0; i < t.R; ++i) {
    int hxp, hxm, hyp, hym, hzp, hzm;
    neighbour_heights(t, w, i, lane, hxp, hxm, hyp, hym, hzp, hzm);
    if (t.e[i] > 0 && t.h[i] < JFC_INF) {
      const int hm = t.h[i] - 1;
      bool adm = (t.rxp[i] > 0 && hxp == hm) | (t.ryp[i] > 0 && hyp == hm) |
                 (t.rym[i] > 0 && hym == hm) | (t.rxm[i] > 0 && hxm == hm);
      if constexpr (DIMS == 3) adm |= (t.rzp[i] > 0 && hzp == hm) | (t.rzm[i] > 0 && hzm == hm);
      if (!adm) {
        int m = JFC_INF;
        if (t.rxp[i] > 0) m = min(m, hxp);
        if (t.ryp[i] > 0) m = min(m, hyp);
        if (t.rym[i] > 0) m = min(m, hym);
        if (t.rxm[i] > 0) m = min(m, hxm);
        if constexpr (DIMS == 3) {
          if (t.rzp[i] > 0) m = min(m, hzp);
          if (t.rzm[i] > 0) m = min(m, hzm);
        }
        t.h[i] = min(m + 1, JFC_INF);
        t.dh |= 1u << i;
        any = true;
      }
    }
  }
  return any;
}

// One row of the push round.  Vertical pushes inside the tile go straight
// into the receiving row's registers; pushes across the tile border are
// accumulated in the warp's shared scratch and sent with global atomics after
// the visit (graphcut_push_relabel.cl:184-195 does the same with __local
// halo cells).  The neighbour tile is of the other parity and not running;
// the atomic covers two same-parity tiles sharing a corner neighbour.
template <int DIMS, int TY, int TZ>
__device__ __forceinline__ bool push_row(TileRegs<DIMS, TY, TZ>& t, WarpSmem<DIMS, TY, TZ>& w, int i,
                                         int lane) {
  const int y = i % TY, z = i / TY;
  int hxp, hxm, hyp, hym, hzp, hzm;
  neighbour_heights(t, w, i, lane, hxp, hxm, hyp, hym, hzp, hzm);
  int pr = 0, pl = 0;
  bool moved = false;
  if (t.e[i] > 0 && t.h[i] < JFC_INF) {
    const int hm = t.h[i] - 1;
    int ex = t.e[i];
    if (t.rxp[i] > 0 && hxp == hm) {
      const int d = min(ex, t.rxp[i]);
      t.rxp[i] -= d; ex -= d; pr = d; t.dxp |= 1u << i;
    }
    if (ex > 0 && t.ryp[i] > 0 && hyp == hm) {
      const int d = min(ex, t.ryp[i]);
      t.ryp[i] -= d; ex -= d; t.dyp |= 1u << i;
      if (y < TY - 1) {
        const int j = (i + 1 < t.R) ? i + 1 : i;
        t.e[j] += d; t.rym[j] += d; t.de |= 1u << j; t.dym |= 1u << j;
      } else {
        w.out_y[1][z * 32 + lane] += d;
      }
    }
    if (ex > 0 && t.rym[i] > 0 && hym == hm) {
      const int d = min(ex, t.rym[i]);
      t.rym[i] -= d; ex -= d; t.dym |= 1u << i;
      if (y > 0) {
        const int j = (i > 0) ? i - 1 : 0;
        t.e[j] += d; t.ryp[j] += d; t.de |= 1u << j; t.dyp |= 1u << j;
      } else {
        w.out_y[0][z * 32 + lane] += d;
      }
    }
    if constexpr (DIMS == 3) {
      if (ex > 0 && t.rzp[i] > 0 && hzp == hm) {
        const int d = min(ex, t.rzp[i]);
        t.rzp[i] -= d; ex -= d; t.dzp |= 1u << i;
        if (z < TZ - 1) {
          const int j = (i + TY < t.R) ? i + TY : i;
          t.e[j] += d; t.rzm[j] += d; t.de |= 1u << j; t.dzm |= 1u << j;
        } else {
          w.out_z[1][y * 32 + lane] += d;
        }
      }
      if (ex > 0 && t.rzm[i] > 0 && hzm == hm) {
        const int d = min(ex, t.rzm[i]);
        t.rzm[i] -= d; ex -= d; t.dzm |= 1u << i;
        if (z > 0) {
          const int j = (i >= TY) ? i - TY : 0;
          t.e[j] += d; t.rzp[j] += d; t.de |= 1u << j; t.dzp |= 1u << j;
        } else {
          w.out_z[0][y * 32 + lane] += d;
        }
      }
    }
    if (ex > 0 && t.rxm[i] > 0 && hxm == hm) {
      const int d = min(ex, t.rxm[i]);
      t.rxm[i] -= d; ex -= d; pl = d; t.dxm |= 1u << i;
    }
    if (ex != t.e[i]) { t.e[i] = ex; t.de |= 1u << i; moved = true; }
  }
  // horizontal exchange: what my left neighbour pushed right arrives here
  int in_l = __shfl_up_sync(FULL, pr, 1);
  int in_r = __shfl_down_sync(FULL, pl, 1);
  if (lane == 0) { if (pl) w.out_x[0][i] += pl; in_l = 0; }
  if (lane == 31) { if (pr) w.out_x[1][i] += pr; in_r = 0; }
  if (in_l | in_r) {
    t.e[i] += in_l + in_r;
    t.rxm[i] += in_l;
    t.rxp[i] += in_r;
    t.de |= 1u << i;
    if (in_l) t.dxm |= 1u << i;
    if (in_r) t.dxp |= 1u << i;
  }
  return moved;
}

template <int DIMS, int TY, int TZ>
__device__ __forceinline__ void pr_tile(const GridDev* __restrict__ gd, int4 ti, int tid,
                                        uint8_t* __restrict__ flags, int local_iters,
                                        WarpSmem<DIMS, TY, TZ>& w) {
  using S = Shape<DIMS, TY, TZ>;
  constexpr int R = S::R;
  const int lane = threadIdx.x & 31;
  const GridDev& g = gd[ti.x];
  const int pitch = g.pitch;
  const int slab = g.pitch * g.Hp;
  const int x0 = ti.y * 32, y0 = ti.z * TY, z0 = ti.w * TZ;
  const long long base = (long long)(x0 + lane) + (long long)y0 * pitch + (long long)z0 * slab;
  int* const E = g.e + base;
  int* const H = g.h + base;
  const bool has_yT = y0 > 0, has_yB = y0 + TY < g.Hp;
  const bool has_zT = z0 > 0, has_zB = (DIMS == 3) && (z0 + TZ < g.Dp);

  TileRegs<DIMS, TY, TZ> t;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int n = row_off<DIMS, TY, TZ>(pitch, slab, i);
    t.e[i] = E[n]; t.h[i] = H[n];
    t.rxp[i] = g.r[S::XP][base + n]; t.ryp[i] = g.r[S::YP][base + n];
    t.rym[i] = g.r[S::YM][base + n]; t.rxm[i] = g.r[S::XM][base + n];
    if constexpr (DIMS == 3) { t.rzp[i] = g.r[S::ZP][base + n]; t.rzm[i] = g.r[S::ZM][base + n]; }
  }
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    const int n = row_off<DIMS, TY, TZ>(pitch, slab, z * TY);
    t.hyT[z] = has_yT ? H[n - pitch] : JFC_INF;
    t.hyB[z] = has_yB ? H[n + TY * pitch] : JFC_INF;
  }
  if constexpr (DIMS == 3) {
#pragma unroll
    for (int y = 0; y < TY; ++y) {
      const int n = row_off<DIMS, TY, TZ>(pitch, slab, y);
      t.hzT[y] = has_zT ? H[n - slab] : JFC_INF;
      t.hzB[y] = has_zB ? H[n + TZ * slab] : JFC_INF;
    }
  }
  {
    // side halos: lane l < R loads the left neighbour of row l, lane 16+l the right one
    const int row = lane & 15;
    const int side = lane >> 4;
    const int xs = side ? x0 + 32 : x0 - 1;
    if (row < R) {
      int v = JFC_INF;
      if (xs >= 0 && xs < pitch) v = H[(xs - x0 - lane) + row_off<DIMS, TY, TZ>(pitch, slab, row)];
      w.side[side][row] = v;
      w.out_x[side][row] = 0;
    }
#pragma unroll
    for (int k = lane; k < TZ * 32; k += 32) { w.out_y[0][k] = 0; w.out_y[1][k] = 0; }
    if constexpr (DIMS == 3) {
#pragma unroll
      for (int k = lane; k < TY * 32; k += 32) { w.out_z[0][k] = 0; w.out_z[1][k] = 0; }
    }
    __syncwarp();
  }
  t.de = t.dh = t.dxp = t.dyp = t.dym = t.dxm = t.dzp = t.dzm = 0u;

  for (int it = 0; it < local_iters; ++it) {
    const bool rl = relabel_round(t, w, lane);
    bool mv = false;
    if ((it & 1) == 0) {
#pragma unroll
      for (int i = 0; i < R; ++i) mv |= push_row(t, w, i, lane);
    } else {
#pragma unroll
      for (int i = R - 1; i >= 0; --i) mv |= push_row(t, w, i, lane);
    }
    if (!__any_sync(FULL, rl | mv)) break;
  }

  // write back rows that changed (whole 128-byte rows)
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int n = row_off<DIMS, TY, TZ>(pitch, slab, i);
    const unsigned b = 1u << i;
    if (__any_sync(FULL, t.de & b)) E[n] = t.e[i];
    if (__any_sync(FULL, t.dh & b)) H[n] = t.h[i];
    if (__any_sync(FULL, t.dxp & b)) g.r[S::XP][base + n] = t.rxp[i];
    if (__any_sync(FULL, t.dyp & b)) g.r[S::YP][base + n] = t.ryp[i];
    if (__any_sync(FULL, t.dym & b)) g.r[S::YM][base + n] = t.rym[i];
    if (__any_sync(FULL, t.dxm & b)) g.r[S::XM][base + n] = t.rxm[i];
    if constexpr (DIMS == 3) {
      if (__any_sync(FULL, t.dzp & b)) g.r[S::ZP][base + n] = t.rzp[i];
      if (__any_sync(FULL, t.dzm & b)) g.r[S::ZM][base + n] = t.rzm[i];
    }
  }
  bool act = false;
#pragma unroll
  for (int i = 0; i < R; ++i) act |= (t.e[i] > 0) & (t.h[i] < JFC_INF);
  act = __any_sync(FULL, act);

  // flush the flow pushed across the tile border into the neighbours' excess
  // and reverse residual arcs
  __syncwarp();
  unsigned out = 0u;
  {
    const int row = lane & 15;
    const int side = lane >> 4;
    int v = (row < R) ? w.out_x[side][row] : 0;
    if (v) {
      const int n = row_off<DIMS, TY, TZ>(pitch, slab, row) + (side ? 32 - lane : -1 - lane);
      atomicAdd(E + n, v);
      atomicAdd(g.r[side ? S::XM : S::XP] + base + n, v);
    }
    const unsigned bl = __ballot_sync(FULL, v != 0);
    if (bl & 0x0000ffffu) out |= 1u;
    if (bl & 0xffff0000u) out |= 2u;
  }
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    const int n = row_off<DIMS, TY, TZ>(pitch, slab, z * TY);
    const int up = w.out_y[0][z * 32 + lane], dn = w.out_y[1][z * 32 + lane];
    if (up) { atomicAdd(E + n - pitch, up); atomicAdd(g.r[S::YP] + base + n - pitch, up); }
    if (dn) { atomicAdd(E + n + TY * pitch, dn); atomicAdd(g.r[S::YM] + base + n + TY * pitch, dn); }
    if (__any_sync(FULL, up != 0)) out |= 4u;
    if (__any_sync(FULL, dn != 0)) out |= 8u;
  }
  if constexpr (DIMS == 3) {
#pragma unroll
    for (int y = 0; y < TY; ++y) {
      const int n = row_off<DIMS, TY, TZ>(pitch, slab, y);
      const int bk = w.out_z[0][y * 32 + lane], fw = w.out_z[1][y * 32 + lane];
      if (bk) { atomicAdd(E + n - slab, bk); atomicAdd(g.r[S::ZP] + base + n - slab, bk); }
      if (fw) { atomicAdd(E + n + TZ * slab, fw); atomicAdd(g.r[S::ZM] + base + n + TZ * slab, fw); }
      if (__any_sync(FULL, bk != 0)) out |= 16u;
      if (__any_sync(FULL, fw != 0)) out |= 32u;
    }
  }
  __syncwarp();
  if (lane == 0) {
    flags[tid] = act ? 1 : 0;
    const int txs = g.tiles_x, tys = g.tiles_y;
    if (out & 1u) flags[tid - 1] = 1;
    if (out & 2u) flags[tid + 1] = 1;
    if (out & 4u) flags[tid - txs] = 1;
    if (out & 8u) flags[tid + txs] = 1;
    if (DIMS == 3) {
      if (out & 16u) flags[tid - txs * tys] = 1;
      if (out & 32u) flags[tid + txs * tys] = 1;
    }
  }
}

template <int DIMS, int TY, int TZ>
__global__ void __launch_bounds__(256, (TY * TZ <= 8) ? 2 : 1) k_pr_sweep(const GridDev* __restrict__ gd,
                                                  const int4* __restrict__ info,
                                                  const int* __restrict__ list, int nlist,
                                                  uint8_t* __restrict__ flags, int local_iters,
                                                  DevCounters* __restrict__ ctr) {
  const int lane = threadIdx.x & 31;
  __shared__ WarpSmem<DIMS, TY, TZ> s_w[8];
  unsigned long long visits = 0;
  for (;;) {
    unsigned chunk = 0;
    if (lane == 0) chunk = atomicAdd(&ctr->tk.chunk, 1u);
    chunk = __shfl_sync(FULL, chunk, 0);
    const long long b = (long long)chunk * 32;
    if (b >= nlist) break;
    const long long li = b + lane;
    int tid = 0;
    bool f = false;
    if (li < nlist) {
      tid = list[li];
      f = flags[tid] != 0;
    }
    unsigned m = __ballot_sync(FULL, f);
    while (m) {
      const int src = __ffs(m) - 1;
      m &= m - 1;
      const int tt = __shfl_sync(FULL, tid, src);
      pr_tile<DIMS, TY, TZ>(gd, info[tt], tt, flags, local_iters, s_w[threadIdx.x >> 5]);
      ++visits;
    }
  }
  // per-block visit count + ticket reset by the last block
  __shared__ unsigned long long s_vis;
  if (threadIdx.x == 0) s_vis = 0;
  __syncthreads();
  if (lane == 0 && visits) atomicAdd(&s_vis, visits);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_vis) atomicAdd(&ctr->visits, s_vis);
    __threadfence();
    const unsigned prev = atomicAdd(&ctr->tk.done, 1u);
    if (prev == gridDim.x - 1) {
      ctr->tk.chunk = 0;
      ctr->tk.done = 0;
      __threadfence();
    }
  }
}

template <int DIMS, int TY, int TZ>
cudaError_t launch_t(const TileSet& ts, int parity, int local_iters, cudaStream_t s) {
  static int blocks = 0;
  if (!blocks) blocks = persistent_blocks((const void*)k_pr_sweep<DIMS, TY, TZ>, 256, 0);
  if (ts.nlist[parity] == 0) return cudaSuccess;
  int nb = blocks;
  const int need = (ts.nlist[parity] + 31) / 32;       // chunks of 32 tiles
  const int max_useful = (need + 7) / 8;               // 8 warps per block
  if (nb > max_useful) nb = max_useful;
  if (nb < 1) nb = 1;
  jfc_note_launch();
  k_pr_sweep<DIMS, TY, TZ><<<nb, 256, 0, s>>>(ts.d_desc, ts.d_info, ts.d_list[parity],
                                              ts.nlist[parity], ts.d_flag_pr, local_iters, ts.d_ctr);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pr_sweep(const TileSet& ts, int parity, int local_iters, cudaStream_t s) {
  if (ts.dims == 2) {
    switch (ts.TR) {
      case 8: return launch_t<2, 8, 1>(ts, parity, local_iters, s);
      case 16: return launch_t<2, 16, 1>(ts, parity, local_iters, s);
      default: return cudaErrorInvalidValue;
    }
  }
  if (ts.TY == 4 && ts.TZ == 4) return launch_t<3, 4, 4>(ts, parity, local_iters, s);
  if (ts.TY == 4 && ts.TZ == 2) return launch_t<3, 4, 2>(ts, parity, local_iters, s);
  return cudaErrorInvalidValue;
}
