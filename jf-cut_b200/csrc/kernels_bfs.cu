// kernels_bfs.cu — global relabel, convergence / cut BFS, reductions and
// layout helpers.
//
// Global relabel — reference graphcut_init_global_relabel / graphcut_global_relabel
// (graphcut_global_relabel.cl:19-124 2D, :128-249 3D) driven by QGCWidget::globalRelabel
// (QGCWidget.cpp:2208-2241): heights = exact BFS distance to the deficit nodes
// (e < 0) over residual arcs, computed by in-tile fixpoint relaxation
// h = min(h, h(v) + 1) with tiles revisited in level sweeps ordered by the
// jump-flooding tile BFS (graphcut_bfs_block.cl).
// Here: the relaxation is monotone (heights only fall from INF), so every tile
// may run at once with no parity and no ordering; a tile whose boundary fell
// flags its neighbours in a double-buffered flag array and passes repeat until
// no tile is flagged.  Each visit relaxes the whole warp tile in registers with
// alternating top-down / bottom-up sweeps (lane = column, shuffles across
// columns), which plays the role of the reference's in-tile fixpoint plus its
// back-and-forth level order.  The first pass is fused with the initialisation
// (h = 0 on deficits, INF elsewhere) and reads neighbour excess for its halo.
// Each visit also records whether the tile holds an active node
// (e > 0 and h < INF): this is the device-side active-tile count
// (graphcut_count_node, graphcut_count_block.cl:19-47) that decides convergence.
//
// Cut — reference graphcut_init_cut / graphcut_compute_cut (graphcut_compute_cut.cl:19-140):
// the source side is every node reachable from {e > 0} along residual arcs.
// Here a warp tile is R rows of 32-bit words (bit = lane); each row's in-arc
// masks are built once with ballots, propagation along a row is a 5-step
// shift-doubling closure and across rows is word AND/OR, so a tile converges
// in a few word operations per row.  Reaching a deficit raises cut_bad (the
// reference's done[1] divergence flag).
#include "jfc_internal.h"

namespace {

constexpr unsigned FULL = 0xffffffffu;

template <int DIMS>
struct Dirs {
  static constexpr int XP = 0, YP = 1;
  static constexpr int ZP = DIMS == 2 ? 0 : 2;
  static constexpr int ZM = DIMS == 2 ? 0 : 3;
  static constexpr int YM = DIMS == 2 ? 2 : 4;
  static constexpr int XM = DIMS == 2 ? 3 : 5;
};

struct Addr {
  long long base, pitch, slab;
  bool has_yT, has_yB, has_zT, has_zB, has_xL, has_xR;
  int x0, y0, z0;
};

template <int DIMS, int TY, int TZ>
__device__ __forceinline__ Addr make_addr(const GridDev& g, int4 ti, int lane) {
  Addr a;
  a.pitch = g.pitch;
  a.slab = (long long)g.pitch * g.Hp;
  a.x0 = ti.y * 32; a.y0 = ti.z * TY; a.z0 = ti.w * TZ;
  a.base = (long long)(a.x0 + lane) + (long long)a.y0 * a.pitch + (long long)a.z0 * a.slab;
  a.has_yT = a.y0 > 0;
  a.has_yB = a.y0 + TY < g.Hp;
  a.has_zT = (DIMS == 3) && a.z0 > 0;
  a.has_zB = (DIMS == 3) && (a.z0 + TZ < g.Dp);
  a.has_xL = a.x0 > 0;
  a.has_xR = a.x0 + 32 < g.pitch;
  return a;
}

template <int TY>
__device__ __forceinline__ long long roff(const Addr& a, int i) {
  return a.base + (long long)(i % TY) * a.pitch + (long long)(i / TY) * a.slab;
}

// ------------------------------------------------------------ global relabel
template <int DIMS, int TY, int TZ, bool FIRST>
__device__ __forceinline__ void relabel_tile(const GridDev& g, int4 ti, int tid,
                                             uint8_t* __restrict__ fnext, uint8_t* __restrict__ fpr,
                                             int* __restrict__ pending, int& act_delta) {
  using D = Dirs<DIMS>;
  constexpr int R = TY * TZ;
  const int lane = threadIdx.x & 31;
  const Addr a = make_addr<DIMS, TY, TZ>(g, ti, lane);
  const int* __restrict__ E = g.e;
  int* __restrict__ H = g.h;
  // residual-arc bits per row: bit k set when arc k is residual
  unsigned arcs[R];
  int h[R];
  bool act_pos[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const long long n = roff<TY>(a, i);
    const int e = E[n];
    unsigned m = 0;
    m |= (g.r[D::XP][n] > 0) ? 1u : 0u;
    m |= (g.r[D::YP][n] > 0) ? 2u : 0u;
    m |= (g.r[D::YM][n] > 0) ? 4u : 0u;
    m |= (g.r[D::XM][n] > 0) ? 8u : 0u;
    if constexpr (DIMS == 3) {
      m |= (g.r[D::ZP][n] > 0) ? 16u : 0u;
      m |= (g.r[D::ZM][n] > 0) ? 32u : 0u;
    }
    arcs[i] = m;
    act_pos[i] = e > 0;
    if constexpr (FIRST) h[i] = (e < 0) ? 0 : JFC_INF;
    else h[i] = H[n];
  }
  // halo heights (FIRST: derived from neighbour excess)
  auto halo = [&](long long n) -> int {
    if constexpr (FIRST) return (E[n] < 0) ? 0 : JFC_INF;
    else return H[n];
  };
  int hyT[TZ], hyB[TZ];
  int hzT[DIMS == 3 ? TY : 1], hzB[DIMS == 3 ? TY : 1];
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    const long long n = roff<TY>(a, z * TY);
    hyT[z] = a.has_yT ? halo(n - a.pitch) : JFC_INF;
    hyB[z] = a.has_yB ? halo(n + (long long)TY * a.pitch) : JFC_INF;
  }
  if constexpr (DIMS == 3) {
#pragma unroll
    for (int y = 0; y < TY; ++y) {
      const long long n = roff<TY>(a, y);
      hzT[y] = a.has_zT ? halo(n - a.slab) : JFC_INF;
      hzB[y] = a.has_zB ? halo(n + (long long)TZ * a.slab) : JFC_INF;
    }
  }
  int hs[R];
  {
    const int row = lane & 15;
    const bool left = lane < 16;
    int v = JFC_INF;
    if (row < R && (left ? a.has_xL : a.has_xR)) {
      const long long n = (long long)(left ? a.x0 - 1 : a.x0 + 32) +
                          (long long)(a.y0 + row % TY) * a.pitch + (long long)(a.z0 + row / TY) * a.slab;
      v = halo(n);
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int lv = __shfl_sync(FULL, v, i);
      const int rv = __shfl_sync(FULL, v, 16 + i);
      hs[i] = (lane == 0) ? lv : rv;
    }
  }

  unsigned dirty = 0;
  bool converged = false;
  auto relax_row = [&](int i) -> bool {
    const int y = i % TY, z = i / TY;
    int hxm = __shfl_up_sync(FULL, h[i], 1);
    int hxp = __shfl_down_sync(FULL, h[i], 1);
    if (lane == 0) hxm = hs[i];
    if (lane == 31) hxp = hs[i];
    const int hyp = (y < TY - 1) ? h[(i + 1 < R) ? i + 1 : i] : hyB[z];
    const int hym = (y > 0) ? h[(i > 0) ? i - 1 : 0] : hyT[z];
    const unsigned m = arcs[i];
    int v = h[i];
    if (m & 1u) v = min(v, hxp + 1);
    if (m & 2u) v = min(v, hyp + 1);
    if (m & 4u) v = min(v, hym + 1);
    if (m & 8u) v = min(v, hxm + 1);
    if constexpr (DIMS == 3) {
      const int hzp = (z < TZ - 1) ? h[(i + TY < R) ? i + TY : i] : hzB[y];
      const int hzm = (z > 0) ? h[(i >= TY) ? i - TY : 0] : hzT[y];
      if (m & 16u) v = min(v, hzp + 1);
      if (m & 32u) v = min(v, hzm + 1);
    }
    if (v < h[i]) { h[i] = v; dirty |= 1u << i; return true; }
    return false;
  };
  for (int it = 0; it < 64; ++it) {
    bool ch = false;
#pragma unroll
    for (int i = 0; i < R; ++i) ch |= relax_row(i);
#pragma unroll
    for (int i = R - 1; i >= 0; --i) ch |= relax_row(i);
    if (!__any_sync(FULL, ch)) { converged = true; break; }
  }

#pragma unroll
  for (int i = 0; i < R; ++i) {
    if (FIRST || __any_sync(FULL, (dirty >> i) & 1u)) H[roff<TY>(a, i)] = h[i];
  }
  // flag neighbours whose halo fell, and myself if not yet at the fixpoint
  unsigned rows_dirty = __reduce_or_sync(FULL, dirty);
  const unsigned lane0 = __shfl_sync(FULL, dirty, 0);
  const unsigned lane31 = __shfl_sync(FULL, dirty, 31);
  bool act = false;
#pragma unroll
  for (int i = 0; i < R; ++i) act |= act_pos[i] & (h[i] < JFC_INF);
  act = __any_sync(FULL, act);
  if (lane == 0) {
    unsigned ymask0 = 0, ymask1 = 0, zmask0 = 0, zmask1 = 0;
#pragma unroll
    for (int z = 0; z < TZ; ++z) { ymask0 |= 1u << (z * TY); ymask1 |= 1u << (z * TY + TY - 1); }
#pragma unroll
    for (int y = 0; y < TY; ++y) { zmask0 |= 1u << y; zmask1 |= 1u << ((TZ - 1) * TY + y); }
    bool any = false;
    const int txs = g.tiles_x, tys = g.tiles_y;
    if ((rows_dirty & ymask0) && a.has_yT) { fnext[tid - txs] = 1; any = true; }
    if ((rows_dirty & ymask1) && a.has_yB) { fnext[tid + txs] = 1; any = true; }
    if (DIMS == 3) {
      if ((rows_dirty & zmask0) && a.has_zT) { fnext[tid - txs * tys] = 1; any = true; }
      if ((rows_dirty & zmask1) && a.has_zB) { fnext[tid + txs * tys] = 1; any = true; }
    }
    if (lane0 && a.has_xL) { fnext[tid - 1] = 1; any = true; }
    if (lane31 && a.has_xR) { fnext[tid + 1] = 1; any = true; }
    if (!converged) { fnext[tid] = 1; any = true; }
    if (any) *pending = 1;
    const int old = FIRST ? 0 : (int)fpr[tid];
    fpr[tid] = act ? 1 : 0;
    act_delta += (act ? 1 : 0) - old;
  }
}

template <int DIMS, int TY, int TZ, bool FIRST>
__global__ void __launch_bounds__(256) k_relabel(const GridDev* __restrict__ gd,
                                                 const int4* __restrict__ info, int ntiles,
                                                 uint8_t* __restrict__ fcur, uint8_t* __restrict__ fnext,
                                                 uint8_t* __restrict__ fpr, int* __restrict__ grid_active,
                                                 DevCounters* __restrict__ ctr, int pass) {
  const int lane = threadIdx.x & 31;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctr->pending[(pass + 1) & 1] = 0;
  int* pending = &ctr->pending[pass & 1];
  int cur_grid = -1, delta = 0;
  unsigned long long visits = 0;
  for (;;) {
    unsigned chunk = 0;
    if (lane == 0) chunk = atomicAdd(&ctr->tk.chunk, 1u);
    chunk = __shfl_sync(FULL, chunk, 0);
    const long long b = (long long)chunk * 32;
    if (b >= ntiles) break;
    const long long li = b + lane;
    bool f = li < ntiles;
    if (!FIRST && f) {
      f = fcur[li] != 0;
      if (f) fcur[li] = 0;
    }
    unsigned m = __ballot_sync(FULL, f);
    while (m) {
      const int src = __ffs(m) - 1;
      m &= m - 1;
      const int tt = (int)b + src;
      const int4 ti = info[tt];
      if (ti.x != cur_grid) {
        if (lane == 0 && delta != 0 && cur_grid >= 0) atomicAdd(&grid_active[cur_grid], delta);
        delta = 0;
        cur_grid = ti.x;
      }
      relabel_tile<DIMS, TY, TZ, FIRST>(gd[ti.x], ti, tt, fnext, fpr, pending, delta);
      ++visits;
    }
  }
  if (lane == 0 && delta != 0 && cur_grid >= 0) atomicAdd(&grid_active[cur_grid], delta);
  __shared__ unsigned long long s_vis;
  if (threadIdx.x == 0) s_vis = 0;
  __syncthreads();
  if (lane == 0 && visits) atomicAdd(&s_vis, visits);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_vis) atomicAdd(&ctr->bfs_visits, s_vis);
    __threadfence();
    const unsigned prev = atomicAdd(&ctr->tk.done, 1u);
    if (prev == gridDim.x - 1) {
      ctr->tk.chunk = 0;
      ctr->tk.done = 0;
      __threadfence();
    }
  }
}

// ------------------------------------------------------------------ cut BFS
__device__ __forceinline__ unsigned close_right(unsigned p, unsigned m) {
  // bit x reached from bit x-1 when m bit x is set; closure by doubling
  p |= (p << 1) & m; m &= m << 1;
  p |= (p << 2) & m; m &= m << 2;
  p |= (p << 4) & m; m &= m << 4;
  p |= (p << 8) & m; m &= m << 8;
  p |= (p << 16) & m;
  return p;
}
__device__ __forceinline__ unsigned close_left(unsigned p, unsigned m) {
  p |= (p >> 1) & m; m &= m >> 1;
  p |= (p >> 2) & m; m &= m >> 2;
  p |= (p >> 4) & m; m &= m >> 4;
  p |= (p >> 8) & m; m &= m >> 8;
  p |= (p >> 16) & m;
  return p;
}

template <int DIMS, int TY, int TZ, bool FIRST>
__device__ __forceinline__ void cut_tile(const GridDev& g, int4 ti, int tid,
                                         uint8_t* __restrict__ fnext, int* __restrict__ pending,
                                         int* __restrict__ bad) {
  using D = Dirs<DIMS>;
  constexpr int R = TY * TZ;
  const int lane = threadIdx.x & 31;
  const Addr a = make_addr<DIMS, TY, TZ>(g, ti, lane);
  const int* __restrict__ E = g.e;
  uint8_t* __restrict__ Lb = g.label;
  unsigned L[R], L0[R], IXL[R], IXR[R], IYU[R], IYD[R];
  unsigned IZU[DIMS == 3 ? R : 1], IZD[DIMS == 3 ? R : 1];
  unsigned NEG[R];
  {
    int rxp[R], ryp[R], rym[R], rxm[R], rzp[DIMS == 3 ? R : 1], rzm[DIMS == 3 ? R : 1];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const long long n = roff<TY>(a, i);
      rxp[i] = g.r[D::XP][n]; ryp[i] = g.r[D::YP][n]; rym[i] = g.r[D::YM][n]; rxm[i] = g.r[D::XM][n];
      if constexpr (DIMS == 3) { rzp[i] = g.r[D::ZP][n]; rzm[i] = g.r[D::ZM][n]; }
      const int e = E[n];
      NEG[i] = __ballot_sync(FULL, e < 0);
      if constexpr (FIRST) L[i] = __ballot_sync(FULL, e > 0);
      else L[i] = __ballot_sync(FULL, Lb[n] != 0);
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int y = i % TY, z = i / TY;
      const int fl = __shfl_up_sync(FULL, rxp[i], 1);
      const int fr = __shfl_down_sync(FULL, rxm[i], 1);
      IXL[i] = __ballot_sync(FULL, lane > 0 && fl > 0);
      IXR[i] = __ballot_sync(FULL, lane < 31 && fr > 0);
      IYU[i] = (y > 0) ? __ballot_sync(FULL, ryp[(i > 0) ? i - 1 : 0] > 0) : 0u;
      IYD[i] = (y < TY - 1) ? __ballot_sync(FULL, rym[(i + 1 < R) ? i + 1 : i] > 0) : 0u;
      if constexpr (DIMS == 3) {
        IZU[i] = (z > 0) ? __ballot_sync(FULL, rzp[(i >= TY) ? i - TY : 0] > 0) : 0u;
        IZD[i] = (z < TZ - 1) ? __ballot_sync(FULL, rzm[(i + TY < R) ? i + TY : i] > 0) : 0u;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i) L0[i] = L[i];
  // sources entering through the halo: neighbour reached and its arc toward us residual
  auto halo_lab = [&](long long n) -> bool {
    if constexpr (FIRST) return E[n] > 0;
    else return Lb[n] != 0;
  };
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    const long long n = roff<TY>(a, z * TY);
    bool s = false;
    if (a.has_yT) { const long long m = n - a.pitch; s = halo_lab(m) && g.r[D::YP][m] > 0; }
    L[z * TY] |= __ballot_sync(FULL, s);
    s = false;
    if (a.has_yB) { const long long m = n + (long long)TY * a.pitch; s = halo_lab(m) && g.r[D::YM][m] > 0; }
    L[z * TY + TY - 1] |= __ballot_sync(FULL, s);
  }
  if constexpr (DIMS == 3) {
#pragma unroll
    for (int y = 0; y < TY; ++y) {
      const long long n = roff<TY>(a, y);
      bool s = false;
      if (a.has_zT) { const long long m = n - a.slab; s = halo_lab(m) && g.r[D::ZP][m] > 0; }
      L[y] |= __ballot_sync(FULL, s);
      s = false;
      if (a.has_zB) { const long long m = n + (long long)TZ * a.slab; s = halo_lab(m) && g.r[D::ZM][m] > 0; }
      L[(TZ - 1) * TY + y] |= __ballot_sync(FULL, s);
    }
  }
  {
    const int row = lane & 15;
    const bool left = lane < 16;
    bool s = false;
    if (row < R && (left ? a.has_xL : a.has_xR)) {
      const long long n = (long long)(left ? a.x0 - 1 : a.x0 + 32) +
                          (long long)(a.y0 + row % TY) * a.pitch + (long long)(a.z0 + row / TY) * a.slab;
      s = halo_lab(n) && (left ? g.r[D::XP][n] : g.r[D::XM][n]) > 0;
    }
    const unsigned sb = __ballot_sync(FULL, s);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      L[i] |= (sb >> i) & 1u;
      L[i] |= ((sb >> (16 + i)) & 1u) << 31;
    }
  }
  bool converged = false;
  for (int it = 0; it < 64; ++it) {
    unsigned ch = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const unsigned p = close_left(close_right(L[i], IXL[i]), IXR[i]);
      ch |= p ^ L[i];
      L[i] = p;
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      if (i % TY > 0) { const unsigned p = L[i] | (L[(i > 0) ? i - 1 : 0] & IYU[i]); ch |= p ^ L[i]; L[i] = p; }
    }
#pragma unroll
    for (int i = R - 1; i >= 0; --i) {
      if (i % TY < TY - 1) { const unsigned p = L[i] | (L[(i + 1 < R) ? i + 1 : i] & IYD[i]); ch |= p ^ L[i]; L[i] = p; }
    }
    if constexpr (DIMS == 3) {
#pragma unroll
      for (int i = TY; i < R; ++i) { const unsigned p = L[i] | (L[i - TY] & IZU[i]); ch |= p ^ L[i]; L[i] = p; }
#pragma unroll
      for (int i = R - TY - 1; i >= 0; --i) { const unsigned p = L[i] | (L[i + TY] & IZD[i]); ch |= p ^ L[i]; L[i] = p; }
    }
    if (!ch) { converged = true; break; }
  }
  unsigned rows_changed = 0, col0 = 0, col31 = 0;
  bool hit = false;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const unsigned c = L[i] ^ L0[i];
    if (c) rows_changed |= 1u << i;
    col0 |= c & 1u;
    col31 |= c >> 31;
    hit |= (L[i] & NEG[i]) != 0u;
    if (FIRST || c) Lb[roff<TY>(a, i)] = (uint8_t)((L[i] >> lane) & 1u);
  }
  if (lane == 0) {
    unsigned ymask0 = 0, ymask1 = 0, zmask0 = 0, zmask1 = 0;
#pragma unroll
    for (int z = 0; z < TZ; ++z) { ymask0 |= 1u << (z * TY); ymask1 |= 1u << (z * TY + TY - 1); }
#pragma unroll
    for (int y = 0; y < TY; ++y) { zmask0 |= 1u << y; zmask1 |= 1u << ((TZ - 1) * TY + y); }
    // boundary labels that differ from what the neighbours last read (their
    // halo read our labels, or our excess in the first pass)
    const unsigned bnd = rows_changed;
    const bool c0 = col0, c31 = col31;
    bool any = false;
    const int txs = g.tiles_x, tys = g.tiles_y;
    if ((bnd & ymask0) && a.has_yT) { fnext[tid - txs] = 1; any = true; }
    if ((bnd & ymask1) && a.has_yB) { fnext[tid + txs] = 1; any = true; }
    if (DIMS == 3) {
      if ((bnd & zmask0) && a.has_zT) { fnext[tid - txs * tys] = 1; any = true; }
      if ((bnd & zmask1) && a.has_zB) { fnext[tid + txs * tys] = 1; any = true; }
    }
    if (c0 && a.has_xL) { fnext[tid - 1] = 1; any = true; }
    if (c31 && a.has_xR) { fnext[tid + 1] = 1; any = true; }
    if (!converged) { fnext[tid] = 1; any = true; }
    if (any) *pending = 1;
    if (hit) *bad = 1;
  }
}

template <int DIMS, int TY, int TZ, bool FIRST>
__global__ void __launch_bounds__(256) k_cut(const GridDev* __restrict__ gd,
                                             const int4* __restrict__ info, int ntiles,
                                             uint8_t* __restrict__ fcur, uint8_t* __restrict__ fnext,
                                             DevCounters* __restrict__ ctr, int pass) {
  const int lane = threadIdx.x & 31;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctr->pending[(pass + 1) & 1] = 0;
  int* pending = &ctr->pending[pass & 1];
  unsigned long long visits = 0;
  for (;;) {
    unsigned chunk = 0;
    if (lane == 0) chunk = atomicAdd(&ctr->tk.chunk, 1u);
    chunk = __shfl_sync(FULL, chunk, 0);
    const long long b = (long long)chunk * 32;
    if (b >= ntiles) break;
    const long long li = b + lane;
    bool f = li < ntiles;
    if (!FIRST && f) {
      f = fcur[li] != 0;
      if (f) fcur[li] = 0;
    }
    unsigned m = __ballot_sync(FULL, f);
    while (m) {
      const int src = __ffs(m) - 1;
      m &= m - 1;
      const int tt = (int)b + src;
      const int4 ti = info[tt];
      cut_tile<DIMS, TY, TZ, FIRST>(gd[ti.x], ti, tt, fnext, pending, &ctr->cut_bad);
      ++visits;
    }
  }
  __shared__ unsigned long long s_vis;
  if (threadIdx.x == 0) s_vis = 0;
  __syncthreads();
  if (lane == 0 && visits) atomicAdd(&s_vis, visits);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_vis) atomicAdd(&ctr->bfs_visits, s_vis);
    __threadfence();
    const unsigned prev = atomicAdd(&ctr->tk.done, 1u);
    if (prev == gridDim.x - 1) {
      ctr->tk.chunk = 0;
      ctr->tk.done = 0;
      __threadfence();
    }
  }
}

// per-grid sum of min(e, 0) and count of source-side nodes (reduce_flow,
// bin/x64/cl/Infrastructures/reduce.cl:92-117, in int64 instead of int32 partials)
template <int TY, int TZ>
__global__ void __launch_bounds__(256) k_grid_sums(const GridDev* __restrict__ gd,
                                                   const int4* __restrict__ info, int ntiles,
                                                   long long* __restrict__ sums) {
  constexpr int R = TY * TZ;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  int cur = -1;
  long long s_neg = 0, s_lab = 0;
  for (int t = warp; t < ntiles; t += nwarps) {
    const int4 ti = info[t];
    if (ti.x != cur) {
      if (cur >= 0) {
        for (int o = 16; o; o >>= 1) { s_neg += __shfl_xor_sync(FULL, s_neg, o); s_lab += __shfl_xor_sync(FULL, s_lab, o); }
        if (lane == 0) { atomicAdd((unsigned long long*)&sums[2 * cur], (unsigned long long)s_neg);
                         atomicAdd((unsigned long long*)&sums[2 * cur + 1], (unsigned long long)s_lab); }
      }
      s_neg = 0; s_lab = 0; cur = ti.x;
    }
    const GridDev& g = gd[ti.x];
    const long long pitch = g.pitch, slab = (long long)g.pitch * g.Hp;
    const long long base = (long long)(ti.y * 32 + lane) + (long long)ti.z * TY * pitch + (long long)ti.w * TZ * slab;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const long long n = base + (long long)(i % TY) * pitch + (long long)(i / TY) * slab;
      const int e = g.e[n];
      s_neg += e < 0 ? e : 0;
      s_lab += g.label[n];
    }
  }
  if (cur >= 0) {
    for (int o = 16; o; o >>= 1) { s_neg += __shfl_xor_sync(FULL, s_neg, o); s_lab += __shfl_xor_sync(FULL, s_lab, o); }
    if (lane == 0) { atomicAdd((unsigned long long*)&sums[2 * cur], (unsigned long long)s_neg);
                     atomicAdd((unsigned long long*)&sums[2 * cur + 1], (unsigned long long)s_lab); }
  }
}

template <int DIMS, int TY, int TZ>
cudaError_t relabel_t(const TileSet& ts, int pass, bool first, cudaStream_t s) {
  static int blocks_first = 0, blocks = 0;
  uint8_t* fcur = ts.d_flag_bfs[pass & 1];
  uint8_t* fnext = ts.d_flag_bfs[(pass + 1) & 1];
  if (first) {
    if (!blocks_first) blocks_first = persistent_blocks((const void*)k_relabel<DIMS, TY, TZ, true>, 256, 0);
    jfc_note_launch();
    k_relabel<DIMS, TY, TZ, true><<<blocks_first, 256, 0, s>>>(ts.d_desc, ts.d_info, ts.ntiles, fcur, fnext,
                                                              ts.d_flag_pr, ts.d_grid_active, ts.d_ctr, pass);
  } else {
    if (!blocks) blocks = persistent_blocks((const void*)k_relabel<DIMS, TY, TZ, false>, 256, 0);
    jfc_note_launch();
    k_relabel<DIMS, TY, TZ, false><<<blocks, 256, 0, s>>>(ts.d_desc, ts.d_info, ts.ntiles, fcur, fnext,
                                                         ts.d_flag_pr, ts.d_grid_active, ts.d_ctr, pass);
  }
  return cudaGetLastError();
}

template <int DIMS, int TY, int TZ>
cudaError_t cut_t(const TileSet& ts, int pass, bool first, cudaStream_t s) {
  static int blocks_first = 0, blocks = 0;
  uint8_t* fcur = ts.d_flag_bfs[pass & 1];
  uint8_t* fnext = ts.d_flag_bfs[(pass + 1) & 1];
  if (first) {
    if (!blocks_first) blocks_first = persistent_blocks((const void*)k_cut<DIMS, TY, TZ, true>, 256, 0);
    jfc_note_launch();
    k_cut<DIMS, TY, TZ, true><<<blocks_first, 256, 0, s>>>(ts.d_desc, ts.d_info, ts.ntiles, fcur, fnext, ts.d_ctr, pass);
  } else {
    if (!blocks) blocks = persistent_blocks((const void*)k_cut<DIMS, TY, TZ, false>, 256, 0);
    jfc_note_launch();
    k_cut<DIMS, TY, TZ, false><<<blocks, 256, 0, s>>>(ts.d_desc, ts.d_info, ts.ntiles, fcur, fnext, ts.d_ctr, pass);
  }
  return cudaGetLastError();
}

template <int TY, int TZ>
cudaError_t sums_t(const TileSet& ts, cudaStream_t s) {
  static int blocks = 0;
  if (!blocks) blocks = persistent_blocks((const void*)k_grid_sums<TY, TZ>, 256, 0);
  jfc_note_launch();
  k_grid_sums<TY, TZ><<<blocks, 256, 0, s>>>(ts.d_desc, ts.d_info, ts.ntiles, ts.d_grid_sum);
  return cudaGetLastError();
}

// ---------------------------------------------------------- layout helpers
// Zero arcs that leave the grid and flag inputs the int32 solver cannot hold
// (negative capacities).
__global__ void k_fix_boundary(GridDev g, int conn, int* bad) {
  const long long total = g.plane;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < total;
       n += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(n % g.pitch);
    const long long yz = n / g.pitch;
    const int y = (int)(yz % g.Hp), z = (int)(yz / g.Hp);
    const bool real = x < g.W && y < g.H && z < g.D;
    if (!real) {
      g.e[n] = 0;
      for (int k = 0; k < conn; ++k) g.r[k][n] = 0;
      g.label[n] = 0;
      continue;
    }
    bool ok[6];
    if (g.dims == 2) {
      ok[0] = x + 1 < g.W; ok[1] = y + 1 < g.H; ok[2] = y > 0; ok[3] = x > 0;
    } else {
      ok[0] = x + 1 < g.W; ok[1] = y + 1 < g.H; ok[2] = z + 1 < g.D;
      ok[3] = z > 0; ok[4] = y > 0; ok[5] = x > 0;
    }
    for (int k = 0; k < conn; ++k) {
      const int v = g.r[k][n];
      if (!ok[k]) g.r[k][n] = 0;
      else if (v < 0) *bad = 1;
    }
    g.label[n] = 0;
  }
}

__global__ void k_pack_u8(GridDev g, const uint8_t* __restrict__ src, uint8_t* __restrict__ dst) {
  const long long n = (long long)g.W * g.H * g.D;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.W);
    const long long yz = i / g.W;
    const int y = (int)(yz % g.H), z = (int)(yz / g.H);
    dst[i] = src[(long long)x + (long long)g.pitch * (y + (long long)g.Hp * z)];
  }
}

__global__ void k_pack_i32(GridDev g, const int* __restrict__ src, int* __restrict__ dst) {
  const long long n = (long long)g.W * g.H * g.D;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.W);
    const long long yz = i / g.W;
    const int y = (int)(yz % g.H), z = (int)(yz / g.H);
    dst[i] = src[(long long)x + (long long)g.pitch * (y + (long long)g.Hp * z)];
  }
}

__global__ void k_edit_tlinks(GridDev g, const uint32_t* __restrict__ idx, const int32_t* __restrict__ dcs,
                              const int32_t* __restrict__ dct, long long n, long long* dsink) {
  long long acc = 0;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const long long i = idx[j];
    const int x = (int)(i % g.W);
    const long long yz = i / g.W;
    const int y = (int)(yz % g.H), z = (int)(yz / g.H);
    const long long p = (long long)x + (long long)g.pitch * (y + (long long)g.Hp * z);
    atomicAdd(g.e + p, dcs[j] - dct[j]);
    acc += dct[j];
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd((unsigned long long*)dsink, (unsigned long long)acc);
}

}  // namespace

int persistent_blocks(const void* kernel, int threads, size_t smem) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
  if (per < 1) per = 1;
  return sms * per;
}

cudaError_t launch_relabel_pass(const TileSet& ts, int pass, bool first, cudaStream_t s) {
  if (ts.dims == 2) {
    if (ts.TR == 8) return relabel_t<2, 8, 1>(ts, pass, first, s);
    if (ts.TR == 16) return relabel_t<2, 16, 1>(ts, pass, first, s);
    return cudaErrorInvalidValue;
  }
  if (ts.TY == 4 && ts.TZ == 4) return relabel_t<3, 4, 4>(ts, pass, first, s);
  if (ts.TY == 4 && ts.TZ == 2) return relabel_t<3, 4, 2>(ts, pass, first, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_cut_pass(const TileSet& ts, int pass, bool first, cudaStream_t s) {
  if (ts.dims == 2) {
    if (ts.TR == 8) return cut_t<2, 8, 1>(ts, pass, first, s);
    if (ts.TR == 16) return cut_t<2, 16, 1>(ts, pass, first, s);
    return cudaErrorInvalidValue;
  }
  if (ts.TY == 4 && ts.TZ == 4) return cut_t<3, 4, 4>(ts, pass, first, s);
  if (ts.TY == 4 && ts.TZ == 2) return cut_t<3, 4, 2>(ts, pass, first, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_grid_sums(const TileSet& ts, cudaStream_t s) {
  cudaError_t err = cudaMemsetAsync(ts.d_grid_sum, 0, sizeof(long long) * 2 * ts.ngrids, s);
  if (err != cudaSuccess) return err;
  if (ts.dims == 2) {
    if (ts.TR == 8) return sums_t<8, 1>(ts, s);
    if (ts.TR == 16) return sums_t<16, 1>(ts, s);
    return cudaErrorInvalidValue;
  }
  if (ts.TY == 4 && ts.TZ == 4) return sums_t<4, 4>(ts, s);
  if (ts.TY == 4 && ts.TZ == 2) return sums_t<4, 2>(ts, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_clear_counters(const TileSet& ts, cudaStream_t s) {
  return cudaMemsetAsync(ts.d_ctr, 0, sizeof(DevCounters), s);
}

static int grid_blocks(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

cudaError_t launch_fix_boundary(const GridDev& g, int conn, int* d_bad, cudaStream_t s) {
  jfc_note_launch();
  k_fix_boundary<<<grid_blocks(g.plane), 256, 0, s>>>(g, conn, d_bad);
  return cudaGetLastError();
}

cudaError_t launch_pack_labels(const GridDev& g, uint8_t* d_dense, cudaStream_t s) {
  jfc_note_launch();
  k_pack_u8<<<grid_blocks((long long)g.W * g.H * g.D), 256, 0, s>>>(g, g.label, d_dense);
  return cudaGetLastError();
}

cudaError_t launch_pack_plane(const GridDev& g, const int* d_plane, int* d_dense, cudaStream_t s) {
  jfc_note_launch();
  k_pack_i32<<<grid_blocks((long long)g.W * g.H * g.D), 256, 0, s>>>(g, d_plane, d_dense);
  return cudaGetLastError();
}

cudaError_t launch_edit_tlinks(const GridDev& g, const uint32_t* d_idx, const int32_t* d_dcs,
                               const int32_t* d_dct, size_t n, long long* d_dsink, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  jfc_note_launch();
  k_edit_tlinks<<<grid_blocks((long long)n), 256, 0, s>>>(g, d_idx, d_dcs, d_dct, (long long)n, d_dsink);
  return cudaGetLastError();
}
