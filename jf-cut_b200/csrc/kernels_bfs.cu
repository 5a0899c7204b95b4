// kernels_bfs.cu — global relabel, convergence / cut BFS, reductions and
// layout helpers.
//
// Global relabel — reference graphcut_init_global_relabel / graphcut_global_relabel
// (graphcut_global_relabel.cl:19-124 2D, :128-249 3D) driven by QGCWidget::globalRelabel
// (QGCWidget.cpp:2208-2241): heights = exact BFS distance to the deficit nodes
// (e < 0) over residual arcs, by in-tile fixpoint relaxation with tiles
// revisited in level sweeps ordered by the jump-flooding tile BFS
// (graphcut_bfs_block.cl).  Here the relaxation is monotone (heights only fall
// from INF), so tiles need no parity and no order: a persistent cooperative
// kernel runs a first pass over every tile (fused initialisation, one warp
// per tile, bit-parallel level BFS) and then the frontier (a tile whose
// boundary fell queues its neighbours).  In 2D the frontier starts with a
// one-warp border check of the tiles the first pass queued and continues as
// an asynchronous worklist: one CTA per queued tile closes the in-tile
// distances with warp min-plus scans along rows and columns.  In 3D it runs in
// passes separated by grid barriers, one warp per queued tile (level BFS
// seeded by the halo heights).  Each visit records whether the tile holds an
// active node (e > 0, h < INF): the device-side active-tile count
// (graphcut_count_node, graphcut_count_block.cl:19-47) that decides
// convergence, and the queue of tiles the next push-relabel phase visits.
//
// Cut — reference graphcut_init_cut / graphcut_compute_cut (graphcut_compute_cut.cl:19-140):
// the source side is every node reachable from {e > 0} along residual arcs.
// One warp per tile: R rows of 32-bit words (bit = lane), in-arc masks built
// once with ballots, row closure by 5-step shift doubling, rows combined by
// word AND/OR.  Reaching a deficit raises cut_bad (the reference's done[1]
// divergence flag).
#include "jfc_relax.cuh"
#include "jfc_tma.cuh"

namespace {

using jfc::FULL;

// Frontier the tile visits feed (next pass), deduplicated by its flags.
struct BfsQ {
  int* flags;
  int* q;
  int* qn;
  // staging in shared memory (null: appends go straight to the queue): the
  // items that won their flag are collected in sbuf (count *scnt) and the
  // caller moves them to the queue with one counter update per batch, so
  // thousands of warps do not all serialise on the queue's one counter
  // (the warp form of the 3D frontier passes)
  int* sbuf = nullptr;
  int* scnt = nullptr;
};

// Move a warp's staged items of Q to its queue with one counter update (all
// lanes, after a __syncwarp; the caller resets the count).
__device__ __forceinline__ void flush_staged(const BfsQ& Q, int lane) {
  const int cnt = *(volatile int*)Q.scnt;
  if (cnt == 0) return;
  int base = 0;
  if (lane == 0) base = atomicAdd(Q.qn, cnt);
  base = __shfl_sync(FULL, base, 0);
  for (int i = lane; i < cnt; i += 32) Q.q[base + i] = Q.sbuf[i];
}

// Worklist of the asynchronous 2D relabel: a ring of `cap` tile slots (-1 =
// empty) with the queued flags of BfsQ, a tail counter and the count of
// items queued and not yet fully visited (zero = the relaxation is done).
struct RlRing {
  int* ring;
  unsigned cap;
  unsigned long long* tail_out;   // ring positions reserved (high 32 bits), items outstanding (low 32)
  int* err;
  unsigned long long max_spins;   // polls before a wait gives up
};

// Append the tiles offered by the lanes of a warp that win their queued
// flag: count them as outstanding first (so the count never reaches zero
// while one is on its way), then reserve ring positions and claim each slot
// (free, or freed by its reader within a few polls; bounded: after
// W.max_spins polls the error flag is raised).  Returns false after an error.
// Returns false after an error.  `folded` tells whether the appending visit's
// own completion was counted in the same update (it appended something): the
// update adds m positions and m - 1 outstanding items, made before the items
// are published, so the count cannot reach zero while they wait.
__device__ __forceinline__ bool ring_append(bool want, int tile, int* flags, const RlRing& W, bool& folded) {
  bool won = false;
  if (want) won = atomicExch(flags + tile, 1) == 0;
  const unsigned m = __ballot_sync(jfc::FULL, won);
  folded = m != 0;
  if (!m) return true;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  unsigned base = 0;
  if (lane == leader) {
    const unsigned c = (unsigned)__popc(m);
    base = (unsigned)(atomicAdd(W.tail_out, ((unsigned long long)c << 32) + (c - 1u)) >> 32);
  }
  base = __shfl_sync(jfc::FULL, base, leader);
  bool ok = true;
  if (won) {
    int* slot = W.ring + (base + __popc(m & ((1u << lane) - 1u))) % W.cap;
    __threadfence();
    unsigned long long spins = 0;
    while (atomicCAS(slot, -1, tile) != -1) {
      if (++spins > W.max_spins || *(volatile int*)W.err) { atomicExch(W.err, 1); ok = false; break; }
      __nanosleep(64);
    }
  }
  return __all_sync(jfc::FULL, ok);
}

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

// Queue the neighbour tiles whose halo changed (rows_changed: rows of this
// tile that changed; c0 / c31: a change in the first / last column) and the
// tile itself when its in-tile fixpoint is not reached yet.
template <int DIMS, int TY, int TZ>
__device__ __forceinline__ void flag_neighbours(const GridDev& g, const Addr& a, int tid, unsigned rows_changed,
                                                bool c0, bool c31, bool again, const BfsQ& Q) {
  const int lane = threadIdx.x & 31;
  unsigned ymask0 = 0, ymask1 = 0, zmask0 = 0, zmask1 = 0;
#pragma unroll
  for (int z = 0; z < TZ; ++z) { ymask0 |= 1u << (z * TY); ymask1 |= 1u << (z * TY + TY - 1); }
#pragma unroll
  for (int y = 0; y < TY; ++y) { zmask0 |= 1u << y; zmask1 |= 1u << ((TZ - 1) * TY + y); }
  const int txs = g.tiles_x, tys = g.tiles_y;
  bool want = false;
  int nb = tid;
  switch (lane) {
    case 0: want = (rows_changed & ymask0) && a.has_yT; nb = tid - txs; break;
    case 1: want = (rows_changed & ymask1) && a.has_yB; nb = tid + txs; break;
    case 2: want = c0 && a.has_xL; nb = tid - 1; break;
    case 3: want = c31 && a.has_xR; nb = tid + 1; break;
    case 4: want = DIMS == 3 && (rows_changed & zmask0) && a.has_zT; nb = tid - txs * tys; break;
    case 5: want = DIMS == 3 && (rows_changed & zmask1) && a.has_zB; nb = tid + txs * tys; break;
    case 6: want = again; nb = tid; break;
    default: break;
  }
  if (Q.sbuf) {
    if (want && atomicExch(Q.flags + nb, 1) == 0) Q.sbuf[atomicAdd(Q.scnt, 1)] = nb;
  } else {
    jfc::warp_append(want, nb, Q.flags, Q.q, Q.qn);
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

// TAG: the reference's tag post-process (graphcut_compute_tag.cl) on the same
// machinery: reachability from the foreground seeds through object nodes
// (any direction), kept in bit 1 of the label byte; `seeds` is the dense
// seed array (JFC_SEED_FG = 1).
template <int DIMS, int TY, int TZ, bool FIRST, bool TAG = false>
__device__ __forceinline__ void cut_tile(const GridDev& g, int4 ti, int tid, const BfsQ& Q,
                                         int* __restrict__ bad, const uint8_t* __restrict__ seeds = nullptr) {
  using D = Dirs<DIMS>;
  constexpr int R = TY * TZ;
  const int lane = threadIdx.x & 31;
  const Addr a = make_addr<DIMS, TY, TZ>(g, ti, lane);
  const int* __restrict__ E = g.e;
  uint8_t* __restrict__ Lb = g.label;
  unsigned L[R], L0[R], IXL[R], IXR[R], IYU[R], IYD[R];
  unsigned IZU[DIMS == 3 ? R : 1], IZD[DIMS == 3 ? R : 1];
  unsigned NEG[R];
  // dense index of this lane's node in row i (seed lookup of the tag pass)
  auto dense = [&](int i) -> long long {
    return (long long)(a.x0 + lane) + (long long)g.W * ((a.y0 + i % TY) + (long long)g.H * (a.z0 + i / TY));
  };
  auto is_seed = [&](int i) -> bool {
    const int x = a.x0 + lane, y = a.y0 + i % TY, z = a.z0 + i / TY;
    return x < g.W && y < g.H && z < g.D && seeds[dense(i)] == JFC_SEED_FG;
  };
  unsigned OBJ[TAG ? R : 1];   // object nodes (tag mode)
  if constexpr (TAG) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const unsigned lb = Lb[roff<TY>(a, i)];
      OBJ[i] = __ballot_sync(FULL, lb & 1u);
      NEG[i] = 0u;
      if constexpr (FIRST) L[i] = __ballot_sync(FULL, is_seed(i));
      else L[i] = __ballot_sync(FULL, (lb & 2u) != 0);
    }
    // a node takes the tag from any tagged neighbour when it is an object node
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int y = i % TY, z = i / TY;
      IXL[i] = OBJ[i] & ~1u;
      IXR[i] = OBJ[i] & 0x7fffffffu;
      IYU[i] = y > 0 ? OBJ[i] : 0u;
      IYD[i] = y < TY - 1 ? OBJ[i] : 0u;
      if constexpr (DIMS == 3) {
        IZU[i] = z > 0 ? OBJ[i] : 0u;
        IZD[i] = z < TZ - 1 ? OBJ[i] : 0u;
      }
    }
  } else {
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
  // sources entering through the halo: neighbour reached and its arc toward us
  // residual (cut), or neighbour tagged (tag; the receiving node must be an
  // object node, applied through the in-masks below)
  auto halo_lab = [&](long long n) -> bool {
    if constexpr (TAG) {
      if constexpr (FIRST) {
        const long long x = n % g.pitch, yz = n / g.pitch, y = yz % g.Hp, z = yz / g.Hp;
        return x < g.W && y < g.H && z < g.D && seeds[x + (long long)g.W * (y + (long long)g.H * z)] == JFC_SEED_FG;
      } else {
        return (Lb[n] & 2u) != 0;
      }
    } else {
      if constexpr (FIRST) return E[n] > 0;
      else return Lb[n] != 0;
    }
  };
  // residual arc from halo node m toward the tile (cut); any neighbour (tag)
  auto halo_arc = [&](int dir, long long m) -> bool {
    if constexpr (TAG) return true;
    else return g.r[dir][m] > 0;
  };
  // nodes a halo source may reach: all (cut: the arc decides) or objects (tag)
  auto objm = [&](int i) -> unsigned {
    if constexpr (TAG) return OBJ[i];
    else return FULL;
  };
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    const long long n = roff<TY>(a, z * TY);
    bool s = false;
    if (a.has_yT) { const long long m = n - a.pitch; s = halo_lab(m) && halo_arc(D::YP, m); }
    L[z * TY] |= __ballot_sync(FULL, s) & objm(z * TY);
    s = false;
    if (a.has_yB) { const long long m = n + (long long)TY * a.pitch; s = halo_lab(m) && halo_arc(D::YM, m); }
    L[z * TY + TY - 1] |= __ballot_sync(FULL, s) & objm(z * TY + TY - 1);
  }
  if constexpr (DIMS == 3) {
#pragma unroll
    for (int y = 0; y < TY; ++y) {
      const long long n = roff<TY>(a, y);
      bool s = false;
      if (a.has_zT) { const long long m = n - a.slab; s = halo_lab(m) && halo_arc(D::ZP, m); }
      L[y] |= __ballot_sync(FULL, s) & objm(y);
      s = false;
      if (a.has_zB) { const long long m = n + (long long)TZ * a.slab; s = halo_lab(m) && halo_arc(D::ZM, m); }
      L[(TZ - 1) * TY + y] |= __ballot_sync(FULL, s) & objm((TZ - 1) * TY + y);
    }
  }
  {
    const int row = lane & 15;
    const bool left = lane < 16;
    bool s = false;
    if (row < R && (left ? a.has_xL : a.has_xR)) {
      const long long n = (long long)(left ? a.x0 - 1 : a.x0 + 32) +
                          (long long)(a.y0 + row % TY) * a.pitch + (long long)(a.z0 + row / TY) * a.slab;
      s = halo_lab(n) && halo_arc(left ? D::XP : D::XM, n);
    }
    const unsigned sb = __ballot_sync(FULL, s);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      L[i] |= ((sb >> i) & 1u) & objm(i);
      L[i] |= (((sb >> (16 + i)) & 1u) << 31) & objm(i);
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
    if constexpr (TAG) {
      if (FIRST || c) {
        uint8_t* p = Lb + roff<TY>(a, i);
        *p = (uint8_t)((*p & 1u) | (((L[i] >> lane) & 1u) << 1));
      }
    } else {
      if (FIRST || c) Lb[roff<TY>(a, i)] = (uint8_t)((L[i] >> lane) & 1u);
    }
  }
  if (lane == 0 && hit) *bad = 1;
  // boundary labels that differ from what the neighbours last read (their
  // halo read our labels, or our excess in the first pass)
  flag_neighbours<DIMS, TY, TZ>(g, a, tid, rows_changed, col0 != 0, col31 != 0, !converged, Q);
}

// Persistent cut BFS: pass 0 visits every tile (labels start as e > 0),
// later passes drain the frontier built by the previous one (one tile per
// warp ticket), grid barriers in between, until a pass queues nothing or the
// pass budget runs out.
template <int DIMS, int TY, int TZ, bool TAG = false>
__global__ void __launch_bounds__(256) k_cut(TileSet ts, int max_passes, const uint8_t* seeds) {
  DevCounters* ctr = ts.d_ctr;
  const int lane = threadIdx.x & 31;
  unsigned long long visits = 0;
  bool ok = true;
  int pass = 0;
  {
    BfsQ Q{ts.d_flag_bfs[1], ts.d_q_bfs[1], &ctr->qn_bfs[1]};
    for (;;) {
      const unsigned c = jfc::warp_ticket(&ctr->ticket[0]);
      const long long b = (long long)c * 32;
      if (b >= ts.ntiles) break;
      const int cnt = (int)min(32ll, (long long)ts.ntiles - b);
      for (int k = 0; k < cnt; ++k) {
        const int tt = (int)b + k;
        const int4 ti = ts.d_info[tt];
        cut_tile<DIMS, TY, TZ, true, TAG>(ts.d_desc[ti.x], ti, tt, Q, &ctr->cut_bad, seeds);
        ++visits;
      }
    }
    ok = jfc::grid_sync(ctr, [&]() { ctr->ticket[0] = 0; });
  }
  for (pass = 1; ok; ++pass) {
    const int cb = pass & 1;
    const int n = jfc::vload(&ctr->qn_bfs[cb]);
    if (n == 0) break;
    if (pass > max_passes) {
      if (blockIdx.x == 0 && threadIdx.x == 0) ctr->bfs_status = 2;
      break;
    }
    BfsQ Q{ts.d_flag_bfs[cb ^ 1], ts.d_q_bfs[cb ^ 1], &ctr->qn_bfs[cb ^ 1]};
    const int* queue = ts.d_q_bfs[cb];
    int* fcur = ts.d_flag_bfs[cb];
    for (;;) {
      const unsigned k = jfc::warp_ticket(&ctr->ticket[cb]);
      if ((int)k >= n) break;
      const int tt = queue[k];
      if (lane == 0) fcur[tt] = 0;
      __syncwarp();
      const int4 ti = ts.d_info[tt];
      cut_tile<DIMS, TY, TZ, false, TAG>(ts.d_desc[ti.x], ti, tt, Q, &ctr->cut_bad, seeds);
      ++visits;
    }
    ok = jfc::grid_sync(ctr, [&]() {
      ctr->ticket[cb] = 0;
      ctr->qn_bfs[cb] = 0;
    });
  }
  __shared__ unsigned long long s_vis;
  if (threadIdx.x == 0) s_vis = 0;
  __syncthreads();
  if (lane == 0 && visits) atomicAdd(&s_vis, visits);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_vis) atomicAdd(&ctr->bfs_visits, s_vis);
    if (blockIdx.x == 0) {
      ctr->bfs_passes = pass;
      if (ctr->bfs_status == 0) ctr->bfs_status = 1;
    }
  }
}

// ------------------------------------------------------------ global relabel
template <int DIMS, int TY, int TZ>
using RTile = jfc::CtaTile<DIMS, TY, TZ>;

template <int DIMS, int TY, int TZ>
struct RlSmem {
  int h[RTile<DIMS, TY, TZ>::HN];
  uint8_t arc[RTile<DIMS, TY, TZ>::NT];
  int ntile;
  int face[6];
  int folded;   // worklist: the visit's completion was counted with its appends
};

// One frontier visit, one CTA per tile, one thread per node (the reference's
// work-group layout, graphcut_global_relabel.cl:50-124): stage the tile's
// heights and the halo, close the in-tile distances (relax_cta), write the
// heights that fell, queue the neighbours whose halo fell and the tile itself
// when its fixpoint was not reached.
// W.ring non-null: the asynchronous worklist (neighbours go to the ring).
template <int DIMS, int TY, int TZ>
__device__ __forceinline__ void relabel_visit(const TileSet& ts, int tid, RlSmem<DIMS, TY, TZ>& s,
                                              const BfsQ& Q, int& cur_grid, int& delta,
                                              const RlRing& W = RlRing{nullptr, 0, nullptr, nullptr, 0}) {
  using T = RTile<DIMS, TY, TZ>;
  using D = Dirs<DIMS>;
  const int t = threadIdx.x;
  const int x = t & 31, row = t >> 5, y = row % TY, z = row / TY;
  const int4 ti = ts.d_info[tid];
  const GridDev& g = ts.d_desc[ti.x];
  const int pitch = g.pitch;
  const long long slab = (long long)g.pitch * g.Hp;
  const int x0 = ti.y * 32, y0 = ti.z * TY, z0 = ti.w * TZ;
  const long long tbase = (long long)x0 + (long long)y0 * pitch + (long long)z0 * slab;
  const long long n = tbase + x + (long long)y * pitch + (long long)z * slab;
  const int hi = T::hidx(x, y, z);
  // residual-arc bits and the excess sign, written by the first pass
  const unsigned ab = g.label[n];
  const unsigned arcs = ab & 63u;
  const bool pos = (ab & 128u) != 0;
  s.arc[t] = (uint8_t)arcs;
  // heights other CTAs write while the worklist runs are read from L2 (the
  // SM's L1 may hold an older copy of the line)
  const bool fresh = W.ring != nullptr;
  // (thread 0) the tile's activity byte as its last visit left it, read early
  unsigned act_old = 0;
  if (t == 0) act_old = fresh ? __ldcg(ts.d_act + tid) : ts.d_act[tid];
  const int hstart = fresh ? __ldcg(g.h + n) : g.h[n];
  s.h[hi] = hstart;
  for (int c = t; c < T::NHALO; c += T::NT) {
    int hx, hy, hz, f;
    T::halo_cell(c, hx, hy, hz, f);
    const int gx = x0 + hx, gy = y0 + hy, gz = z0 + hz;
    int v = JFC_INF;
    if (gx >= 0 && gx < pitch && gy >= 0 && gy < g.Hp && gz >= 0 && gz < g.Dp) {
      const int* p = g.h + (long long)gx + (long long)gy * pitch + (long long)gz * slab;
      v = fresh ? __ldcg(p) : *p;
    }
    s.h[T::hidx(hx, hy, hz)] = v;
  }
  if (t < 6) s.face[t] = 0;
  __syncthreads();
  // a tile is queued when a neighbour's boundary heights changed, which may
  // not lower anything here: relax only when some residual arc (in the tile
  // or into the halo) still offers a shorter distance
  int m = JFC_INF;
  if (arcs & jfc::A_XP) m = min(m, s.h[hi + 1]);
  if (arcs & jfc::A_XM) m = min(m, s.h[hi - 1]);
  if (arcs & jfc::A_YP) m = min(m, s.h[hi + T::SY]);
  if (arcs & jfc::A_YM) m = min(m, s.h[hi - T::SY]);
  if constexpr (DIMS == 3) {
    if (arcs & jfc::A_ZP) m = min(m, s.h[hi + T::SZ]);
    if (arcs & jfc::A_ZM) m = min(m, s.h[hi - T::SZ]);
  }
  const int cap = jfc::cap_of(g, ts.d_ctr);
  const bool need = __syncthreads_or(m + 1 < hstart && m + 1 < cap);
  const bool converged = need ? jfc::relax_cta<DIMS, TY, TZ>(s.h, s.arc, 16) : true;
  // distances at or above the cap stay unreachable (every stored height is
  // below the cap or JFC_INF, so the capped closure is the closure clamped)
  const int hf = s.h[hi] < cap ? s.h[hi] : hstart;
  const bool changed = hf != hstart;
  if (changed) {
    g.h[n] = hf;
    if (W.ring) __threadfence();   // visible before any neighbour is queued
    if (x == 0) s.face[0] = 1;
    if (x == 31) s.face[1] = 1;
    if (y == 0) s.face[2] = 1;
    if (y == TY - 1) s.face[3] = 1;
    if (DIMS == 3 && z == 0) s.face[4] = 1;
    if (DIMS == 3 && z == TZ - 1) s.face[5] = 1;
  }
  // activity per 8-row half of a 2D 32x16 tile (bit 0 rows 0-7, bit 1 rows
  // 8-15: the push-relabel work items of split tile sets), else bit 0
  const bool live = pos & (hf < JFC_INF);
  bool act_lo, act_hi = false;
  if constexpr (DIMS == 2 && TY == 16) {
    act_lo = __syncthreads_or(live && y < 8);
    act_hi = __syncthreads_or(live && y >= 8);
  } else {
    act_lo = __syncthreads_or(live);
  }
  const bool act = act_lo || act_hi;
  if (t < 32) {
    const int txs = g.tiles_x, tys = g.tiles_y;
    bool want = false;
    int nb = tid;
    switch (t) {
      case 0: want = s.face[0] && x0 > 0; nb = tid - 1; break;
      case 1: want = s.face[1] && x0 + 32 < pitch; nb = tid + 1; break;
      case 2: want = s.face[2] && y0 > 0; nb = tid - txs; break;
      case 3: want = s.face[3] && y0 + TY < g.Hp; nb = tid + txs; break;
      case 4: want = DIMS == 3 && s.face[4] && z0 > 0; nb = tid - txs * tys; break;
      case 5: want = DIMS == 3 && s.face[5] && z0 + TZ < g.Dp; nb = tid + txs * tys; break;
      case 6: want = !converged; nb = tid; break;
      default: break;
    }
    if (W.ring) {
      bool folded = false;
      ring_append(want, nb, Q.flags, W, folded);
      if (t == 0) s.folded = folded ? 1 : 0;
    } else {
      jfc::warp_append(want, nb, Q.flags, Q.q, Q.qn);
    }
    if (t == 0) {
      const int old = (act_old & 3u) != 0 ? 1 : 0;
      ts.d_act[tid] = (uint8_t)((act_lo ? 1 : 0) | (act_hi ? 2 : 0));
      if (ti.x != cur_grid) {
        if (delta && cur_grid >= 0) atomicAdd(&ts.d_grid_active[cur_grid], delta);
        delta = 0;
        cur_grid = ti.x;
      }
      delta += (act ? 1 : 0) - old;
    }
  }
  __syncthreads();
}

// x-direction closure of one tile row (lane = x): h(p) = min(h(p), h(q) + |p - q|)
// over the runs of residual arcs p -> p+1 -> ... -> q (axp) and p -> p-1 ->
// ... -> q (axm), by doubling.  The arc runs are read from the row's arc
// masks, so only the values move between lanes.
__device__ __forceinline__ int row_close(int v, unsigned axp, unsigned axm, int lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int nv = __shfl_down_sync(FULL, v, off);
    const unsigned run = (1u << off) - 1u;
    if (lane + off < 32 && ((~axp >> lane) & run) == 0u) v = min(v, nv + off);
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int nv = __shfl_up_sync(FULL, v, off);
    const unsigned run = (1u << off) - 1u;
    if (lane >= off && ((~axm >> (lane - off + 1)) & run) == 0u) v = min(v, nv + off);
  }
  return v;
}

// In-tile closure of a warp's tile (lane = x, hv[i] = row i's height, lab[i]
// its arc byte, AXP / AXM the rows' x-arc masks): h(u) = min(h(u), h(v) + 1)
// over residual arcs u -> v inside the tile, to the fixpoint.  Row closures
// by doubling shuffles, y and z runs in registers (a backward and a forward
// sweep per line); bounded by the tile's nodes (every pass but the last
// lowers some height, and heights are bounded below by 0).
template <int DIMS, int TY, int TZ>
__device__ __forceinline__ void tile_close(int (&hv)[TY * TZ], const unsigned (&lab)[TY * TZ],
                                           const unsigned (&AXP)[TY * TZ], const unsigned (&AXM)[TY * TZ], int lane) {
  constexpr int R = TY * TZ;
  for (int pass = 0; pass < 32 * R; ++pass) {
    bool ch = false;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int v = row_close(hv[i], AXP[i], AXM[i], lane);
      ch |= v < hv[i];
      hv[i] = v;
    }
#pragma unroll
    for (int z = 0; z < TZ; ++z) {
#pragma unroll
      for (int y = TY - 2; y >= 0; --y) {
        const int i = z * TY + y;
        if ((lab[i] & jfc::A_YP) && hv[i + 1] + 1 < hv[i]) { hv[i] = hv[i + 1] + 1; ch = true; }
      }
#pragma unroll
      for (int y = 1; y < TY; ++y) {
        const int i = z * TY + y;
        if ((lab[i] & jfc::A_YM) && hv[i - 1] + 1 < hv[i]) { hv[i] = hv[i - 1] + 1; ch = true; }
      }
    }
    if constexpr (DIMS == 3) {
#pragma unroll
      for (int y = 0; y < TY; ++y) {
#pragma unroll
        for (int z = TZ - 2; z >= 0; --z) {
          const int i = z * TY + y;
          if ((lab[i] & jfc::A_ZP) && hv[i + TY] + 1 < hv[i]) { hv[i] = hv[i + TY] + 1; ch = true; }
        }
#pragma unroll
        for (int z = 1; z < TZ; ++z) {
          const int i = z * TY + y;
          if ((lab[i] & jfc::A_ZM) && hv[i - TY] + 1 < hv[i]) { hv[i] = hv[i - TY] + 1; ch = true; }
        }
      }
    }
    if (!__any_sync(FULL, ch)) break;
  }
}

// First pass of the global relabel, one warp per tile: a bit-parallel BFS
// from the deficit nodes.  Each tile row is a 32-bit word (bit = lane); the
// level-d frontier expands through the residual-arc masks in a few word
// operations per row, so a tile costs (levels x rows) word ops and no block
// barrier.  Halo nodes count as sources only when they are deficits
// (h = 0 in this pass); everything later passes refine.  (A min-plus closure
// of the tile instead of the level steps measured slower here: the deficits
// lie close, so few levels run, and the pass streams its loads.)
template <int DIMS, int TY, int TZ>
__device__ __forceinline__ void relabel_first_warp(const TileSet& ts, int tid, const BfsQ& Q, int& cur_grid,
                                                   int& delta) {
  using D = Dirs<DIMS>;
  constexpr int R = TY * TZ;
  const int lane = threadIdx.x & 31;
  const int4 ti = ts.d_info[tid];
  const GridDev& g = ts.d_desc[ti.x];
  const Addr a = make_addr<DIMS, TY, TZ>(g, ti, lane);
  unsigned AXP[R], AXM[R], AYP[R], AYM[R], AZP[DIMS == 3 ? R : 1], AZM[DIMS == 3 ? R : 1];
  unsigned DEF[R], POS[R], V[R], F[R];
  // each node as one byte (arc bits, bit 6 e < 0, bit 7 e > 0); the row
  // masks come from it
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const long long n = roff<TY>(a, i);
    const int e = g.e[n];
    unsigned b = (g.r[D::XP][n] > 0 ? jfc::A_XP : 0u) | (g.r[D::YP][n] > 0 ? jfc::A_YP : 0u) |
                 (g.r[D::YM][n] > 0 ? jfc::A_YM : 0u) | (g.r[D::XM][n] > 0 ? jfc::A_XM : 0u) |
                 (e < 0 ? 64u : 0u) | (e > 0 ? 128u : 0u);
    if constexpr (DIMS == 3)
      b |= (g.r[D::ZP][n] > 0 ? jfc::A_ZP : 0u) | (g.r[D::ZM][n] > 0 ? jfc::A_ZM : 0u);
    AXP[i] = __ballot_sync(FULL, b & jfc::A_XP);
    AXM[i] = __ballot_sync(FULL, b & jfc::A_XM);
    AYP[i] = __ballot_sync(FULL, b & jfc::A_YP);
    AYM[i] = __ballot_sync(FULL, b & jfc::A_YM);
    if constexpr (DIMS == 3) {
      AZP[i] = __ballot_sync(FULL, b & jfc::A_ZP);
      AZM[i] = __ballot_sync(FULL, b & jfc::A_ZM);
    }
    DEF[i] = __ballot_sync(FULL, b & 64u);
    POS[i] = __ballot_sync(FULL, b & 128u);
    V[i] = DEF[i];
    F[i] = DEF[i];
  }
  // level-1 seeds: nodes with a residual arc into a deficit halo node
  unsigned S1[R];
#pragma unroll
  for (int i = 0; i < R; ++i) S1[i] = 0u;
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    const long long n = roff<TY>(a, z * TY);
    const bool t0 = a.has_yT && g.e[n - a.pitch] < 0;
    const bool t1 = a.has_yB && g.e[n + (long long)TY * a.pitch] < 0;
    S1[z * TY] |= __ballot_sync(FULL, t0) & AYM[z * TY];
    S1[z * TY + TY - 1] |= __ballot_sync(FULL, t1) & AYP[z * TY + TY - 1];
  }
  if constexpr (DIMS == 3) {
#pragma unroll
    for (int y = 0; y < TY; ++y) {
      const long long n = roff<TY>(a, y);
      const bool t0 = a.has_zT && g.e[n - a.slab] < 0;
      const bool t1 = a.has_zB && g.e[n + (long long)TZ * a.slab] < 0;
      S1[y] |= __ballot_sync(FULL, t0) & AZM[y];
      S1[(TZ - 1) * TY + y] |= __ballot_sync(FULL, t1) & AZP[(TZ - 1) * TY + y];
    }
  }
  {
    const int row = lane & 15;
    const bool left = lane < 16;
    bool sdef = false;
    if (row < R && (left ? a.has_xL : a.has_xR)) {
      const long long n = (long long)(left ? a.x0 - 1 : a.x0 + 32) +
                          (long long)(a.y0 + row % TY) * a.pitch + (long long)(a.z0 + row / TY) * a.slab;
      sdef = g.e[n] < 0;
    }
    const unsigned sb = __ballot_sync(FULL, sdef);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      S1[i] |= ((sb >> i) & 1u) & AXM[i];
      S1[i] |= (((sb >> (16 + i)) & 1u) << 31) & AXP[i];
    }
  }
  // the frontier passes read one byte per node instead of e and the residual
  // planes: bits 0-5 residual arcs (jfc::A_*), bit 6 e < 0, bit 7 e > 0 (the
  // label plane is free until the cut BFS writes it)
#pragma unroll
  for (int i = 0; i < R; ++i) {
    unsigned b = ((AXP[i] >> lane) & 1u) * jfc::A_XP | ((AYP[i] >> lane) & 1u) * jfc::A_YP |
                 ((AYM[i] >> lane) & 1u) * jfc::A_YM | ((AXM[i] >> lane) & 1u) * jfc::A_XM |
                 ((DEF[i] >> lane) & 1u) * 64u | ((POS[i] >> lane) & 1u) * 128u;
    if constexpr (DIMS == 3) b |= ((AZP[i] >> lane) & 1u) * jfc::A_ZP | ((AZM[i] >> lane) & 1u) * jfc::A_ZM;
    g.label[roff<TY>(a, i)] = (uint8_t)b;
  }
  int h[R];
#pragma unroll
  for (int i = 0; i < R; ++i) h[i] = ((DEF[i] >> lane) & 1u) ? 0 : JFC_INF;
  // level-synchronous expansion: u reaches level d+1 through an arc to a level-d node
  // (levels at or above the relabel's distance cap stay unreachable)
  const int dmax = min(32 * R, jfc::cap_of(g, ts.d_ctr) - 1);
  for (int d = 0; d < dmax; ++d) {
    unsigned any = 0;
    unsigned N[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int y = i % TY, z = i / TY;
      unsigned m = ((F[i] >> 1) & AXP[i]) | ((F[i] << 1) & AXM[i]);
      if (y < TY - 1) m |= F[(i + 1 < R) ? i + 1 : i] & AYP[i];
      if (y > 0) m |= F[(i > 0) ? i - 1 : 0] & AYM[i];
      if constexpr (DIMS == 3) {
        if (z < TZ - 1) m |= F[(i + TY < R) ? i + TY : i] & AZP[i];
        if (z > 0) m |= F[(i >= TY) ? i - TY : 0] & AZM[i];
      }
      if (d == 0) m |= S1[i];
      N[i] = m & ~V[i];
      any |= N[i];
    }
    if (!any) break;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      V[i] |= N[i];
      F[i] = N[i];
      if ((N[i] >> lane) & 1u) h[i] = d + 1;
    }
  }
  unsigned rows_fin = 0, c0 = 0, c31 = 0, act = 0, act_hi = 0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    g.h[roff<TY>(a, i)] = h[i];
    const unsigned fin = V[i] & ~DEF[i];   // finite and above 0: news for the neighbours
    if (fin) rows_fin |= 1u << i;
    c0 |= fin & 1u;
    c31 |= fin >> 31;
    // activity per 8-row half of a 2D 32x16 tile (push-relabel work items)
    if (DIMS == 2 && TY == 16 && i >= 8) act_hi |= POS[i] & V[i];
    else act |= POS[i] & V[i];
  }
  if (lane == 0) {
    const int old = 0;
    ts.d_act[tid] = (uint8_t)((act ? 1 : 0) | (act_hi ? 2 : 0));
    act |= act_hi;
    if (ti.x != cur_grid) {
      if (delta && cur_grid >= 0) atomicAdd(&ts.d_grid_active[cur_grid], delta);
      delta = 0;
      cur_grid = ti.x;
    }
    delta += (act ? 1 : 0) - old;
  }
  flag_neighbours<DIMS, TY, TZ>(g, a, tid, rows_fin, c0 != 0, c31 != 0, false, Q);
}

// Frontier visit, one warp per tile: a level BFS over the tile (bit-parallel
// rows as in the first pass) seeded by the halo heights, keeping only strict
// improvements (heights only fall during a relabel, and a node is assigned
// at the first level that reaches it).  Levels with an empty frontier jump
// to the next halo seed that could improve its node, so a visit costs one
// level per improved BFS layer plus one per distinct useful seed value:
// bounded by the tile's nodes plus its halo cells.
template <int DIMS, int TY, int TZ>
__device__ __forceinline__ void relabel_frontier_warp(const TileSet& ts, int tid, const BfsQ& Q, int& cur_grid,
                                                      int& delta) {
  constexpr int R = TY * TZ;
  constexpr int kMaxLevels = 4096;   // above the bound (nodes + halo cells); never reached
  const int lane = threadIdx.x & 31;
  const int4 ti = ts.d_info[tid];
  const GridDev& g = ts.d_desc[ti.x];
  const Addr a = make_addr<DIMS, TY, TZ>(g, ti, lane);
  unsigned AXP[R], AXM[R], AYP[R], AYM[R];
  unsigned AZP[DIMS == 3 ? R : 1], AZM[DIMS == 3 ? R : 1];
  int hv[R];
  unsigned posm = 0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const long long n = roff<TY>(a, i);
    const unsigned b = g.label[n];   // arc byte written by the first pass
    hv[i] = g.h[n];
    AXP[i] = __ballot_sync(FULL, b & jfc::A_XP);
    AXM[i] = __ballot_sync(FULL, b & jfc::A_XM);
    AYP[i] = __ballot_sync(FULL, b & jfc::A_YP);
    AYM[i] = __ballot_sync(FULL, b & jfc::A_YM);
    if constexpr (DIMS == 3) {
      AZP[i] = __ballot_sync(FULL, b & jfc::A_ZP);
      AZM[i] = __ballot_sync(FULL, b & jfc::A_ZM);
    }
    if (b & 128u) posm |= 1u << i;
  }
  // halo heights: y faces per z slice (lane = x), z faces per row y, x faces
  // in lanes r (left of row r) and 16 + r (right of row r)
  int HT[TZ], HB[TZ];
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    const long long n = roff<TY>(a, z * TY);
    HT[z] = a.has_yT ? g.h[n - a.pitch] : JFC_INF;
    HB[z] = a.has_yB ? g.h[n + (long long)TY * a.pitch] : JFC_INF;
  }
  int HZT[DIMS == 3 ? TY : 1], HZB[DIMS == 3 ? TY : 1];
  if constexpr (DIMS == 3) {
#pragma unroll
    for (int y = 0; y < TY; ++y) {
      const long long n = roff<TY>(a, y);
      HZT[y] = a.has_zT ? g.h[n - a.slab] : JFC_INF;
      HZB[y] = a.has_zB ? g.h[n + (long long)TZ * a.slab] : JFC_INF;
    }
  }
  int HX = JFC_INF;
  const int xrow = lane & 15;
  {
    const bool left = lane < 16;
    if (xrow < R && (left ? a.has_xL : a.has_xR))
      HX = g.h[(long long)(left ? a.x0 - 1 : a.x0 + 32) + (long long)(a.y0 + xrow % TY) * a.pitch +
               (long long)(a.z0 + xrow / TY) * a.slab];
  }
  // smallest seed level above d that could still improve its node
  auto next_level = [&](int d) -> int {
    int c = JFC_INF;
#pragma unroll
    for (int z = 0; z < TZ; ++z) {
      const int it = z * TY, ib = z * TY + TY - 1;
      int v = HT[z] + 1;
      if (v > d && v < hv[it] && ((AYM[it] >> lane) & 1u)) c = min(c, v);
      v = HB[z] + 1;
      if (v > d && v < hv[ib] && ((AYP[ib] >> lane) & 1u)) c = min(c, v);
    }
    if constexpr (DIMS == 3) {
#pragma unroll
      for (int y = 0; y < TY; ++y) {
        const int it = y, ib = (TZ - 1) * TY + y;
        int v = HZT[y] + 1;
        if (v > d && v < hv[it] && ((AZM[it] >> lane) & 1u)) c = min(c, v);
        v = HZB[y] + 1;
        if (v > d && v < hv[ib] && ((AZP[ib] >> lane) & 1u)) c = min(c, v);
      }
    }
    if (xrow < R && HX + 1 > d) c = min(c, HX + 1);
    return __reduce_min_sync(FULL, c);
  };
  unsigned F[R];
#pragma unroll
  for (int i = 0; i < R; ++i) F[i] = 0u;
  unsigned rows_changed = 0, c0 = 0, c31 = 0;
  bool again = false;
  const int cap = jfc::cap_of(g, ts.d_ctr);   // levels at or above it stay unreachable
  int d = next_level(-1);
  for (int level = 0; d < cap; ++level) {
    if (level >= kMaxLevels) { again = true; break; }
    const unsigned sx = __ballot_sync(FULL, HX + 1 == d);
    unsigned N[R];
    unsigned any = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int y = i % TY, z = i / TY;
      unsigned m = ((F[i] >> 1) & AXP[i]) | ((F[i] << 1) & AXM[i]);
      if (y < TY - 1) m |= F[(i + 1 < R) ? i + 1 : i] & AYP[i];
      if (y > 0) m |= F[(i > 0) ? i - 1 : 0] & AYM[i];
      if constexpr (DIMS == 3) {
        if (z < TZ - 1) m |= F[(i + TY < R) ? i + TY : i] & AZP[i];
        if (z > 0) m |= F[(i >= TY) ? i - TY : 0] & AZM[i];
        if (z == 0) m |= __ballot_sync(FULL, HZT[y] + 1 == d) & AZM[i];
        if (z == TZ - 1) m |= __ballot_sync(FULL, HZB[y] + 1 == d) & AZP[i];
      }
      if (y == 0) m |= __ballot_sync(FULL, HT[z] + 1 == d) & AYM[i];
      if (y == TY - 1) m |= __ballot_sync(FULL, HB[z] + 1 == d) & AYP[i];
      m |= ((sx >> i) & 1u) & AXM[i];
      m |= (((sx >> (16 + i)) & 1u) << 31) & AXP[i];
      N[i] = m & __ballot_sync(FULL, hv[i] > d);
      any |= N[i];
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      F[i] = N[i];
      if (N[i]) {
        rows_changed |= 1u << i;
        c0 |= N[i] & 1u;
        c31 |= N[i] >> 31;
        if ((N[i] >> lane) & 1u) {
          hv[i] = d;
          g.h[roff<TY>(a, i)] = d;
        }
      }
    }
    d = any ? d + 1 : next_level(d);
  }
  // activity per 8-row half of a 2D 32x16 tile (bit 0 rows 0-7, bit 1 rows
  // 8-15: the push-relabel work items of split tile sets), else bit 0
  bool act_lo = false, act_hi = false;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const bool live = ((posm >> i) & 1u) && hv[i] < JFC_INF;
    if (DIMS == 2 && TY == 16 && i >= 8) act_hi |= live;
    else act_lo |= live;
  }
  act_lo = __any_sync(FULL, act_lo);
  act_hi = __any_sync(FULL, act_hi);
  const bool act = act_lo || act_hi;
  if (lane == 0) {
    const int old = (__ldcg(ts.d_act + tid) & 3u) != 0 ? 1 : 0;
    ts.d_act[tid] = (uint8_t)((act_lo ? 1 : 0) | (act_hi ? 2 : 0));
    if (ti.x != cur_grid) {
      if (delta && cur_grid >= 0) atomicAdd(&ts.d_grid_active[cur_grid], delta);
      delta = 0;
      cur_grid = ti.x;
    }
    delta += (act ? 1 : 0) - old;
  }
  flag_neighbours<DIMS, TY, TZ>(g, a, tid, rows_changed, c0 != 0, c31 != 0, again, Q);
}

// Frontier visit, one warp per tile, min-plus form: the tile's heights in
// registers (lane = x, one register per row), lowered by the halo heights
// across residual arcs, then closed in place: row closures by doubling
// shuffles, y and z runs in registers (a forward and a backward sweep per
// line), repeated until nothing falls.  Monotone, so the fixpoint is the
// exact in-tile distance given the halo, as the level BFS gives; a visit
// costs one closure per turn a shortest path takes instead of one step per
// level.  Improvements at or above the distance cap are dropped (those
// nodes stay unreachable).
// Staged tile of a 3D frontier visit, filled by two tensor copies: the h
// plane over the tile and its one-cell halo (40 columns from x0 - 4, as the
// push-relabel staging) and the tile's arc bytes.
template <int TY, int TZ>
struct alignas(128) RlStage {
  using T = jfc::CtaTile<3, TY, TZ, 40, 4>;
  static constexpr unsigned kHb = sizeof(int) * T::HN, kLb = 32u * TY * TZ;
  static constexpr unsigned kBytes = kHb + kLb;   // bytes the two copies deliver
  int hb[T::HN];
  alignas(128) uint8_t lb[32 * TY * TZ];
};

// hb / lb non-null: the tile comes from a staged copy (RlStage) instead of
// global loads.
template <int DIMS, int TY, int TZ, bool STAGED = false>
__device__ __forceinline__ void relabel_frontier_minplus(const TileSet& ts, int tid, int4 ti, const BfsQ& Q,
                                                         int& cur_grid, int& delta, const int* hb = nullptr,
                                                         const uint8_t* lb = nullptr) {
  constexpr int R = TY * TZ;
  using ST = jfc::CtaTile<3, TY, TZ, 40, 4>;
  const int lane = threadIdx.x & 31;
  const GridDev& g = ts.d_desc[ti.x];
  const Addr a = make_addr<DIMS, TY, TZ>(g, ti, lane);
  // the tile's activity byte as the last visit left it (another SM's write of
  // an earlier pass: read from L2, and early, so its latency overlaps the
  // closure)
  const unsigned act_old = lane == 0 ? (unsigned)__ldcg(ts.d_act + tid) : 0u;
  unsigned lab[R];
  int hv[R], h0[R];
  unsigned AXP[R], AXM[R];
  unsigned posm = 0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    if constexpr (STAGED) {
      lab[i] = lb[i * 32 + lane];
      h0[i] = hb[ST::hidx(lane, i % TY, i / TY)];
    } else {
      const long long n = roff<TY>(a, i);
      lab[i] = g.label[n];   // arc byte written by the first pass
      h0[i] = g.h[n];
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i) {
    hv[i] = h0[i];
    AXP[i] = __ballot_sync(FULL, lab[i] & jfc::A_XP);
    AXM[i] = __ballot_sync(FULL, lab[i] & jfc::A_XM);
    if (lab[i] & 128u) posm |= 1u << i;
  }
  // the halo, fixed during the visit: y faces per z slice (lane = x), z
  // faces per row y, x faces in lanes r (left of row r) and 16 + r (right);
  // loaded together with the tile (no load waits for the arc bytes)
  int HT[TZ], HB[TZ], HZT[DIMS == 3 ? TY : 1], HZB[DIMS == 3 ? TY : 1];
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    if constexpr (STAGED) {
      HT[z] = a.has_yT ? hb[ST::hidx(lane, -1, z)] : JFC_INF;
      HB[z] = a.has_yB ? hb[ST::hidx(lane, TY, z)] : JFC_INF;
    } else {
      const long long n = roff<TY>(a, z * TY);
      HT[z] = a.has_yT ? g.h[n - a.pitch] : JFC_INF;
      HB[z] = a.has_yB ? g.h[n + (long long)TY * a.pitch] : JFC_INF;
    }
  }
  if constexpr (DIMS == 3) {
#pragma unroll
    for (int y = 0; y < TY; ++y) {
      if constexpr (STAGED) {
        HZT[y] = a.has_zT ? hb[ST::hidx(lane, y, -1)] : JFC_INF;
        HZB[y] = a.has_zB ? hb[ST::hidx(lane, y, TZ)] : JFC_INF;
      } else {
        const long long n = roff<TY>(a, y);
        HZT[y] = a.has_zT ? g.h[n - a.slab] : JFC_INF;
        HZB[y] = a.has_zB ? g.h[n + (long long)TZ * a.slab] : JFC_INF;
      }
    }
  }
  const int xrow = lane & 15;
  int hx = JFC_INF;
  if (xrow < R && (lane < 16 ? a.has_xL : a.has_xR))
    hx = STAGED ? hb[ST::hidx(lane < 16 ? -1 : 32, xrow % TY, xrow / TY)]
                : g.h[(long long)(lane < 16 ? a.x0 - 1 : a.x0 + 32) + (long long)(a.y0 + xrow % TY) * a.pitch +
                  (long long)(a.z0 + xrow / TY) * a.slab];
  // the tile's interior is at its fixpoint (the dense pass or its last
  // visit closed it, and only its own visits write it), so only a halo seed
  // that lowers a border node can change anything
  bool seeded = false;
  auto seed = [&](int& v, bool arc, int hn) {
    if (arc && hn + 1 < v) { v = hn + 1; seeded = true; }
  };
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    const int it = z * TY, ib = z * TY + TY - 1;
    seed(hv[it], lab[it] & jfc::A_YM, HT[z]);
    seed(hv[ib], lab[ib] & jfc::A_YP, HB[z]);
  }
  if constexpr (DIMS == 3) {
#pragma unroll
    for (int y = 0; y < TY; ++y) {
      const int it = y, ib = (TZ - 1) * TY + y;
      seed(hv[it], lab[it] & jfc::A_ZM, HZT[y]);
      seed(hv[ib], lab[ib] & jfc::A_ZP, HZB[y]);
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int hl = __shfl_sync(FULL, hx, i), hr = __shfl_sync(FULL, hx, 16 + i);
    seed(hv[i], lane == 0 && (lab[i] & jfc::A_XM), hl);
    seed(hv[i], lane == 31 && (lab[i] & jfc::A_XP), hr);
  }
  if (__any_sync(FULL, seeded)) tile_close<DIMS, TY, TZ>(hv, lab, AXP, AXM, lane);
  const int cap = jfc::cap_of(g, ts.d_ctr);
  unsigned rows_changed = 0;
  bool c0 = false, c31 = false, act_lo = false, act_hi = false;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    if (hv[i] >= cap) hv[i] = h0[i];   // at or above the cap: stays as it was (unreachable)
    const bool chg = hv[i] < h0[i];
    const unsigned m = __ballot_sync(FULL, chg);
    if (m) {
      rows_changed |= 1u << i;
      c0 |= (m & 1u) != 0;
      c31 |= (m >> 31) != 0;
    }
    if (chg) g.h[roff<TY>(a, i)] = hv[i];
    // activity per 8-row half of a 2D 32x16 tile (bit 0 rows 0-7, bit 1
    // rows 8-15: the push-relabel work items of split tile sets), else bit 0
    const bool live = ((posm >> i) & 1u) && hv[i] < JFC_INF;
    if (DIMS == 2 && TY == 16 && i >= 8) act_hi |= live;
    else act_lo |= live;
  }
  act_lo = __any_sync(FULL, act_lo);
  act_hi = __any_sync(FULL, act_hi);
  const bool act = act_lo || act_hi;
  if (lane == 0) {
    const int old = (act_old & 3u) != 0 ? 1 : 0;
    ts.d_act[tid] = (uint8_t)((act_lo ? 1 : 0) | (act_hi ? 2 : 0));
    if (ti.x != cur_grid) {
      if (delta && cur_grid >= 0) atomicAdd(&ts.d_grid_active[cur_grid], delta);
      delta = 0;
      cur_grid = ti.x;
    }
    delta += (act ? 1 : 0) - old;
  }
  flag_neighbours<DIMS, TY, TZ>(g, a, tid, rows_changed, c0, c31, false, Q);
}

// 1: frontier visits of the warp form use the min-plus closure, 0: the level BFS
#ifndef JFC_RELABEL_MINPLUS
#define JFC_RELABEL_MINPLUS 1
#endif

#ifndef JFC_GR_ASYNC
#define JFC_GR_ASYNC 1
#endif

// Refill of the push-relabel queues (buffer 0 of each parity) from the
// active-tile bits, warp-aggregated.  Split tile sets queue the active 8-row
// halves as work items 2 * tile + half, half 0 with the tile's checkerboard
// parity in the 32x8 tiling and half 1 with the other.
__device__ __forceinline__ void refill_pr_queues(const TileSet& ts, DevCounters* ctr, int lane) {
  for (;;) {
    const unsigned c = jfc::warp_ticket(&ctr->ticket[0]);
    const long long b = (long long)c * 32;
    if (b >= ts.ntiles) break;
    const long long t = b + lane;
    bool w[2][2] = {{false, false}, {false, false}};   // [half][parity queue]
    if (t < ts.ntiles) {
      const unsigned bits = ts.d_act[t] & 3u;
      int par = 0;
      if (bits) { const int4 ti = ts.d_info[t]; par = (ti.y + (ts.pr_split ? 2 * ti.z : ti.z) + ti.w) & 1; }
      if (ts.pr_split) {
        const bool a0 = (bits & 1u) != 0, a1 = (bits & 2u) != 0;
        ts.d_flag_pr[2 * t] = a0 ? 1 : 0;
        ts.d_flag_pr[2 * t + 1] = a1 ? 1 : 0;
        w[0][par] = a0;
        w[1][par ^ 1] = a1;
      } else {
        ts.d_flag_pr[t] = bits ? 1 : 0;
        w[0][par] = bits != 0;
      }
    }
    const int item0 = ts.pr_split ? (int)(2 * t) : (int)t;
    jfc::warp_append(w[0][0], item0, nullptr, ts.d_q_pr[0][0], &ctr->qn_pr[0][0]);
    jfc::warp_append(w[0][1], item0, nullptr, ts.d_q_pr[1][0], &ctr->qn_pr[1][0]);
    if (ts.pr_split) {
      jfc::warp_append(w[1][0], item0 + 1, nullptr, ts.d_q_pr[0][0], &ctr->qn_pr[0][0]);
      jfc::warp_append(w[1][1], item0 + 1, nullptr, ts.d_q_pr[1][0], &ctr->qn_pr[1][0]);
    }
  }
}

// Global relabel, pass 0: every tile, one warp per tile (bit-parallel level
// BFS from the deficits, fused initialisation).  A plain launch: its many
// registers do not limit the occupancy of the frontier kernel.
// (32 x 8 2D tiles fit in 64 registers without spills: 4 CTAs per SM keep
// twice the loads in flight of the 2-CTA bound the larger tiles need)
template <int DIMS, int TY, int TZ>
__global__ void __launch_bounds__(256, (DIMS == 3 && TY * TZ > 8) ? 1 : (DIMS == 2 && TY == 8) ? 4 : 2)
    k_relabel_first(TileSet ts) {
  DevCounters* ctr = ts.d_ctr;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctr->t_gr_start = jfc::global_ns();
  const int lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= ts.ntiles) return;
  // (appends straight to the queue: gathering a CTA's appends behind a block
  // barrier measured slower, the barrier holds the CTA's slot to its
  // slowest warp)
  BfsQ Q{ts.d_flag_bfs[1], ts.d_q_bfs[1], &ctr->qn_bfs[1]};
  int wgrid = -1, wdelta = 0;
  relabel_first_warp<DIMS, TY, TZ>(ts, (int)w, Q, wgrid, wdelta);
  if (lane == 0 && wdelta && wgrid >= 0) atomicAdd(&ts.d_grid_active[wgrid], wdelta);
}

// Global relabel, frontier passes (persistent, cooperative): one CTA per
// queued tile, grid barrier between passes, until a pass queues nothing; then
// the push-relabel queues are refilled with every tile holding an active node
// (the reference's graphcut_count_node + clogs scan + graphcut_scatter_node,
// graphcut_count_block.cl:19-65, as one warp-aggregated append).
// Warp form of the frontier passes: one warp per queued tile (3D: many
// tiles per pass, so the visit throughput counts).
// (level-BFS form: one CTA per SM, its registers; min-plus form: 2 CTAs per
// SM, the registers the two-ahead ticket pipeline holds without spills: 3
// CTAs per SM spilled and measured slower, 116.5 vs 104-108.5 ms of frontier
// per video solve)
#ifndef JFC_RELABEL_WARP_MINB
#define JFC_RELABEL_WARP_MINB 1
#endif
#ifndef JFC_RL3D_MINB
#define JFC_RL3D_MINB 2
#endif
// 1: 3D frontier tiles of up to 8 rows are staged by tensor copies
#ifndef JFC_RL3D_STAGE
#define JFC_RL3D_STAGE 1
#endif
template <int DIMS, int TY, int TZ>
__global__ void __launch_bounds__(256, JFC_RELABEL_MINPLUS ? (TY * TZ > 8 ? 2 : JFC_RL3D_MINB) : JFC_RELABEL_WARP_MINB)
    k_relabel_warp(TileSet ts, int max_passes) {
  __shared__ int s_items[8][64];   // per-warp staged queue appends (at most 38 before a flush)
  __shared__ int s_cnt[8];
  // 3D tiles of up to 8 rows with tensor maps: each warp stages its tiles by
  // tensor copies into two buffers of its own (dynamic shared memory), the
  // next ticket's tile copied while the current one is visited
  using Stage = RlStage<TY, TZ>;
  constexpr bool kStage = JFC_RL3D_STAGE && JFC_RELABEL_MINPLUS && DIMS == 3 && TY * TZ <= 8;
  __shared__ uint64_t s_bar[8][2];
  extern __shared__ __align__(128) unsigned char s_dyn[];
  DevCounters* ctr = ts.d_ctr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool tma = kStage && ts.d_tmap != nullptr;
  Stage* stage = reinterpret_cast<Stage*>(s_dyn + ((128u - (jfc::smem_addr(s_dyn) & 127u)) & 127u)) + 2 * warp;
  if (lane == 0) s_cnt[warp] = 0;
  if (tma && lane == 0) {
    jfc::mbar_init(&s_bar[warp][0], 1);
    jfc::mbar_init(&s_bar[warp][1], 1);
    jfc::fence_mbar_init();
  }
  __syncthreads();
  const unsigned long long spin = jfc::spin_cap(ctr);
  unsigned parity = 0;      // bit b: phase parity of buffer b's next fill (warp-uniform)
  int acquired_grid = -1;   // lane 0: grid whose maps it acquired
  // lane 0: copy tile t4 (grid, tile x / y / z) into buffer b
  auto issue = [&](int4 t4, int b) {
    if (lane == 0) {
      const char* maps = (const char*)ts.d_tmap + (size_t)t4.x * 384;
      if (t4.x != acquired_grid) {
        jfc::fence_tmap_acquire(maps + 128);
        jfc::fence_tmap_acquire(maps + 256);
        acquired_grid = t4.x;
      }
      jfc::fence_async_shared();
      jfc::mbar_arrive_tx(&s_bar[warp][b], Stage::kBytes);
      jfc::tma_load_3d(stage[b].hb, maps + 128, t4.y * 32 - 4, t4.z * TY - 1, t4.w * TZ - 1, &s_bar[warp][b]);
      jfc::tma_load_3d(stage[b].lb, maps + 256, t4.y * 32, t4.z * TY, t4.w * TZ, &s_bar[warp][b]);
    }
  };
  unsigned long long visits = 0;
  int cur_grid = -1, delta = 0;
  bool ok = true;
  int pass = 1;
  const unsigned long long t1 = jfc::global_ns();
  for (pass = 1; ok; ++pass) {
    const int cb = pass & 1;
    const int n = jfc::vload(&ctr->qn_bfs[cb]);
    if (n == 0) break;
    if (pass > max_passes) {
      if (blockIdx.x == 0 && threadIdx.x == 0) ctr->bfs_status = 2;
      break;
    }
    BfsQ Q{ts.d_flag_bfs[cb ^ 1], ts.d_q_bfs[cb ^ 1], &ctr->qn_bfs[cb ^ 1], s_items[warp], &s_cnt[warp]};
    const int* queue = ts.d_q_bfs[cb];
    int* fcur = ts.d_flag_bfs[cb];
    // Tickets come in chunks of kChunk while the pass holds a full round of
    // chunks beyond the warp's (one counter update per chunk: the ticket
    // and queue counters are single addresses every warp updates, which
    // serialises them), singly near the end of the pass.  The next ticket,
    // its queue entry and its tile are fetched while the current tile is
    // visited.  Queue appends are staged per warp and published 32 or more
    // at a time.
    constexpr unsigned kChunk = 4;
    const long long round = (long long)gridDim.x * (blockDim.x >> 5);
    unsigned k = 0, kend = 0;   // tickets [k, kend) held by the warp
    auto take = [&]() -> int {
      if (k >= kend) {
        unsigned v = 0;
        // chunk size from the warp's last ticket (a lower bound on the
        // counter): no extra read of the counter on the way to its update
        const unsigned c = (long long)k + round * kChunk < n ? kChunk : 1u;
        if (lane == 0) v = atomicAdd(&ctr->ticket[cb], c);
        k = __shfl_sync(FULL, v, 0);
        kend = k + c;
      }
      const unsigned kk = k++;
      return (int)kk < n ? queue[kk] : -1;
    };
    // the previous pass's writes (seen through the grid barrier) come before
    // this pass's tensor reads
    if (tma && lane == 0) jfc::fence_async_global();
    // Two tickets ahead: the current tile tt is staged in `buf`, the next
    // one tn is being copied into the other buffer, and the ticket and tile
    // of the one after (tnn) are fetched while tt is visited; tnn's copy goes
    // into `buf` once tt's visit has read it.
    int tt = take();
    int4 ti = tt >= 0 ? ts.d_info[tt] : make_int4(0, 0, 0, 0);
    int buf = 0;
    if (tma && tt >= 0) issue(ti, buf);
    int tn = tt >= 0 ? take() : -1;
    int4 tin = tn >= 0 ? ts.d_info[tn] : make_int4(0, 0, 0, 0);
    if (tma && tn >= 0) issue(tin, buf ^ 1);
    while (tt >= 0) {
      const int tnn = tn >= 0 ? take() : -1;
      const int4 tinn = tnn >= 0 ? ts.d_info[tnn] : make_int4(0, 0, 0, 0);
      if (lane == 0) fcur[tt] = 0;
      __syncwarp();
      if (tma) {
        const unsigned ph = (parity >> buf) & 1u;
        const bool got = __all_sync(FULL, jfc::mbar_wait(&s_bar[warp][buf], ph, spin));
        parity ^= 1u << buf;
        if (!got) {
          if (lane == 0) {
            atomicExch(&ctr->error, 1);
            // copies in flight land before the warp leaves (fixed bound)
            constexpr unsigned long long kDrainPolls = 1ull << 26;
            jfc::mbar_wait(&s_bar[warp][buf], ph, kDrainPolls);
            if (tn >= 0) jfc::mbar_wait(&s_bar[warp][buf ^ 1], (parity >> (buf ^ 1)) & 1u, kDrainPolls);
          }
          __syncwarp();
          break;   // the grid barrier below sees the error: every CTA leaves
        }
        relabel_frontier_minplus<DIMS, TY, TZ, true>(ts, tt, ti, Q, cur_grid, delta, stage[buf].hb, stage[buf].lb);
        __syncwarp();   // every lane has read `buf` before it is refilled
        if (tnn >= 0) issue(tinn, buf);
      } else if (JFC_RELABEL_MINPLUS) {
        relabel_frontier_minplus<DIMS, TY, TZ>(ts, tt, ti, Q, cur_grid, delta);
      } else {
        relabel_frontier_warp<DIMS, TY, TZ>(ts, tt, Q, cur_grid, delta);
      }
      buf ^= 1;
      ++visits;
      __syncwarp();
      if (*(volatile int*)Q.scnt >= 32) {
        flush_staged(Q, lane);
        __syncwarp();
        if (lane == 0) *Q.scnt = 0;
        __syncwarp();
      }
      tt = tn;
      ti = tin;
      tn = tnn;
      tin = tinn;
    }
    __syncwarp();
    flush_staged(Q, lane);
    __syncwarp();
    if (lane == 0) *Q.scnt = 0;
    __syncwarp();
    ok = jfc::grid_sync(ctr, [&]() {
      ctr->ticket[cb] = 0;
      ctr->qn_bfs[cb] = 0;
    });
  }
  if (lane == 0 && delta && cur_grid >= 0) atomicAdd(&ts.d_grid_active[cur_grid], delta);
  // refill the push-relabel queues (buffer 0 of each parity) from the
  // active-tile flags
  if (ok) ok = jfc::grid_sync(ctr, [&]() {
    ctr->qn_pr[0][0] = ctr->qn_pr[0][1] = ctr->qn_pr[1][0] = ctr->qn_pr[1][1] = 0;
    ctr->cur_pr[0] = ctr->cur_pr[1] = 0;
  });
  if (ok) {
    refill_pr_queues(ts, ctr, lane);
    ok = jfc::grid_sync(ctr, [&]() { ctr->ticket[0] = 0; });
  }
  // frontier visits are counted per warp (lane 0); pass 0 visited every tile
  __shared__ unsigned long long s_vis;
  if (threadIdx.x == 0) s_vis = 0;
  __syncthreads();
  if (lane == 0 && visits) atomicAdd(&s_vis, visits);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_vis) atomicAdd(&ctr->bfs_visits, s_vis);
    if (blockIdx.x == 0) {
      ctr->bfs_passes = pass;
      ctr->bfs_visits += (unsigned long long)ts.ntiles;
      if (ctr->bfs_status == 0) ctr->bfs_status = 1;
      const unsigned long long t2 = jfc::global_ns();
      ctr->ns_gr_first += t1 - ctr->t_gr_start;
      ctr->ns_gr_frontier += t2 - t1;
    }
  }
}

// Global relabel, frontier passes (persistent, cooperative), CTA form: one
// CTA per queued tile (2D: few tiles per pass, so the visit latency counts), grid barrier between passes, until a pass queues nothing; then
// the push-relabel queues are refilled with every tile holding an active node
// (the reference's graphcut_count_node + clogs scan + graphcut_scatter_node,
// graphcut_count_block.cl:19-65, as one warp-aggregated append).
// After the dense first pass every tile's heights are the exact in-tile
// distances (halo unknown), so a tile can only fall through an arc leaving
// it: one warp checks the tile's border nodes against the halo (2D) and
// queues the tile for a full visit only when some residual arc u -> v out of
// the tile has h(v) + 1 < h(u).
template <int TY>
__device__ __forceinline__ bool border_improvable(const TileSet& ts, int tid, int lane) {
  const int4 ti = ts.d_info[tid];
  const GridDev& g = ts.d_desc[ti.x];
  const int cap = jfc::cap_of(g, ts.d_ctr);
  const long long pitch = g.pitch;
  const int x0 = ti.y * 32, y0 = ti.z * TY;
  const long long base = (long long)x0 + (long long)y0 * pitch;
  // a distance offered through the arc counts only below the relabel's cap
  auto better = [&](long long n, long long m) { const int v = g.h[m] + 1; return v < g.h[n] && v < cap; };
  bool imp = false;
  if (y0 > 0) {   // top row, arcs -y
    const long long n = base + lane;
    if ((g.label[n] & jfc::A_YM) && better(n, n - pitch)) imp = true;
  }
  if (y0 + TY < g.Hp) {   // bottom row, arcs +y
    const long long n = base + lane + (TY - 1) * pitch;
    if ((g.label[n] & jfc::A_YP) && better(n, n + pitch)) imp = true;
  }
  if (lane < TY && x0 > 0) {   // left column, arcs -x
    const long long n = base + lane * pitch;
    if ((g.label[n] & jfc::A_XM) && better(n, n - 1)) imp = true;
  } else if (lane >= 16 && lane < 16 + TY && x0 + 32 < pitch) {   // right column, arcs +x
    const long long n = base + 31 + (lane - 16) * pitch;
    if ((g.label[n] & jfc::A_XP) && better(n, n + 1)) imp = true;
  }
  return __any_sync(jfc::FULL, imp);
}

// (32 x 8 tiles: 6 CTAs per SM, the worklist's pollers and the border check's warps)
#ifndef JFC_RL2D_MINB
#define JFC_RL2D_MINB 6
#endif
template <int DIMS, int TY, int TZ>
__global__ void __launch_bounds__(RTile<DIMS, TY, TZ>::NT,
                                  (DIMS == 2 && TY == 8) ? JFC_RL2D_MINB : RTile<DIMS, TY, TZ>::NT > 256 ? 2 : 3)
    k_relabel_cta(TileSet ts, int max_passes) {
  __shared__ RlSmem<DIMS, TY, TZ> sm;
  DevCounters* ctr = ts.d_ctr;
  const int lane = threadIdx.x & 31;
  unsigned long long visits = 0;
  int cur_grid = -1, delta = 0;
  bool ok = true;
  int pass = 1;
  bool to_worklist = false;
  const unsigned long long t1 = jfc::global_ns();
  for (pass = 1; ok; ++pass) {
    const int cb = pass & 1;
    const int n = jfc::vload(&ctr->qn_bfs[cb]);
    if (n == 0) break;
    if (pass > max_passes) {
      if (blockIdx.x == 0 && threadIdx.x == 0) ctr->bfs_status = 2;
      break;
    }
    BfsQ Q{ts.d_flag_bfs[cb ^ 1], ts.d_q_bfs[cb ^ 1], &ctr->qn_bfs[cb ^ 1]};
    const int* queue = ts.d_q_bfs[cb];
    int* fcur = ts.d_flag_bfs[cb];
    to_worklist = JFC_GR_ASYNC && DIMS == 2 && pass == 1;
    if (DIMS == 2 && pass == 1) {
      // the tiles the dense pass queued: a warp-level border check, full
      // visits from pass 2 on for the tiles that can fall
      for (;;) {
        const unsigned k = jfc::warp_ticket(&ctr->ticket[cb]);
        if ((int)k >= n) break;
        const int tt = queue[k];
        if (lane == 0) fcur[tt] = 0;
        const bool imp = border_improvable<TY>(ts, tt, lane);
        jfc::warp_append(imp && lane == 0, tt, Q.flags, Q.q, Q.qn);
      }
    } else {
      for (;;) {
        if (threadIdx.x == 0) {
          const unsigned k = atomicAdd(&ctr->ticket[cb], 1u);
          sm.ntile = (int)k < n ? queue[k] : -1;
          if ((int)k < n) fcur[sm.ntile] = 0;
        }
        __syncthreads();
        const int tt = sm.ntile;
        __syncthreads();
        if (tt < 0) break;
        relabel_visit<DIMS, TY, TZ>(ts, tt, sm, Q, cur_grid, delta);
        if (threadIdx.x < 32) ++visits;
      }
    }
    ok = jfc::grid_sync(ctr, [&]() {
      ctr->ticket[cb] = 0;
      ctr->qn_bfs[cb] = 0;
      if (to_worklist) {
        ctr->wl_head = 0;
        const unsigned long long q = (unsigned)ctr->qn_bfs[cb ^ 1];
        ctr->wl_tail_out = (q << 32) | q;
      }
    });
    if (to_worklist) { ++pass; break; }
  }
  if (ok && to_worklist) {
    // 2D passes 2..: an asynchronous worklist instead of barrier-separated
    // passes.  A tile whose boundary fell queues its neighbours at once and
    // any free CTA takes them, so a distance wave crosses one tile per visit
    // instead of one tile per pass (the relaxation is monotone: any order
    // reaches the same exact distances).  A per-tile lock keeps two visits of
    // one tile apart; the work is done when no queued item is left.
    const unsigned cap = (unsigned)ts.ntiles;
    int* ring = ts.d_q_bfs[0];          // the border check queued into buffer 0
    int* busy = ts.d_flag_bfs[1];       // free after the border check
    const unsigned n0 = (unsigned)(*(volatile unsigned long long*)&ctr->wl_tail_out >> 32);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap; i += (long long)gridDim.x * blockDim.x) {
      if (i >= n0) ring[i] = -1;
      busy[i] = 0;
    }
    ok = jfc::grid_sync(ctr, [&]() {});
    const unsigned long long max_spins = jfc::spin_cap(ctr);
    const RlRing W{ring, cap, &ctr->wl_tail_out, &ctr->error, max_spins};
    const BfsQ Q{ts.d_flag_bfs[0], nullptr, nullptr};
    while (ok) {
      if (threadIdx.x == 0) {
        int tile = -1;
        const unsigned k = atomicAdd(&ctr->wl_head, 1u);
        int* slot = ring + k % cap;
        // bounded: the item arrives, or the work is done, or an error; the
        // count measures a stall (it restarts whenever the worklist moves:
        // items appended or finished), not the length of the relabel
        unsigned long long spins = 0;
        volatile unsigned long long* vto = &ctr->wl_tail_out;
        unsigned long long seen = *vto;
        for (;;) {
          if (*(volatile int*)slot >= 0) {
            const int v = atomicExch(slot, -1);
            if (v >= 0) { tile = v; break; }
          }
          const unsigned long long to = *vto;
          if ((unsigned)to == 0u || *(volatile int*)&ctr->error) break;
          if (to != seen) {
            seen = to;
            spins = 0;
          } else if (++spins > max_spins) {
            atomicExch(&ctr->error, 1);
            break;
          }
          __nanosleep(32);
        }
        if (tile >= 0) {
          spins = 0;
          while (atomicCAS(busy + tile, 0, 1) != 0) {
            if (++spins > max_spins || *(volatile int*)&ctr->error) { atomicExch(&ctr->error, 1); tile = -1; break; }
            __nanosleep(32);
          }
        }
        if (tile >= 0) {
          __threadfence();
          atomicExch(Q.flags + tile, 0);   // dequeued before its heights are read
          __threadfence();
        }
        sm.ntile = tile;
      }
      __syncthreads();
      const int tt = sm.ntile;
      __syncthreads();
      if (tt < 0) break;
      relabel_visit<DIMS, TY, TZ>(ts, tt, sm, Q, cur_grid, delta, W);   // ends with a block barrier
      if (threadIdx.x == 0) {
        __threadfence();
        atomicExch(busy + tt, 0);
        if (!sm.folded) atomicAdd(&ctr->wl_tail_out, ~0ull);   // - 1 outstanding
      }
      if (threadIdx.x < 32) ++visits;
    }
  }
  // per-grid activity deltas: thread 0 holds the CTA visits', lane 0 of
  // each warp the warp visits'
  if (lane == 0 && delta && cur_grid >= 0) atomicAdd(&ts.d_grid_active[cur_grid], delta);
  // refill the push-relabel queues (buffer 0 of each parity) from the
  // active-tile flags
  if (ok) ok = jfc::grid_sync(ctr, [&]() {
    ctr->qn_pr[0][0] = ctr->qn_pr[0][1] = ctr->qn_pr[1][0] = ctr->qn_pr[1][1] = 0;
    ctr->cur_pr[0] = ctr->cur_pr[1] = 0;
  });
  if (ok) {
    refill_pr_queues(ts, ctr, lane);
    ok = jfc::grid_sync(ctr, [&]() { ctr->ticket[0] = 0; });
  }
  // frontier visits are counted by warp 0 of each CTA; pass 0 visited every tile
  __shared__ unsigned long long s_vis;
  if (threadIdx.x == 0) s_vis = 0;
  __syncthreads();
  if (lane == 0 && visits) atomicAdd(&s_vis, visits);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_vis) atomicAdd(&ctr->bfs_visits, s_vis);
    if (blockIdx.x == 0) {
      ctr->bfs_passes = pass;
      ctr->bfs_visits += (unsigned long long)ts.ntiles;
      if (ctr->bfs_status == 0) ctr->bfs_status = 1;
      const unsigned long long t2 = jfc::global_ns();
      ctr->ns_gr_first += t1 - ctr->t_gr_start;
      ctr->ns_gr_frontier += t2 - t1;
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

// MODE 0: global relabel, 1: cut, 2: tag
template <int DIMS, int TY, int TZ, int MODE>
cudaError_t bfs_t(const TileSet& ts, int max_passes, const uint8_t* seeds, cudaStream_t s) {
  constexpr bool CUT = MODE != 0;
  // global relabel frontier passes: CTA per tile in 2D, warp per tile in 3D
  const void* fn;
  if constexpr (MODE == 1) fn = (const void*)k_cut<DIMS, TY, TZ, false>;
  else if constexpr (MODE == 2) fn = (const void*)k_cut<DIMS, TY, TZ, true>;
  else if constexpr (DIMS == 2) fn = (const void*)k_relabel_cta<DIMS, TY, TZ>;
  else fn = (const void*)k_relabel_warp<DIMS, TY, TZ>;
  const int nt = (CUT || DIMS == 3) ? 256 : RTile<DIMS, TY, TZ>::NT;
  // the 3D frontier's staging buffers: two per warp (dynamic shared memory)
  const size_t dyn = (!CUT && DIMS == 3 && JFC_RL3D_STAGE && JFC_RELABEL_MINPLUS && TY * TZ <= 8)
                         ? 2 * 8 * sizeof(RlStage<TY, TZ>) + 128 : 0;
  if (dyn > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
  }
  static int cache[64] = {0};
  const int blocks = persistent_blocks_cached(cache, fn, nt, dyn);
  if (!CUT) {
    const long long fb = ((long long)ts.ntiles * 32 + 255) / 256;
    jfc_note_launch();
    k_relabel_first<DIMS, TY, TZ><<<(unsigned)fb, 256, 0, s>>>(ts);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  TileSet arg = ts;
  void* params[] = {(void*)&arg, (void*)&max_passes, (void*)&seeds};   // relabel kernels take two
  jfc_note_launch();
  return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(nt), params, dyn, s);
}

template <int TY, int TZ>
cudaError_t sums_t(const TileSet& ts, cudaStream_t s) {
  static int cache[64] = {0};
  const int blocks = persistent_blocks_cached(cache, (const void*)k_grid_sums<TY, TZ>, 256);
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

int persistent_blocks_cached(int* cache, const void* kernel, int threads, size_t smem) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return persistent_blocks(kernel, threads, smem);
  // two threads filling one entry at once compute the same value; the
  // atomic store keeps the write whole
  int v = __atomic_load_n(cache + dev, __ATOMIC_RELAXED);
  if (!v) {
    v = persistent_blocks(kernel, threads, smem);
    __atomic_store_n(cache + dev, v, __ATOMIC_RELAXED);
  }
  return v;
}

static cudaError_t bfs_dispatch(const TileSet& ts, int mode, int max_passes, const uint8_t* seeds, cudaStream_t s) {
#define JFC_BFS(D, Y, Z)                                                       \
  (mode == 1 ? bfs_t<D, Y, Z, 1>(ts, max_passes, seeds, s)                     \
             : mode == 2 ? bfs_t<D, Y, Z, 2>(ts, max_passes, seeds, s)         \
                         : bfs_t<D, Y, Z, 0>(ts, max_passes, seeds, s))
  if (ts.dims == 2) {
    if (ts.TR == 8) return JFC_BFS(2, 8, 1);
    if (ts.TR == 16) return JFC_BFS(2, 16, 1);
    return cudaErrorInvalidValue;
  }
  if (ts.TY == 4 && ts.TZ == 4) return JFC_BFS(3, 4, 4);
  if (ts.TY == 4 && ts.TZ == 2) return JFC_BFS(3, 4, 2);
  if (ts.TY == 16 && ts.TZ == 1) return JFC_BFS(3, 16, 1);
  if (ts.TY == 8 && ts.TZ == 2) return JFC_BFS(3, 8, 2);
  if (ts.TY == 8 && ts.TZ == 1) return JFC_BFS(3, 8, 1);
#undef JFC_BFS
  return cudaErrorInvalidValue;
}

cudaError_t launch_bfs(const TileSet& ts, bool cut, int max_passes, cudaStream_t s) {
  return bfs_dispatch(ts, cut ? 1 : 0, max_passes, nullptr, s);
}

cudaError_t launch_tag(const TileSet& ts, const uint8_t* d_seeds, int max_passes, cudaStream_t s) {
  return bfs_dispatch(ts, 2, max_passes, d_seeds, s);
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
  if (ts.TY == 16 && ts.TZ == 1) return sums_t<16, 1>(ts, s);
  if (ts.TY == 8 && ts.TZ == 2) return sums_t<8, 2>(ts, s);
  if (ts.TY == 8 && ts.TZ == 1) return sums_t<8, 1>(ts, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_clear_counters(const TileSet& ts, cudaStream_t s) {
  return cudaMemsetAsync(ts.d_ctr, 0, sizeof(DevCounters), s);
}

namespace {
__global__ void k_set_limits(DevCounters* ctr, unsigned long long polls, int h_cap) {
  ctr->spin_limit = polls;
  ctr->h_cap = h_cap;
}
}  // namespace

cudaError_t launch_set_limits(const TileSet& ts, unsigned long long polls, int h_cap, cudaStream_t s) {
  jfc_note_launch();
  k_set_limits<<<1, 1, 0, s>>>(ts.d_ctr, polls, h_cap);
  return cudaGetLastError();
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
