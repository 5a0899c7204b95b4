// kernels_pr.cu — block-wise push-relabel (the JF-Cut core).
//
// Reference: graphcut_relabel_push (src/QVisualizer/cl/GraphCut/graphcut_push_relabel.cl:25-203
// for 2D, :215-439 for 3D) driven by QGCWidget::relabelPush (QGCWidget.cpp:2136-2154):
// one work-group per 16x16 / 8x8x4 tile with the tile + a one-cell halo in
// __local memory, {relabel even, relabel odd, push even, push odd} to a local
// fixpoint, boundary flow sent out with global atomics, even and odd tiles of
// the checkerboard in separate launches so adjacent tiles never run at once.
//
// B200 design:
//  * one CTA per tile of 32 x TY (x TZ) nodes, one thread per node, one warp per
//    tile row (128-byte coalesced row loads / stores); excess, heights (with
//    the halo) and residual arcs live in shared memory for the visit.  With 2D
//    32 x 16 relabel tiles the visits work on their 32 x 8 halves (SPLIT),
//    which keep a checkerboard parity of their own;
//  * a round = one relabel step and one push step for all nodes at once
//    (two block barriers per round):
//    under a fixed height vector two neighbours never push to each other, so a
//    node's own arcs are only written by itself, the reverse arc of a push only
//    by the pusher, and excess arrives through shared-memory atomics;
//  * rounds repeat until a round moves nothing (__syncthreads_or) or
//    `local_iters` rounds ran; the visit then writes back only words that
//    changed and sends the flow pushed across the border with global atomics;
//  * persistent cooperative launch: `sweeps` x (even tiles, odd tiles) with a
//    grid barrier between parities; each parity drains a compact device queue
//    of active tiles (one tile per CTA ticket), tiles still active re-queue
//    themselves, neighbours that received flow are queued for the other
//    parity (deduplicated).  The phase stops early when both queues are empty.
// Heights only grow between global relabels (relabel = 1 + min over residual
// arcs, applied to active nodes without an admissible arc).
#include "jfc_relax.cuh"
#include "jfc_tma.cuh"


// Iteration cap of the exact local relabel at the start of a visit (0: none).
#ifndef JFC_LOCAL_RELABEL_ITERS
#define JFC_LOCAL_RELABEL_ITERS 8
#endif

namespace {

using jfc::FULL;

template <int DIMS, int TY, int TZ>
using Tile = jfc::CtaTile<DIMS, TY, TZ>;

// Geometry of a visit's height box: 40 columns, node x at column x + 4 (the
// box the tensor copy of the halo lands in: x0 - 4 .. x0 + 35 keeps its
// first column on a 16-byte boundary).
template <int DIMS, int TY, int TZ>
using PrTile = jfc::CtaTile<DIMS, TY, TZ, 40, 4>;

// Staging buffer of one visit, the working copy of the tile during it:
// the tile's planes {e, h, r[0..K-1]} (plane-major, thread order) and the h
// plane over the tile plus its one-cell halo.  The visit pushes and relabels
// in place here.
template <int DIMS, int TY, int TZ>
struct alignas(128) PrStage {
  using T = PrTile<DIMS, TY, TZ>;
  static constexpr int P = 2 + T::K;
  static constexpr unsigned kBytes = (unsigned)(sizeof(int) * (P * T::NT + T::HN));   // bytes one fill copies
  int pl[P][T::NT];
  int hb[T::HN];
};

template <int DIMS, int TY, int TZ>
struct PrSmem {
  using T = PrTile<DIMS, TY, TZ>;
  int out[T::NHALO];      // flow pushed into each halo cell during the visit
  uint8_t arc[T::NT];     // residual-arc bits for the local relabel
  int tile;
  int buf;                // staging buffer of the item being visited
  int gen;                // worklist: generation of the item being visited
  int face[6];            // any flow left through face: x-, x+, y-, y+, z-, z+
  int q_nb[6];            // after a visit: the work item behind each face that received flow, or -1
  int active;             // after a visit: the item still holds an active node
};

template <int DIMS, int TY, int TZ>
__device__ __forceinline__ void halo_cell(int c, int& x, int& y, int& z, int& face) {
  Tile<DIMS, TY, TZ>::halo_cell(c, x, y, z, face);
}

// SPLIT: the work item `tid` is half `tid & 1` (rows 0-7 / 8-15) of the 2D
// 32x16 tile `tid >> 1`, visited as a 32x8 tile; the halves keep their own
// checkerboard parity, so the two halves of a tile never run at once.
// The work items behind the faces of item `tid` (x-, x+, y-, y+, z-, z+),
// -1 where the face is the grid's border.
template <int DIMS, int TY, int TZ, bool SPLIT>
__device__ __forceinline__ int face_item(const TileSet& ts, int tid, int f) {
  const int tile = SPLIT ? tid >> 1 : tid, half = SPLIT ? tid & 1 : 0;
  const int4 ti = ts.d_info[tile];
  const GridDev& g = ts.d_desc[ti.x];
  const int txs = g.tiles_x, tys = g.tiles_y, tzs = g.tiles_z;
  switch (f) {
    case 0: return ti.y > 0 ? (SPLIT ? tid - 2 : tid - 1) : -1;
    case 1: return ti.y < txs - 1 ? (SPLIT ? tid + 2 : tid + 1) : -1;
    case 2: return SPLIT ? (half ? tid - 1 : (ti.z > 0 ? 2 * (tile - txs) + 1 : -1)) : (ti.z > 0 ? tid - txs : -1);
    case 3: return SPLIT ? (half ? (ti.z < tys - 1 ? 2 * (tile + txs) : -1) : tid + 1)
                         : (ti.z < tys - 1 ? tid + txs : -1);
    case 4: return DIMS == 3 && ti.w > 0 ? tid - txs * tys : -1;
    case 5: return DIMS == 3 && ti.w < tzs - 1 ? tid + txs * tys : -1;
    default: return -1;
  }
}

// Tile origin of work item `tid` (elements) and its grid.
template <int DIMS, int TY, int TZ, bool SPLIT>
__device__ __forceinline__ int4 item_origin(const TileSet& ts, int tid) {
  const int tile = SPLIT ? tid >> 1 : tid, half = SPLIT ? tid & 1 : 0;
  const int4 ti = ts.d_info[tile];
  return make_int4(ti.x, ti.y * 32, SPLIT ? (2 * ti.z + half) * TY : ti.z * TY, ti.w * TZ);
}

// Fill staging buffer `st` with work item `tid` by two tensor copies (the
// tile's planes, and the h plane over the tile and its halo), completed on
// `bar`.  Issued by one thread.  Box cells outside the grid arrive as zeros;
// the visit sets the halo ones to INF.
template <int DIMS, int TY, int TZ, bool SPLIT>
__device__ __forceinline__ void pr_stage_issue(const TileSet& ts, int tid, PrStage<DIMS, TY, TZ>& st, uint64_t* bar,
                                               int& acquired_grid) {
  const int4 o = item_origin<DIMS, TY, TZ, SPLIT>(ts, tid);
  const char* maps = (const char*)ts.d_tmap + (size_t)o.x * 384;   // three maps per grid
  if (o.x != acquired_grid) {
    jfc::fence_tmap_acquire(maps);
    jfc::fence_tmap_acquire(maps + 128);
    acquired_grid = o.x;
  }
  jfc::fence_async_shared();   // the buffer's previous visit wrote it through the generic proxy
  jfc::mbar_arrive_tx(bar, PrStage<DIMS, TY, TZ>::kBytes);
  jfc::tma_load_4d(&st.pl[0][0], maps, o.y, o.z, o.w, 0, bar);
  jfc::tma_load_3d(&st.hb[0], maps + 128, o.y - 4, o.z - 1, DIMS == 3 ? o.w - 1 : 0, bar);
}

// One visit of work item `tid` on staging buffer `st`; staged: the tensor
// copies already filled it, otherwise the visit loads the tile itself.  On
// return s.active tells whether the item still holds an active node and
// s.q_nb[f] the item behind each face f that received flow (-1: none).  The
// caller queues them.
template <int DIMS, int TY, int TZ, bool SPLIT>
__device__ __forceinline__ int pr_visit(const TileSet& ts, int tid, int local_iters, bool local_relabel,
                                        PrSmem<DIMS, TY, TZ>& s, PrStage<DIMS, TY, TZ>& st, bool staged) {
  using T = PrTile<DIMS, TY, TZ>;
  const int t = threadIdx.x;
  const int x = t & 31, row = t >> 5, y = row % TY, z = row / TY;
  const int4 o = item_origin<DIMS, TY, TZ, SPLIT>(ts, tid);
  const GridDev& g = ts.d_desc[o.x];
  const int pitch = g.pitch;
  const long long slab = (long long)g.pitch * g.Hp;
  const int x0 = o.y, y0 = o.z, z0 = o.w;
  const long long tbase = (long long)x0 + (long long)y0 * pitch + (long long)z0 * slab;
  const long long n = tbase + x + (long long)y * pitch + (long long)z * slab;
  const int hi = T::hidx(x, y, z);
  int* const se = st.pl[0];
  int* const sh = st.hb;
  JFC_PCLK_DECL

  // ---- the tile and its halo heights
  if (!staged) {
    st.pl[0][t] = g.e[n];
    st.pl[1][t] = g.h[n];
#pragma unroll
    for (int k = 0; k < T::K; ++k) st.pl[2 + k][t] = g.r[k][n];
  }
  const int e0 = st.pl[0][t], h0 = st.pl[1][t];
  int r0[T::K];
#pragma unroll
  for (int k = 0; k < T::K; ++k) r0[k] = st.pl[2 + k][t];
  for (int c = t; c < T::NHALO; c += T::NT) {
    int hx, hy, hz, f;
    halo_cell<DIMS, TY, TZ>(c, hx, hy, hz, f);
    const int gx = x0 + hx, gy = y0 + hy, gz = z0 + hz;
    const bool in = gx >= 0 && gx < pitch && gy >= 0 && gy < g.Hp && gz >= 0 && gz < g.Dp;
    if (!staged || !in)
      sh[T::hidx(hx, hy, hz)] = in ? g.h[(long long)gx + (long long)gy * pitch + (long long)gz * slab] : JFC_INF;
    s.out[c] = 0;
  }
  if (t < 6) s.face[t] = 0;
  {
    unsigned a = 0;
    a |= r0[T::XP] > 0 ? jfc::A_XP : 0u;
    a |= r0[T::YP] > 0 ? jfc::A_YP : 0u;
    a |= r0[T::YM] > 0 ? jfc::A_YM : 0u;
    a |= r0[T::XM] > 0 ? jfc::A_XM : 0u;
    if constexpr (DIMS == 3) {
      a |= r0[T::ZP] > 0 ? jfc::A_ZP : 0u;
      a |= r0[T::ZM] > 0 ? jfc::A_ZM : 0u;
    }
    s.arc[t] = (uint8_t)a;
    // local relabel: distance to the nearest in-tile deficit or halo node
    // over residual arcs (halo heights fixed), then h = max(h, distance).
    // The pointwise max of two valid labellings is valid, so heights stay
    // monotone (push-relabel termination holds) while excess trapped in the
    // tile jumps straight to INF instead of climbing one level per round.
    sh[hi] = e0 < 0 ? 0 : JFC_INF;
  }
  __syncthreads();
  JFC_PCLK(ts.d_ctr, 0);
  // the node's own height lives in a register for the rounds (only its owner
  // writes it); the shared copy is what the neighbours read
  int hown = h0;
  if (JFC_LOCAL_RELABEL_ITERS > 0 && local_relabel) {
    // a partial relaxation overestimates distances, so the local labelling
    // is only applied when the in-tile fixpoint was reached
    const bool exact = jfc::relax_cta_t<T>(sh, s.arc, JFC_LOCAL_RELABEL_ITERS);
    hown = exact ? max(sh[hi], h0) : h0;
#ifdef JFC_PHASE_CLOCK
    if (threadIdx.x == 0 && exact) atomicAdd(&ts.d_ctr->prof[5], 1ull);
#endif
  }
  sh[hi] = hown;
  __syncthreads();
  JFC_PCLK(ts.d_ctr, 1);

  // in-tile neighbours, or the halo cell a push across the border lands in
  const bool in_xp = x < 31, in_xm = x > 0, in_yp = y < TY - 1, in_ym = y > 0;
  const bool in_zp = DIMS == 3 && z < TZ - 1, in_zm = DIMS == 3 && z > 0;
  const int hc_xm = T::NHY + row, hc_xp = T::NHY + T::R + row;
  const int hc_ym = z * 32 + x, hc_yp = TZ * 32 + z * 32 + x;
  const int hc_zm = T::NHY + T::NHX + y * 32 + x, hc_zp = T::NHY + T::NHX + TY * 32 + y * 32 + x;

  // push order: +x, +y, -y, (+z, -z,) -x; q is a constant after unrolling
  constexpr int NP = DIMS == 3 ? 6 : 4;
  auto slot = [](int q) { return q == 0 ? T::XP : q == 1 ? T::YP : q == 2 ? T::YM
                                        : q == NP - 1 ? T::XM : q == 3 ? T::ZP : T::ZM; };
  auto hoff = [](int q) { return q == 0 ? 1 : q == 1 ? T::HX : q == 2 ? -T::HX
                                       : q == NP - 1 ? -1 : q == 3 ? T::HX * T::HY : -T::HX * T::HY; };
  auto toff = [](int q) { return q == 0 ? 1 : q == 1 ? 32 : q == 2 ? -32
                                       : q == NP - 1 ? -1 : q == 3 ? 32 * TY : -32 * TY; };
  int it = 0;
  for (; it < local_iters; ++it) {
    bool did = false;
    // the node's excess and residual arcs, read once per round: nothing
    // changes them between the relabel step and the push step, and the
    // credits neighbours add during the push step only raise them, so these
    // values bound what the node may push from below
    const int e = se[t];
    const bool act = e > 0 && hown < JFC_INF;
    int rk[NP];
    // relabel every active node without an admissible arc, in place
    // (graphcut_push_relabel.cl:80-99 relabels two colours in turn).  A node
    // reading a neighbour that relabels in the same step sees its old or new
    // height; heights only grow, so either value keeps the labelling valid.
    if (act) {
      int hn[NP];
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        rk[q] = st.pl[2 + slot(q)][t];
        hn[q] = sh[hi + hoff(q)];
      }
      const int hm = hown - 1;
      bool adm = false;
      int m = JFC_INF;
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        adm |= rk[q] > 0 && hn[q] == hm;
        m = min(m, rk[q] > 0 ? hn[q] : JFC_INF);
      }
      if (!adm) {
        hown = max(hown, min(m + 1, JFC_INF));
        sh[hi] = hown;
        did = true;
      }
    }
    __syncthreads();
    // push: every node with excess, along admissible arcs in reference order.
    // All operands are loaded first and the pushes are computed in registers,
    // then issued as independent shared-memory updates: a push u->v needs
    // h(u) = h(v) + 1, so in one step nothing else writes u's own arcs or the
    // reverse arc v->u that u credits (the credits are reductions, no load).
    {
      if (act && hown < JFC_INF) {
        const int hm = hown - 1;
        const bool inside[6] = {in_xp, in_yp, in_ym, DIMS == 3 ? in_zp : in_xm, in_zm, in_xm};
        const int hcell[6] = {hc_xp, hc_yp, hc_ym, DIMS == 3 ? hc_zp : hc_xm, hc_zm, hc_xm};
        int hn[NP], d[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) hn[q] = sh[hi + hoff(q)];
        int ex = e;
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          d[q] = (ex > 0 && rk[q] > 0 && hn[q] == hm) ? min(ex, rk[q]) : 0;
          ex -= d[q];
        }
        if (ex != e) {
#pragma unroll
          for (int q = 0; q < NP; ++q) {
            if (d[q]) {
              st.pl[2 + slot(q)][t] = rk[q] - d[q];
              if (inside[q == NP - 1 ? 5 : q]) {
                atomicAdd(&se[t + toff(q)], d[q]);
                atomicAdd(&st.pl[2 + T::K - 1 - slot(q)][t + toff(q)], d[q]);
              } else {
                s.out[hcell[q == NP - 1 ? 5 : q]] += d[q];
              }
            }
          }
          atomicAdd(&se[t], ex - e);
          did = true;
        }
      }
    }
    if (!__syncthreads_or(did)) break;
  }
  const int rounds = it < local_iters ? it + 1 : local_iters;
  JFC_PCLK(ts.d_ctr, 2);

  // ---- write back: each row's 4-node groups holding a changed word, as
  //      128-bit stores (nothing else writes the tile while it is visited, so
  //      the unchanged words of a group are rewritten with their own values)
  const int e1 = se[t], h1 = hown;
  {
    const long long nrow = n - x;
    const int grp = x & ~3;
    auto put = [&](int* gplane, const int* srow, bool changed) {
      const unsigned m = __ballot_sync(jfc::FULL, changed);
      if ((x & 3) == 0 && ((m >> grp) & 0xFu))
        *reinterpret_cast<int4*>(gplane + nrow + grp) = *reinterpret_cast<const int4*>(srow + grp);
    };
    put(g.e, se + row * 32, e1 != e0);
    put(g.h, sh + T::hidx(0, y, z), h1 != h0);
#pragma unroll
    for (int k = 0; k < T::K; ++k) put(g.r[k], st.pl[2 + k] + row * 32, st.pl[2 + k][t] != r0[k]);
  }
  // ---- send the flow pushed across the border into the neighbours' excess
  //      and reverse arcs (only halo cells inside the grid can receive flow:
  //      arcs leaving the grid are zero)
  for (int c = t; c < T::NHALO; c += T::NT) {
    const int v = s.out[c];
    if (v) {
      int hx, hy, hz, f;
      halo_cell<DIMS, TY, TZ>(c, hx, hy, hz, f);
      const long long m = tbase + hx + (long long)hy * pitch + (long long)hz * slab;
      // the halo node's arc pointing back into the tile
      const int rev = f == 0 ? T::XP : f == 1 ? T::XM : f == 2 ? T::YP : f == 3 ? T::YM : f == 4 ? T::ZP : T::ZM;
      atomicAdd(g.e + m, v);
      atomicAdd(g.r[rev] + m, v);
      s.face[f] = 1;
    }
  }
  const bool active = __syncthreads_or((e1 > 0) & (h1 < JFC_INF));
  // flow crossed face f only toward an item inside the grid (arcs leaving
  // the grid are zero)
  if (t < 6) {
    const int nb = s.face[t] ? face_item<DIMS, TY, TZ, SPLIT>(ts, tid, t) : -1;
    s.q_nb[t] = nb;
  }
  if (t == 0) s.active = active ? 1 : 0;
  __syncthreads();
  JFC_PCLK(ts.d_ctr, 3);
  return rounds;
}

// Persistent push-relabel phase: 2*sweeps alternating parity sweeps separated
// by grid barriers.  Sweep s of parity p drains queue q_pr[p][cur_pr[p]] one
// tile per CTA ticket; tiles still active go to q_pr[p][1-cur], neighbours
// that received flow to the other parity's pending buffer.
//
// Staging (ts.d_tmap set): tensor copies fill one of two staging buffers in
// dynamic shared memory.  While a visit runs, the CTA's next ticket is
// already being copied into the other buffer, as long as the sweep holds at
// least a grid's worth of tickets beyond the current one (in a short sweep
// a second ticket would only keep another CTA idle).  A prefetched item is
// safe to read early: items of one sweep are never adjacent, so nothing
// writes its tile or its halo heights until the sweep ends.
// CTAs per SM the phase is compiled for (its registers): the 2D 32 x 8 form
// JFC_PR2D_MINB, other 256-node tiles 3, 512-node tiles 2
#ifndef JFC_PR2D_MINB
#define JFC_PR2D_MINB 4
#endif
template <int DIMS, int TY, int TZ, bool SPLIT>
__global__ void __launch_bounds__(Tile<DIMS, TY, TZ>::NT,
                                  (DIMS == 2 && TY == 8) ? JFC_PR2D_MINB : Tile<DIMS, TY, TZ>::NT > 256 ? 2 : 3)
    k_pr_phase(TileSet ts, int sweeps, int local_iters) {
  using Stage = PrStage<DIMS, TY, TZ>;
  __shared__ PrSmem<DIMS, TY, TZ> sm;
  __shared__ uint64_t s_bar[2];
  extern __shared__ __align__(128) unsigned char s_dyn[];
  Stage* stage = reinterpret_cast<Stage*>(s_dyn + ((128u - (jfc::smem_addr(s_dyn) & 127u)) & 127u));
  DevCounters* ctr = ts.d_ctr;
  const bool tma = ts.d_tmap != nullptr;
  unsigned long long visits = 0, rounds = 0;
  const unsigned long long t0 = jfc::global_ns();
  const unsigned long long cap = jfc::spin_cap(ctr);
  if (tma && threadIdx.x == 0) {
    jfc::mbar_init(&s_bar[0], 1);
    jfc::mbar_init(&s_bar[1], 1);
    jfc::fence_mbar_init();
  }
  __syncthreads();
  unsigned parity = 0;      // bit b: phase parity of buffer b's next fill
  int acquired_grid = -1;   // thread 0: grid whose tensor maps it acquired
  int next_buf = 0;         // thread 0: buffer of the next fill
  int s = 0;
  const int npairs = sweeps > 0 ? sweeps : jfc::vload(&ctr->pr_sweeps);
  for (; s < 2 * npairs; ++s) {
    const int p = s & 1;
    const int b = jfc::vload(&ctr->cur_pr[p]);
    const int bo = jfc::vload(&ctr->cur_pr[p ^ 1]);
    const int n = jfc::vload(&ctr->qn_pr[p][b]);
    if (n == 0 && jfc::vload(&ctr->qn_pr[p ^ 1][bo]) == 0) break;  // nothing left anywhere
    const int* queue = ts.d_q_pr[p][b];
    // the previous sweep's writes (seen through the grid barrier) come before
    // this sweep's tensor reads
    if (tma && threadIdx.x == 0) jfc::fence_async_global();
    int pre = -1, pre_buf = 0;   // thread 0: the prefetched item and its buffer
    unsigned pre_k = 0;
    bool failed = false;
    for (;;) {
      if (threadIdx.x == 0) {
        int item, buf = 0;
        unsigned k;
        if (pre >= 0) {
          item = pre; buf = pre_buf; k = pre_k; pre = -1;
        } else {
          k = atomicAdd(&ctr->ticket[s & 1], 1u);
          item = (int)k < n ? queue[k] : -1;
          if (item >= 0) {
            ts.d_flag_pr[item] = 0;
            if (tma) {
              buf = next_buf; next_buf ^= 1;
              pr_stage_issue<DIMS, TY, TZ, SPLIT>(ts, item, stage[buf], &s_bar[buf], acquired_grid);
            }
          }
        }
        if (tma && item >= 0 && (long long)k + gridDim.x < n) {
          const unsigned k2 = atomicAdd(&ctr->ticket[s & 1], 1u);
          if ((int)k2 < n) {
            pre = queue[k2];
            pre_k = k2;
            ts.d_flag_pr[pre] = 0;
            pre_buf = next_buf; next_buf ^= 1;
            pr_stage_issue<DIMS, TY, TZ, SPLIT>(ts, pre, stage[pre_buf], &s_bar[pre_buf], acquired_grid);
          }
        }
        sm.tile = item;
        sm.buf = buf;
      }
      __syncthreads();
      const int tid = sm.tile, buf = sm.buf;
      if (tid < 0) break;
      if (tma) {
        const bool ok = jfc::mbar_wait(&s_bar[buf], (parity >> buf) & 1u, cap);
        parity ^= 1u << buf;
        if (__syncthreads_or(!ok)) {
          if (threadIdx.x == 0) {
            atomicExch(&ctr->error, 1);
            // copies still in flight land before the CTA leaves its shared
            // memory: bounded by a fixed poll count of its own, not by the
            // (possibly tiny) spin limit that gave up above
            constexpr unsigned long long kDrainPolls = 1ull << 26;
            jfc::mbar_wait(&s_bar[buf], ((parity >> buf) & 1u) ^ 1u, kDrainPolls);
            if (pre >= 0) jfc::mbar_wait(&s_bar[pre_buf], (parity >> pre_buf) & 1u, kDrainPolls);
          }
          failed = true;
          break;
        }
      }
      // first sweep of a phase: nothing moved since the exact global relabel
      // (the halo tiles have the other parity), so the local relabel would
      // reproduce the heights it finds
      rounds += pr_visit<DIMS, TY, TZ, SPLIT>(ts, tid, local_iters, s > 0, sm, stage[buf], tma);
      ++visits;
      // queue: myself for my parity's next sweep, neighbours for the other parity
      if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const int nb = lane < 6 ? sm.q_nb[lane] : -1;
        jfc::warp_append(nb >= 0, nb, ts.d_flag_pr, ts.d_q_pr[p ^ 1][bo], &ctr->qn_pr[p ^ 1][bo]);
        const bool active = sm.active != 0;
        if (active && lane == 0) ts.d_flag_pr[tid] = 1;
        jfc::warp_append(active && lane == 0, tid, nullptr, ts.d_q_pr[p][b ^ 1], &ctr->qn_pr[p][b ^ 1]);
      }
      __syncthreads();
    }
    if (failed) break;   // a staging copy never completed (error raised): leave
    JFC_PCLK_DECL
    const bool ok = jfc::grid_sync(ctr, [&]() {
      ctr->ticket[s & 1] = 0;
      ctr->qn_pr[p][b] = 0;
      ctr->cur_pr[p] = b ^ 1;
    });
    JFC_PCLK(ctr, 4);
    if (!ok) break;
  }
  if (threadIdx.x == 0) {
    if (visits) atomicAdd(&ctr->visits, visits);
    if (rounds) atomicAdd(&ctr->rounds, rounds);
    if (blockIdx.x == 0) {
      ctr->sweeps_done = s;
      ctr->ns_pr += jfc::global_ns() - t0;
    }
  }
}

// ---------------------------------------------------------------------------
// Asynchronous push-relabel phase: a worklist instead of parity sweeps.
//
// The sweeps keep adjacent work items apart by running one checkerboard
// colour at a time, with a grid barrier between colours; in the tail of a
// solve a sweep holds a few items and every CTA waits at the barrier for the
// slowest visit.  Here the items live in a ring (one entry per queued item:
// the queued flags dedupe), any free CTA takes the next entry, and adjacency
// is kept apart by per-item locks instead: a visit takes its item's lock,
// then (after a sequentially consistent fence) checks that no item behind
// its faces holds one; of two adjacent items that try at once at least one
// sees the other and backs off (the entry goes back to the ring).  So a visit
// sees exactly what it would see in a sweep: its item and halo untouched by
// any other visit while it runs.  An entry carries a generation that plays
// the role of the sweep index: a visit of generation k queues the items it
// fed for k + 1 (the other colour's next sweep) and itself for k + 2 (its own
// colour's next sweep), and a phase of `npairs` sweep pairs visits
// generations 0 .. 2 * npairs - 1 (the sweeps' budget); items past it stay
// active for the next global relabel.  The phase ends when
// no queued item is left (every wait is bounded, see jfc::spin_cap).
constexpr unsigned long long kRingEmpty = ~0ull;

__device__ __forceinline__ unsigned long long ring_entry(int item, int gen) {
  return ((unsigned long long)(unsigned)gen << 32) | (unsigned)item;
}

// Put one entry into the ring (a position reserved at the tail; the slot is
// free, or freed by its reader within a few polls).  Returns false after an
// error.
__device__ __forceinline__ bool pr_ring_put(unsigned long long* ring, unsigned cap, unsigned* tail, int* err,
                                            unsigned long long max_spins, unsigned long long v) {
  const unsigned pos = atomicAdd(tail, 1u);
  unsigned long long* slot = ring + pos % cap;
  unsigned long long spins = 0;
  while (atomicCAS(slot, kRingEmpty, v) != kRingEmpty) {
    if (++spins > max_spins || jfc::vload(err)) { atomicExch(err, 1); return false; }
    __nanosleep(32);
  }
  return true;
}

template <int DIMS, int TY, int TZ, bool SPLIT>
__global__ void __launch_bounds__(Tile<DIMS, TY, TZ>::NT)
    k_pr_async(TileSet ts, int sweeps, int local_iters) {
  __shared__ PrSmem<DIMS, TY, TZ> sm;
  extern __shared__ __align__(128) unsigned char s_dyn[];
  PrStage<DIMS, TY, TZ>& stage =
      *reinterpret_cast<PrStage<DIMS, TY, TZ>*>(s_dyn + ((128u - (jfc::smem_addr(s_dyn) & 127u)) & 127u));
  DevCounters* ctr = ts.d_ctr;
  const unsigned long long t0 = jfc::global_ns();
  const int npairs = sweeps > 0 ? sweeps : jfc::vload(&ctr->pr_sweeps);
  const int gens = 2 * npairs;
  const unsigned cap = (unsigned)(SPLIT ? 2 * ts.ntiles : ts.ntiles);
  unsigned long long* ring = ts.d_pr_ring;
  int* lock = ts.d_pr_lock;
  // ---- the ring starts with the items the global relabel queued (both
  //      parity queues, colour 0 first: the first wave of takers is
  //      conflict-free), generation 0; locks clear
  const int b0 = jfc::vload(&ctr->cur_pr[0]), b1 = jfc::vload(&ctr->cur_pr[1]);
  const int n0 = jfc::vload(&ctr->qn_pr[0][b0]), n1 = jfc::vload(&ctr->qn_pr[1][b1]);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap; i += (long long)gridDim.x * blockDim.x) {
    unsigned long long v = kRingEmpty;
    if (i < n0) v = ring_entry(ts.d_q_pr[0][b0][i], 0);
    else if (i < n0 + n1) v = ring_entry(ts.d_q_pr[1][b1][i - n0], 0);
    ring[i] = v;
    lock[i] = 0;
  }
  const bool ok = jfc::grid_sync(ctr, [&]() {
    ctr->pr_head = 0;
    ctr->pr_tail = (unsigned)(n0 + n1);
    ctr->pr_out = n0 + n1;
    ctr->sweeps_done = 0;
  });
  const unsigned long long max_spins = jfc::spin_cap(ctr);
  unsigned long long visits = 0, rounds = 0;
  int maxgen = -1;
  while (ok) {
    if (threadIdx.x == 0) {
      int item = -1, gen = 0;
      const unsigned k = atomicAdd(&ctr->pr_head, 1u);
      unsigned long long* slot = ring + k % cap;
      // bounded: the entry arrives, or no item is left, or an error; the
      // count restarts whenever the worklist moves
      unsigned long long spins = 0, v = kRingEmpty;
      unsigned seen_tail = (unsigned)jfc::vload((const int*)&ctr->pr_tail);
      int seen_out = jfc::vload(&ctr->pr_out);
      for (;;) {
        if (*(volatile unsigned long long*)slot != kRingEmpty) {
          v = atomicExch(slot, kRingEmpty);
          if (v != kRingEmpty) break;
        }
        const int out = jfc::vload(&ctr->pr_out);
        if (out == 0 || jfc::vload(&ctr->error)) break;
        const unsigned tl = (unsigned)jfc::vload((const int*)&ctr->pr_tail);
        if (out != seen_out || tl != seen_tail) {
          seen_out = out;
          seen_tail = tl;
          spins = 0;
        } else if (++spins > max_spins) {
          atomicExch(&ctr->error, 1);
          break;
        }
        __nanosleep(32);
      }
      if (v != kRingEmpty) {
        item = (int)(unsigned)(v & 0xffffffffu);
        gen = (int)(v >> 32);
        // neighbour exclusion (see above)
        bool conflict = atomicCAS(lock + item, 0, 1) != 0;
        if (!conflict) {
          asm volatile("fence.sc.gpu;" ::: "memory");
#pragma unroll
          for (int f = 0; f < (DIMS == 3 ? 6 : 4); ++f) {
            const int nb = face_item<DIMS, TY, TZ, SPLIT>(ts, item, f);
            if (nb >= 0 && jfc::vload(lock + nb) != 0) conflict = true;
          }
          if (conflict) atomicExch(lock + item, 0);
        }
        if (conflict) {
          // back to the ring, same generation, still flagged as queued (it
          // stays outstanding); -2: take the next entry
          if (!pr_ring_put(ring, cap, &ctr->pr_tail, &ctr->error, max_spins, v)) item = -1;
          else item = -2;
        } else {
          ts.d_flag_pr[item] = 0;   // dequeued: a neighbour may queue it again once we unlock
          __threadfence();
        }
      }
      sm.tile = item;
      sm.gen = gen;
    }
    __syncthreads();
    const int item = sm.tile, gen = sm.gen;
    if (item == -1) break;
    if (item == -2) {
      __syncthreads();   // sm.tile is rewritten only after every thread read it
      continue;
    }
    // generation 0: nothing around the item moved since the exact global
    // relabel unless a neighbour was visited first; the local relabel is an
    // improvement only, so skipping it is safe either way
    rounds += pr_visit<DIMS, TY, TZ, SPLIT>(ts, item, local_iters, gen > 0, sm, stage, false);
    ++visits;
    maxgen = max(maxgen, gen);
    // release the item (its writes visible first), then queue what it fed
    // and itself for generation gen + 1, then count it done
    if (threadIdx.x == 0) {
      __threadfence();
      atomicExch(lock + item, 0);
    }
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      int nb = -1, ng = gen + 1;
      if (lane < 6) nb = sm.q_nb[lane];
      else if (lane == 6 && sm.active) { nb = item; ng = gen + 2; }
      bool won = false;
      if (ng < gens && nb >= 0) won = atomicExch(ts.d_flag_pr + nb, 1) == 0;
      const unsigned m = __ballot_sync(jfc::FULL, won);
      if (m && lane == 0) atomicAdd(&ctr->pr_out, __popc(m));   // counted before they can finish
      // (a failed put raises the error flag; the next dequeue sees it and
      // every thread of the CTA leaves the loop together)
      if (won) pr_ring_put(ring, cap, &ctr->pr_tail, &ctr->error, max_spins, ring_entry(nb, ng));
      __syncwarp();
      if (lane == 0) atomicSub(&ctr->pr_out, 1);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (visits) atomicAdd(&ctr->visits, visits);
    if (rounds) atomicAdd(&ctr->rounds, rounds);
    // "sweeps" of the phase: generations reached (the engine's schedule reads it)
    atomicMax(&ctr->sweeps_done, maxgen + 1);
  }
  // the phase clock: the last CTA to leave adds the elapsed time
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&ctr->bar_count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_last) {
    ctr->bar_count = 0;
    ctr->ns_pr += jfc::global_ns() - t0;
  }
}

template <int DIMS, int TY, int TZ, bool SPLIT = false>
cudaError_t launch_t(const TileSet& ts, int sweeps, int local_iters, cudaStream_t st, int sched) {
  constexpr int NT = Tile<DIMS, TY, TZ>::NT;
  const bool async = sched == 2 && ts.d_pr_ring != nullptr;
  const void* fn = async ? (const void*)k_pr_async<DIMS, TY, TZ, SPLIT> : (const void*)k_pr_phase<DIMS, TY, TZ, SPLIT>;
  // staging buffers in dynamic shared memory: two for the sweeps (one being
  // visited, one being filled), one for the worklist; + 128 B to align them
  const size_t dyn = sizeof(PrStage<DIMS, TY, TZ>) * (async ? 1 : 2) + 128;
  static int cache_sweeps[64] = {0}, cache_async[64] = {0};
  // without this opt-in a kernel's dynamic shared memory is limited to 48 KB
  // minus its static shared memory
  {
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
  }
  const int blocks = persistent_blocks_cached(async ? cache_async : cache_sweeps, fn, NT, dyn);
  TileSet arg = ts;
  void* params[] = {(void*)&arg, (void*)&sweeps, (void*)&local_iters};
  jfc_note_launch();
  return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(NT), params, dyn, st);
}

// Local pre-push before the first relabel of a solve, one CTA per tile, the
// tile in shared memory: along one arc slot at a time, every node with excess
// pushes to its in-tile neighbour across that slot when the neighbour is a
// deficit, at most the arc's residual and the deficit.  Along one slot a node
// either sends (e > 0) or receives (e < 0, from its one neighbour on the other
// side), so each step is race-free; JFC_PREPUSH_ROUNDS rounds over all slots.
// These are ordinary preflow pushes (the exact relabel that follows gives
// valid heights), so the maximum flow and the canonical cut do not change;
// most of the excess that meets a deficit a step or two away cancels here, in
// one read and one write of the tile, instead of in push-relabel visits.
#ifndef JFC_PREPUSH_ROUNDS
#define JFC_PREPUSH_ROUNDS 2
#endif
template <int DIMS, int TY, int TZ>
__global__ void __launch_bounds__(Tile<DIMS, TY, TZ>::NT) k_prepush(TileSet ts) {
  using T = Tile<DIMS, TY, TZ>;
  __shared__ int se[T::NT];
  __shared__ int sr[T::K][T::NT];
  const int t = threadIdx.x;
  const int x = t & 31, row = t >> 5, y = row % TY, z = row / TY;
  const int4 ti = ts.d_info[blockIdx.x];
  const GridDev& g = ts.d_desc[ti.x];
  const long long pitch = g.pitch, slab = (long long)g.pitch * g.Hp;
  const long long n = (long long)ti.y * 32 + x + ((long long)ti.z * TY + y) * pitch + ((long long)ti.w * TZ + z) * slab;
  const int e0 = g.e[n];
  int r0[T::K];
#pragma unroll
  for (int k = 0; k < T::K; ++k) r0[k] = g.r[k][n];
  // nothing to do unless the tile holds both excess and a deficit
  const bool pos = __syncthreads_or(e0 > 0);
  const bool neg = __syncthreads_or(e0 < 0);
  if (!pos || !neg) return;
  se[t] = e0;
#pragma unroll
  for (int k = 0; k < T::K; ++k) sr[k][t] = r0[k];
  __syncthreads();
  for (int rnd = 0; rnd < JFC_PREPUSH_ROUNDS; ++rnd) {
#pragma unroll
    for (int k = 0; k < T::K; ++k) {
      const bool inside = k == T::XP ? x < 31 : k == T::XM ? x > 0 : k == T::YP ? y < TY - 1
                        : k == T::YM ? y > 0 : k == T::ZP ? z < TZ - 1 : z > 0;
      const int off = k == T::XP ? 1 : k == T::XM ? -1 : k == T::YP ? 32 : k == T::YM ? -32
                    : k == T::ZP ? 32 * TY : -32 * TY;
      const int e = se[t];
      if (inside && e > 0) {
        const int r = sr[k][t], ev = se[t + off];
        if (r > 0 && ev < 0) {
          const int d = min(min(e, r), -ev);
          se[t] = e - d;
          sr[k][t] = r - d;
          se[t + off] = ev + d;
          sr[T::K - 1 - k][t + off] += d;
        }
      }
      __syncthreads();
    }
  }
  const int e1 = se[t];
  if (e1 != e0) g.e[n] = e1;
#pragma unroll
  for (int k = 0; k < T::K; ++k) {
    const int v = sr[k][t];
    if (v != r0[k]) g.r[k][n] = v;
  }
}

template <int DIMS, int TY, int TZ>
cudaError_t prepush_t(const TileSet& ts, cudaStream_t st) {
  jfc_note_launch();
  k_prepush<DIMS, TY, TZ><<<(unsigned)ts.ntiles, Tile<DIMS, TY, TZ>::NT, 0, st>>>(ts);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_prepush(const TileSet& ts, cudaStream_t s) {
  if (ts.ntiles <= 0) return cudaSuccess;
  if (ts.dims == 2) return ts.TR == 8 ? prepush_t<2, 8, 1>(ts, s) : prepush_t<2, 16, 1>(ts, s);
  if (ts.TY == 4 && ts.TZ == 4) return prepush_t<3, 4, 4>(ts, s);
  if (ts.TY == 4 && ts.TZ == 2) return prepush_t<3, 4, 2>(ts, s);
  if (ts.TY == 16 && ts.TZ == 1) return prepush_t<3, 16, 1>(ts, s);
  if (ts.TY == 8 && ts.TZ == 2) return prepush_t<3, 8, 2>(ts, s);
  if (ts.TY == 8 && ts.TZ == 1) return prepush_t<3, 8, 1>(ts, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_pr_phase(const TileSet& ts, int sweeps, int local_iters, cudaStream_t s, int sched) {
  if (ts.dims == 2) {
    if (ts.pr_split && ts.TR == 16) return launch_t<2, 8, 1, true>(ts, sweeps, local_iters, s, sched);
    switch (ts.TR) {
      case 8: return launch_t<2, 8, 1>(ts, sweeps, local_iters, s, sched);
      case 16: return launch_t<2, 16, 1>(ts, sweeps, local_iters, s, sched);
      default: return cudaErrorInvalidValue;
    }
  }
  if (ts.TY == 4 && ts.TZ == 4) return launch_t<3, 4, 4>(ts, sweeps, local_iters, s, sched);
  if (ts.TY == 4 && ts.TZ == 2) return launch_t<3, 4, 2>(ts, sweeps, local_iters, s, sched);
  if (ts.TY == 16 && ts.TZ == 1) return launch_t<3, 16, 1>(ts, sweeps, local_iters, s, sched);
  if (ts.TY == 8 && ts.TZ == 2) return launch_t<3, 8, 2>(ts, sweeps, local_iters, s, sched);
  if (ts.TY == 8 && ts.TZ == 1) return launch_t<3, 8, 1>(ts, sweeps, local_iters, s, sched);
  return cudaErrorInvalidValue;
}
