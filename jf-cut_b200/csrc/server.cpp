// server.cpp — serving: continuous batching of interactive graph-cut sessions
// with HBM-budget admission and warm stroke edits.
//
// No reference counterpart: JF-Cut re-models and re-solves one volume per
// user action on the GUI thread (QGCWidget::slotModelClicked / slotCutClicked,
// QGCWidget.cpp:2560, 2364).  Here each session keeps its residual graph,
// excess and heights resident on the device; a stroke edit only re-derives
// the t-links of the edited nodes (e += delta(cs - ct)) and re-solves warm
// from the previous preflow.
//
// Two host threads:
//   builder — admits cold sessions in FIFO order while their device bytes fit
//             the HBM budget, allocates their state and runs the capacity
//             build on its own stream (overlapping the solver's kernels);
//   solver  — the continuous-batching loop.  The solving set is one tile set
//             per dimensionality over the grids of every admitted request, so
//             each push-relabel phase and each global relabel is one
//             persistent launch over all of them.  Membership changes only
//             between a push-relabel phase and the global relabel that
//             follows it (the relabel rebuilds every work queue, so tiles can
//             be renumbered there):
//               loop { push-relabel phase over the set (if any tile active)
//                      leave: finished / cancelled members; join: requests
//                      waiting for a slot (edits applied now)
//                      global relabel over the set -> active tiles per grid
//                      grids with no active tile: cut BFS -> result }
// A request's arithmetic is the plain solver's: the same kernels on the same
// grid, and the max-flow / canonical cut do not depend on what else shares
// the launches (tests check alone vs in the mix).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
  bool cold = true;                 // a new session (build + solve) or a stroke edit
  std::vector<uint32_t> idx;
  std::vector<uint8_t> seed;
  Clock::time_point t_submit, t_admit;
};

enum Phase { WAIT_BUILD, BUILDING, READY, SOLVING, IDLE, DEAD };

struct Session {
  int sid = -1;
  int dims = 2, w = 0, h = 0, d = 1, pixfmt = 0;
  jfc_model model{};
  std::vector<uint8_t> img, seeds;  // host copies until the cold build
  jfc_graph* G = nullptr;
  size_t charge = 0;                // bytes the session needs on the device
  size_t held = 0;                  // bytes held against the budget (after admission)
  Phase phase = WAIT_BUILD;
  std::deque<Request> reqs;         // front = the request being served
  jfc_request_info last{};
  bool has_last = false;
  long long sweeps = 0;             // sweeps of the current request
  bool cancel = false, close = false;
  int lane_refs = 0;                // lane entries that hold this session (joining, solving, or
                                    // done but not yet removed; a finished session can be
                                    // re-admitted before its old entry leaves).  Guarded by mu; a
                                    // closed session is freed only once none is left
};

}  // namespace

struct jfc_server {
  int device = 0;
  jfc_params params{};
  jfc_ctx* solve_ctx = nullptr;
  jfc_ctx* build_ctx = nullptr;
  cudaStream_t read_stream = nullptr;
  cudaStream_t solve_stream = nullptr;   // the solver context's stream (highest priority)
  Clock::time_point t0 = Clock::now();   // (verbose logs) server start
  cudaMemPool_t pool = nullptr;          // the device's default pool (graph memory)
  unsigned long long pool_threshold0 = 0;   // its release threshold before the server
  std::mutex read_mu;
  size_t budget = 0, used = 0;
  int max_slots = 64;

  std::mutex mu;
  std::condition_variable cv_build, cv_work, cv_done;
  std::map<int, std::unique_ptr<Session>> sessions;
  int next_sid = 0;
  std::deque<int> build_q;          // sessions waiting for admission + cold build
  std::deque<int> ready_q;          // sessions with a request waiting for a slot
  std::vector<Session*> to_free;    // closed sessions whose device state the solver frees
  bool stop = false;
  std::thread builder, solver;
  int fatal = JFC_OK;               // a device error stops the server
  size_t peak_used = 0;
  int solving = 0, peak_solving = 0;
  long long loops = 0, requests_done = 0;

  TileSet cut_ts[2];                // converged grids of a cycle, [0] 2D, [1] 3D
};

namespace {

size_t session_bytes(int dims, int w, int h, int d, int pixfmt, size_t nseeds) {
  const size_t n = (size_t)w * h * d;
  const size_t nlut = pixfmt == JFC_PIX_RGB8 ? 3 * 255 * 255 + 1 : (pixfmt == JFC_PIX_I16 ? 65536 : 256);
  return state_bytes(dims, w, h, d) + align256(n * jfc_pix_bytes(pixfmt)) + align256(n) +
         2 * align256(sizeof(int) * (JFC_TQ + 1)) +
         // capacity-build temporaries: seed lists, n-link tables, scratch
         align256(4 * nseeds) + 2 * align256(sizeof(int) * nlut) + 4096;
}

// Finish the front request of a session (lock held).
void finish_front(jfc_server* S, Session* s, int status, long long flow, Clock::time_point now) {
  if (s->reqs.empty()) return;
  Request& r = s->reqs.front();
  jfc_request_info& in = s->last;
  in.status = status;
  in.flow = flow;
  const Clock::time_point admit = r.t_admit == Clock::time_point() ? now : r.t_admit;
  in.ms_queue = ms_between(r.t_submit, admit);
  in.ms_solve = ms_between(admit, now);
  in.ms_total = ms_between(r.t_submit, now);
  in.warm = r.cold ? 0 : 1;
  s->has_last = true;
  s->reqs.pop_front();
  ++S->requests_done;
  s->sweeps = 0;
}

// Finish every queued request of a session as cancelled (lock held).
void cancel_all(jfc_server* S, Session* s, Clock::time_point now) {
  while (!s->reqs.empty()) finish_front(S, s, JFC_ERR_CANCELLED, 0, now);
}

// Release a session's device state and budget (solver thread; no tile set
// references its grid any more).  Label reads hold read_mu while they copy.
// Called by the solver thread only, for a session in no tile set: its last
// kernels ran on the solver stream (before a read-back the thread waited
// for), its build finished on the builder stream before it was handed over,
// and read_mu keeps label reads out, so the release is ordered on the solver
// stream and synchronises nothing else (a device-wide wait here would stall
// the solver for the builder's work in flight).
void free_session(jfc_server* S, Session* s) {
  std::lock_guard<std::mutex> rl(S->read_mu);
  if (s->G) {
    graph_release(s->G, S->solve_ctx->stream);
    s->G = nullptr;
  }
  std::lock_guard<std::mutex> lk(S->mu);
  S->used -= s->held;
  s->held = 0;
  S->cv_build.notify_all();
}

void builder_loop(jfc_server* S) {
  cudaSetDevice(S->device);
  for (;;) {
    Session* s = nullptr;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_build.wait(lk, [&] {
        if (S->stop) return true;
        if (S->build_q.empty()) return false;
        const Session* f = S->sessions.at(S->build_q.front()).get();
        return S->used + f->charge <= S->budget;
      });
      if (S->stop) return;
      s = S->sessions.at(S->build_q.front()).get();
      S->build_q.pop_front();
      S->used += s->charge;
      S->peak_used = std::max(S->peak_used, S->used);
      s->held = s->charge;
      s->phase = BUILDING;
      s->reqs.front().t_admit = Clock::now();
    }
    jfc_graph* G = nullptr;
    const Clock::time_point tb = Clock::now();
    int rc = jfc_graph_create_grid(S->build_ctx, s->dims, s->w, s->h, s->d, s->dims == 2 ? 4 : 6, &G);
    if (rc == JFC_OK) rc = build_core(G, s->img.data(), s->pixfmt, s->seeds.data(), &s->model, cudaMemcpyHostToDevice);
    if (S->params.verbose) {
      const Clock::time_point te = Clock::now();
      auto ms = [](Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
      fprintf(stderr, "{\"build\": %d, \"nodes\": %lld, \"ms\": %.3f, \"t_end_ms\": %.1f}\n", s->sid,
              (long long)s->w * s->h * s->d, ms(tb, te), ms(S->t0, te));
    }
    std::unique_lock<std::mutex> lk(S->mu);
    s->G = G;
    std::vector<uint8_t>().swap(s->img);
    std::vector<uint8_t>().swap(s->seeds);
    if (G) G->ctx = S->solve_ctx;   // later launches on this graph come from the solver
    if (rc != JFC_OK || s->cancel) {
      const Clock::time_point now = Clock::now();
      if (rc != JFC_OK) finish_front(S, s, rc, 0, now);
      cancel_all(S, s, now);
      s->phase = G && rc == JFC_OK ? IDLE : DEAD;
      if (s->close) S->to_free.push_back(s);
      S->cv_done.notify_all();
      S->cv_work.notify_all();
      continue;
    }
    s->phase = READY;
    S->ready_q.push_back(s->sid);
    S->cv_work.notify_all();
  }
}

struct Member {
  Session* s;
  bool done = false;      // result delivered; leaves at the next membership change
};

// A solving set: one tile set per dimensionality over its members' grids.
// The server runs two: interactive (warm stroke edits) and bulk (cold
// requests); the interactive lane gets its cycles first, so an edit does not
// wait behind the relabels of large cold solves.
struct Lane {
  std::vector<Member> mem[2];       // members of ts[0] / ts[1], in grid order
  std::vector<int> active[2];       // active tiles per grid after the last relabel
  TileSet ts[2];
  int interval = 4;
  std::vector<Session*> joining;    // admitted requests, join at the next relabel
  std::vector<Session*> freeing;    // closed members, freed once ts[] no longer holds them
  bool empty() const { return mem[0].empty() && mem[1].empty() && joining.empty(); }
  long long active_tiles() const {
    long long a = 0;
    for (int k = 0; k < 2; ++k)
      for (size_t i = 0; i < mem[k].size(); ++i)
        if (!mem[k][i].done) a += active[k][i];
    return a;
  }
};

// Finish every request of the lane's members with a device error.
void fail_lane(jfc_server* S, Lane& L, int rc) {
  std::lock_guard<std::mutex> lk(S->mu);
  S->fatal = rc;
  const Clock::time_point now = Clock::now();
  for (int k = 0; k < 2; ++k)
    for (Member& m : L.mem[k]) {
      if (!m.done) finish_front(S, m.s, rc, 0, now);
      cancel_all(S, m.s, now);
      m.s->phase = IDLE;
    }
  S->cv_done.notify_all();
}

// One relabel cycle of a lane: push-relabel phase over its members, then
// membership (leave / join), then one global relabel over the re-formed set,
// then the cut of every converged grid.  Returns a status (device errors).
int lane_cycle(jfc_server* S, Lane& L, int lane_id, int max_interval = 1 << 30) {
  jfc_ctx* ctx = S->solve_ctx;
  const jfc_params& p = S->params;
  const Clock::time_point t_start = Clock::now();
  Clock::time_point t_form = t_start, t_relabel = t_start;   // host-side phase ends (verbose)
  // 1. push-relabel phase over the current members
  bool ran_pr[2] = {false, false};
  for (int k = 0; k < 2; ++k) {
    long long a = 0;
    for (size_t i = 0; i < L.mem[k].size(); ++i)
      if (!L.mem[k][i].done) a += L.active[k][i];
    if (a == 0) continue;
    cudaMemsetAsync(L.ts[k].d_ctr->ticket, 0, sizeof(L.ts[k].d_ctr->ticket), ctx->stream);
    const cudaError_t e = launch_pr_phase(L.ts[k], std::min(L.interval, max_interval), p.local_iters, ctx->stream);
    if (e != cudaSuccess) return cuda_status(e, "push-relabel phase");
    ran_pr[k] = true;
  }
  // 2. membership: done / cancelled members leave, admitted requests join
  bool changed[2] = {false, false};
  {
    std::lock_guard<std::mutex> lk(S->mu);
    const Clock::time_point now = Clock::now();
    for (int k = 0; k < 2; ++k) {
      std::vector<Member> keep;
      std::vector<int> keep_act;
      for (size_t i = 0; i < L.mem[k].size(); ++i) {
        Member& m = L.mem[k][i];
        if (!m.done && m.s->cancel) {
          cancel_all(S, m.s, now);
          m.s->phase = IDLE;
          m.done = true;
          S->cv_done.notify_all();
        }
        if (m.done) {
          changed[k] = true;
          if (--m.s->lane_refs == 0 && m.s->close) L.freeing.push_back(m.s);
          continue;
        }
        keep.push_back(m);
        keep_act.push_back(L.active[k][i]);
      }
      L.mem[k].swap(keep);
      L.active[k].swap(keep_act);
    }
  }
  for (Session* s : L.joining) {
    const int k = s->dims == 3 ? 1 : 0;
    L.mem[k].push_back(Member{s});
    L.active[k].push_back(0);
    changed[k] = true;
  }
  L.joining.clear();
  // 3. global relabel over the (re-formed) set
  double ms_build = 0.0, ms_bfs = 0.0;   // (verbose) tile-set builds; phase + relabel to its read-back
  for (int k = 0; k < 2; ++k) {
    if (k == 0) t_form = Clock::now();
    const Clock::time_point t_k = Clock::now();
    if (L.mem[k].empty()) {
      L.active[k].clear();
      continue;
    }
    if (changed[k]) {
      std::vector<GridDev> grids;
      for (Member& m : L.mem[k]) grids.push_back(m.s->G->g);
      int rc = tileset_build(L.ts[k], k ? 3 : 2, p.tile_rows, p.tile_depth, grids, ctx->stream,
                             pr_split_for(p, k ? 3 : 2));
      if (rc) return rc;
    }
    const Clock::time_point t_built = Clock::now();
    int passes = 0, sw = 0;
    int rc = engine_bfs(ctx, L.ts[k], p, false, passes, &L.active[k], nullptr, &sw);
    if (rc) return rc;
    ms_build += std::chrono::duration<double, std::milli>(t_built - t_k).count();
    ms_bfs += std::chrono::duration<double, std::milli>(Clock::now() - t_built).count();
    if (ran_pr[k])
      for (Member& m : L.mem[k]) m.s->sweeps += sw;
  }
  // closed members are no longer in any tile set of this lane (rebuilt above,
  // or the lane is empty and launches nothing): free their device state
  for (Session* s : L.freeing) {
    free_session(S, s);
    std::lock_guard<std::mutex> lk(S->mu);
    S->sessions.erase(s->sid);
  }
  L.freeing.clear();
  t_relabel = Clock::now();
  // 4. converged grids: cut BFS on a tile set of those grids alone
  long long still = 0;
  for (int k = 0; k < 2; ++k) {
    std::vector<size_t> conv;
    for (size_t i = 0; i < L.mem[k].size(); ++i) {
      GridDev& gd = L.mem[k][i].s->G->g;
      if (L.active[k][i] == 0 && gd.h_cap > 0) {
        // no active tile under the cap: the grid's next relabel is exact and
        // decides (excess farther than the cap keeps it solving)
        gd.h_cap = 0;
        const cudaError_t e = cudaMemsetAsync(&L.ts[k].d_desc[i].h_cap, 0, sizeof(int), ctx->stream);
        if (e != cudaSuccess) return cuda_status(e, "relabel cap");
        continue;
      }
      if (L.active[k][i] == 0) conv.push_back(i);
      else if (L.mem[k][i].s->sweeps >= p.max_sweeps) conv.push_back(i);
      else still += L.active[k][i];
    }
    if (conv.empty()) continue;
    std::vector<GridDev> grids;
    for (size_t i : conv) grids.push_back(L.mem[k][i].s->G->g);
    int rc = tileset_build(S->cut_ts[k], k ? 3 : 2, p.tile_rows, p.tile_depth, grids, ctx->stream);
    if (rc) return rc;
    std::vector<GridResult> res;
    int passes = 0;
    rc = engine_cut(ctx, S->cut_ts[k], p, res, passes);
    if (rc && rc != JFC_ERR_NOT_CONVERGED) return rc;
    std::lock_guard<std::mutex> lk(S->mu);
    const Clock::time_point now = Clock::now();
    for (size_t j = 0; j < conv.size(); ++j) {
      Member& m = L.mem[k][conv[j]];
      Session* s = m.s;
      jfc_graph* G = s->G;
      int st = res[j].status;
      if (L.active[k][conv[j]] > 0) st = JFC_ERR_NOT_CONVERGED;
      G->flow = G->sink_total + res[j].neg_sum;
      G->source_nodes = res[j].labels;
      G->state = st == JFC_OK ? 2 : 1;
      finish_front(S, s, st, G->flow, now);
      m.done = true;
      if (s->cancel) cancel_all(S, s, now);
      if (!s->reqs.empty() && !s->close) {
        s->phase = READY;
        S->ready_q.push_back(s->sid);
      } else {
        s->phase = IDLE;
      }
    }
    S->cv_done.notify_all();
  }
  // adaptive interval as in the plain solve: a sliver of active tiles makes
  // the dense relabel dominate, so relabel less often
  const long long nt = (long long)L.ts[0].ntiles * (L.mem[0].empty() ? 0 : 1) +
                       (long long)L.ts[1].ntiles * (L.mem[1].empty() ? 0 : 1);
  if (p.verbose) {
    const Clock::time_point t_end = Clock::now();
    auto ms = [](Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    fprintf(stderr, "{\"lane\": \"%s\", \"members\": %zu, \"active_tiles\": %lld, \"tiles\": %lld, \"interval\": %d, "
                    "\"ms_phase_membership\": %.3f, \"ms_form_relabel\": %.3f, \"ms_build\": %.3f, \"ms_bfs\": %.3f, "
                    "\"ms_cut\": %.3f, \"t_end_ms\": %.1f}\n",
            lane_id == 0 ? "interactive" : lane_id == 1 ? "interactive-large" : "bulk",
            L.mem[0].size() + L.mem[1].size(), still, nt, L.interval,
            ms(t_start, t_form), ms(t_form, t_relabel), ms_build, ms_bfs, ms(t_relabel, t_end), ms(S->t0, t_end));
  }
  if (still > 0 && still * 256 < nt) L.interval = std::min(L.interval * 2, p.relabel_interval_max);
  else L.interval = interval_for(p, 2);
  return JFC_OK;
}

void solver_loop(jfc_server* S) {
  cudaSetDevice(S->device);
  const jfc_params& p = S->params;
  // [0] interactive: warm edits of 2D grids up to 4096^2 nodes; [1] interactive
  // large: warm edits of volumes and larger images (their relabels take tens
  // of milliseconds, which an edit of a small image should not wait for);
  // [2] bulk: cold requests
  Lane lanes[3];
  constexpr int kSmall = 0, kLarge = 1, kBulk = 2;
  for (Lane& L : lanes) L.interval = interval_for(p, 2);
  constexpr long long kSmallEditNodes = 4096ll * 4096ll;
  constexpr int kLargeEvery = 4;            // one large-edit cycle per this many small-edit cycles
  constexpr int kInteractiveCycles = 16;   // interactive cycles per bulk cycle, at most
  // The bulk lane's size bounds how long one bulk cycle (a push-relabel phase
  // and a relabel over every member) keeps a warm edit waiting: cold requests
  // join while the lane holds fewer nodes than this (always at least one),
  // and its push-relabel phases run at most kBulkPairsBusy sweep pairs while
  // the interactive lane has work.
  constexpr long long kBulkNodes = 1ll << 28;
  constexpr int kBulkPairsBusy = 2;
  auto nodes_of = [](const Session* s) { return (long long)s->w * s->h * s->d; };
  // admission: requests waiting for a slot join their lane at its next
  // relabel.  Runs at the top of every round and again between interactive
  // cycles (an edit that arrives during a round does not wait for the round
  // to end); `idle_wait` blocks while every lane is empty.  Returns false
  // when the server stops.
  auto admit = [&](bool idle_wait) -> bool {
    std::vector<Session*> admitted, frees;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (idle_wait && lanes[0].empty() && lanes[1].empty() && lanes[2].empty())
        S->cv_work.wait(lk, [&] { return S->stop || !S->ready_q.empty() || !S->to_free.empty(); });
      if (S->stop) return false;
      if (!idle_wait && S->ready_q.empty() && S->to_free.empty()) return true;
      const Clock::time_point now = Clock::now();
      frees.swap(S->to_free);   // idle sessions: in no lane
      int members = 0;
      for (Lane& L : lanes) members += (int)(L.mem[0].size() + L.mem[1].size() + L.joining.size());
      int slots = S->max_slots - members;
      // a quarter of the slots stays free for edits: cold requests take at
      // most the rest, so a warm edit never waits for a bulk solve to finish
      // before it is admitted
      const int bulk_slots = std::max(1, S->max_slots - std::max(1, S->max_slots / 4));
      int bulk_members = (int)lanes[kBulk].joining.size();
      for (int k = 0; k < 2; ++k)
        for (const Member& m : lanes[kBulk].mem[k])
          if (!m.done) ++bulk_members;
      long long bulk_nodes = 0;
      for (int k = 0; k < 2; ++k)
        for (const Member& m : lanes[kBulk].mem[k])
          if (!m.done) bulk_nodes += nodes_of(m.s);
      for (const Session* s : lanes[kBulk].joining) bulk_nodes += nodes_of(s);
      // in queue order; a cold request that would overfill the bulk lane
      // keeps its place (and the cold ones behind it theirs), edits go ahead
      std::deque<int> keep;
      bool bulk_full = false;
      while (slots > 0 && !S->ready_q.empty()) {
        Session* s = S->sessions.at(S->ready_q.front()).get();
        const int sid = S->ready_q.front();
        S->ready_q.pop_front();
        const bool cold = !s->reqs.empty() && s->reqs.front().cold && !s->cancel;
        if (cold && (bulk_full || bulk_members >= bulk_slots ||
                     (bulk_nodes > 0 && bulk_nodes + nodes_of(s) > kBulkNodes))) {
          bulk_full = true;
          keep.push_back(sid);
          continue;
        }
        if (cold) {
          bulk_nodes += nodes_of(s);
          ++bulk_members;
        }
        if (s->cancel || s->reqs.empty()) {
          cancel_all(S, s, now);
          s->phase = IDLE;
          if (s->close && s->lane_refs == 0) frees.push_back(s);   // else its lane frees it
          S->cv_done.notify_all();
          continue;
        }
        s->phase = SOLVING;
        ++s->lane_refs;
        if (!s->reqs.front().cold) s->reqs.front().t_admit = now;
        admitted.push_back(s);
        --slots;
      }
      while (!keep.empty()) {   // back to the front, in order
        S->ready_q.push_front(keep.back());
        keep.pop_back();
      }
      if (idle_wait) ++S->loops;
    }
    for (Session* s : frees) {
      free_session(S, s);
      std::lock_guard<std::mutex> lk(S->mu);
      S->sessions.erase(s->sid);
    }
    if (!admitted.empty()) {
      // a label read in progress finishes before an edit changes a graph
      std::lock_guard<std::mutex> rl(S->read_mu);
      for (Session* s : admitted) {
        Request& r = s->reqs.front();
        int rc = JFC_OK;
        if (!r.cold) rc = jfc_graph_edit_seeds(s->G, r.idx.data(), r.seed.data(), r.idx.size());
        if (rc != JFC_OK) {
          std::lock_guard<std::mutex> lk(S->mu);
          --s->lane_refs;   // admitted, but it joins no lane
          finish_front(S, s, rc, 0, Clock::now());
          s->phase = s->reqs.empty() ? IDLE : READY;
          if (!s->reqs.empty()) S->ready_q.push_back(s->sid);
          else if (s->close && s->lane_refs == 0) S->to_free.push_back(s);   // closed meanwhile
          S->cv_done.notify_all();
          continue;
        }
        // capped relabels while the request solves (the plain solve's
        // schedule); dropped for the grid once it has no active tile left
        s->G->g.h_cap = relabel_cap_for(S->params, s->dims);
        const bool small = s->dims == 2 && nodes_of(s) <= kSmallEditNodes;
        lanes[r.cold ? kBulk : small ? kSmall : kLarge].joining.push_back(s);
      }
    }
    {
      std::lock_guard<std::mutex> lk(S->mu);
      int solving = 0;
      for (Lane& L : lanes) solving += (int)(L.mem[0].size() + L.mem[1].size() + L.joining.size());
      S->solving = solving;
      S->peak_solving = std::max(S->peak_solving, solving);
    }
    return true;
  };
  for (;;) {
    if (!admit(true)) break;
    // interactive lane first (until it drains, bounded), then one bulk cycle
    auto fail_all = [&](int rc) { for (Lane& L : lanes) fail_lane(S, L, rc); };
    // edits first (until they drain, bounded): small-edit cycles, with a
    // large-edit cycle every kLargeEvery of them (every cycle when no small
    // edit waits); then one bulk cycle, short while any edit waits
    for (int c = 0; c < kInteractiveCycles; ++c) {
      const bool small = !lanes[kSmall].empty(), large = !lanes[kLarge].empty();
      if (!small && !large) break;
      if (small) {
        const int rc = lane_cycle(S, lanes[kSmall], kSmall);
        if (rc) { fail_all(rc); return; }
      }
      if (!admit(false)) break;
      if (large && (!small || c % kLargeEvery == kLargeEvery - 1)) {
        const int rc = lane_cycle(S, lanes[kLarge], kLarge, small ? kBulkPairsBusy : 1 << 30);
        if (rc) { fail_all(rc); return; }
      }
      if (lanes[kSmall].active_tiles() == 0 && lanes[kSmall].joining.empty() &&
          lanes[kLarge].active_tiles() == 0 && lanes[kLarge].joining.empty()) {
        // converged members leave at the next cycle; run it now only if
        // someone is waiting for a slot
        break;
      }
    }
    if (!lanes[kBulk].empty()) {
      const bool busy = !lanes[kSmall].empty() || !lanes[kLarge].empty();
      const int rc = lane_cycle(S, lanes[kBulk], kBulk, busy ? kBulkPairsBusy : 1 << 30);
      if (rc) { fail_all(rc); return; }
    }
  }
  for (Lane& L : lanes)
    for (int k = 0; k < 2; ++k) tileset_free(L.ts[k]);
}

Session* find(jfc_server* S, int sid) {
  auto it = S->sessions.find(sid);
  return it == S->sessions.end() || it->second->close ? nullptr : it->second.get();
}

}  // namespace

extern "C" {

int jfc_server_create(jfc_ctx* ctx, size_t hbm_budget_bytes, int max_slots, jfc_server** out) {
  if (!ctx || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (max_slots <= 0) max_slots = 64;
  JFC_CUDA(cudaSetDevice(ctx->device));
  if (hbm_budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    JFC_CUDA(cudaMemGetInfo(&fr, &tot));
    hbm_budget_bytes = fr / 10 * 8;
  }
  std::unique_ptr<jfc_server> S(new jfc_server());
  S->device = ctx->device;
  S->params = ctx->params;
  fill_defaults(S->params);
  S->budget = hbm_budget_bytes;
  S->max_slots = max_slots;
  int rc = jfc_create(ctx->device, &S->params, &S->solve_ctx);
  if (rc == JFC_OK) rc = jfc_create(ctx->device, &S->params, &S->build_ctx);
  if (rc == JFC_OK && cudaStreamCreateWithFlags(&S->read_stream, cudaStreamNonBlocking) != cudaSuccess)
    rc = set_error(JFC_ERR_CUDA, "cudaStreamCreate");
  // the solver's launches get the device's highest stream priority: its
  // persistent phases need every SM at once, and the builder's kernels
  // (capacity builds and k-means of large volumes) would otherwise keep
  // taking the SMs that free up while a phase waits to start
  if (rc == JFC_OK) {
    int lo = 0, hi = 0;
    if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&S->solve_stream, cudaStreamNonBlocking, hi) != cudaSuccess)
      rc = set_error(JFC_ERR_CUDA, "cudaStreamCreateWithPriority");
    else
      rc = jfc_set_stream(S->solve_ctx, S->solve_stream);
  }
  if (rc != JFC_OK) {
    if (S->solve_ctx) jfc_destroy(S->solve_ctx);
    if (S->build_ctx) jfc_destroy(S->build_ctx);
    if (S->read_stream) cudaStreamDestroy(S->read_stream);
    if (S->solve_stream) cudaStreamDestroy(S->solve_stream);
    return rc;
  }
  // graph memory comes from the device's default pool (stream-ordered): keep
  // up to the budget mapped in the pool between sessions, so a new session's
  // allocation reuses memory instead of mapping fresh pages while the solver's
  // kernels run (restored when the server goes)
  if (cudaDeviceGetDefaultMemPool(&S->pool, S->device) == cudaSuccess) {
    cudaMemPoolGetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &S->pool_threshold0);
    unsigned long long thr = std::max<unsigned long long>(S->pool_threshold0, S->budget);
    cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  jfc_server* raw = S.release();
  raw->builder = std::thread(builder_loop, raw);
  raw->solver = std::thread(solver_loop, raw);
  *out = raw;
  return JFC_OK;
}

void jfc_server_destroy(jfc_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv_build.notify_all();
    S->cv_work.notify_all();
  }
  S->builder.join();
  S->solver.join();
  cudaSetDevice(S->device);
  cudaDeviceSynchronize();   // the threads' last frees and launches complete first
  for (int k = 0; k < 2; ++k) tileset_free(S->cut_ts[k]);
  for (auto& kv : S->sessions)
    if (kv.second->G) jfc_graph_destroy(kv.second->G);
  S->sessions.clear();
  if (S->read_stream) cudaStreamDestroy(S->read_stream);
  jfc_destroy(S->solve_ctx);
  jfc_destroy(S->build_ctx);
  if (S->solve_stream) cudaStreamDestroy(S->solve_stream);
  if (S->pool) {
    cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &S->pool_threshold0);
    cudaMemPoolTrimTo(S->pool, 0);
  }
  delete S;
}

int jfc_server_submit(jfc_server* S, int dims, int w, int h, int d, const void* img, int pixfmt,
                      const uint8_t* seeds, const jfc_model* model, int* sid) {
  if (!S || !img || !seeds || !sid) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  *sid = -1;
  if (dims == 2) d = 1;
  if ((dims != 2 && dims != 3) || w < 1 || h < 1 || d < 1)
    return set_error(JFC_ERR_INVALID_ARG, "bad grid shape");
  if (pixfmt < JFC_PIX_GRAY8 || pixfmt > JFC_PIX_I16) return set_error(JFC_ERR_INVALID_ARG, "bad pixel format");
  if ((long long)w * h * d > (1ll << 32) - 1) return set_error(JFC_ERR_INVALID_ARG, "grid larger than 2^32 nodes");
  const size_t n = (size_t)w * h * d;
  size_t nseeds = 0;
  for (size_t i = 0; i < n; ++i) nseeds += (seeds[i] == JFC_SEED_FG || seeds[i] == JFC_SEED_BG);
  std::unique_ptr<Session> s(new Session());
  s->dims = dims; s->w = w; s->h = h; s->d = d; s->pixfmt = pixfmt;
  if (model) s->model = *model;
  model_defaults(s->model);
  s->charge = session_bytes(dims, w, h, d, pixfmt, nseeds);
  if (s->charge > S->budget) return set_error(JFC_ERR_OOM, "session needs more device memory than the server budget");
  // the copies (up to hundreds of MB) are made before the server lock is
  // taken: the solver thread takes it between every two relabel cycles
  s->img.assign((const uint8_t*)img, (const uint8_t*)img + n * jfc_pix_bytes(pixfmt));
  s->seeds.assign(seeds, seeds + n);
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal) return set_error(S->fatal, "server stopped after a device error");
  Request r;
  r.cold = true;
  r.t_submit = Clock::now();
  s->reqs.push_back(std::move(r));
  s->sid = S->next_sid++;
  *sid = s->sid;
  S->build_q.push_back(s->sid);
  S->sessions[s->sid] = std::move(s);
  S->cv_build.notify_all();
  return JFC_OK;
}

int jfc_server_edit(jfc_server* S, int sid, const uint32_t* idx, const uint8_t* new_seed, size_t n) {
  if (!S || (n && (!idx || !new_seed))) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  // the edit is copied and its seed values checked before the server lock
  // is taken (the solver thread takes it between every two relabel cycles)
  Request r;
  r.cold = false;
  r.idx.assign(idx, idx + n);
  r.seed.assign(new_seed, new_seed + n);
  uint32_t max_idx = 0;
  for (size_t j = 0; j < n; ++j) {
    if (new_seed[j] > 2) return set_error(JFC_ERR_INVALID_ARG, "bad edit");
    max_idx = std::max(max_idx, idx[j]);
  }
  std::lock_guard<std::mutex> lk(S->mu);
  Session* s = find(S, sid);
  if (!s) return set_error(JFC_ERR_INVALID_ARG, "unknown session");
  if (s->phase == DEAD) return set_error(JFC_ERR_STATE, "session has no graph (build failed or cancelled)");
  const unsigned long long N = (unsigned long long)s->w * s->h * s->d;
  if (n && max_idx >= N) return set_error(JFC_ERR_INVALID_ARG, "bad edit");
  r.t_submit = Clock::now();
  s->cancel = false;
  s->reqs.push_back(std::move(r));
  if (s->phase == IDLE) {
    s->phase = READY;
    S->ready_q.push_back(sid);
    S->cv_work.notify_all();
  }
  return JFC_OK;
}

int jfc_server_wait(jfc_server* S, int sid, int timeout_ms, jfc_request_info* info) {
  if (!S) return set_error(JFC_ERR_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lk(S->mu);
  if (!find(S, sid)) return set_error(JFC_ERR_INVALID_ARG, "unknown session");
  // the session may be closed (and freed) while this thread waits
  auto idle = [&] {
    const Session* x = find(S, sid);
    return !x || x->reqs.empty() || S->fatal;
  };
  if (timeout_ms < 0) S->cv_done.wait(lk, idle);
  else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), idle))
    return set_error(JFC_ERR_BUSY, "request not finished");
  Session* s = find(S, sid);
  if (!s) return set_error(JFC_ERR_CANCELLED, "session closed");
  if (!s->reqs.empty()) return set_error(S->fatal, "server stopped after a device error");
  if (info) *info = s->last;
  if (!s->has_last) return set_error(JFC_ERR_STATE, "no request finished");
  return s->last.status == JFC_OK ? JFC_OK : set_error(s->last.status, "request failed");
}

int jfc_server_read_labels(jfc_server* S, int sid, uint8_t* out) {
  if (!S || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  // read_mu first: while it is held no graph is freed and no edit joins the
  // solving set, so a session without unfinished requests stays untouched
  std::lock_guard<std::mutex> rl(S->read_mu);
  jfc_graph* G = nullptr;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    Session* s = find(S, sid);
    if (!s) return set_error(JFC_ERR_INVALID_ARG, "unknown session");
    if (!s->reqs.empty()) return set_error(JFC_ERR_BUSY, "session has unfinished requests");
    if (!s->G || s->G->state != 2) return set_error(JFC_ERR_STATE, "not solved");
    G = s->G;
  }
  JFC_CUDA(cudaSetDevice(S->device));
  JFC_CUDA(copy_plane(G->g.label, out, 1, G, true, cudaMemcpyDeviceToHost, S->read_stream));
  JFC_CUDA(cudaStreamSynchronize(S->read_stream));
  return JFC_OK;
}

int jfc_server_get_stats(jfc_server* S, jfc_server_stats* out) {
  if (!S || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  std::memset(out, 0, sizeof(*out));
  out->budget = S->budget;
  out->used = S->used;
  out->peak_used = S->peak_used;
  out->sessions = (int)S->sessions.size();
  out->waiting = (int)(S->build_q.size() + S->ready_q.size());
  out->solving = S->solving;
  out->peak_solving = S->peak_solving;
  out->loops = S->loops;
  out->requests_done = S->requests_done;
  return JFC_OK;
}

int jfc_server_cancel(jfc_server* S, int sid) {
  if (!S) return set_error(JFC_ERR_INVALID_ARG, "null server");
  std::lock_guard<std::mutex> lk(S->mu);
  Session* s = find(S, sid);
  if (!s) return set_error(JFC_ERR_INVALID_ARG, "unknown session");
  if (s->phase == WAIT_BUILD) {
    S->build_q.erase(std::remove(S->build_q.begin(), S->build_q.end(), sid), S->build_q.end());
    cancel_all(S, s, Clock::now());
    s->phase = DEAD;
  } else {
    s->cancel = true;   // the thread that owns the session finishes its requests
  }
  S->cv_done.notify_all();
  S->cv_work.notify_all();
  return JFC_OK;
}

int jfc_server_close(jfc_server* S, int sid) {
  if (!S) return set_error(JFC_ERR_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lk(S->mu);
  Session* s = find(S, sid);
  if (!s) return set_error(JFC_ERR_INVALID_ARG, "unknown session");
  s->cancel = true;
  s->close = true;
  const Clock::time_point now = Clock::now();
  if (s->phase == WAIT_BUILD) {
    S->build_q.erase(std::remove(S->build_q.begin(), S->build_q.end(), sid), S->build_q.end());
    cancel_all(S, s, now);
    S->sessions.erase(sid);   // nothing on the device yet
  } else if ((s->phase == IDLE || s->phase == DEAD) && s->lane_refs == 0) {
    cancel_all(S, s, now);
    S->to_free.push_back(s);  // freed by the solver between launches
    S->cv_work.notify_all();
  }
  // READY / BUILDING / SOLVING, or a finished request whose lane still holds
  // the session: the owner thread finishes and frees it (a lane drops its
  // done members at its next membership change and frees the closed ones)
  S->cv_done.notify_all();
  return JFC_OK;
}

}  // extern "C"
