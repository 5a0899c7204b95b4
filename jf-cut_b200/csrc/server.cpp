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
};

}  // namespace

struct jfc_server {
  int device = 0;
  jfc_params params{};
  jfc_ctx* solve_ctx = nullptr;
  jfc_ctx* build_ctx = nullptr;
  cudaStream_t read_stream = nullptr;
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

  TileSet ts[2], cut_ts[2];         // solving set / converged grids, [0] 2D, [1] 3D
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
void free_session(jfc_server* S, Session* s) {
  std::lock_guard<std::mutex> rl(S->read_mu);
  if (s->G) {
    jfc_graph_destroy(s->G);
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
    int rc = jfc_graph_create_grid(S->build_ctx, s->dims, s->w, s->h, s->d, s->dims == 2 ? 4 : 6, &G);
    if (rc == JFC_OK) rc = build_core(G, s->img.data(), s->pixfmt, s->seeds.data(), &s->model, cudaMemcpyHostToDevice);
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

void solver_loop(jfc_server* S) {
  cudaSetDevice(S->device);
  jfc_ctx* ctx = S->solve_ctx;
  const jfc_params& p = S->params;
  std::vector<Member> mem[2];       // members of ts[0] / ts[1], in grid order
  std::vector<int> active[2];       // active tiles per grid after the last relabel
  int interval = p.relabel_interval;
  auto fail_all = [&](int rc) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->fatal = rc;
    const Clock::time_point now = Clock::now();
    for (int k = 0; k < 2; ++k)
      for (Member& m : mem[k]) {
        if (!m.done) finish_front(S, m.s, rc, 0, now);
        cancel_all(S, m.s, now);
        m.s->phase = IDLE;
      }
    S->cv_done.notify_all();
  };
  for (;;) {
    // 1. push-relabel phase over the current solving set
    long long total_active = 0;
    for (int k = 0; k < 2; ++k)
      for (size_t i = 0; i < mem[k].size(); ++i)
        if (!mem[k][i].done) total_active += active[k][i];
    bool ran_pr[2] = {false, false};
    for (int k = 0; k < 2; ++k) {
      long long a = 0;
      for (size_t i = 0; i < mem[k].size(); ++i)
        if (!mem[k][i].done) a += active[k][i];
      if (a == 0) continue;
      cudaMemsetAsync(S->ts[k].d_ctr->ticket, 0, sizeof(S->ts[k].d_ctr->ticket), ctx->stream);
      const cudaError_t e = launch_pr_phase(S->ts[k], interval, p.local_iters, ctx->stream);
      if (e != cudaSuccess) { fail_all(cuda_status(e, "push-relabel phase")); return; }
      ran_pr[k] = true;
    }
    // 2. membership: leave (done / cancelled), free closed sessions, join
    bool changed[2] = {false, false};
    std::vector<Session*> joining, frees;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (total_active == 0 && mem[0].empty() && mem[1].empty())
        S->cv_work.wait(lk, [&] { return S->stop || !S->ready_q.empty() || !S->to_free.empty(); });
      if (S->stop) break;
      const Clock::time_point now = Clock::now();
      for (int k = 0; k < 2; ++k) {
        std::vector<Member> keep;
        std::vector<int> keep_act;
        for (size_t i = 0; i < mem[k].size(); ++i) {
          Member& m = mem[k][i];
          if (!m.done && m.s->cancel) {
            cancel_all(S, m.s, now);
            m.done = true;
            S->cv_done.notify_all();
          }
          if (m.done) {
            changed[k] = true;
            if (m.s->close) S->to_free.push_back(m.s);
            continue;
          }
          keep.push_back(m);
          keep_act.push_back(active[k][i]);
        }
        mem[k].swap(keep);
        active[k].swap(keep_act);
      }
      frees.swap(S->to_free);
      int slots = S->max_slots - (int)(mem[0].size() + mem[1].size());
      while (slots > 0 && !S->ready_q.empty()) {
        Session* s = S->sessions.at(S->ready_q.front()).get();
        S->ready_q.pop_front();
        if (s->cancel || s->reqs.empty()) {
          cancel_all(S, s, now);
          s->phase = IDLE;
          if (s->close) frees.push_back(s);
          S->cv_done.notify_all();
          continue;
        }
        s->phase = SOLVING;
        if (!s->reqs.front().cold) s->reqs.front().t_admit = now;
        joining.push_back(s);
        --slots;
      }
    }
    for (Session* s : frees) {
      free_session(S, s);
      std::lock_guard<std::mutex> lk(S->mu);
      S->sessions.erase(s->sid);
    }
    // a label read in progress finishes before any joining edit changes a graph
    std::unique_lock<std::mutex> rl(S->read_mu, std::defer_lock);
    if (!joining.empty()) rl.lock();
    for (Session* s : joining) {
      int rc = JFC_OK;
      Request& r = s->reqs.front();
      if (!r.cold) rc = jfc_graph_edit_seeds(s->G, r.idx.data(), r.seed.data(), r.idx.size());
      if (rc != JFC_OK) {
        std::lock_guard<std::mutex> lk(S->mu);
        finish_front(S, s, rc, 0, Clock::now());
        s->phase = s->reqs.empty() ? IDLE : READY;
        if (!s->reqs.empty()) S->ready_q.push_back(s->sid);
        S->cv_done.notify_all();
        continue;
      }
      const int k = s->dims == 3 ? 1 : 0;
      mem[k].push_back(Member{s});
      active[k].push_back(0);
      changed[k] = true;
    }
    if (rl.owns_lock()) rl.unlock();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      ++S->loops;
      S->solving = (int)(mem[0].size() + mem[1].size());
      S->peak_solving = std::max(S->peak_solving, S->solving);
    }
    // 3. global relabel over the (re-formed) solving set
    for (int k = 0; k < 2; ++k) {
      if (mem[k].empty()) {
        active[k].clear();
        continue;
      }
      if (changed[k]) {
        std::vector<GridDev> grids;
        for (Member& m : mem[k]) grids.push_back(m.s->G->g);
        int rc = tileset_build(S->ts[k], k ? 3 : 2, p.tile_rows, p.tile_depth, grids, ctx->stream);
        if (rc) { fail_all(rc); return; }
      }
      int passes = 0, sw = 0;
      int rc = engine_bfs(ctx, S->ts[k], p, false, passes, &active[k], nullptr, &sw);
      if (rc) { fail_all(rc); return; }
      if (ran_pr[k])
        for (Member& m : mem[k]) m.s->sweeps += sw;
    }
    // 4. converged grids: cut BFS on a tile set of those grids alone
    long long still = 0;
    for (int k = 0; k < 2; ++k) {
      std::vector<size_t> conv;
      for (size_t i = 0; i < mem[k].size(); ++i) {
        if (active[k][i] == 0) conv.push_back(i);
        else if (mem[k][i].s->sweeps >= p.max_sweeps) conv.push_back(i);
        else still += active[k][i];
      }
      if (conv.empty()) continue;
      std::vector<GridDev> grids;
      for (size_t i : conv) grids.push_back(mem[k][i].s->G->g);
      int rc = tileset_build(S->cut_ts[k], k ? 3 : 2, p.tile_rows, p.tile_depth, grids, ctx->stream);
      if (rc) { fail_all(rc); return; }
      std::vector<GridResult> res;
      int passes = 0;
      rc = engine_cut(ctx, S->cut_ts[k], p, res, passes);
      if (rc && rc != JFC_ERR_NOT_CONVERGED) { fail_all(rc); return; }
      std::lock_guard<std::mutex> lk(S->mu);
      const Clock::time_point now = Clock::now();
      for (size_t j = 0; j < conv.size(); ++j) {
        Member& m = mem[k][conv[j]];
        Session* s = m.s;
        jfc_graph* G = s->G;
        int st = res[j].status;
        if (active[k][conv[j]] > 0) st = JFC_ERR_NOT_CONVERGED;
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
    // adaptive interval as in the plain solve: a sliver of active tiles
    // makes the dense relabel dominate, so relabel less often
    long long nt = (long long)S->ts[0].ntiles * (mem[0].empty() ? 0 : 1) +
                   (long long)S->ts[1].ntiles * (mem[1].empty() ? 0 : 1);
    if (still > 0 && still * 256 < nt) interval = std::min(interval * 2, p.relabel_interval_max);
    else interval = p.relabel_interval;
  }
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
  if (rc != JFC_OK) {
    if (S->solve_ctx) jfc_destroy(S->solve_ctx);
    if (S->build_ctx) jfc_destroy(S->build_ctx);
    return rc;
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
  for (int k = 0; k < 2; ++k) {
    tileset_free(S->ts[k]);
    tileset_free(S->cut_ts[k]);
  }
  for (auto& kv : S->sessions)
    if (kv.second->G) jfc_graph_destroy(kv.second->G);
  S->sessions.clear();
  if (S->read_stream) cudaStreamDestroy(S->read_stream);
  jfc_destroy(S->solve_ctx);
  jfc_destroy(S->build_ctx);
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
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal) return set_error(S->fatal, "server stopped after a device error");
  if (s->charge > S->budget) return set_error(JFC_ERR_OOM, "session needs more device memory than the server budget");
  s->img.assign((const uint8_t*)img, (const uint8_t*)img + n * jfc_pix_bytes(pixfmt));
  s->seeds.assign(seeds, seeds + n);
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
  std::lock_guard<std::mutex> lk(S->mu);
  Session* s = find(S, sid);
  if (!s) return set_error(JFC_ERR_INVALID_ARG, "unknown session");
  if (s->phase == DEAD) return set_error(JFC_ERR_STATE, "session has no graph (build failed or cancelled)");
  const unsigned long long N = (unsigned long long)s->w * s->h * s->d;
  for (size_t j = 0; j < n; ++j)
    if (idx[j] >= N || new_seed[j] > 2) return set_error(JFC_ERR_INVALID_ARG, "bad edit");
  Request r;
  r.cold = false;
  r.idx.assign(idx, idx + n);
  r.seed.assign(new_seed, new_seed + n);
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
  } else if (s->phase == IDLE || s->phase == DEAD) {
    cancel_all(S, s, now);
    S->to_free.push_back(s);  // freed by the solver between launches
    S->cv_work.notify_all();
  }
  // READY / BUILDING / SOLVING: the owner thread finishes and frees it
  S->cv_done.notify_all();
  return JFC_OK;
}

}  // extern "C"
