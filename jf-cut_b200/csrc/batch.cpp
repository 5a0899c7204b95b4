// batch.cpp — batched solver: many independent grids of uneven sizes share
// every launch.
//
// No reference counterpart: JF-Cut solves one volume at a time
// (QGCWidget::slotCutClicked, QGCWidget.cpp:2364).  The per-grid arithmetic is
// unchanged; what changes is that all grids' tiles form one tile set, so every
// sweep / BFS pass is one persistent launch whose warps pull tiles of any grid
// from the device work queue, and the host loop runs once for the whole batch
// (converged grids simply stop producing flagged tiles).  The autotuner times
// candidate schedules (tile height, rounds per visit, relabel interval) on the
// batch itself and restores the graphs' state after each trial; its choice
// belongs to the batch (the context's parameters stay as the caller set them).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "engine.h"

struct jfc_batch {
  jfc_ctx* ctx = nullptr;
  std::vector<jfc_graph*> graphs;
  TileSet ts[2];          // [0] 2D grids, [1] 3D grids
  int shape[2] = {-1, -1};
  bool dirty = true;
  bool tuned = false;     // params below were chosen by jfc_batch_autotune
  jfc_params params{};
};

namespace {

// The schedule this batch solves with: its tuned one, else the context's.
const jfc_params& batch_params(const jfc_batch* b) { return b->tuned ? b->params : b->ctx->params; }

int rebuild(jfc_batch* b) {
  const jfc_params& bp = batch_params(b);
  const int tr = bp.tile_rows;
  for (int k = 0; k < 2; ++k) {
    const int dims = k ? 3 : 2;
    const int td = bp.tile_depth;
    const bool split = pr_split_for(bp, dims);
    const int code = shape_code(dims, tr, td, split);
    if (!b->dirty && b->shape[k] == code) continue;
    std::vector<GridDev> v;
    for (jfc_graph* g : b->graphs)
      if (g->dims == dims) v.push_back(g->g);
    tileset_free(b->ts[k]);
    b->shape[k] = -1;
    if (v.empty()) continue;
    int rc = tileset_build(b->ts[k], dims, tr, td, v, nullptr, split);
    if (rc) return rc;
    b->shape[k] = code;
  }
  b->dirty = false;
  return JFC_OK;
}

// Device snapshot of every graph's e and residual planes (autotuner).
struct Snapshot {
  std::vector<void*> bufs;
  ~Snapshot() { for (void* p : bufs) cudaFree(p); }
};

int snapshot(jfc_batch* b, Snapshot& s, bool restore) {
  cudaStream_t st = b->ctx->stream;
  for (size_t i = 0; i < b->graphs.size(); ++i) {
    jfc_graph* g = b->graphs[i];
    const size_t bytes = (size_t)g->g.plane * 4 * (1 + g->conn);
    if (!restore) {
      void* p = nullptr;
      JFC_CUDA(cudaMalloc(&p, bytes));
      s.bufs.push_back(p);
    }
    char* p = (char*)s.bufs[i];
    const size_t pb = (size_t)g->g.plane * 4;
    int* planes[7] = {g->g.e, g->g.r[0], g->g.r[1], g->g.r[2], g->g.r[3], g->g.r[4], g->g.r[5]};
    for (int k = 0; k < 1 + g->conn; ++k) {
      if (restore) JFC_CUDA(cudaMemcpyAsync(planes[k], p + k * pb, pb, cudaMemcpyDeviceToDevice, st));
      else JFC_CUDA(cudaMemcpyAsync(p + k * pb, planes[k], pb, cudaMemcpyDeviceToDevice, st));
    }
  }
  JFC_CUDA(cudaStreamSynchronize(st));
  return JFC_OK;
}

}  // namespace

extern "C" {

int jfc_batch_create(jfc_ctx* ctx, jfc_batch** out) {
  if (!ctx || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  jfc_batch* b = new jfc_batch();
  b->ctx = ctx;
  *out = b;
  return JFC_OK;
}

void jfc_batch_destroy(jfc_batch* b) {
  if (!b) return;
  cudaSetDevice(b->ctx->device);
  tileset_free(b->ts[0]);
  tileset_free(b->ts[1]);
  delete b;
}

int jfc_batch_add(jfc_batch* b, jfc_graph* g) {
  if (!b || !g) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (g->ctx != b->ctx) return set_error(JFC_ERR_INVALID_ARG, "graph belongs to another context");
  if (g->state == 0) return set_error(JFC_ERR_STATE, "graph is empty");
  b->graphs.push_back(g);
  b->dirty = true;
  return JFC_OK;
}

int jfc_batch_clear(jfc_batch* b) {
  if (!b) return set_error(JFC_ERR_INVALID_ARG, "null batch");
  b->graphs.clear();
  b->dirty = true;
  b->tuned = false;       // a schedule tuned for the old graphs does not carry over
  return JFC_OK;
}

int jfc_batch_size(jfc_batch* b) { return b ? (int)b->graphs.size() : 0; }

int jfc_batch_solve(jfc_batch* b, jfc_stats* stats) {
  if (!b) return set_error(JFC_ERR_INVALID_ARG, "null batch");
  JFC_CUDA(cudaSetDevice(b->ctx->device));
  for (jfc_graph* g : b->graphs)
    if (g->state == 0) return set_error(JFC_ERR_STATE, "graph is empty");
  int rc = rebuild(b);
  if (rc) return rc;
  int first_bad = JFC_OK;
  for (int k = 0; k < 2; ++k) {
    if (b->shape[k] < 0) continue;
    const int dims = k ? 3 : 2;
    std::vector<GridResult> res;
    jfc_stats st;
    rc = engine_solve(b->ctx, b->ts[k], batch_params(b), res, st);
    if (rc && rc != JFC_ERR_NOT_CONVERGED) return rc;
    int gi = 0;
    for (size_t i = 0; i < b->graphs.size(); ++i) {
      jfc_graph* g = b->graphs[i];
      if (g->dims != dims) continue;
      const GridResult& r = res[gi++];
      g->flow = g->sink_total + r.neg_sum;
      g->source_nodes = r.labels;
      g->state = r.status ? 1 : 2;
      jfc_stats gs = st;
      gs.status = r.status;
      gs.flow = g->flow;
      gs.source_nodes = g->source_nodes;
      g->last = gs;
      if (stats) stats[i] = gs;
      if (r.status && !first_bad) first_bad = r.status;
    }
  }
  return first_bad;
}

int jfc_batch_autotune(jfc_batch* b, jfc_params* chosen) {
  if (!b) return set_error(JFC_ERR_INVALID_ARG, "null batch");
  if (b->graphs.empty()) return set_error(JFC_ERR_STATE, "empty batch");
  JFC_CUDA(cudaSetDevice(b->ctx->device));
  Snapshot snap;
  int rc = snapshot(b, snap, false);
  if (rc) return rc;
  const bool was_tuned = b->tuned;
  const jfc_params was = b->params;
  const jfc_params base = batch_params(b);
  auto give_up = [&](int r) { b->tuned = was_tuned; b->params = was; b->dirty = true; return r; };
  // a trial: the batch solved from the snapshot under schedule p, twice; its
  // time is the faster of the two device-clock solve times (one sample can
  // be slowed by anything else on the host or device)
  std::vector<jfc_stats> st(b->graphs.size());
  auto trial = [&](const jfc_params& p, double& ms) -> int {
    b->params = p;
    b->params.relabel_interval_max = 0;   // re-derived from the trial interval
    fill_defaults(b->params);
    b->tuned = true;
    ms = 1e30;
    for (int rep = 0; rep < 2; ++rep) {
      int r = snapshot(b, snap, true);
      if (r) return r;
      r = jfc_batch_solve(b, st.data());
      if (r == JFC_ERR_NOT_CONVERGED) return JFC_OK;   // this schedule ran out of budget: not chosen
      if (r) return r;
      // the batch's solves are one engine run per dimensionality; each
      // graph's stats carry the time of the run it was part of
      double t2 = 0.0, t3 = 0.0;
      for (size_t i = 0; i < b->graphs.size(); ++i)
        (b->graphs[i]->dims == 2 ? t2 : t3) = st[i].ms_total;
      ms = std::min(ms, t2 + t3);
    }
    return JFC_OK;
  };
  // Coordinate descent from the context's schedule: relabel interval, then
  // rounds per visit, then tile height (then 3D tile depth when the batch has
  // volumes); each axis keeps its best value.  The
  // first trial also pays one-time costs (tile set, graph capture), so the
  // starting point is timed twice.
  jfc_params best = base;
  double best_ms = 1e30, ms = 0.0;
  rc = trial(best, ms);
  if (rc) return give_up(rc);
  rc = trial(best, best_ms);
  if (rc) return give_up(rc);
  const int intervals[] = {2, 3, 4, 8, 16};
  const int iters[] = {8, 12, 16, 32};
  const int rows[] = {8, 16};
  const int depths[] = {0, 1, 2, 4};   // 3D tile depth (0 = automatic 32x4x2)
  bool has3d = false;
  for (jfc_graph* g : b->graphs) has3d |= g->dims == 3;
  for (int axis = 0; axis < (has3d ? 4 : 3); ++axis) {
    const int* vals = axis == 0 ? intervals : axis == 1 ? iters : axis == 2 ? rows : depths;
    const int nv = axis == 0 ? 5 : axis == 1 ? 4 : axis == 2 ? 2 : 4;
    const jfc_params center = best;
    for (int i = 0; i < nv; ++i) {
      jfc_params p = center;
      if (axis == 3 && vals[i] == 4 && p.tile_rows != 16) continue;
      int& field = axis == 0 ? p.relabel_interval : axis == 1 ? p.local_iters : axis == 2 ? p.tile_rows : p.tile_depth;
      if (field == vals[i]) continue;
      field = vals[i];
      rc = trial(p, ms);
      if (rc) return give_up(rc);
      if (ms < best_ms) { best_ms = ms; best = p; }
    }
  }
  best.relabel_interval_max = 0;
  fill_defaults(best);
  b->params = best;
  b->tuned = true;
  rc = snapshot(b, snap, true);
  for (jfc_graph* g : b->graphs) g->state = 1;
  if (chosen) *chosen = best;
  return rc;
}

}  // extern "C"
