// engine.cpp — the solve loop shared by plain, batched and served solves.
//
// Reference: QGCWidget::slotCutClicked (QGCWidget.cpp:2364-2558): optional
// global relabel, then { countActiveBlock every countIterations; relabelPush;
// computeCut every cutIterations } until the cut BFS finds no augmenting path
// or totalIterations runs out (then the cut is returned silently, :2413).
// The reference reads back a few ints per step with blocking calls
// (:2122-2123, 2237, 3267).
//
// Here: one loop for any set of grids (a plain solve is a set of one):
//   global relabel (exact sink distances; also counts active tiles per grid)
//   while any grid has an active tile:
//     relabel_interval x { sweep even tiles, sweep odd tiles }
//     global relabel
//   cut BFS; per-grid int64 sums of min(e, 0) and of the labels.
// Convergence is the device-side active-tile count (zero active tiles after an
// exact global relabel means no residual path from excess to a deficit: a
// maximum preflow), read once per relabel, never per sweep.  The budget
// (max_sweeps, max_bfs_passes) ends the loop with JFC_ERR_NOT_CONVERGED
// instead of returning a non-converged cut.
#include "engine.h"

#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>

static thread_local std::string g_err;
static std::atomic<unsigned long long> g_launches{0};

void jfc_note_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

extern "C" unsigned long long jfc_kernel_launches(void) { return g_launches.load(); }

int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_status(cudaError_t e, const char* where) {
  g_err = std::string(where) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return JFC_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return JFC_ERR_NO_DEVICE;
  return JFC_ERR_CUDA;
}

extern "C" const char* jfc_last_error(void) { return g_err.c_str(); }

void fill_defaults(jfc_params& p) {
  if (p.tile_rows != 8 && p.tile_rows != 16) p.tile_rows = 16;
  if (p.local_iters <= 0) p.local_iters = 16;
  if (p.relabel_interval <= 0) p.relabel_interval = 8;
  if (p.max_sweeps <= 0) p.max_sweeps = 1 << 20;
  if (p.max_bfs_passes <= 0) p.max_bfs_passes = 1 << 20;
}

double elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return (double)ms;
}

int shape_code(int dims, int tile_rows) { return dims * 100 + tile_rows; }

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

void tileset_free(TileSet& ts) {
  if (ts.d_block) cudaFree(ts.d_block);
  ts = TileSet();
}

int tileset_build(TileSet& ts, int dims, int tile_rows, const std::vector<GridDev>& grids_in) {
  tileset_free(ts);
  ts.dims = dims;
  if (dims == 2) {
    ts.TR = tile_rows; ts.TY = tile_rows; ts.TZ = 1;
  } else {
    ts.TR = tile_rows; ts.TY = 4; ts.TZ = tile_rows >= 16 ? 4 : 2;
  }
  std::vector<GridDev> grids = grids_in;
  std::vector<int4> info;
  std::vector<int> list[2];
  int base = 0;
  for (size_t gi = 0; gi < grids.size(); ++gi) {
    GridDev& g = grids[gi];
    if (g.dims != dims) return set_error(JFC_ERR_INVALID_ARG, "tile set mixes 2D and 3D grids");
    g.tiles_x = g.pitch / JFC_TW;
    g.tiles_y = g.Hp / ts.TY;
    g.tiles_z = g.Dp / ts.TZ;
    g.tile_base = base;
    for (int tz = 0; tz < g.tiles_z; ++tz)
      for (int ty = 0; ty < g.tiles_y; ++ty)
        for (int tx = 0; tx < g.tiles_x; ++tx) {
          info.push_back(make_int4((int)gi, tx, ty, tz));
          list[(tx + ty + tz) & 1].push_back(base + tx + g.tiles_x * (ty + g.tiles_y * tz));
        }
    base += g.tiles_x * g.tiles_y * g.tiles_z;
  }
  ts.ngrids = (int)grids.size();
  ts.ntiles = base;
  ts.nlist[0] = (int)list[0].size();
  ts.nlist[1] = (int)list[1].size();
  size_t off = 0;
  const size_t o_desc = off; off = align_up(off + sizeof(GridDev) * grids.size(), 256);
  const size_t o_info = off; off = align_up(off + sizeof(int4) * info.size(), 256);
  const size_t o_l0 = off; off = align_up(off + sizeof(int) * list[0].size(), 256);
  const size_t o_l1 = off; off = align_up(off + sizeof(int) * list[1].size(), 256);
  const size_t o_fpr = off; off = align_up(off + (size_t)ts.ntiles, 256);
  const size_t o_fb0 = off; off = align_up(off + (size_t)ts.ntiles, 256);
  const size_t o_fb1 = off; off = align_up(off + (size_t)ts.ntiles, 256);
  const size_t o_act = off; off = align_up(off + sizeof(int) * grids.size(), 256);
  const size_t o_sum = off; off = align_up(off + sizeof(long long) * 2 * grids.size(), 256);
  const size_t o_ctr = off; off = align_up(off + sizeof(DevCounters), 256);
  char* blk = nullptr;
  JFC_CUDA(cudaMalloc((void**)&blk, off));
  ts.d_block = blk;
  ts.block_bytes = off;
  ts.d_desc = (GridDev*)(blk + o_desc);
  ts.d_info = (int4*)(blk + o_info);
  ts.d_list[0] = (int*)(blk + o_l0);
  ts.d_list[1] = (int*)(blk + o_l1);
  ts.d_flag_pr = (uint8_t*)(blk + o_fpr);
  ts.d_flag_bfs[0] = (uint8_t*)(blk + o_fb0);
  ts.d_flag_bfs[1] = (uint8_t*)(blk + o_fb1);
  ts.d_grid_active = (int*)(blk + o_act);
  ts.d_grid_sum = (long long*)(blk + o_sum);
  ts.d_ctr = (DevCounters*)(blk + o_ctr);
  JFC_CUDA(cudaMemset(blk, 0, off));
  JFC_CUDA(cudaMemcpy(ts.d_desc, grids.data(), sizeof(GridDev) * grids.size(), cudaMemcpyHostToDevice));
  JFC_CUDA(cudaMemcpy(ts.d_info, info.data(), sizeof(int4) * info.size(), cudaMemcpyHostToDevice));
  if (!list[0].empty())
    JFC_CUDA(cudaMemcpy(ts.d_list[0], list[0].data(), sizeof(int) * list[0].size(), cudaMemcpyHostToDevice));
  if (!list[1].empty())
    JFC_CUDA(cudaMemcpy(ts.d_list[1], list[1].data(), sizeof(int) * list[1].size(), cudaMemcpyHostToDevice));
  return JFC_OK;
}

// Pinned read-back buffer of the context (grown on demand).
static int pin_reserve(jfc_ctx* ctx, size_t bytes) {
  if (ctx->h_pin_bytes >= bytes) return JFC_OK;
  if (ctx->h_pin) cudaFreeHost(ctx->h_pin);
  ctx->h_pin = nullptr;
  ctx->h_pin_bytes = 0;
  JFC_CUDA(cudaMallocHost(&ctx->h_pin, bytes));
  ctx->h_pin_bytes = bytes;
  return JFC_OK;
}

// Run one BFS (global relabel when !cut, cut otherwise) to its fixpoint.
// On return (relabel) active[g] holds the active tiles of every grid.
static int run_bfs(jfc_ctx* ctx, TileSet& ts, const jfc_params& p, bool cut, int& passes,
                   std::vector<int>* active, int* cut_bad) {
  cudaStream_t s = ctx->stream;
  JFC_CUDA(cudaMemsetAsync(ts.d_flag_bfs[0], 0, (size_t)ts.ntiles, s));
  JFC_CUDA(cudaMemsetAsync(ts.d_flag_bfs[1], 0, (size_t)ts.ntiles, s));
  if (!cut) JFC_CUDA(cudaMemsetAsync(ts.d_grid_active, 0, sizeof(int) * ts.ngrids, s));
  else JFC_CUDA(cudaMemsetAsync(&ts.d_ctr->cut_bad, 0, sizeof(int), s));
  JFC_CUDA(cut ? launch_cut_pass(ts, 0, true, s) : launch_relabel_pass(ts, 0, true, s));
  int pass = 1, batch = 2;
  const size_t need = sizeof(int) * (4 + (size_t)ts.ngrids);
  int rc = pin_reserve(ctx, need);
  if (rc) return rc;
  int* hp = (int*)ctx->h_pin;
  for (;;) {
    for (int k = 0; k < batch; ++k)
      JFC_CUDA(cut ? launch_cut_pass(ts, pass + k, false, s) : launch_relabel_pass(ts, pass + k, false, s));
    pass += batch;
    JFC_CUDA(cudaMemcpyAsync(hp, &ts.d_ctr->pending[(pass - 1) & 1], sizeof(int), cudaMemcpyDeviceToHost, s));
    JFC_CUDA(cudaStreamSynchronize(s));
    if (hp[0] == 0) break;
    if (pass > p.max_bfs_passes) {
      passes += pass;
      return set_error(JFC_ERR_NOT_CONVERGED, "BFS pass budget exhausted");
    }
    if (batch < 16) batch *= 2;
  }
  passes += pass;
  if (!cut && active) {
    active->resize(ts.ngrids);
    JFC_CUDA(cudaMemcpyAsync(hp + 4, ts.d_grid_active, sizeof(int) * ts.ngrids, cudaMemcpyDeviceToHost, s));
    JFC_CUDA(cudaStreamSynchronize(s));
    for (int g = 0; g < ts.ngrids; ++g) (*active)[g] = hp[4 + g];
  }
  if (cut && cut_bad) {
    JFC_CUDA(cudaMemcpyAsync(hp, &ts.d_ctr->cut_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    JFC_CUDA(cudaStreamSynchronize(s));
    *cut_bad = hp[0];
  }
  return JFC_OK;
}

namespace {
struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() { cudaEventCreate(&a); cudaEventCreate(&b); }
  ~Timer() { cudaEventDestroy(a); cudaEventDestroy(b); }
};
}  // namespace

int engine_solve(jfc_ctx* ctx, TileSet& ts, const jfc_params& p_in, std::vector<GridResult>& res,
                 jfc_stats& st) {
  jfc_params p = p_in;
  fill_defaults(p);
  cudaStream_t s = ctx->stream;
  std::memset(&st, 0, sizeof(st));
  res.assign(ts.ngrids, GridResult());
  Timer t_all, t_ph;
  JFC_CUDA(cudaEventRecord(t_all.a, s));
  JFC_CUDA(launch_clear_counters(ts, s));
  std::vector<int> active;
  int rc;

  JFC_CUDA(cudaEventRecord(t_ph.a, s));
  rc = run_bfs(ctx, ts, p, false, st.bfs_passes, &active, nullptr);
  JFC_CUDA(cudaEventRecord(t_ph.b, s));
  JFC_CUDA(cudaEventSynchronize(t_ph.b));
  st.ms_global_relabel += elapsed_ms(t_ph.a, t_ph.b);
  st.global_relabels = 1;
  if (rc) return rc;

  auto total = [&]() { long long t = 0; for (int v : active) t += v; return t; };
  int status = JFC_OK;
  while (total() > 0) {
    if (st.sweeps >= p.max_sweeps) {
      status = set_error(JFC_ERR_NOT_CONVERGED, "sweep budget exhausted");
      break;
    }
    JFC_CUDA(cudaEventRecord(t_ph.a, s));
    for (int k = 0; k < p.relabel_interval; ++k) {
      JFC_CUDA(launch_pr_sweep(ts, 0, p.local_iters, s));
      JFC_CUDA(launch_pr_sweep(ts, 1, p.local_iters, s));
      ++st.sweeps;
    }
    JFC_CUDA(cudaEventRecord(t_ph.b, s));
    JFC_CUDA(cudaEventSynchronize(t_ph.b));
    st.ms_push_relabel += elapsed_ms(t_ph.a, t_ph.b);

    JFC_CUDA(cudaEventRecord(t_ph.a, s));
    rc = run_bfs(ctx, ts, p, false, st.bfs_passes, &active, nullptr);
    JFC_CUDA(cudaEventRecord(t_ph.b, s));
    JFC_CUDA(cudaEventSynchronize(t_ph.b));
    st.ms_global_relabel += elapsed_ms(t_ph.a, t_ph.b);
    ++st.global_relabels;
    if (rc) return rc;
  }
  if (status != JFC_OK) {
    for (int g = 0; g < ts.ngrids; ++g)
      if (active[g] > 0) res[g].status = status;
  }

  // canonical cut: nodes reachable from excess in the final residual graph
  int bad = 0;
  JFC_CUDA(cudaEventRecord(t_ph.a, s));
  rc = run_bfs(ctx, ts, p, true, st.bfs_passes, nullptr, &bad);
  if (rc) return rc;
  JFC_CUDA(launch_grid_sums(ts, s));
  JFC_CUDA(cudaEventRecord(t_ph.b, s));
  rc = pin_reserve(ctx, sizeof(long long) * 2 * (size_t)ts.ngrids + 64);
  if (rc) return rc;
  long long* hs = (long long*)ctx->h_pin;
  JFC_CUDA(cudaMemcpyAsync(hs, ts.d_grid_sum, sizeof(long long) * 2 * ts.ngrids, cudaMemcpyDeviceToHost, s));
  unsigned long long visits = 0;
  JFC_CUDA(cudaMemcpyAsync(&visits, &ts.d_ctr->visits, sizeof(visits), cudaMemcpyDeviceToHost, s));
  JFC_CUDA(cudaEventRecord(t_all.b, s));
  JFC_CUDA(cudaStreamSynchronize(s));
  st.ms_cut = elapsed_ms(t_ph.a, t_ph.b);
  st.ms_total = elapsed_ms(t_all.a, t_all.b);
  st.tile_visits = (long long)visits;
  for (int g = 0; g < ts.ngrids; ++g) {
    res[g].neg_sum = hs[2 * g];
    res[g].labels = hs[2 * g + 1];
  }
  if (bad && status == JFC_OK) {
    status = set_error(JFC_ERR_NOT_CONVERGED, "cut BFS reached a deficit node");
    for (auto& r : res) r.status = status;
  }
  st.status = status;
  return status;
}
