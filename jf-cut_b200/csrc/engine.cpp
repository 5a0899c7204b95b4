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

#include <cuda.h>   // CUtensorMap and the tensor-map encode function's types

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>

static thread_local std::string g_err;
static std::atomic<unsigned long long> g_launches{0};

// launches recorded while a stream is captured run later as graph nodes and
// are counted when the graph is launched
static thread_local bool g_capturing = false;

void jfc_note_launch(int n) {
  if (!g_capturing) g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed);
}

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
  // 2D tiles 32 x 8 by default: with the relabel worklist the small tiles no
  // longer cost relabel passes, and their visits are the shortest
  if (p.tile_rows != 8 && p.tile_rows != 16) p.tile_rows = 8;
  // 3D tile depth: 0 = automatic (32 x 4 x 2 tiles); 4 needs tile_rows 16
  if (p.tile_depth == 4 && p.tile_rows == 8) p.tile_depth = 2;
  if (p.tile_depth != 1 && p.tile_depth != 2 && p.tile_depth != 4) p.tile_depth = 0;
  if (p.pr_mode != 1 && p.pr_mode != 2) p.pr_mode = 0;
  if (p.local_iters <= 0) p.local_iters = 12;
  if (p.relabel_interval < 0) p.relabel_interval = 0;   // 0: automatic per dimensionality
  if (p.relabel_interval_max <= 0 || p.relabel_interval_max < p.relabel_interval)
    p.relabel_interval_max = std::max(64, 16 * p.relabel_interval);
  if (p.max_sweeps <= 0) p.max_sweeps = 1 << 20;
  if (p.max_bfs_passes <= 0) p.max_bfs_passes = 1 << 20;
  if (p.spin_limit < 0) p.spin_limit = 0;   // 0: the device default (2^26 polls)
}

double elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return (double)ms;
}

int shape_code(int dims, int tile_rows, int tile_depth, bool pr_split) {
  return dims * 1000 + tile_rows * 10 + (dims == 3 ? tile_depth : 0) + (pr_split ? 100000 : 0);
}

bool pr_split_for(const jfc_params& p, int dims) { return dims == 2 && p.tile_rows == 16 && p.pr_mode != 2; }

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// (blocks from the stream-ordered allocator are freed without a device
// synchronisation: nothing may still run on them)
void tileset_free(TileSet& ts) {
  tileset_drop_graphs(ts);
  if (ts.d_block) cudaFree(ts.d_block);
  if (ts.h_stage) cudaFreeHost(ts.h_stage);
  ts = TileSet();
}

// Tensor maps of one grid (three CUtensorMap): the push-relabel staging
// ([0] planes, [1] h with halo) and the 3D relabel frontier's ([1] and [2]
// the arc-byte plane).
constexpr size_t kTmapBytes = 3 * sizeof(CUtensorMap);
// 0: visits load their tiles with ordinary loads (a comparison build)
#ifndef JFC_PR_TMA
#define JFC_PR_TMA 1
#endif

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tiled tensor-map encoder (resolved once; null when absent).
static EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Encode grid g's staging maps for visits of 32 x ty x tz nodes into out[3]:
//  [0] the planes {e, h, r[0..K-1]} as one 4D tensor {pitch, Hp, Dp, planes},
//      box {32, ty, tz, planes};
//  [1] the h plane {pitch, Hp, Dp}, box {40, ty + 2, tz + 2 (1 in 2D)} (the
//      tile and its one-cell halo, starting 4 columns left of the tile);
//  [2] the arc-byte (label) plane {pitch, Hp, Dp} of bytes, box {32, ty, tz}.
// Returns false when the planes are not one evenly spaced run or a map is
// refused; the tile set then stages with ordinary loads.
static bool encode_pr_maps(const GridDev& g, int ty, int tz, CUtensorMap* out) {
  const EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const int K = g.dims == 2 ? 4 : 6;
  const long long pb = (long long)((const char*)g.h - (const char*)g.e);
  if (pb < g.plane * 4 || pb % 16 || (size_t)g.e % 16 || (g.pitch * 4) % 16) return false;
  for (int k = 0; k < K; ++k)
    if ((const char*)g.r[k] != (const char*)g.e + (2 + k) * pb) return false;
  const cuuint64_t row = (cuuint64_t)g.pitch * 4, slab = row * (cuuint64_t)g.Hp;
  const cuuint64_t dims4[4] = {(cuuint64_t)g.pitch, (cuuint64_t)g.Hp, (cuuint64_t)g.Dp, (cuuint64_t)(2 + K)};
  const cuuint64_t str4[3] = {row, slab, (cuuint64_t)pb};
  const cuuint32_t box4[4] = {32u, (cuuint32_t)ty, (cuuint32_t)tz, (cuuint32_t)(2 + K)};
  const cuuint32_t unit[4] = {1u, 1u, 1u, 1u};
  if (fn(&out[0], CU_TENSOR_MAP_DATA_TYPE_INT32, 4, g.e, dims4, str4, box4, unit, CU_TENSOR_MAP_INTERLEAVE_NONE,
         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  const cuuint32_t box3[3] = {40u, (cuuint32_t)(ty + 2), (cuuint32_t)(g.dims == 3 ? tz + 2 : 1)};
  if (fn(&out[1], CU_TENSOR_MAP_DATA_TYPE_INT32, 3, g.h, dims4, str4, box3, unit, CU_TENSOR_MAP_INTERLEAVE_NONE,
         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  if ((size_t)g.label % 16 || g.pitch % 16) return false;
  const cuuint64_t strb[2] = {(cuuint64_t)g.pitch, (cuuint64_t)g.pitch * (cuuint64_t)g.Hp};
  const cuuint32_t boxb[3] = {32u, (cuuint32_t)ty, (cuuint32_t)tz};
  if (fn(&out[2], CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, g.label, dims4, strb, boxb, unit, CU_TENSOR_MAP_INTERLEAVE_NONE,
         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  return true;
}

// Carve the control block for cap_tiles tiles / cap_grids grids.
static void tileset_carve(TileSet& ts, char* blk, size_t* total) {
  const size_t nt = (size_t)ts.cap_tiles, ng = (size_t)ts.cap_grids;
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off = align_up(off + bytes, 256); return o; };
  const size_t o_desc = take(sizeof(GridDev) * ng);
  const size_t o_info = take(sizeof(int4) * nt);
  const size_t o_fpr = take(sizeof(int) * nt * 2);   // half-tile work items
  size_t o_qpr[2][2];
  for (int p = 0; p < 2; ++p)
    for (int b = 0; b < 2; ++b) o_qpr[p][b] = take(sizeof(int) * nt);
  const size_t o_fb0 = take(sizeof(int) * nt);
  const size_t o_fb1 = take(sizeof(int) * nt);
  const size_t o_qb0 = take(sizeof(int) * nt);
  const size_t o_qb1 = take(sizeof(int) * nt);
  const size_t o_act = take(nt);
  const size_t o_gact = take(sizeof(int) * ng);
  const size_t o_sum = take(sizeof(long long) * 2 * ng);
  const size_t o_ctr = take(sizeof(DevCounters));
  const size_t o_ring = take(sizeof(unsigned long long) * nt * 2);   // work items: halves of split tiles
  const size_t o_lock = take(sizeof(int) * nt * 2);
  const size_t o_tmap = take(kTmapBytes * ng);
  *total = off;
  if (!blk) return;
  ts.d_desc = (GridDev*)(blk + o_desc);
  ts.d_info = (int4*)(blk + o_info);
  ts.d_flag_pr = (int*)(blk + o_fpr);
  for (int p = 0; p < 2; ++p)
    for (int b = 0; b < 2; ++b) ts.d_q_pr[p][b] = (int*)(blk + o_qpr[p][b]);
  ts.d_flag_bfs[0] = (int*)(blk + o_fb0);
  ts.d_flag_bfs[1] = (int*)(blk + o_fb1);
  ts.d_q_bfs[0] = (int*)(blk + o_qb0);
  ts.d_q_bfs[1] = (int*)(blk + o_qb1);
  ts.d_act = (uint8_t*)(blk + o_act);
  ts.d_grid_active = (int*)(blk + o_gact);
  ts.d_grid_sum = (long long*)(blk + o_sum);
  ts.d_ctr = (DevCounters*)(blk + o_ctr);
  ts.d_pr_ring = (unsigned long long*)(blk + o_ring);
  ts.d_pr_lock = (int*)(blk + o_lock);
  ts.tmap_slot = blk + o_tmap;
}

int tileset_build(TileSet& ts, int dims, int tile_rows, int tile_depth, const std::vector<GridDev>& grids_in,
                  cudaStream_t s, bool pr_split) {
  int TY, TZ;
  if (dims == 2) {
    TY = tile_rows; TZ = 1;
  } else {
    // automatic 3D shape: 32 x 4 x 2 (measured best on the video workload:
    // small tiles in y and z keep the relabel and push waves moving)
    TZ = tile_depth > 0 ? tile_depth : 2;
    TY = tile_depth > 0 ? tile_rows / tile_depth : 4;
  }
  std::vector<GridDev> grids = grids_in;
  int base = 0, npar[2] = {0, 0};
  for (size_t gi = 0; gi < grids.size(); ++gi) {
    GridDev& g = grids[gi];
    if (g.dims != dims) return set_error(JFC_ERR_INVALID_ARG, "tile set mixes 2D and 3D grids");
    g.tiles_x = g.pitch / JFC_TW;
    g.tiles_y = g.Hp / TY;
    g.tiles_z = g.Dp / TZ;
    g.tile_base = base;
    base += g.tiles_x * g.tiles_y * g.tiles_z;
  }
  const int ntiles = base, ngrids = (int)grids.size();
  // reuse the control block while it is large enough (the server re-forms its
  // tile sets between relabels); otherwise allocate with headroom when asked
  // to stage asynchronously
  if (!ts.d_block || ts.cap_tiles < ntiles || ts.cap_grids < ngrids) {
    if (s) {
      // stream-ordered: the old block goes back to the pool when `s` reaches
      // the free, and nothing waits for the other streams' work (the server
      // grows its tile sets while builds run); the pinned staging is kept
      tileset_drop_graphs(ts);
      if (ts.d_block) JFC_CUDA(cudaFreeAsync(ts.d_block, s));
      ts.d_block = nullptr;
    } else {
      tileset_free(ts);
    }
    ts.cap_tiles = s ? ntiles + ntiles / 4 + 64 : ntiles;
    ts.cap_grids = s ? ngrids + ngrids / 4 + 8 : ngrids;
    if (ts.cap_tiles < 1) ts.cap_tiles = 1;
    if (ts.cap_grids < 1) ts.cap_grids = 1;
    size_t total = 0;
    tileset_carve(ts, nullptr, &total);
    char* blk = nullptr;
    if (s) JFC_CUDA(cudaMallocAsync((void**)&blk, total, s));
    else JFC_CUDA(cudaMalloc((void**)&blk, total));
    ts.d_block = blk;
    ts.block_bytes = total;
    tileset_carve(ts, blk, &total);
    // on the caller's stream when staging asynchronously: the table uploads
    // below are ordered after it (a legacy-stream memset is not ordered with a
    // non-blocking stream)
    if (s) JFC_CUDA(cudaMemsetAsync(blk, 0, total, s));
    else JFC_CUDA(cudaMemset(blk, 0, total));
  }
  tileset_drop_graphs(ts);   // captured launches hold the old tile set by value
  ts.dims = dims;
  ts.TR = tile_rows; ts.TY = TY; ts.TZ = TZ;
  ts.pr_split = pr_split && dims == 2 && TY == 16 ? 1 : 0;
  ts.ngrids = ngrids;
  ts.ntiles = ntiles;
  const size_t desc_bytes = sizeof(GridDev) * (size_t)ngrids, info_bytes = sizeof(int4) * (size_t)ntiles;
  const size_t tmap_bytes = kTmapBytes * (size_t)ngrids;
  const size_t o_maps = align_up(align_up(desc_bytes, 256) + info_bytes, 256);
  const size_t stage = o_maps + tmap_bytes;
  int4* info;
  if (s) {
    if (ts.h_stage_bytes < stage) {
      if (ts.h_stage) cudaFreeHost(ts.h_stage);
      ts.h_stage = nullptr;
      ts.h_stage_bytes = 0;
      JFC_CUDA(cudaMallocHost(&ts.h_stage, stage + stage / 4));
      ts.h_stage_bytes = stage + stage / 4;
    }
    std::memcpy(ts.h_stage, grids.data(), desc_bytes);
    info = (int4*)((char*)ts.h_stage + align_up(desc_bytes, 256));
  } else {
    static thread_local std::vector<int4> v;
    v.resize(ntiles);
    info = v.data();
  }
  // staging tensor maps (visits of the push-relabel shape: 32 x 8 halves of
  // split 32 x 16 tiles)
  static thread_local std::vector<CUtensorMap> mv;
  CUtensorMap* maps;
  if (s) {
    maps = (CUtensorMap*)((char*)ts.h_stage + o_maps);
  } else {
    mv.resize(3 * (size_t)ngrids);
    maps = mv.data();
  }
  bool tma = JFC_PR_TMA && ngrids > 0;
  for (int gi = 0; gi < ngrids && tma; ++gi)
    tma = encode_pr_maps(grids[gi], ts.pr_split ? 8 : TY, TZ, maps + 3 * gi);
  npar[0] = npar[1] = 0;
  size_t k = 0;
  for (size_t gi = 0; gi < grids.size(); ++gi) {
    const GridDev& g = grids[gi];
    for (int tz = 0; tz < g.tiles_z; ++tz)
      for (int ty = 0; ty < g.tiles_y; ++ty)
        for (int tx = 0; tx < g.tiles_x; ++tx) {
          info[k++] = make_int4((int)gi, tx, ty, tz);
          ++npar[(tx + ty + tz) & 1];
        }
  }
  ts.nlist[0] = npar[0];
  ts.nlist[1] = npar[1];
  ts.d_tmap = tma ? ts.tmap_slot : nullptr;
  if (s) {
    // the staging buffer is rewritten only after the next host sync on `s`
    if (desc_bytes) JFC_CUDA(cudaMemcpyAsync(ts.d_desc, ts.h_stage, desc_bytes, cudaMemcpyHostToDevice, s));
    if (info_bytes) JFC_CUDA(cudaMemcpyAsync(ts.d_info, info, info_bytes, cudaMemcpyHostToDevice, s));
    if (tma) JFC_CUDA(cudaMemcpyAsync((void*)ts.d_tmap, maps, tmap_bytes, cudaMemcpyHostToDevice, s));
  } else {
    if (desc_bytes) JFC_CUDA(cudaMemcpy(ts.d_desc, grids.data(), desc_bytes, cudaMemcpyHostToDevice));
    if (info_bytes) JFC_CUDA(cudaMemcpy(ts.d_info, info, info_bytes, cudaMemcpyHostToDevice));
    if (tma) JFC_CUDA(cudaMemcpy((void*)ts.d_tmap, maps, tmap_bytes, cudaMemcpyHostToDevice));
  }
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

static size_t pin_need(const TileSet& ts) {
  return sizeof(DevCounters) + sizeof(long long) * 2 * (size_t)ts.ngrids + 64;
}

// pinned slot holding the sweep pairs of the next push-relabel phase and the
// distance cap of the relabel after it (after the read-back area); copied to
// the control block (pr_sweeps, h_cap) by the cycle itself
static int* pin_sweeps(jfc_ctx* ctx, const TileSet& ts) {
  return (int*)((char*)ctx->h_pin + (pin_need(ts) + 255) / 256 * 256);
}
static size_t pin_need_cycle(const TileSet& ts) { return (pin_need(ts) + 255) / 256 * 256 + 64; }

// Enqueue one BFS (global relabel when !cut, cut otherwise) and the read-back
// of its counters (+ per-grid active tiles) into pinned memory `pin`.
static cudaError_t enqueue_bfs(TileSet& ts, bool cut, int max_passes, cudaStream_t s, void* pin) {
  cudaError_t e;
#define JFC_E(call) do { e = (call); if (e != cudaSuccess) return e; } while (0)
  JFC_E(cudaMemsetAsync(ts.d_flag_bfs[0], 0, sizeof(int) * (size_t)ts.ntiles, s));
  JFC_E(cudaMemsetAsync(ts.d_flag_bfs[1], 0, sizeof(int) * (size_t)ts.ntiles, s));
  if (!cut) JFC_E(cudaMemsetAsync(ts.d_grid_active, 0, sizeof(int) * ts.ngrids, s));
  // reset the BFS part of the control block: tickets, frontiers, status, cut flag
  JFC_E(cudaMemsetAsync(ts.d_ctr->ticket, 0, sizeof(ts.d_ctr->ticket), s));
  JFC_E(cudaMemsetAsync(ts.d_ctr->qn_bfs, 0, sizeof(ts.d_ctr->qn_bfs), s));
  JFC_E(cudaMemsetAsync(&ts.d_ctr->bfs_status, 0, sizeof(int), s));
  if (cut) JFC_E(cudaMemsetAsync(&ts.d_ctr->cut_bad, 0, sizeof(int), s));
  JFC_E(launch_bfs(ts, cut, max_passes, s));
  JFC_E(cudaMemcpyAsync(pin, ts.d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
  if (!cut)
    JFC_E(cudaMemcpyAsync((char*)pin + sizeof(DevCounters), ts.d_grid_active, sizeof(int) * ts.ngrids,
                          cudaMemcpyDeviceToHost, s));
#undef JFC_E
  return cudaSuccess;
}

// Outcome of a BFS from the pinned read-back (after the stream sync).
static int finish_bfs(const TileSet& ts, bool cut, const void* pin, int& passes, std::vector<int>* active,
                      int* cut_bad, int* sweeps_done) {
  const DevCounters* hc = (const DevCounters*)pin;
  const int* hact = (const int*)((const char*)pin + sizeof(DevCounters));
  passes += hc->bfs_passes;
  if (sweeps_done) *sweeps_done = hc->sweeps_done;
  if (hc->error) return set_error(JFC_ERR_CUDA, "a device-side wait timed out in a persistent kernel (grid barrier, worklist or tile staging)");
  if (hc->bfs_status == 2) return set_error(JFC_ERR_NOT_CONVERGED, "BFS pass budget exhausted");
  if (!cut && active) {
    active->resize(ts.ngrids);
    for (int g = 0; g < ts.ngrids; ++g) (*active)[g] = hact[g];
  }
  if (cut && cut_bad) *cut_bad = hc->cut_bad;
  return JFC_OK;
}

// Run one BFS to its fixpoint in one persistent launch, then read back its
// outcome (the only host sync of a relabel cycle).  On return (relabel)
// active[g] holds the active tiles of every grid.
int engine_bfs(jfc_ctx* ctx, TileSet& ts, const jfc_params& p, bool cut, int& passes,
               std::vector<int>* active, int* cut_bad, int* sweeps_done) {
  cudaStream_t s = ctx->stream;
  int rc = pin_reserve(ctx, pin_need(ts));
  if (rc) return rc;
  JFC_CUDA(enqueue_bfs(ts, cut, p.max_bfs_passes, s, ctx->h_pin));
  JFC_CUDA(cudaStreamSynchronize(s));
  return finish_bfs(ts, cut, ctx->h_pin, passes, active, cut_bad, sweeps_done);
}

// ---- CUDA graphs of the relabel cycle -------------------------------------
// One cycle = { push-relabel phase (interval sweeps), global relabel, counter
// read-back }: ~10 stream operations between two host syncs.  They are
// captured once per (interval, local_iters, pass budget, read-back buffer)
// and replayed with one graph launch.  The cache belongs to the tile set and
// is dropped whenever the tile set changes.
namespace {
struct CycleGraphs {
  struct Entry {
    int local_iters, max_passes, sched;
    void* pin;
    cudaGraphExec_t exec;
  };
  std::vector<Entry> v;
  bool broken = false;   // capture not available on this stream: direct launches
};
}  // namespace

void tileset_drop_graphs(TileSet& ts) {
  if (!ts.gcache) return;
  CycleGraphs* c = (CycleGraphs*)ts.gcache;
  for (auto& e : c->v) cudaGraphExecDestroy(e.exec);
  delete c;
  ts.gcache = nullptr;
}

static cudaError_t enqueue_cycle(TileSet& ts, const int* pin_sw, int local_iters, int max_passes, int sched,
                                 cudaStream_t s, void* pin) {
  cudaError_t e = cudaMemsetAsync(ts.d_ctr->ticket, 0, sizeof(ts.d_ctr->ticket), s);
  static_assert(offsetof(DevCounters, h_cap) == offsetof(DevCounters, pr_sweeps) + sizeof(int),
                "pr_sweeps and h_cap are copied together");
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ts.d_ctr->pr_sweeps, pin_sw, 2 * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = launch_pr_phase(ts, 0, local_iters, s, sched);
  if (e == cudaSuccess) e = enqueue_bfs(ts, false, max_passes, s, pin);
  return e;
}

static cudaGraphExec_t cycle_graph(TileSet& ts, const int* pin_sw, int local_iters, int max_passes, int sched,
                                   cudaStream_t s, void* pin) {
  if (!ts.gcache) ts.gcache = new CycleGraphs();
  CycleGraphs* c = (CycleGraphs*)ts.gcache;
  if (c->broken) return nullptr;
  for (auto& e : c->v)
    if (e.local_iters == local_iters && e.max_passes == max_passes && e.sched == sched && e.pin == pin)
      return e.exec;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    c->broken = true;   // the caller is capturing this stream itself
    return nullptr;
  }
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    c->broken = true;
    return nullptr;
  }
  g_capturing = true;
  const cudaError_t e1 = enqueue_cycle(ts, pin_sw, local_iters, max_passes, sched, s, pin);
  g_capturing = false;
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(s, &g);
  cudaGraphExec_t x = nullptr;
  if (e1 == cudaSuccess && e2 == cudaSuccess && g) {
    if (cudaGraphInstantiate(&x, g, 0) != cudaSuccess) x = nullptr;
  }
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();   // a refused capture leaves no sticky error
  if (!x) {
    c->broken = true;
    return nullptr;
  }
  c->v.push_back({local_iters, max_passes, sched, pin, x});
  return x;
}

// One relabel cycle, replayed from a graph when enabled; returns the outcome
// of its global relabel.
static int run_cycle(jfc_ctx* ctx, TileSet& ts, const jfc_params& p, int interval, int h_cap, int local_iters,
                     int sched, int& passes, std::vector<int>& active, int* sweeps_done, bool* used_graph) {
  cudaStream_t s = ctx->stream;
  int rc = pin_reserve(ctx, pin_need_cycle(ts));
  if (rc) return rc;
  int* pin_sw = pin_sweeps(ctx, ts);
  pin_sw[0] = interval;   // the previous cycle's copies finished at its sync
  pin_sw[1] = h_cap;
  cudaGraphExec_t x = p.use_graph ? cycle_graph(ts, pin_sw, local_iters, p.max_bfs_passes, sched, s, ctx->h_pin)
                                  : nullptr;
  if (x) {
    JFC_CUDA(cudaGraphLaunch(x, s));
    jfc_note_launch(2);
    if (used_graph) *used_graph = true;
  } else {
    JFC_CUDA(enqueue_cycle(ts, pin_sw, local_iters, p.max_bfs_passes, sched, s, ctx->h_pin));
  }
  JFC_CUDA(cudaStreamSynchronize(s));
  return finish_bfs(ts, false, ctx->h_pin, passes, &active, nullptr, sweeps_done);
}

int engine_cut(jfc_ctx* ctx, TileSet& ts, const jfc_params& p, std::vector<GridResult>& res, int& passes) {
  cudaStream_t s = ctx->stream;
  res.assign(ts.ngrids, GridResult());
  int bad = 0;
  int rc = engine_bfs(ctx, ts, p, true, passes, nullptr, &bad, nullptr);
  if (rc) return rc;
  JFC_CUDA(launch_grid_sums(ts, s));
  rc = pin_reserve(ctx, pin_need(ts));
  if (rc) return rc;
  long long* hs = (long long*)ctx->h_pin;
  JFC_CUDA(cudaMemcpyAsync(hs, ts.d_grid_sum, sizeof(long long) * 2 * ts.ngrids, cudaMemcpyDeviceToHost, s));
  JFC_CUDA(cudaStreamSynchronize(s));
  for (int g = 0; g < ts.ngrids; ++g) {
    res[g].neg_sum = hs[2 * g];
    res[g].labels = hs[2 * g + 1];
  }
  if (bad) {
    rc = set_error(JFC_ERR_NOT_CONVERGED, "cut BFS reached a deficit node");
    for (auto& r : res) r.status = rc;
  }
  return rc;
}

int engine_solve(jfc_ctx* ctx, TileSet& ts, const jfc_params& p_in, std::vector<GridResult>& res,
                 jfc_stats& st, const GridDev* fast_grid) {
  jfc_params p = p_in;
  fill_defaults(p);
  cudaStream_t s = ctx->stream;
  std::memset(&st, 0, sizeof(st));
  res.assign(ts.ngrids, GridResult());
  cudaEvent_t ev[4];
  for (auto& e : ev) cudaEventCreate(&e);
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() { for (int i = 0; i < 4; ++i) cudaEventDestroy(e[i]); }
  } ev_free{ev};
  JFC_CUDA(cudaEventRecord(ev[0], s));
  JFC_CUDA(launch_clear_counters(ts, s));
  // capped relabels while solving (the first one included), then one exact
  // relabel certifies the result
  int h_cap = relabel_cap_for(p, ts.dims);   // cap of the next relabel
  int last_cap = h_cap;                       // cap the last relabel ran with
  if (p.spin_limit > 0 || h_cap > 0)
    JFC_CUDA(launch_set_limits(ts, (unsigned long long)p.spin_limit, h_cap, s));
#ifndef JFC_NO_PREPUSH
  if (p.pr_mode != 1) JFC_CUDA(launch_prepush(ts, s));   // the Fast-Cut comparison stays as it was
#endif
  std::vector<int> active;
  int rc;

  // initial global relabel (exact sink distances; fills the work queues)
  rc = engine_bfs(ctx, ts, p, false, st.bfs_passes, &active, nullptr, nullptr);
  if (rc) return rc;
  st.global_relabels = 1;

  auto total = [&]() { long long t = 0; for (int v : active) t += v; return t; };
  const DevCounters* hc = (const DevCounters*)ctx->h_pin;
  double prev_pr = 0.0, prev_gr = 0.0, prev_grf = 0.0;
  unsigned long long prev_vis = 0;
  if (p.verbose) {   // the first relabel's share
    const DevCounters* c0 = (const DevCounters*)ctx->h_pin;
    prev_gr = (c0->ns_gr_first + c0->ns_gr_frontier) * 1e-6;
    prev_grf = c0->ns_gr_first * 1e-6;
    prev_vis = c0->bfs_visits;
    fprintf(stderr, "{\"relabel\": 1, \"active_tiles\": %lld, \"ms_gr\": %.3f, \"ms_gr_dense\": %.3f, "
                    "\"gr_passes\": %d, \"gr_visits\": %llu}\n",
            [&]() { long long t = 0; for (int v : active) t += v; return t; }(), prev_gr, prev_grf, c0->bfs_passes,
            c0->bfs_visits);
  }
  int status = JFC_OK;
  // Adaptive schedule: while a large part of the grid is active, frequent
  // global relabels pay off; once only a sliver is active (long transport
  // paths, few tiles), the dense relabel dominates, so the interval doubles
  // (the push-relabel phase still stops as soon as its queues drain).
  //  The interval also doubles while the last relabel cost more than twice
  // the push-relabel phase before it (device clocks) and that phase used all
  // its sweeps: the relabel is then the bottleneck and is amortised.
  const int interval0 = interval_for(p, ts.dims);
  int interval = interval0;
  const int tail_iters = p.local_iters_tail > 0 ? p.local_iters_tail
                         : p.local_iters_tail < 0 ? p.local_iters : std::min(2 * p.local_iters, 64);
  bool graphs = false;
  double fast_ms = 0.0;   // Fast-Cut iterations (event-timed: many small launches)
  unsigned long long last_pr = 0, last_gr = 0;
  bool post_exact = false;   // the exact relabel ran and found reachable excess
  {
    const DevCounters* c0 = (const DevCounters*)ctx->h_pin;
    last_pr = c0->ns_pr;
    last_gr = c0->ns_gr_first + c0->ns_gr_frontier;
  }
  for (;;) {
  while (total() > 0) {
    if (st.sweeps >= p.max_sweeps) {
      status = set_error(JFC_ERR_NOT_CONVERGED, "sweep budget exhausted");
      break;
    }
    // relabel_interval x (even sweep, odd sweep), global relabel, active-tile
    // count: one host read-back per cycle
    int sw = 0;
    if (p.pr_mode == 1 && fast_grid) {
      // Fast-Cut comparison: `interval` line-sweep iterations, then the
      // exact global relabel and convergence test
      cudaEvent_t f0 = ev[2], f1 = ev[3];
      JFC_CUDA(cudaEventRecord(f0, s));
      for (int it = 0; it < interval; ++it) JFC_CUDA(launch_fast_iteration(*fast_grid, &ts.d_ctr->fast_moved, s));
      JFC_CUDA(cudaEventRecord(f1, s));
      rc = engine_bfs(ctx, ts, p, false, st.bfs_passes, &active, nullptr, nullptr);
      if (rc) return rc;
      const double fms = elapsed_ms(f0, f1);
      fast_ms += fms;
      last_pr -= (unsigned long long)(fms * 1e6);   // the cost rule below sees the sweeps' time
      sw = 2 * interval;
    } else {
      // the long-path tail (a sliver of the tiles active): longer visits, so
      // excess crosses a whole tile per visit instead of per several sweeps
      const bool tail = total() * 256 < (long long)ts.ntiles;
      const int li = tail ? tail_iters : p.local_iters;
      // pr_sched 3: parity sweeps in the bulk, the worklist in the tail;
      // automatic: the worklist once the exact relabel found excess farther
      // than the cap from every deficit (a few tiles whose excess crosses
      // many tiles, where the sweeps would idle at their barriers)
      const int sched = pr_sched_for(p) == 3 ? (tail ? 2 : 1) : (p.pr_sched == 0 && post_exact) ? 2
                                                                                               : pr_sched_for(p);
      rc = run_cycle(ctx, ts, p, interval, h_cap, li, sched, st.bfs_passes, active, &sw, &graphs);
      last_cap = h_cap;
      ++st.pr_phases;
      if (rc) return rc;
    }
    st.sweeps += sw;
    {
      const DevCounters* c1 = (const DevCounters*)ctx->h_pin;
      const unsigned long long pr = c1->ns_pr - last_pr, gr = c1->ns_gr_first + c1->ns_gr_frontier - last_gr;
      last_pr = c1->ns_pr;
      last_gr = c1->ns_gr_first + c1->ns_gr_frontier;
      const bool sliver = total() * 256 < (long long)ts.ntiles;
      const bool relabel_bound = gr > 2 * pr && sw >= 2 * interval;
      if (sliver || relabel_bound) interval = std::min(interval * 2, p.relabel_interval_max);
      else interval = interval0;
    }
    ++st.global_relabels;
    if (p.verbose) {
      hc = (const DevCounters*)ctx->h_pin;
      const double pr = hc->ns_pr * 1e-6, gr = (hc->ns_gr_first + hc->ns_gr_frontier) * 1e-6;
      const double grf = hc->ns_gr_first * 1e-6;
      fprintf(stderr, "{\"relabel\": %d, \"sweeps\": %d, \"active_tiles\": %lld, \"ms_pr\": %.3f, \"ms_gr\": %.3f, "
                      "\"ms_gr_dense\": %.3f, \"gr_passes\": %d, \"gr_visits\": %llu}\n",
              st.global_relabels, st.sweeps, total(), pr - prev_pr, gr - prev_gr, grf - prev_grf, hc->bfs_passes,
              hc->bfs_visits - prev_vis);
      prev_vis = hc->bfs_visits;
      prev_pr = pr;
      prev_gr = gr;
      prev_grf = grf;
    }
  }
  // no active tile under the cap: one exact relabel decides.  Excess it finds
  // reachable (farther than the cap from every deficit) keeps the solve going
  // with exact relabels; none means the preflow is maximum.
  if (status != JFC_OK || last_cap == 0) break;
  h_cap = 0;
  last_cap = 0;
  JFC_CUDA(launch_set_limits(ts, (unsigned long long)p.spin_limit, 0, s));
  rc = engine_bfs(ctx, ts, p, false, st.bfs_passes, &active, nullptr, nullptr);
  if (rc) return rc;
  ++st.global_relabels;
  if (p.verbose)
    fprintf(stderr, "{\"relabel\": %d, \"exact\": true, \"active_tiles\": %lld}\n", st.global_relabels, total());
  if (total() == 0) break;
  post_exact = true;
  }
  if (status != JFC_OK) {
    for (int g = 0; g < ts.ngrids; ++g)
      if (active[g] > 0) res[g].status = status;
  }

  // canonical cut: nodes reachable from excess in the final residual graph
  JFC_CUDA(cudaEventRecord(ev[2], s));
  int passes = st.bfs_passes;
  std::vector<GridResult> cut;
  rc = engine_cut(ctx, ts, p, cut, passes);
  if (rc && rc != JFC_ERR_NOT_CONVERGED) return rc;
  st.bfs_passes = passes;
  JFC_CUDA(cudaEventRecord(ev[3], s));
  // device-clock phase times and visit counters
  unsigned long long* hv = (unsigned long long*)ctx->h_pin;
  JFC_CUDA(cudaMemcpyAsync(hv, &ts.d_ctr->visits, 15 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  JFC_CUDA(cudaEventRecord(ev[1], s));
  JFC_CUDA(cudaStreamSynchronize(s));
  st.ms_cut = elapsed_ms(ev[2], ev[3]);
  st.ms_total = elapsed_ms(ev[0], ev[1]);
  st.tile_visits = (long long)hv[0];
  st.bfs_visits = (long long)hv[1];
  st.pr_rounds = (long long)hv[2];
  st.ms_gr_first = hv[3] * 1e-6;
  st.ms_gr_frontier = hv[4] * 1e-6;
  st.ms_global_relabel = st.ms_gr_first + st.ms_gr_frontier;
  st.ms_push_relabel = hv[5] * 1e-6 + fast_ms;
  if (p.verbose >= 2)   // phase-clock split (non-zero in JFC_PHASE_CLOCK builds)
    fprintf(stderr, "{\"pr_cycles\": {\"stage\": %llu, \"local_relabel\": %llu, \"rounds\": %llu, \"exact_local\": %llu, "
                    "\"write_back\": %llu, \"grid_barrier\": %llu}}\n",
            hv[7], hv[8], hv[9], hv[12], hv[10], hv[11]);
  st.used_graph = graphs ? 1 : 0;
  for (int g = 0; g < ts.ngrids; ++g) {
    res[g].neg_sum = cut[g].neg_sum;
    res[g].labels = cut[g].labels;
    if (cut[g].status && !res[g].status) res[g].status = cut[g].status;
  }
  if (rc == JFC_ERR_NOT_CONVERGED && status == JFC_OK) status = rc;
  st.status = status;
  return status;
}
