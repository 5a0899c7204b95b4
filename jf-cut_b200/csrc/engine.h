// engine.h — host-side engine shared by the plain solver, the batch and the
// server (C++ only; not part of the C ABI).
#pragma once

#include <string>
#include <vector>

#include "jfc_internal.h"

struct jfc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;     // the stream every launch of this context uses
  cudaStream_t own_stream = nullptr; // the context's own stream
  jfc_params params{};
  void* h_pin = nullptr;         // pinned host scratch for counter read-back
  size_t h_pin_bytes = 0;
};

// Colour model + inputs kept on the device for warm seed edits.
struct DevModel {
  bool valid = false;
  BuildModelDev m{};
  void* d_img = nullptr;
  uint8_t* d_seeds = nullptr;
  int* d_lut_s = nullptr;        // t-link tables [JFC_TQ + 1]
  int* d_lut_t = nullptr;
  int lut_lambda_t = -1;         // lambda_t the t-link tables hold (-1: none)
  size_t img_bytes = 0;
};

struct jfc_graph {
  jfc_ctx* ctx = nullptr;
  int device = 0;
  int dims = 2, W = 0, H = 0, D = 1, conn = 4;
  GridDev g{};                   // tile fields unset; pointers into d_state
  void* d_state = nullptr;
  size_t state_bytes = 0;
  long long sink_total = 0;      // sum of sink t-link capacities (int64)
  int state = 0;                 // 0 empty, 1 graph loaded, 2 solved
  long long flow = 0;
  long long source_nodes = 0;
  TileSet ts;                    // tile set of this graph alone
  int ts_shape = -1;             // tile shape the tile set was built for
  DevModel model;
  jfc_stats last{};
};

// Per-grid result of an engine run.
struct GridResult {
  long long neg_sum = 0;
  long long labels = 0;
  int status = JFC_OK;
};

// Solve every grid of `ts` to the exact max-flow (engine.cpp).
// fast_grid: with p.pr_mode == 1, the single grid the Fast-Cut line sweeps run
// on instead of the block-wise push-relabel phases.
int engine_solve(jfc_ctx* ctx, TileSet& ts, const jfc_params& p, std::vector<GridResult>& res,
                 jfc_stats& st, const GridDev* fast_grid = nullptr);
// One BFS to its fixpoint in one persistent launch and its read-back: global
// relabel (cut = false; active[g] = active tiles of grid g afterwards) or the
// source-side cut (cut = true).  sweeps_done reports the sweeps of the
// push-relabel phase that ran before it.
int engine_bfs(jfc_ctx* ctx, TileSet& ts, const jfc_params& p, bool cut, int& passes,
               std::vector<int>* active, int* cut_bad, int* sweeps_done);
// Cut BFS + per-grid sums (min(e, 0), source-side count) of every grid of ts.
int engine_cut(jfc_ctx* ctx, TileSet& ts, const jfc_params& p, std::vector<GridResult>& res, int& passes);
// Build / free a tile set over grids (all of one dimensionality).  The control
// block is reused while it is large enough.  With a stream the grid and tile
// tables are uploaded asynchronously from pinned staging (rewrite it only
// after the next host sync on that stream) and a new block gets headroom.
int tileset_build(TileSet& ts, int dims, int tile_rows, int tile_depth, const std::vector<GridDev>& grids,
                  cudaStream_t s = nullptr, bool pr_split = false);
void tileset_free(TileSet& ts);
// Drop the tile set's captured relabel-cycle graphs.
void tileset_drop_graphs(TileSet& ts);
int shape_code(int dims, int tile_rows, int tile_depth, bool pr_split);
// 2D 32x16 tile sets run push-relabel on 32x8 halves unless pr_mode == 2
bool pr_split_for(const jfc_params& p, int dims);
// Sweep pairs between global relabels: relabel_interval, or when it is 0 the
// measured best per dimensionality (2D: relabels are cheap next to the
// push-relabel sweeps; 3D: the relabel dominates and runs less often).
inline int interval_for(const jfc_params& p, int dims) {
  return p.relabel_interval > 0 ? p.relabel_interval : (dims == 2 ? 2 : 3);
}
// Push-relabel visit scheduling (1 sweeps, 2 worklist, 3 sweeps while many
// tiles are active and the worklist in the tail): pr_sched, or the sweeps when
// it is 0 (engine_solve then switches to the worklist after the exact relabel).
inline int pr_sched_for(const jfc_params& p) { return p.pr_sched >= 1 && p.pr_sched <= 3 ? p.pr_sched : 1; }
// Distance cap of the global relabels while solving (0: none): relabel_cap,
// or when it is 0 the measured default per dimensionality.  The Fast-Cut
// comparison mode keeps the reference's exact relabels.
inline int relabel_cap_for(const jfc_params& p, int dims) {
  if (p.pr_mode == 1 || p.relabel_cap < 0) return 0;
  return p.relabel_cap > 0 ? p.relabel_cap : (dims == 2 ? 256 : 128);
}

int set_error(int code, const std::string& msg);
int cuda_status(cudaError_t e, const char* where);
#define JFC_CUDA(call)                                   \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return cuda_status(_e, #call); \
  } while (0)

void fill_defaults(jfc_params& p);

// solver.cpp: graph layout, capacity build and plane copies
size_t align256(size_t v);
size_t state_bytes(int dims, int w, int h, int d);
void model_defaults(jfc_model& m);
int build_core(jfc_graph* G, const void* img, int pixfmt, const uint8_t* seeds, const jfc_model* mdl,
               cudaMemcpyKind kind);
// Free a graph whose last use was ordered on stream `s` (or completed) without
// synchronising the device: its memory goes back to the pool when `s` reaches
// the free (the server's solver thread, while other streams keep running).
void graph_release(jfc_graph* G, cudaStream_t s);
// Copy a dense array into (to_dense false) or out of a padded plane of G.
cudaError_t copy_plane(void* padded, const void* dense, size_t elem, const jfc_graph* G, bool to_dense,
                       cudaMemcpyKind kind, cudaStream_t s);
double elapsed_ms(cudaEvent_t a, cudaEvent_t b);
