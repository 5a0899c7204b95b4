// jfc_internal.h — shared device/host definitions of libjfcut.
//
// Data layout in HBM (one grid instance):
//   planes of int32 e (net excess), h (height), r[conn] (residual capacity of
//   the arc leaving the node in direction k, reference channel order), plus a
//   uint8 label plane.  Every plane is padded to pitch x Hp x Dp with
//   pitch = roundup(W, 32) and Hp / Dp multiples of the largest tile extent, so
//   a warp tile never needs a bounds check.  Padding nodes are inert: e = 0,
//   r = 0, h = INF (they have no residual arc in or out).
// Work is organised in warp tiles: 32 columns (one per lane) x TR rows (2D) or
// 32 x TY x TZ (3D); each lane keeps its column's state in registers.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "../../include/jfcut.h"

#define JFC_INF (1 << 30)
#define JFC_TW 32           // tile width = warp width
#define JFC_PAD_Y2 16       // 2D row padding (covers tile heights 4, 8, 16)
#define JFC_PAD_Y3 16       // 3D y padding (tile heights 4, 8, 16)
#define JFC_PAD_Z3 4        // 3D z padding (tile depths 1, 2, 4)
#define JFC_MAX_K 32        // k-means clusters per class
#define JFC_TQ 65536        // t-link probability quantisation

// Device-side descriptor of one grid instance.
struct GridDev {
  int dims, W, H, D;
  int pitch, Hp, Dp;
  int tiles_x, tiles_y, tiles_z;
  int tile_base;             // global id of this grid's first tile
  int h_cap;                 // distance cap of this grid's global relabels (0: the tile set's, h_cap
                             // of its control block)
  long long plane;           // pitch * Hp * Dp
  int* e;
  int* h;
  int* r[6];
  uint8_t* label;
};

// Device-side control state of one tile set (persistent phase kernels).
struct DevCounters {
  unsigned ticket[2];        // work tickets (alternate between phases)
  unsigned bar_count;        // grid barrier arrivals
  unsigned bar_gen;          // grid barrier generation
  int error;                 // a barrier wait timed out: kernels leave, host reports
  int cut_bad;               // cut BFS reached a deficit node (augmenting path left)
  int qn_pr[2][2];           // push-relabel queue lengths [parity][buffer]
  int cur_pr[2];             // pending buffer per parity
  int qn_bfs[2];             // BFS frontier lengths [buffer]
  int bfs_passes;            // passes of the last BFS
  int bfs_status;            // 1 converged, 2 pass budget exhausted
  int sweeps_done;           // sweeps run by the last push-relabel phase
  int pr_sweeps;             // sweep pairs of the next phase when launched with sweeps <= 0
  int h_cap;                 // global relabels: distances >= h_cap count as unreachable (0: no cap)
                             // (pr_sweeps and h_cap: a relabel cycle copies both at once)
  int fast_moved;            // a Fast-Cut push moved flow (comparison mode)
  unsigned long long visits; // push-relabel tile visits
  unsigned long long bfs_visits;
  unsigned long long rounds; // push/relabel rounds summed over visits
  unsigned long long ns_gr_first;     // global relabel: first (dense) pass, device ns
  unsigned long long ns_gr_frontier;  // global relabel: frontier passes + queue refill
  unsigned long long ns_pr;           // push-relabel phases, device ns
  unsigned long long t_gr_start;      // device clock at the start of the last relabel
  unsigned long long prof[8];         // SM-cycle split of push-relabel visits (JFC_PHASE_CLOCK builds)
  unsigned long long spin_limit;  // polls before a device-side wait gives up (0: 2^26)
  unsigned pr_head;          // push-relabel worklist: tickets taken
  unsigned pr_tail;          // push-relabel worklist: ring positions reserved
  int pr_out;                // push-relabel worklist: items queued and not yet fully visited
  unsigned wl_head;          // 2D relabel worklist: tickets taken
  unsigned long long wl_tail_out;  // 2D relabel worklist, updated together: ring positions
                                   // reserved (high 32 bits) and items queued and not yet fully
                                   // visited (low 32 bits)
};

// A set of grids tiled with one tile shape: the unit every launch works on
// (a plain solve is a set of one grid; a batch concatenates many).
struct TileSet {
  int dims = 2;
  int TR = 16, TY = 4, TZ = 4;       // tile shape (2D: 32xTR, 3D: 32xTYxTZ)
  int pr_split = 0;                  // 2D 32x16 tiles: push-relabel runs on 32x8 halves
                                     // (work item 2 * tile + half; relabel and cut on whole tiles)
  int ngrids = 0;
  int ntiles = 0;
  GridDev* d_desc = nullptr;         // [ngrids]
  int4* d_info = nullptr;            // [ntiles] {grid, tx, ty, tz}
  int nlist[2] = {0, 0};             // tiles of parity 0 / 1
  int* d_flag_pr = nullptr;          // [2 * ntiles] work item waits in a push-relabel queue
  int* d_q_pr[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [parity][buffer]
  int* d_flag_bfs[2] = {nullptr, nullptr};  // [buffer][ntiles] tile waits in a BFS frontier
  int* d_q_bfs[2] = {nullptr, nullptr};     // [buffer] BFS frontiers
  uint8_t* d_act = nullptr;          // [ntiles] bits 0-1: tile (half) held an active node at its last
                                     // relabel visit
  int* d_grid_active = nullptr;      // [ngrids] active tiles after global relabel
  unsigned long long* d_pr_ring = nullptr;  // [work items] push-relabel worklist ring (null: sweeps only)
  int* d_pr_lock = nullptr;          // [work items] a visit of the item is in progress
  const void* d_tmap = nullptr;      // [ngrids][3] tensor maps (128 B each) that stage tile visits:
                                     // the grid's planes {e, h, r...} with a tile box, the h plane
                                     // with a 40-wide tile + halo box, the arc-byte plane with a tile
                                     // box (null: visits load their tiles with ordinary loads)
  void* tmap_slot = nullptr;         // room for d_tmap in the control block
  long long* d_grid_sum = nullptr;   // [ngrids*2] sum min(e,0), source-side count
  DevCounters* d_ctr = nullptr;
  void* d_block = nullptr;           // single allocation backing the above
  size_t block_bytes = 0;
  int cap_tiles = 0, cap_grids = 0;  // capacity of d_block (reused while it fits)
  void* h_stage = nullptr;           // pinned staging of d_desc / d_info uploads
  size_t h_stage_bytes = 0;
  void* gcache = nullptr;            // captured relabel-cycle graphs (engine.cpp)
};

// (kernels_post.cu) labelling energy over dense device arrays: out[0] data,
// out[1] smooth (int64 sums, out zeroed by the caller)
cudaError_t launch_energy(int dims, int w, int h, int d, const int32_t* e, const int32_t* const* caps,
                          const uint8_t* lab, unsigned long long* out, cudaStream_t s);
// (kernels_post.cu) stroke-to-seed mapping through the volume (visibility)
cudaError_t launch_stroke_seeds(const jfc_view& v, int w, int h, int d, const float* vol, const float* tf, int ntf,
                                const uint8_t* mask, uint8_t label, uint8_t* seeds, cudaStream_t s);
// (kernels_post.cu) p[i] &= keep over n bytes
cudaError_t launch_and_bytes(uint8_t* p, long long n, uint8_t keep, cudaStream_t s);

// (kernels_fast.cu) one Fast-Cut iteration on a single grid: relabel in two
// parities, then line-segment pushes along each axis in two parities;
// *moved (device) is raised when anything moved
cudaError_t launch_fast_iteration(const GridDev& g, int* moved, cudaStream_t s);

// Counts every kernel launch of the library (engine.cpp).
void jfc_note_launch(int n = 1);

// ----------------------------------------------------------- kernel launchers
// (kernels_pr.cu) `sweeps` parity sweeps (even tiles, then odd tiles, ...)
// in one persistent launch, draining the device work queues; sweeps <= 0
// reads the count from the control block (pr_sweeps), so one captured graph
// serves every interval
// sched 2: the asynchronous worklist (needs ts.d_pr_ring) instead of the
// parity sweeps
cudaError_t launch_pr_phase(const TileSet& ts, int sweeps, int local_iters, cudaStream_t s, int sched = 1);
// Local pre-push inside every tile before the first relabel of a solve.
cudaError_t launch_prepush(const TileSet& ts, cudaStream_t s);
// (kernels_bfs.cu) one BFS to its fixpoint in one persistent launch:
// global relabel (cut = false; also refills the push-relabel queues) or the
// source-side cut (cut = true)
cudaError_t launch_bfs(const TileSet& ts, bool cut, int max_passes, cudaStream_t s);
// (kernels_bfs.cu) tag post-process: bit 1 of each label byte = object node
// connected through object nodes to a foreground seed (dense d_seeds)
cudaError_t launch_tag(const TileSet& ts, const uint8_t* d_seeds, int max_passes, cudaStream_t s);
cudaError_t launch_grid_sums(const TileSet& ts, cudaStream_t s);
cudaError_t launch_clear_counters(const TileSet& ts, cudaStream_t s);
// Polls before the device-side waits of later launches give up (0: default)
// and the distance cap of the global relabels (0: none).
cudaError_t launch_set_limits(const TileSet& ts, unsigned long long polls, int h_cap, cudaStream_t s);
int persistent_blocks(const void* kernel, int threads, size_t smem);
// persistent_blocks on the current device, cached per device in cache[64]
// (every cooperative launch of one kernel reuses its grid size)
// (smem: dynamic shared memory per block)
int persistent_blocks_cached(int* cache, const void* kernel, int threads, size_t smem = 0);
// layout helpers (kernels_bfs.cu)
cudaError_t launch_fix_boundary(const GridDev& g, int conn, int* d_bad, cudaStream_t s);
cudaError_t launch_pack_labels(const GridDev& g, uint8_t* d_dense, cudaStream_t s);
cudaError_t launch_pack_plane(const GridDev& g, const int* d_plane, int* d_dense, cudaStream_t s);
cudaError_t launch_edit_tlinks(const GridDev& g, const uint32_t* d_idx, const int32_t* d_dcs,
                               const int32_t* d_dct, size_t n, long long* d_dsink, cudaStream_t s);

// (kernels_build.cu) capacity build
struct BuildModelDev {
  int pixfmt, channels;
  int kf, kb;
  int seed_cap;
  int mu_f[JFC_MAX_K * 3];
  int mu_b[JFC_MAX_K * 3];
};
cudaError_t launch_contrast_sum(const GridDev& g, const void* d_img, int pixfmt,
                                unsigned long long* d_sum, cudaStream_t s);
cudaError_t launch_seed_stats(const GridDev& g, const void* d_img, int pixfmt, const uint8_t* d_seeds,
                              int* d_minmax /*[2][3][2]*/, unsigned long long* d_count /*[2]*/,
                              uint32_t* d_list_f, uint32_t* d_list_b, unsigned int* d_fill /*[2]*/,
                              bool fill, cudaStream_t s);
// k-means state of both seed classes, resident on the device across the
// queued iterations (class 0 = foreground list first, class 1 after it).
struct KmeansDev {
  int mu[2][JFC_MAX_K * 3];            // centres, fixed point 1/16
  int k[2];
  int live[2];                         // class still moving
  unsigned long long n[2];             // list lengths
  unsigned long long acc[2][JFC_MAX_K * 4];   // per centre: channel sums, count
  unsigned int done;                   // blocks finished in the current launch
};
cudaError_t launch_kmeans(const uint32_t* d_list, KmeansDev* d_km, int pixfmt, unsigned long long nmax,
                          int iters, cudaStream_t s);
cudaError_t launch_build_graph(const GridDev& g, const void* d_img, const uint8_t* d_seeds,
                               const BuildModelDev& m, const int* d_lut_xy, const int* d_lut_z,
                               const int* d_lut_s, const int* d_lut_t,
                               unsigned long long* d_sink, cudaStream_t s);
cudaError_t launch_edit_seeds(const GridDev& g, const void* d_img, uint8_t* d_seeds,
                              const BuildModelDev& m, const int* d_lut_s, const int* d_lut_t,
                              const uint32_t* d_idx, const uint8_t* d_new, size_t n,
                              long long* d_dsink, cudaStream_t s);

// Pixel feature helpers shared by host and device code.
__host__ __device__ inline int jfc_pix_channels(int pixfmt) { return pixfmt == JFC_PIX_RGB8 ? 3 : 1; }
__host__ __device__ inline size_t jfc_pix_bytes(int pixfmt) {
  return pixfmt == JFC_PIX_RGB8 ? 3 : (pixfmt == JFC_PIX_I16 ? 2 : 1);
}
