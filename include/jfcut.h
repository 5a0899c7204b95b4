/*
 * jfcut.h — C ABI of the B200 grid graph-cut solver (libjfcut.so).
 *
 * The surface keeps JF-Cut's graph-cut operator: build a 4-/6-connected grid
 * graph from an image / video / volume plus seed strokes, compute the exact
 * max-flow, read back the min-cut labels.  In the reference this surface is
 * the QGCWidget class (src/QVisualizer/Graph Cut/QGCWidget.h:160-243) driving
 * OpenCL kernels; there is no FFI there, so every entry point below names the
 * reference method or file format it replaces.
 *
 * Conventions
 *  - Every function returns an int status (JFC_OK = 0) unless stated; no C++
 *    exception crosses this boundary.  Errors replace the reference's
 *    QError(level, code) (infrastructures/QError.h:37-73).
 *  - Host buffers are owned by the caller and are only read/written during the
 *    call.  Device buffers (the *_device variants) are caller-owned device
 *    pointers on the context's device.
 *  - Node order is x-fastest: index = x + W*(y + H*z).
 *  - Residual / capacity arrays follow the reference channel order:
 *      2D: [0]=+x [1]=+y [2]=-y [3]=-x      (cl_ushort2 c1=(+x,+y), c2=(-y,-x);
 *                                            QGCWidget.cpp:2479-2482)
 *      3D: [0]=+x [1]=+y [2]=+z [3]=-z [4]=-y [5]=-x
 *                                           (cl_uchar4 c1=(+x,+y,+z), c2=(-z,-y,-x);
 *                                            QGCWidget.cpp:2503-2508)
 *    ncap[k][i] is the capacity of the arc leaving node i in direction k.
 *    Arcs that would leave the grid must be 0.
 *  - Terminal links use the reference's net-excess form
 *    (graphcut_compute_excessflow.cl:39-44): excess[i] = cs[i] - ct[i].
 *    flow_offset = sum_i min(cs[i], ct[i]) (0 for graphs given as net excess).
 *    Max-flow values are int64.
 *  - Labels: 1 = source side (the reference's cut.object = CHAR_MAX), 0 = sink
 *    side.  The source side is the canonical (minimal) one: the nodes reachable
 *    from excess in the final residual graph (graphcut_compute_cut.cl:36-125).
 */
#ifndef JFCUT_H
#define JFCUT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace QError levels, QGCWidget.cpp:2017, 3112-3116) ---- */
enum {
  JFC_OK = 0,
  JFC_ERR_INVALID_ARG = 1,   /* bad size, null pointer, unsupported connectivity */
  JFC_ERR_NO_SEEDS = 2,      /* "no labels" (QGCWidget.cpp:2017, 3112) */
  JFC_ERR_OOM = 3,           /* device allocation failed / over HBM budget */
  JFC_ERR_NOT_CONVERGED = 4, /* iteration budget hit; never silent (QGCWidget.cpp:2413) */
  JFC_ERR_CUDA = 5,          /* CUDA runtime error */
  JFC_ERR_NO_DEVICE = 6,     /* no CUDA device / extension cannot run here */
  JFC_ERR_STATE = 7,         /* call out of order (e.g. labels before solve) */
  JFC_ERR_CANCELLED = 8,     /* server request cancelled */
  JFC_ERR_BUSY = 9,          /* server queue full / request not finished */
  JFC_ERR_IO = 10            /* a data file could not be opened, read or written */
};

/* Pixel formats of jfc_graph_build_from_image (the reference reads a float
 * volume plus an RGBA8 feature image, QGCWidget.cpp:1309-1368). */
enum {
  JFC_PIX_GRAY8 = 0,   /* uint8, 1 channel */
  JFC_PIX_RGB8 = 1,    /* uint8, 3 channels interleaved */
  JFC_PIX_I16 = 2      /* int16, 1 channel (CT/MR style volumes) */
};

/* Seed byte values (cl_cut.foreground / background, QGCSetting.h:46-52). */
enum { JFC_SEED_NONE = 0, JFC_SEED_FG = 1, JFC_SEED_BG = 2 };

/* Solver schedule.  Replaces the Convergence panel (countIterations,
 * cutIterations, totalIterations: QGCPanel.ui:1494-1658) and the tile
 * constants (QGCSetting.cpp:28-29).  Zero fields take defaults. */
typedef struct jfc_params {
  int tile_rows;         /* 2D tiles are 32 x tile_rows: 8 (default) or 16; 3D tiles
                            see tile_depth */
  int local_iters;       /* push/relabel rounds per tile visit (default 12) */
  int relabel_interval;  /* sweep pairs between global relabels at the start (default 0 =
                            automatic: 2 for 2D grids, 3 for 3D grids) */
  int max_sweeps;        /* budget of sweeps -> JFC_ERR_NOT_CONVERGED (default 1<<20) */
  int max_bfs_passes;    /* budget of tile passes per BFS (default 1<<20) */
  int use_graph;         /* 1: replay each relabel cycle (push-relabel phase + global
                            relabel + read-back) as one CUDA graph launch (default) */
  int verbose;           /* 1: one JSON line per global relabel on stderr */
  int relabel_interval_max; /* adaptive interval cap: the interval doubles while fewer
                               than 1/256 of the tiles are active (default max(64, 16 x interval)) */
  int tile_depth;        /* 3D tiles: 0 = automatic (32 x 4 x 2); 1, 2 or 4 = tiles of
                            32 x (tile_rows / tile_depth) x tile_depth (4 needs tile_rows 16) */
  int pr_mode;           /* 0: block-wise push-relabel (default; with 2D 32 x 16 tiles the
                            push-relabel visits run on 32 x 8 halves, the relabel and cut on
                            whole tiles); 1: the reference's Fast-Cut line sweeps
                            (graphcut_push_relabel_fast.cl), for comparison; plain solves only,
                            relabel_interval iterations between global relabels; 2: block-wise
                            on whole 32 x 16 tiles */
  int spin_limit;        /* polls before a device-side wait gives up (grid barrier, relabel
                            worklist): 0 = default (2^26 polls, seconds); on expiry the
                            kernels leave, the call returns JFC_ERR_CUDA ("timed out") and the
                            context stays usable */
  int relabel_cap;       /* distance cap of the global relabels while solving: nodes farther
                            than this from every deficit count as unreachable until no active
                            tile is left, then one exact (uncapped) relabel certifies the maximum
                            preflow and the solve goes on uncapped if it finds reachable excess;
                            flow and cut are those of the exact solve.  0 = automatic, < 0 = no
                            cap (every relabel exact) */
  int pr_sched;          /* scheduling of the push-relabel visits between two global relabels:
                            1 = checkerboard parity sweeps with a grid barrier between colours,
                            2 = an asynchronous worklist with per-tile neighbour exclusion (no
                            barriers), 3 = sweeps while more than 1/256 of the tiles are active
                            and the worklist in the tail, 0 = automatic (sweeps, and the worklist
                            for the cycles after the exact relabel of relabel_cap when it finds
                            excess left).  Same arithmetic, same results */
  int local_iters_tail;  /* push/relabel rounds per visit once fewer than 1/256 of the tiles are
                            active (the long-path tail of a solve, where excess has to cross
                            whole tiles): 0 = automatic, < 0 = local_iters */
} jfc_params;

/* Capacity model (replaces computeCapacity / kmeans / computeExcessFlowLazy,
 * QGCWidget.cpp:1997-2107, 3182-3235).  All weights are integer by
 * construction (host-built int32 lookup tables), so device and CPU builds are
 * bit-identical. */
typedef struct jfc_model {
  int lambda_n;          /* n-link scale: w = round(lambda_n*exp(-D/(2 sigma^2))) (default 100) */
  int z_weight_pct;      /* 3D z-direction n-link scale in percent (default 100; video 50) */
  int lambda_t;          /* t-link scale: round(lambda_t * -ln p) (default 10) */
  int k_fg;              /* k-means clusters for the object model (default 5) */
  int k_bg;              /* k-means clusters for the background model (default 5) */
  int seed_cap;          /* hard seed t-link capacity (default 1000000) */
  int kmeans_iters;      /* k-means iteration cap (default 32, QGCWidget.cpp:2073) */
} jfc_model;

/* Per-solve statistics (the reference prints these as "> GPU TIME" / "> DATA",
 * QGCWidget.cpp:2522-2524). */
typedef struct jfc_stats {
  int status;
  int sweeps;             /* parity sweeps (one even + one odd = one iteration) */
  int global_relabels;
  int bfs_passes;         /* tile passes summed over all BFS runs */
  long long tile_visits;  /* push-relabel tile visits */
  long long flow;         /* max-flow value (int64) */
  long long source_nodes; /* nodes on the source side */
  double ms_total, ms_build, ms_push_relabel, ms_global_relabel, ms_cut;
  long long pr_rounds;    /* push/relabel rounds summed over tile visits */
  long long bfs_visits;   /* tile visits of all BFS passes */
  double ms_gr_first;     /* global relabel: dense first passes (device clock) */
  double ms_gr_frontier;  /* global relabel: frontier passes (device clock) */
  int used_graph;         /* 1 if the relabel cycles ran as CUDA graph launches */
  int pr_phases;          /* push-relabel phase launches (one per relabel cycle) */
} jfc_stats;

typedef struct jfc_ctx jfc_ctx;
typedef struct jfc_graph jfc_graph;
typedef struct jfc_batch jfc_batch;
typedef struct jfc_server jfc_server;

/* ---- context (replaces QGCWidget::initContext / initOpenCL, QGCWidget.cpp:686-813) ---- */
int  jfc_create(int device, const jfc_params* params, jfc_ctx** out);
void jfc_destroy(jfc_ctx* ctx);
int  jfc_set_params(jfc_ctx* ctx, const jfc_params* params);
int  jfc_get_params(jfc_ctx* ctx, jfc_params* out);
void jfc_default_params(jfc_params* out);
void jfc_default_model(jfc_model* out);
const char* jfc_strerror(int status);
/* Detail of the last error raised on the calling thread (the reference's
 * QError message / cl::Error string, QGCWidget.cpp:2533-2557). */
const char* jfc_last_error(void);
/* Run the context's work on a caller-owned CUDA stream (a cudaStream_t passed
 * as void*; NULL restores the context's own stream).  Lets a caller bracket
 * the library's kernels with its own CUDA events (the reference times every
 * phase with OpenCL profiling events, utilities/QUtilityCL.cpp:341-354). */
int  jfc_set_stream(jfc_ctx* ctx, void* stream);
/* Number of CUDA kernels this library has launched in this process. */
unsigned long long jfc_kernel_launches(void);

/* ---- graph (replaces initConfigurations' buffer sizing, QGCWidget.cpp:815-887) ---- */
/* dims = 2 (conn 4, d = 1) or 3 (conn 6). */
int  jfc_graph_create_grid(jfc_ctx* ctx, int dims, int w, int h, int d, int conn, jfc_graph** out);
void jfc_graph_destroy(jfc_graph* g);
/* Bytes of device memory a grid of this shape holds (HBM-budget admission). */
size_t jfc_graph_bytes(int dims, int w, int h, int d);

/* Build n-links and t-links from an image and seeds (host buffers).
 * Replaces slotModelClicked -> computeCapacity + kmeans + computeExcessFlowLazy
 * (QGCWidget.cpp:2560-2606).  Returns JFC_ERR_NO_SEEDS when either class has
 * no seed.  img: w*h*d pixels in pixfmt; seeds: w*h*d bytes (JFC_SEED_*). */
int jfc_graph_build_from_image(jfc_graph* g, const void* img, int pixfmt,
                               const uint8_t* seeds, const jfc_model* model);
/* Same, with img and seeds already in device memory. */
int jfc_graph_build_from_device(jfc_graph* g, const void* d_img, int pixfmt,
                                const uint8_t* d_seeds, const jfc_model* model);

/* Load an explicit graph (replaces slotLoadGraphClicked's .ef/.c1/.c2 load,
 * QGCWidget.cpp:2631-2736).  excess: n int32; ncap: conn pointers to n int32. */
int jfc_graph_set(jfc_graph* g, const int32_t* excess, const int32_t* const* ncap,
                  int64_t flow_offset);
int jfc_graph_set_device(jfc_graph* g, const int32_t* d_excess,
                         const int32_t* const* d_ncap, int64_t flow_offset);
/* Read the current residual state (net excess, residual arcs, heights).
 * Any pointer may be NULL.  Used for certificates and .ef/.c1/.c2 export. */
int jfc_graph_get_state(jfc_graph* g, int32_t* excess, int32_t* const* ncap, int32_t* height);

/* Solve to the exact max-flow / min-cut.  Replaces slotCutClicked's hot loop
 * (QGCWidget.cpp:2364-2558): global relabel, push/relabel sweeps, device-side
 * convergence, final residual BFS.  Warm: a second call after
 * jfc_edit_tlinks continues from the resident residual graph. */
int jfc_solve(jfc_graph* g, jfc_stats* stats);
int jfc_get_flow(jfc_graph* g, int64_t* flow);
/* Labels (1 = source side).  Replaces the cut read-back (QGCWidget.cpp:2454,
 * slotSaveCutClicked 2990-2996). */
int jfc_read_labels(jfc_graph* g, uint8_t* out);
int jfc_read_labels_device(jfc_graph* g, uint8_t* d_out);

/* Warm-start stroke edit: node idx[j] gets cs += dcs[j], ct += dct[j].
 * (New in this build: the reference re-models from scratch on every stroke,
 * QGCWidget.cpp:2560.)  The residual graph and heights stay resident. */
int jfc_edit_tlinks(jfc_graph* g, const uint32_t* idx, const int32_t* dcs,
                    const int32_t* dct, size_t n);
/* Warm-start stroke edit on a graph built from an image: node idx[j] becomes
 * seed new_seed[j] (JFC_SEED_*) with the colour model kept fixed; the t-link
 * change is applied to the resident residual graph (the reference re-runs
 * slotModelClicked, QGCWidget.cpp:2560-2606, after every brush stroke,
 * QGCWidget.cpp:2243-2287).  Duplicate indices: the last one wins.  The
 * height plane serves as scratch until the next jfc_solve (which recomputes
 * it), so jfc_graph_get_state reports meaningful heights only after a solve. */
int jfc_graph_edit_seeds(jfc_graph* g, const uint32_t* idx, const uint8_t* new_seed, size_t n);

/* Solve a 2D 4-connected grid without allocating anything.  No counterpart in
 * the reference: it exists for callers that cannot allocate device memory
 * when they need a cut (real-time frame loops that must not stall on the
 * allocator, hosts that hand the library a fixed memory budget up front).
 * The working set lives in one fixed file-scope device array of about
 * 13.2 MB that every GPU loading the library holds until exit; grids are
 * limited to 524,288 nodes after padding (width to a multiple of 32, height
 * to a multiple of 16), larger ones return JFC_ERR_INVALID_ARG.
 * Inputs d_excess and d_ncap[4] (reference channel order, dense w*h int32)
 * and the output d_labels (w*h bytes, 1 = source side) are caller-owned
 * device buffers on `device`; *flow receives the int64 max-flow.  stream is
 * a cudaStream_t (NULL = the legacy default stream); the call synchronises
 * it before returning (counters are read back between relabel cycles) and
 * restores the caller's current device.  params may be NULL.  Calls share
 * the array: calls that overlap on the GPU race.  The first call on a device
 * looks up the array's address; make it before any stream capture begins. */
int jfc_solve_grid2d_noalloc(int device, void* stream, const jfc_params* params, int w, int h,
                             const int32_t* d_excess, const int32_t* const* d_ncap,
                             int64_t flow_offset, uint8_t* d_labels, int64_t* flow);

/* ---- batched solver: many independent grids in one persistent launch per
 * phase, fed by a device work queue (no reference counterpart; the reference
 * solves one volume at a time, QGCWidget.cpp:2364). ---- */
int  jfc_batch_create(jfc_ctx* ctx, jfc_batch** out);
void jfc_batch_destroy(jfc_batch* b);
int  jfc_batch_add(jfc_batch* b, jfc_graph* g);     /* graph must be built/set */
int  jfc_batch_clear(jfc_batch* b);
int  jfc_batch_size(jfc_batch* b);
/* Solve every graph of the batch; stats may be NULL or an array of the
 * batch's size.  Returns the first non-OK per-graph status.  The schedule is
 * the one jfc_batch_autotune chose for this batch, else the context's. */
int  jfc_batch_solve(jfc_batch* b, jfc_stats* stats);
/* Pick tile_rows / local_iters / relabel_interval (and 3D tile depth) for
 * this batch by timing candidates on a copy of the batch's graphs (state is
 * restored; each candidate is the faster of two solves).  The choice is
 * written to *chosen (may be NULL) and applies to this batch's later solves;
 * the context's parameters are left unchanged.  jfc_batch_clear drops it. */
int  jfc_batch_autotune(jfc_batch* b, jfc_params* chosen);

/* ---- serving: continuous batching with HBM-budget admission and warm
 * stroke edits (no reference counterpart). ---- */
typedef struct jfc_request_info {
  int status;
  int64_t flow;
  double ms_queue, ms_solve, ms_total;   /* latency split */
  int warm;                              /* 1 if re-solved from resident state */
} jfc_request_info;

/* max_slots: requests solving at once (0: 64); cold requests take at most
 * max_slots - max_slots / 4 of them, the rest stay free for warm edits. */
int  jfc_server_create(jfc_ctx* ctx, size_t hbm_budget_bytes, int max_slots, jfc_server** out);
void jfc_server_destroy(jfc_server* s);
/* Submit a new session from host image + seeds; returns a session id >= 0 in *sid. */
int  jfc_server_submit(jfc_server* s, int dims, int w, int h, int d, const void* img, int pixfmt,
                       const uint8_t* seeds, const jfc_model* model, int* sid);
/* Queue a stroke edit (re-seed nodes) for an existing session; re-solved warm
 * from the session's resident residual graph. */
int  jfc_server_edit(jfc_server* s, int sid, const uint32_t* idx, const uint8_t* new_seed, size_t n);
/* Block until the session's latest request is finished (timeout_ms < 0: forever). */
int  jfc_server_wait(jfc_server* s, int sid, int timeout_ms, jfc_request_info* info);
int  jfc_server_read_labels(jfc_server* s, int sid, uint8_t* out);
int  jfc_server_close(jfc_server* s, int sid);      /* frees the session's device state */
int  jfc_server_cancel(jfc_server* s, int sid);
/* Server counters: budget and bytes held (now / peak), sessions by phase, the
 * largest solving set seen (grids sharing one launch), loop iterations. */
typedef struct jfc_server_stats {
  size_t budget, used, peak_used;
  int sessions, waiting, solving, peak_solving;
  int64_t loops, requests_done;
} jfc_server_stats;
int  jfc_server_get_stats(jfc_server* s, jfc_server_stats* out);

/* Tag post-process of a solved graph (QGCWidget::computeTag,
 * QGCWidget.cpp:3275-3308; graphcut_compute_tag.cl): tag[i] = 1 for object
 * nodes connected through object nodes (4 / 6-neighbourhood) to a foreground
 * seed, else 0.  seeds: host dense JFC_SEED_* array, or NULL for the seeds of
 * the graph's image build. */
int jfc_graph_compute_tag(jfc_graph* g, const uint8_t* seeds, uint8_t* tag);

/* Energy of a labelling over a graph given as dense device arrays (the
 * reference's energy check after a solve, QGCWidget.cpp:2452-2520):
 * data = sum over background nodes of max(e, 0) + sum over object nodes of
 * max(-e, 0); smooth = sum of the capacities of arcs from object to background
 * nodes.  With the original capacities and the canonical cut, data + smooth
 * equals the (net-excess) max-flow: an independent certificate.  stream is a
 * cudaStream_t (NULL = legacy default stream). */
int jfc_energy_device(int device, void* stream, int dims, int w, int h, int d, const int32_t* d_excess,
                      const int32_t* const* d_ncap, const uint8_t* d_labels, int64_t* data, int64_t* smooth);

/* Stroke-to-seed mapping through a volume (graphcut_compute_visibility,
 * graphcut_render_ray_casting.cl:275-346; compute only, no graphics): every
 * pixel of the stroke mask (image_w x image_h, non-zero = stroke) casts a ray
 * through the inverse view-projection (column-major, as the reference passes
 * it) into the box [-box, box]; samples of the volume (trilinear, clamp to
 * edge) are classified by the RGBA transfer function (tf_size entries,
 * linear, after the intensity window) and composited front to back; each
 * sample more opaque than alpha marks the 8 surrounding voxels with `label`
 * in the dense seed array.  All arrays are device pointers; 3D volumes. */
typedef struct jfc_view {
  float inverse_mvp[16];
  float box[3];                        /* volumeBoundingBox half extents */
  int image_w, image_h;
  int samples;                         /* sampleNumber (>= 3) */
  float sample_ratio, sample_step_scale;
  float window_width, window_level;
  float alpha;
} jfc_view;
int jfc_stroke_to_seeds(int device, void* stream, const jfc_view* view, int w, int h, int d,
                        const float* d_volume, const float* d_tf_rgba, int tf_size, const uint8_t* d_mask,
                        uint8_t label, uint8_t* d_seeds);

/* ---- the reference's data files (host only; no device work) ----
 * Dense arrays (w*h*d, x fastest) in the solver's channel order. */
enum { JFC_FMT_UCHAR = 0, JFC_FMT_CHAR, JFC_FMT_USHORT, JFC_FMT_SHORT, JFC_FMT_UINT, JFC_FMT_INT, JFC_FMT_FLOAT };
typedef struct jfc_volume_info {
  char object_file[256];     /* "Object File Name" (the .raw next to the header) */
  int w, h, d;               /* "Resolution" */
  float thickness[3];        /* "Slice Thickness" */
  int format;                /* JFC_FMT_* ("Format") */
  int big_endian;            /* "Endian" */
  float intensity_min, intensity_max;  /* "Intensity Extremums" */
} jfc_volume_info;
/* .dat volume header (QGCWidget::parseDataFile / saveDataFile, QGCWidget.cpp:296-683). */
int jfc_read_dat(const char* path, jfc_volume_info* out);
int jfc_write_dat(const char* path, const jfc_volume_info* info);
/* .raw samples in the header's format and endianness, widened to float. */
int jfc_read_raw(const char* path, const jfc_volume_info* info, float* out);
/* <base>.ef / .c1 / .c2 graph files (slotLoadGraphClicked / slotSaveGraphClicked,
 * QGCWidget.cpp:2631-2736): int32 net excess; 2D ushort2 (+x, +y), (-y, -x);
 * 3D uchar4 (+x, +y, +z, -), (-z, -y, -x, -).  ncap[conn] receive / give the
 * capacities; saving rejects capacities that do not fit the file's type. */
int jfc_load_graph_files(const char* base, int dims, int w, int h, int d, int32_t* excess, int32_t* const* ncap);
int jfc_save_graph_files(const char* base, int dims, int w, int h, int d, const int32_t* excess,
                         const int32_t* const* ncap);
/* .cut: 4 bytes per node {foreground seed, background seed, object, tag}
 * (cl_cut, QGCSetting.h:46-51).  seeds in JFC_SEED_*, labels 1 = object;
 * either pointer may be NULL. */
int jfc_read_cut(const char* path, size_t n, uint8_t* seeds, uint8_t* labels);
int jfc_write_cut(const char* path, size_t n, const uint8_t* seeds, const uint8_t* labels);
/* .mfi max-flow instances of the GridCut benchmark (3rdParty/bench/mfi.cpp,
 * QGCWidget::saveMFI, QGCWidget.cpp:3339-3474), 2D/4 and 3D/6 only. */
typedef struct jfc_mfi_info {
  int dims, conn, w, h, d;
  int64_t maxflow;           /* the file's recorded max-flow */
  int active_count;
  int type_terminal, type_neighbor;   /* 0 uint8, 1 uint16, 2 uint32 */
} jfc_mfi_info;
int jfc_read_mfi_info(const char* path, jfc_mfi_info* out);
/* Net excess e = cs - ct, neighbour capacities, *flow_offset = sum min(cs, ct)
 * (pass it to jfc_graph_set); mask (n bytes) may be NULL. */
int jfc_load_mfi(const char* path, int32_t* excess, int32_t* const* ncap, int64_t* flow_offset, uint8_t* mask);
/* Terminal caps as max(e, 0) / max(-e, 0) in uint32 (as the reference writes
 * them); neighbour caps uint16 (2D) / uint8 (3D), or uint32 when one does
 * not fit; mask may be NULL (zeros). */
int jfc_save_mfi(const char* path, int dims, int w, int h, int d, const int32_t* excess, const int32_t* const* ncap,
                 int64_t maxflow, const uint8_t* mask);

#ifdef __cplusplus
}
#endif
#endif /* JFCUT_H */
