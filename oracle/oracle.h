/*
 * oracle.h — CPU restatement of JF-Cut's graph-cut path.  TEST INFRASTRUCTURE
 * ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it
 * as the checker.  The product (libjfcut.so) never links or calls it.
 *
 * Graph convention (same as include/jfcut.h): x-fastest node order, per-node
 * outgoing arc arrays in the reference channel order
 *   2D: +x +y -y -x          (QGCWidget.cpp:2479-2482)
 *   3D: +x +y +z -z -y -x    (QGCWidget.cpp:2503-2508)
 * and terminal links in net-excess form e = cs - ct
 * (graphcut_compute_excessflow.cl:39-44).
 */
#ifndef JFC_ORACLE_H
#define JFC_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Model constants, identical in meaning to jfc_model. */
typedef struct orc_model {
  int lambda_n, z_weight_pct, lambda_t, k_fg, k_bg, seed_cap, kmeans_iters;
} orc_model;

/* Capacity build (n-links, k-means colour models, t-links).  Writes e[n],
 * caps[conn][n] and *sink_total = sum_i ct[i].  Returns 0, or 2 when a seed
 * class is empty ("no labels", QGCWidget.cpp:2017).  centroids_out (may be
 * NULL) receives k_fg+k_bg centroids x 3 channels in 1/16 fixed point. */
int orc_build_graph(int dims, int w, int h, int d, int pixfmt, const void* img,
                    const uint8_t* seeds, const orc_model* m, int32_t* e,
                    int32_t* const* caps, int64_t* sink_total, int32_t* centroids_out);

/* The same build with the colour models fit on `seeds` and the t-links set
 * from `seeds_tl` (the graph a session holds after warm stroke edits). */
int orc_build_graph_ex(int dims, int w, int h, int d, int pixfmt, const void* img,
                       const uint8_t* seeds, const uint8_t* seeds_tl, const orc_model* m, int32_t* e,
                       int32_t* const* caps, int64_t* sink_total, int32_t* centroids_out);

/* Sum of squared neighbour differences and pair count (sigma^2 = sum/count). */
void orc_contrast_sum(int dims, int w, int h, int d, int pixfmt, const void* img,
                      uint64_t* sum, uint64_t* count);

/* Max-flow of the folded grid graph by sequential FIFO push-relabel with
 * global relabelling.  e and caps are modified in place into the final
 * residual state.  labels[n] = 1 for the minimal source side.  Returns the
 * folded flow value (sum of absorbed deficits); the full max-flow is
 * sink_total + sum_i min(e_final[i], 0). */
int64_t orc_maxflow(int dims, int w, int h, int d, int32_t* e, int32_t* const* caps,
                    uint8_t* labels);

/* Exact BFS distance of every node to the nearest deficit (e < 0) along
 * residual arcs (the global relabel, graphcut_global_relabel.cl:19-124);
 * unreachable nodes get 0x3fffffff. */
void orc_sink_distances(int dims, int w, int h, int d, const int32_t* e, const int32_t* const* r,
                        int32_t* dist);

/* Reachability from {e > 0} along residual arcs (graphcut_compute_cut.cl).
 * Returns the number of reached nodes with e < 0 (0 for a maximum preflow). */
int64_t orc_cut_from_residual(int dims, int w, int h, int d, const int32_t* e,
                              const int32_t* const* r, uint8_t* labels);

/* Cut capacity of labels on the ORIGINAL graph (energy check,
 * QGCWidget.cpp:2452-2520): sum_{i sink side} max(e0,0) + sum_{i source side}
 * max(-e0,0) + sum of arcs source->sink. */
int64_t orc_cut_energy(int dims, int w, int h, int d, const int32_t* e0,
                       const int32_t* const* caps0, const uint8_t* labels);

/* sum_i min(e[i], 0) and sum_i max(e[i], 0) in int64 (reduce_flow). */
void orc_excess_sums(const int32_t* e, size_t n, int64_t* neg_sum, int64_t* pos_sum);

/* Validity of a residual state against the original graph: r >= 0,
 * r(u,v) + r(v,u) = c(u,v) + c(v,u), and e = e0 + net inflow.  Returns the
 * number of violations. */
int64_t orc_check_residual(int dims, int w, int h, int d, const int32_t* e0,
                           const int32_t* const* c0, const int32_t* e,
                           const int32_t* const* r);

#ifdef __cplusplus
}
#endif
#endif
