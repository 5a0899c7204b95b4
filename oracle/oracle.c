/*
 * oracle.c — CPU restatement of JF-Cut's graph-cut path, written from the
 * reference's behaviour (not its code).  TEST INFRASTRUCTURE ONLY: the
 * checker for the CUDA path; libjfcut.so never links it.
 *
 * Parity is pinned by tests/test_oracle.py against (a) the max-flow values of
 * the three graphs that ship with the reference (flower 1208089, person
 * 880461, sponge 343591; latex/sources/section-5-results.tex:31-41), (b) the
 * reference GPU's own cut of flower (normalized_flower.raw.cut, object byte),
 * and (c) the reference's CPU solver BK 3.03 built from its sources under
 * oracle/_ref (benchmark/GridCut/code/BK303) on generated graphs.
 *
 * Functions follow these reference parts:
 *   orc_contrast_sum / n-links  graphcut_compute_capacity.cl:21-120 (2D), 124-254 (3D)
 *   k-means                     QGCWidget.cpp:1997-2107, graphcut_kmeans.cl:21-159
 *   t-links (net excess)        graphcut_compute_excessflow.cl:47-77, 109-139
 *   global relabel              graphcut_global_relabel.cl:19-124
 *   push / relabel              graphcut_push_relabel.cl:25-203 (sequential form)
 *   cut (residual reachability) graphcut_compute_cut.cl:19-140
 *   flow reduction              bin/x64/cl/Infrastructures/reduce.cl:92-117
 *   energy check                QGCWidget.cpp:2452-2520
 * The integer model (lookup tables, fixed-point k-means, quantised t-link
 * probability) is this build's own exact-by-construction restatement of the
 * reference's float formulas; the CUDA build implements the same definition.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_INF 0x3fffffff
#define ORC_Q 65536

typedef struct {
  int dims, w, h, d, conn;
  int64_t n;
  int64_t off[6];
} grid_t;

static void grid_init(grid_t* g, int dims, int w, int h, int d) {
  g->dims = dims; g->w = w; g->h = h; g->d = (dims == 2) ? 1 : d;
  g->conn = (dims == 2) ? 4 : 6;
  g->n = (int64_t)w * h * g->d;
  int64_t wh = (int64_t)w * h;
  if (dims == 2) {
    g->off[0] = 1; g->off[1] = w; g->off[2] = -w; g->off[3] = -1;
  } else {
    g->off[0] = 1; g->off[1] = w; g->off[2] = wh; g->off[3] = -wh; g->off[4] = -w; g->off[5] = -1;
  }
}

/* Is the arc of node i in direction k inside the grid? */
static int arc_ok(const grid_t* g, int64_t i, int k) {
  int64_t x = i % g->w, y = (i / g->w) % g->h, z = i / ((int64_t)g->w * g->h);
  if (g->dims == 2) {
    switch (k) {
      case 0: return x + 1 < g->w;
      case 1: return y + 1 < g->h;
      case 2: return y > 0;
      default: return x > 0;
    }
  }
  switch (k) {
    case 0: return x + 1 < g->w;
    case 1: return y + 1 < g->h;
    case 2: return z + 1 < g->d;
    case 3: return z > 0;
    case 4: return y > 0;
    default: return x > 0;
  }
}

/* ------------------------------------------------------------------ model */

static int pix_channels(int pixfmt) { return pixfmt == 1 ? 3 : 1; }

/* Feature vector of pixel i (non-negative integers). */
static void pix_feat(int pixfmt, const void* img, int64_t i, int* f) {
  if (pixfmt == 0) {
    f[0] = ((const uint8_t*)img)[i];
  } else if (pixfmt == 1) {
    const uint8_t* p = (const uint8_t*)img + 3 * i;
    f[0] = p[0]; f[1] = p[1]; f[2] = p[2];
  } else {
    f[0] = (int)((const int16_t*)img)[i] + 32768;
  }
}

/* Contrast index of a pair: |dI| for scalar images, ||dI||^2 for RGB; and the
 * squared difference D that enters exp(-D / 2 sigma^2). */
static void pair_contrast(int pixfmt, const void* img, int64_t p, int64_t q,
                          int64_t* index, uint64_t* dsq) {
  int a[3], b[3];
  pix_feat(pixfmt, img, p, a);
  pix_feat(pixfmt, img, q, b);
  if (pixfmt == 1) {
    int64_t s = 0;
    for (int c = 0; c < 3; ++c) s += (int64_t)(a[c] - b[c]) * (a[c] - b[c]);
    *index = s; *dsq = (uint64_t)s;
  } else {
    int64_t t = a[0] - b[0];
    if (t < 0) t = -t;
    *index = t; *dsq = (uint64_t)(t * t);
  }
}

void orc_contrast_sum(int dims, int w, int h, int d, int pixfmt, const void* img,
                      uint64_t* sum, uint64_t* count) {
  grid_t g; grid_init(&g, dims, w, h, d);
  uint64_t s = 0, c = 0;
  int npos = g.conn / 2;   /* +x, +y (, +z) */
#pragma omp parallel for schedule(static) reduction(+ : s, c)
  for (int64_t i = 0; i < g.n; ++i)
    for (int k = 0; k < npos; ++k) {
      if (!arc_ok(&g, i, k)) continue;
      int64_t idx; uint64_t dsq;
      pair_contrast(pixfmt, img, i, i + g.off[k], &idx, &dsq);
      s += dsq; ++c;
    }
  *sum = s; *count = c;
}

/* n-link weight for a squared difference: round(scale * exp(-D / (2 sigma^2))). */
static int32_t nlink_weight(double scale, double sigma2, uint64_t dsq) {
  if (sigma2 <= 0.0) return (int32_t)floor(scale + 0.5);
  return (int32_t)floor(scale * exp(-(double)dsq / (2.0 * sigma2)) + 0.5);
}

static int64_t feat_dist(const int* x, const int32_t* mu, int C) {
  int64_t s = 0;
  for (int c = 0; c < C; ++c) {
    int64_t t = (int64_t)16 * x[c] - mu[c];
    s += t * t;
  }
  return s;
}

/* Fixed-point k-means over the seed pixels of one class (QGCWidget.cpp:1997-2107
 * iterates assignment + centroid update until the shift is small; here the
 * update is exact integer arithmetic and stops when no centroid moves). */
static void kmeans_class(int pixfmt, const void* img, const uint8_t* seeds, int64_t n,
                         uint8_t cls, int k, int iters, int32_t* mu /* k*3 */) {
  int C = pix_channels(pixfmt);
  int mn[3] = {1 << 30, 1 << 30, 1 << 30}, mx[3] = {-1, -1, -1};
  int f[3];
  /* the class's seed features, gathered once (node order) */
  int64_t m = 0;
  for (int64_t i = 0; i < n; ++i) m += seeds[i] == cls;
  int* feats = (int*)malloc(sizeof(int) * 3 * (size_t)(m ? m : 1));
  m = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (seeds[i] != cls) continue;
    pix_feat(pixfmt, img, i, feats + 3 * m);
    ++m;
  }
  for (int64_t j = 0; j < m; ++j) {
    const int* fj = feats + 3 * j;
    for (int c = 0; c < C; ++c) {
      if (fj[c] < mn[c]) mn[c] = fj[c];
      if (fj[c] > mx[c]) mx[c] = fj[c];
    }
  }
  for (int j = 0; j < k; ++j)
    for (int c = 0; c < 3; ++c)
      mu[j * 3 + c] = (c < C) ? (int32_t)(16 * (int64_t)mn[c] +
                                          (16 * (int64_t)(mx[c] - mn[c]) * (2 * j + 1)) / (2 * k))
                              : 0;
  int64_t* sums = (int64_t*)calloc((size_t)k * 4, sizeof(int64_t));
  for (int it = 0; it < iters; ++it) {
    memset(sums, 0, (size_t)k * 4 * sizeof(int64_t));
    for (int64_t j = 0; j < m; ++j) {
      for (int c = 0; c < 3; ++c) f[c] = feats[3 * j + c];
      int best = 0;
      int64_t bd = feat_dist(f, mu, C);
      for (int j = 1; j < k; ++j) {
        int64_t dj = feat_dist(f, mu + 3 * j, C);
        if (dj < bd) { bd = dj; best = j; }
      }
      sums[best * 4 + 3] += 1;
      for (int c = 0; c < C; ++c) sums[best * 4 + c] += f[c];
    }
    int moved = 0;
    for (int j = 0; j < k; ++j) {
      int64_t cnt = sums[j * 4 + 3];
      if (cnt == 0) continue;
      for (int c = 0; c < C; ++c) {
        int32_t v = (int32_t)((16 * sums[j * 4 + c] + cnt / 2) / cnt);
        if (v != mu[j * 3 + c]) { mu[j * 3 + c] = v; moved = 1; }
      }
    }
    if (!moved) break;
  }
  free(sums);
  free(feats);
}

static int64_t min_dist(const int* f, const int32_t* mu, int k, int C) {
  int64_t bd = feat_dist(f, mu, C);
  for (int j = 1; j < k; ++j) {
    int64_t dj = feat_dist(f, mu + 3 * j, C);
    if (dj < bd) bd = dj;
  }
  return bd;
}

/* Capacity build with the colour models fit on seeds_model and the t-links
 * set from seeds_tl.  With seeds_tl == seeds_model this is the plain build;
 * with the seeds of a session after stroke edits it is the graph the warm
 * edit path holds (an edit recomputes the edited nodes' t-links with the
 * session's colour model, which stays the one of the original strokes). */
int orc_build_graph_ex(int dims, int w, int h, int d, int pixfmt, const void* img,
                       const uint8_t* seeds, const uint8_t* seeds_tl, const orc_model* m, int32_t* e,
                       int32_t* const* caps, int64_t* sink_total, int32_t* centroids_out) {
  grid_t g; grid_init(&g, dims, w, h, d);
  int C = pix_channels(pixfmt);
  int64_t nfg = 0, nbg = 0;
  for (int64_t i = 0; i < g.n; ++i) {
    nfg += seeds[i] == 1;
    nbg += seeds[i] == 2;
  }
  if (nfg == 0 || nbg == 0) return 2;

  /* n-links: contrast-weighted, symmetric (graphcut_compute_capacity.cl). */
  uint64_t ssum, scnt;
  orc_contrast_sum(dims, w, h, d, pixfmt, img, &ssum, &scnt);
  double sigma2 = scnt ? (double)ssum / (double)scnt : 0.0;
  double scale_xy = (double)m->lambda_n;
  double scale_z = (double)m->lambda_n * (double)m->z_weight_pct / 100.0;
  /* 8-bit images: D < 3 * 256^2, so the weights are tabulated once (the same
   * values nlink_weight gives); int16 volumes evaluate it per arc */
  const int64_t dmax = pixfmt == 2 ? 0 : 3 * 256 * 256;
  int32_t* wt_xy = dmax ? (int32_t*)malloc(sizeof(int32_t) * (size_t)dmax) : NULL;
  int32_t* wt_z = dmax ? (int32_t*)malloc(sizeof(int32_t) * (size_t)dmax) : NULL;
  for (int64_t v = 0; v < dmax; ++v) {
    wt_xy[v] = nlink_weight(scale_xy, sigma2, (uint64_t)v);
    wt_z[v] = nlink_weight(scale_z, sigma2, (uint64_t)v);
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < g.n; ++i)
    for (int k = 0; k < g.conn; ++k) {
      if (!arc_ok(&g, i, k)) { caps[k][i] = 0; continue; }
      int64_t idx; uint64_t dsq;
      pair_contrast(pixfmt, img, i, i + g.off[k], &idx, &dsq);
      int zdir = (g.dims == 3) && (k == 2 || k == 3);
      caps[k][i] = (int64_t)dsq < dmax ? (zdir ? wt_z : wt_xy)[dsq]
                                       : nlink_weight(zdir ? scale_z : scale_xy, sigma2, dsq);
    }
  free(wt_xy);
  free(wt_z);

  /* colour models (fg / bg) */
  int kf = m->k_fg < 1 ? 1 : m->k_fg, kb = m->k_bg < 1 ? 1 : m->k_bg;
  if (kf > 32) kf = 32;
  if (kb > 32) kb = 32;
  if (kf > nfg) kf = (int)nfg;
  if (kb > nbg) kb = (int)nbg;
  int32_t muF[32 * 3], muB[32 * 3];
  kmeans_class(pixfmt, img, seeds, g.n, 1, kf, m->kmeans_iters, muF);
  kmeans_class(pixfmt, img, seeds, g.n, 2, kb, m->kmeans_iters, muB);
  if (centroids_out) {
    memcpy(centroids_out, muF, sizeof(int32_t) * 3 * kf);
    memcpy(centroids_out + 3 * kf, muB, sizeof(int32_t) * 3 * kb);
  }

  /* t-link tables over the quantised probability q in [0, Q]. */
  int32_t* lut_s = (int32_t*)malloc(sizeof(int32_t) * (ORC_Q + 1));
  int32_t* lut_t = (int32_t*)malloc(sizeof(int32_t) * (ORC_Q + 1));
  for (int q = 0; q <= ORC_Q; ++q) {
    double pb = ((double)q + 0.5) / (double)(ORC_Q + 1);
    double pf = ((double)ORC_Q + 0.5 - (double)q) / (double)(ORC_Q + 1);
    lut_s[q] = (int32_t)floor((double)m->lambda_t * -log(pb) + 0.5);
    lut_t[q] = (int32_t)floor((double)m->lambda_t * -log(pf) + 0.5);
  }
  int64_t st = 0;
#pragma omp parallel for schedule(static) reduction(+ : st)
  for (int64_t i = 0; i < g.n; ++i) {
    int f[3];
    int32_t cs, ct;
    if (seeds_tl[i] == 1) { cs = m->seed_cap; ct = 0; }
    else if (seeds_tl[i] == 2) { cs = 0; ct = m->seed_cap; }
    else {
      pix_feat(pixfmt, img, i, f);
      uint64_t dF = (uint64_t)min_dist(f, muF, kf, C);
      uint64_t dB = (uint64_t)min_dist(f, muB, kb, C);
      uint64_t q = (dF + dB == 0) ? ORC_Q / 2 : (uint64_t)ORC_Q * dF / (dF + dB);
      cs = lut_s[q]; ct = lut_t[q];
    }
    e[i] = cs - ct;
    st += ct;
  }
  free(lut_s); free(lut_t);
  *sink_total = st;
  return 0;
}

int orc_build_graph(int dims, int w, int h, int d, int pixfmt, const void* img,
                    const uint8_t* seeds, const orc_model* m, int32_t* e,
                    int32_t* const* caps, int64_t* sink_total, int32_t* centroids_out) {
  return orc_build_graph_ex(dims, w, h, d, pixfmt, img, seeds, seeds, m, e, caps, sink_total, centroids_out);
}

/* ------------------------------------------------------------- max-flow */

/* Exact sink distances over residual arcs: h = 0 on deficits (e < 0), BFS
 * backwards (graphcut_init_global_relabel / graphcut_global_relabel). */
static void global_relabel(const grid_t* g, const int64_t* e, int32_t* const* r, int32_t* h,
                           int64_t* queue) {
  int64_t qh = 0, qt = 0;
  for (int64_t i = 0; i < g->n; ++i) {
    if (e[i] < 0) { h[i] = 0; queue[qt++] = i; }
    else h[i] = ORC_INF;
  }
  while (qh < qt) {
    int64_t v = queue[qh++];
    for (int k = 0; k < g->conn; ++k) {
      if (!arc_ok(g, v, k)) continue;
      int64_t u = v + g->off[k];
      int rk = g->conn - 1 - k;            /* arc u -> v */
      if (h[u] == ORC_INF && r[rk][u] > 0) { h[u] = h[v] + 1; queue[qt++] = u; }
    }
  }
}

void orc_sink_distances(int dims, int w, int h, int d, const int32_t* e32, const int32_t* const* r,
                        int32_t* dist) {
  grid_t g; grid_init(&g, dims, w, h, d);
  int64_t* e = (int64_t*)malloc(sizeof(int64_t) * g.n);
  int64_t* queue = (int64_t*)malloc(sizeof(int64_t) * (g.n + 1));
  for (int64_t i = 0; i < g.n; ++i) e[i] = e32[i];
  global_relabel(&g, e, (int32_t* const*)r, dist, queue);
  free(e);
  free(queue);
}

int64_t orc_maxflow(int dims, int w, int h, int d, int32_t* e32, int32_t* const* r,
                    uint8_t* labels) {
  grid_t g; grid_init(&g, dims, w, h, d);
  int64_t n = g.n;
  /* arcs leaving the grid carry nothing */
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < g.conn; ++k)
      if (!arc_ok(&g, i, k)) r[k][i] = 0;
  int64_t* e = (int64_t*)malloc(sizeof(int64_t) * n);
  int32_t* hh = (int32_t*)malloc(sizeof(int32_t) * n);
  int64_t* queue = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
  uint8_t* inq = (uint8_t*)calloc((size_t)n, 1);
  int64_t pos0 = 0;
  for (int64_t i = 0; i < n; ++i) { e[i] = e32[i]; if (e[i] > 0) pos0 += e[i]; }

  int64_t qh = 0, qt = 0;   /* circular FIFO of active nodes */
  int64_t relabels = 0;
  global_relabel(&g, e, r, hh, queue);
  for (int64_t i = 0; i < n; ++i)
    if (e[i] > 0 && hh[i] < ORC_INF) { queue[qt++] = i; inq[i] = 1; }
  int64_t cap = n + 1;
  int64_t count = qt;
  while (count > 0) {
    int64_t u = queue[qh]; qh = (qh + 1) % cap; --count; inq[u] = 0;
    /* discharge u (graphcut_push_relabel.cl pushes along h(u) = h(v) + 1) */
    while (e[u] > 0 && hh[u] < ORC_INF) {
      int pushed = 0;
      for (int k = 0; k < g.conn && e[u] > 0; ++k) {
        int32_t rk = r[k][u];
        if (rk <= 0) continue;
        int64_t v = u + g.off[k];
        if (hh[u] != hh[v] + 1) continue;
        int64_t delta = e[u] < rk ? e[u] : rk;
        r[k][u] -= (int32_t)delta;
        r[g.conn - 1 - k][v] += (int32_t)delta;
        e[u] -= delta;
        int64_t before = e[v];
        e[v] += delta;
        if (before <= 0 && e[v] > 0 && !inq[v] && hh[v] < ORC_INF) {
          queue[(qh + count) % cap] = v; ++count; inq[v] = 1;
        }
        pushed = 1;
      }
      if (e[u] <= 0) break;
      if (!pushed || e[u] > 0) {
        /* relabel: h = 1 + min over residual arcs */
        int32_t m = ORC_INF;
        for (int k = 0; k < g.conn; ++k)
          if (r[k][u] > 0) {
            int32_t hv = hh[u + g.off[k]];
            if (hv + 1 < m) m = hv + 1;
          }
        hh[u] = m >= ORC_INF ? ORC_INF : m;
        ++relabels;
      }
      if (relabels > n) {
        /* periodic global relabel; rebuild the active queue */
        relabels = 0;
        global_relabel(&g, e, r, hh, queue);
        memset(inq, 0, (size_t)n);
        qh = 0; count = 0;
        for (int64_t i = 0; i < n; ++i)
          if (e[i] > 0 && hh[i] < ORC_INF && i != u) { queue[count++] = i; inq[i] = 1; }
        /* u itself continues below if still active */
      }
    }
  }
  int64_t pos1 = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (e[i] > 0) pos1 += e[i];
    e32[i] = (int32_t)e[i];
  }
  free(e); free(hh); free(queue); free(inq);
  if (labels) orc_cut_from_residual(dims, w, h, d, e32, (const int32_t* const*)r, labels);
  return pos0 - pos1;
}

int64_t orc_cut_from_residual(int dims, int w, int h, int d, const int32_t* e,
                              const int32_t* const* r, uint8_t* labels) {
  grid_t g; grid_init(&g, dims, w, h, d);
  int64_t* queue = (int64_t*)malloc(sizeof(int64_t) * (g.n + 1));
  int64_t qh = 0, qt = 0, bad = 0;
  for (int64_t i = 0; i < g.n; ++i) {
    labels[i] = e[i] > 0;
    if (labels[i]) queue[qt++] = i;
  }
  while (qh < qt) {
    int64_t u = queue[qh++];
    for (int k = 0; k < g.conn; ++k) {
      if (!arc_ok(&g, u, k) || r[k][u] <= 0) continue;
      int64_t v = u + g.off[k];
      if (!labels[v]) {
        labels[v] = 1; queue[qt++] = v;
        if (e[v] < 0) ++bad;
      }
    }
  }
  free(queue);
  return bad;
}

int64_t orc_cut_energy(int dims, int w, int h, int d, const int32_t* e0,
                       const int32_t* const* c0, const uint8_t* labels) {
  grid_t g; grid_init(&g, dims, w, h, d);
  int64_t data = 0, smooth = 0;
  for (int64_t i = 0; i < g.n; ++i) {
    if (labels[i]) {
      if (e0[i] < 0) data += -(int64_t)e0[i];
      for (int k = 0; k < g.conn; ++k)
        if (arc_ok(&g, i, k) && !labels[i + g.off[k]]) smooth += c0[k][i];
    } else if (e0[i] > 0) {
      data += e0[i];
    }
  }
  return data + smooth;
}

void orc_excess_sums(const int32_t* e, size_t n, int64_t* neg_sum, int64_t* pos_sum) {
  int64_t a = 0, b = 0;
  for (size_t i = 0; i < n; ++i) {
    if (e[i] < 0) a += e[i];
    else b += e[i];
  }
  *neg_sum = a; *pos_sum = b;
}

int64_t orc_check_residual(int dims, int w, int h, int d, const int32_t* e0,
                           const int32_t* const* c0, const int32_t* e,
                           const int32_t* const* r) {
  grid_t g; grid_init(&g, dims, w, h, d);
  int64_t bad = 0;
  for (int64_t i = 0; i < g.n; ++i) {
    int64_t inflow = 0;
    for (int k = 0; k < g.conn; ++k) {
      if (!arc_ok(&g, i, k)) continue;
      if (r[k][i] < 0) ++bad;
      int64_t v = i + g.off[k];
      int rk = g.conn - 1 - k;
      if ((int64_t)r[k][i] + r[rk][v] != (int64_t)c0[k][i] + c0[rk][v]) ++bad;
      inflow += (int64_t)r[k][i] - c0[k][i];
    }
    if ((int64_t)e0[i] + inflow != e[i]) ++bad;
  }
  return bad;
}
