// ref_api.cpp — C entry points over the reference's own CPU max-flow solvers,
// compiled from their sources under the reference tree by oracle/Makefile into
// oracle/_ref/libjfcref.so.  TEST INFRASTRUCTURE ONLY: the checker and the
// timed CPU baseline; the product never links it.
//
// The graph construction mirrors the reference harness
// (benchmark/GridCut/bench-BK303.cpp:18-108 and bench-GridCut.cpp:26-216):
// net excess e is split into cs = max(e,0), ct = max(-e,0) as QGCWidget::saveMFI
// does (QGCWidget.cpp:3380-3393), every arc pair goes in with add_edge /
// set_caps, and the minimal source side is what_segment(i, SINK) == SOURCE
// (BK303/graph.h:136,486).
#include <graph.h>
#include <GridCut/GridGraph_2D_4C_MT.h>
#include <GridCut/GridGraph_3D_6C_MT.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {
double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
}  // namespace

extern "C" {

// BK 3.03 with Graph<int,int,long long>.  Returns the folded max-flow (the
// caller adds sum min(cs,ct)).  times[3] = init, maxflow, output seconds.
long long ref_bk_maxflow(int dims, int w, int h, int d, const int32_t* e,
                         const int32_t* const* caps, uint8_t* labels, double* times) {
  typedef Graph<int, int, long long> G;
  if (dims == 2) d = 1;
  const long long n = (long long)w * h * d;
  const long long wh = (long long)w * h;
  double t0 = now_s();
  G* g = new G((int)n, (int)(n * (dims == 2 ? 2 : 3)));
  g->add_node((int)n);
  for (int z = 0; z < d; ++z)
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        long long i = x + (long long)w * y + wh * z;
        int ei = e[i];
        g->add_tweights((int)i, ei > 0 ? ei : 0, ei < 0 ? -ei : 0);
        if (dims == 2) {
          // caps order +x +y -y -x
          if (x < w - 1) g->add_edge((int)i, (int)(i + 1), caps[0][i], caps[3][i + 1]);
          if (y < h - 1) g->add_edge((int)i, (int)(i + w), caps[1][i], caps[2][i + w]);
        } else {
          // caps order +x +y +z -z -y -x
          if (x < w - 1) g->add_edge((int)i, (int)(i + 1), caps[0][i], caps[5][i + 1]);
          if (y < h - 1) g->add_edge((int)i, (int)(i + w), caps[1][i], caps[4][i + w]);
          if (z < d - 1) g->add_edge((int)i, (int)(i + wh), caps[2][i], caps[3][i + wh]);
        }
      }
  double t1 = now_s();
  long long flow = g->maxflow();
  double t2 = now_s();
  if (labels)
    for (long long i = 0; i < n; ++i) labels[i] = g->what_segment((int)i, G::SINK) == G::SOURCE;
  delete g;
  double t3 = now_s();
  if (times) { times[0] = t1 - t0; times[1] = t2 - t1; times[2] = t3 - t2; }
  return flow;
}

// GridCut 1.1 multi-threaded (the reference harness's MT path,
// bench-GridCut.cpp:76-216, block_size rule from :92/:192).  Folded flow.
// labels (may be NULL): 1 where get_segment reports the source side
// (GridGraph_2D_4C_MT.h:1152-1157); times[2] covers that read-back.
long long ref_gridcut_maxflow(int dims, int w, int h, int d, const int32_t* e,
                              const int32_t* const* caps, int threads, uint8_t* labels, double* times) {
  if (dims == 2) d = 1;
  const long long n = (long long)w * h * d;
  if (threads < 1) threads = 1;
  double t0 = now_s();
  std::vector<int> cs(n), ct(n);
  for (long long i = 0; i < n; ++i) {
    cs[i] = e[i] > 0 ? e[i] : 0;
    ct[i] = e[i] < 0 ? -e[i] : 0;
  }
  long long flow;
  double t1, t2;
  if (dims == 2) {
    typedef GridGraph_2D_4C_MT<int, int, long long> G;
    int bs = (int)(std::exp(std::log((double)w * h / threads) / 2) + 0.5);
    if (bs < 1) bs = 1;
    G* g = new G(w, h, threads, bs);
    g->set_caps(cs.data(), ct.data(), caps[3], caps[0], caps[2], caps[1]);
    t1 = now_s();
    g->compute_maxflow();
    t2 = now_s();
    flow = g->get_flow();
    if (labels)
      for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) labels[(long long)y * w + x] = g->get_segment(g->node_id(x, y)) == 0;
    delete g;
  } else {
    typedef GridGraph_3D_6C_MT<int, int, long long> G;
    int bs = (int)(std::exp(std::log((double)w * h * d / threads) / 3) + 0.5);
    if (bs < 1) bs = 1;
    G* g = new G(w, h, d, threads, bs);
    g->set_caps(cs.data(), ct.data(), caps[5], caps[0], caps[4], caps[1], caps[3], caps[2]);
    t1 = now_s();
    g->compute_maxflow();
    t2 = now_s();
    flow = g->get_flow();
    if (labels)
      for (int z = 0; z < d; ++z)
        for (int y = 0; y < h; ++y)
          for (int x = 0; x < w; ++x)
            labels[(long long)w * h * z + (long long)y * w + x] = g->get_segment(g->node_id(x, y, z)) == 0;
    delete g;
  }
  double t3 = now_s();
  if (times) { times[0] = t1 - t0; times[1] = t2 - t1; times[2] = t3 - t2; }
  return flow;
}

}  // extern "C"
