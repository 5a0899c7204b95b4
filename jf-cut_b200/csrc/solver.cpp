// solver.cpp — C ABI of the plain solver: context, grid graph, capacity build,
// solve, read-back, warm edits.
//
// Reference: QGCWidget (src/QVisualizer/Graph Cut/QGCWidget.h:160-243):
// initOpenCL / initConfigurations (QGCWidget.cpp:727-887) -> jfc_create /
// jfc_graph_create_grid; slotModelClicked (:2560-2606) -> jfc_graph_build_*;
// slotLoadGraphClicked (:2631-2736) -> jfc_graph_set; slotCutClicked
// (:2364-2558) -> jfc_solve; the cut read-back (:2454, 2990-2996) ->
// jfc_read_labels; reduceFlow + the energy print (:2406-2438, 2519) ->
// jfc_get_flow.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "engine.h"

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

void grid_layout(int dims, int w, int h, int d, int& pitch, int& Hp, int& Dp) {
  pitch = (w + JFC_TW - 1) / JFC_TW * JFC_TW;
  if (dims == 2) {
    Hp = (h + JFC_PAD_Y2 - 1) / JFC_PAD_Y2 * JFC_PAD_Y2;
    Dp = 1;
  } else {
    Hp = (h + JFC_PAD_Y3 - 1) / JFC_PAD_Y3 * JFC_PAD_Y3;
    Dp = (d + JFC_PAD_Z3 - 1) / JFC_PAD_Z3 * JFC_PAD_Z3;
  }
}

size_t state_bytes(int dims, int w, int h, int d) {
  int pitch, Hp, Dp;
  grid_layout(dims, w, h, d, pitch, Hp, Dp);
  const size_t plane = (size_t)pitch * Hp * Dp;
  const int conn = dims == 2 ? 4 : 6;
  return align256(plane * 4) * (2 + conn) + align256(plane);
}

void model_defaults(jfc_model& m) {
  if (m.lambda_n <= 0) m.lambda_n = 100;
  if (m.z_weight_pct <= 0) m.z_weight_pct = 100;
  if (m.lambda_t <= 0) m.lambda_t = 10;
  if (m.k_fg <= 0) m.k_fg = 5;
  if (m.k_bg <= 0) m.k_bg = 5;
  if (m.seed_cap <= 0) m.seed_cap = 1000000;
  if (m.kmeans_iters <= 0) m.kmeans_iters = 32;
}

// Copy a dense host / device array into (or out of) a padded plane.
cudaError_t copy_plane(void* padded, const void* dense, size_t elem, const jfc_graph* G, bool to_dense,
                       cudaMemcpyKind kind, cudaStream_t s) {
  cudaMemcpy3DParms p{};
  cudaPitchedPtr pad = make_cudaPitchedPtr(padded, (size_t)G->g.pitch * elem, (size_t)G->g.pitch, (size_t)G->g.Hp);
  cudaPitchedPtr den = make_cudaPitchedPtr(const_cast<void*>(dense), (size_t)G->W * elem, (size_t)G->W, (size_t)G->H);
  p.srcPtr = to_dense ? pad : den;
  p.dstPtr = to_dense ? den : pad;
  p.extent = make_cudaExtent((size_t)G->W * elem, (size_t)G->H, (size_t)G->D);
  p.kind = kind;
  return cudaMemcpy3DAsync(&p, s);
}

int ensure_tileset(jfc_graph* G) {
  const bool split = pr_split_for(G->ctx->params, G->dims);
  const int code = shape_code(G->dims, G->ctx->params.tile_rows, G->ctx->params.tile_depth, split);
  if (G->ts_shape == code) return JFC_OK;
  std::vector<GridDev> v{G->g};
  int rc = tileset_build(G->ts, G->dims, G->ctx->params.tile_rows, G->ctx->params.tile_depth, v, nullptr, split);
  if (rc) return rc;
  G->ts_shape = code;
  return JFC_OK;
}

struct BuildScratch {
  unsigned long long sum;
  unsigned long long sink;
  unsigned long long count[2];
  int minmax[12];
  unsigned int fill[2];
  KmeansDev km;
};

// n-link table: w(t) = round(scale * exp(-D(t) / (2 sigma^2))) with D(t) = t
// for RGB (t = ||dI||^2) and t^2 for scalar images (t = |dI|).
std::vector<int> nlink_table(int pixfmt, double scale, double sigma2) {
  const size_t n = pixfmt == JFC_PIX_RGB8 ? 3 * 255 * 255 + 1 : (pixfmt == JFC_PIX_I16 ? 65536 : 256);
  std::vector<int> lut(n);
  for (size_t t = 0; t < n; ++t) {
    const unsigned long long dsq = pixfmt == JFC_PIX_RGB8 ? t : (unsigned long long)t * t;
    if (sigma2 <= 0.0) lut[t] = (int)std::floor(scale + 0.5);
    else lut[t] = (int)std::floor(scale * std::exp(-(double)dsq / (2.0 * sigma2)) + 0.5);
  }
  return lut;
}

// Device buffers of the capacity build (kept for warm edits).
int ensure_model_buffers(jfc_graph* G, int pixfmt) {
  DevModel& M = G->model;
  const size_t n = (size_t)G->W * G->H * G->D;
  const size_t ib = n * jfc_pix_bytes(pixfmt);
  // stream-ordered allocations (no device-wide synchronisation when a server
  // frees a session while other work runs)
  cudaStream_t s = G->ctx->stream;
  if (M.d_img && M.img_bytes != ib) { JFC_CUDA(cudaFreeAsync(M.d_img, s)); M.d_img = nullptr; }
  if (!M.d_img) { JFC_CUDA(cudaMallocAsync(&M.d_img, ib, s)); M.img_bytes = ib; }
  if (!M.d_seeds) JFC_CUDA(cudaMallocAsync((void**)&M.d_seeds, n, s));
  if (!M.d_lut_s) JFC_CUDA(cudaMallocAsync((void**)&M.d_lut_s, sizeof(int) * (JFC_TQ + 1), s));
  if (!M.d_lut_t) JFC_CUDA(cudaMallocAsync((void**)&M.d_lut_t, sizeof(int) * (JFC_TQ + 1), s));
  return JFC_OK;
}

int build_core(jfc_graph* G, const void* img, int pixfmt, const uint8_t* seeds, const jfc_model* mdl,
               cudaMemcpyKind kind) {
  if (!G || !img || !seeds) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (pixfmt < JFC_PIX_GRAY8 || pixfmt > JFC_PIX_I16) return set_error(JFC_ERR_INVALID_ARG, "bad pixel format");
  jfc_model m{};
  if (mdl) m = *mdl;
  model_defaults(m);
  if (m.seed_cap > (1 << 28)) return set_error(JFC_ERR_INVALID_ARG, "seed_cap too large for int32 excess");
  cudaStream_t s = G->ctx->stream;
  int rc = ensure_model_buffers(G, pixfmt);
  if (rc) return rc;
  DevModel& M = G->model;
  const size_t n = (size_t)G->W * G->H * G->D;
  JFC_CUDA(cudaMemcpyAsync(M.d_img, img, M.img_bytes, kind, s));
  JFC_CUDA(cudaMemcpyAsync(M.d_seeds, seeds, n, kind, s));
  M.valid = false;

  // build temporaries are stream-ordered (no device-wide sync on free, so a
  // build overlaps other streams' kernels)
  BuildScratch* d_bs = nullptr;
  JFC_CUDA(cudaMallocAsync((void**)&d_bs, sizeof(BuildScratch), s));
  BuildScratch hbs;
  std::memset(&hbs, 0, sizeof(hbs));
  for (int i = 0; i < 12; ++i) hbs.minmax[i] = (i & 1) ? -1 : 0x7fffffff;
  std::vector<void*> temps{d_bs};
  auto cleanup = [&]() { for (void* p : temps) cudaFreeAsync(p, s); };
  auto fail = [&](int code) { cleanup(); return code; };
#define JFC_B(call) do { cudaError_t _e = (call); if (_e != cudaSuccess) return fail(cuda_status(_e, #call)); } while (0)

  JFC_B(cudaMemcpyAsync(d_bs, &hbs, sizeof(hbs), cudaMemcpyHostToDevice, s));
  // 1. contrast statistics -> sigma^2 -> n-link tables
  JFC_B(launch_contrast_sum(G->g, M.d_img, pixfmt, &d_bs->sum, s));
  JFC_B(launch_seed_stats(G->g, M.d_img, pixfmt, M.d_seeds, d_bs->minmax, d_bs->count, nullptr, nullptr,
                          d_bs->fill, false, s));
  JFC_B(cudaMemcpyAsync(&hbs, d_bs, sizeof(hbs), cudaMemcpyDeviceToHost, s));
  JFC_B(cudaStreamSynchronize(s));
  const unsigned long long W = G->W, H = G->H, D = G->D;
  const unsigned long long pairs = (W - 1) * H * D + W * (H - 1) * D + (G->dims == 3 ? W * H * (D - 1) : 0ull);
  const double sigma2 = pairs ? (double)hbs.sum / (double)pairs : 0.0;
  const double scale_xy = (double)m.lambda_n;
  const double scale_z = (double)m.lambda_n * (double)m.z_weight_pct / 100.0;
  // 2. seed lists
  const unsigned long long nf = hbs.count[0], nb = hbs.count[1];
  if (nf == 0 || nb == 0) { cleanup(); return set_error(JFC_ERR_NO_SEEDS, "no labels: a seed class is empty"); }
  uint32_t* d_list = nullptr;
  JFC_B(cudaMallocAsync((void**)&d_list, sizeof(uint32_t) * (nf + nb), s));
  temps.push_back(d_list);
  JFC_B(launch_seed_stats(G->g, M.d_img, pixfmt, M.d_seeds, d_bs->minmax, d_bs->count, d_list, d_list + nf,
                          d_bs->fill, true, s));

  // 3. k-means per class (fixed point 1/16, integer distances, order-free
  // sums), all iterations queued on the device; centres start evenly spaced
  // between the per-channel seed minimum and maximum
  const int C = jfc_pix_channels(pixfmt);
  KmeansDev& km = hbs.km;
  std::memset(&km, 0, sizeof(km));
  km.k[0] = std::min<int>(std::min(m.k_fg, JFC_MAX_K), (int)std::min<unsigned long long>(nf, JFC_MAX_K));
  km.k[1] = std::min<int>(std::min(m.k_bg, JFC_MAX_K), (int)std::min<unsigned long long>(nb, JFC_MAX_K));
  km.n[0] = nf;
  km.n[1] = nb;
  km.live[0] = km.live[1] = 1;
  for (int cls = 0; cls < 2; ++cls)
    for (int j = 0; j < km.k[cls]; ++j)
      for (int c = 0; c < C; ++c) {
        const long long mn = hbs.minmax[(cls * 3 + c) * 2], mx = hbs.minmax[(cls * 3 + c) * 2 + 1];
        km.mu[cls][j * 3 + c] = (int)(16 * mn + (16 * (mx - mn) * (2 * j + 1)) / (2 * km.k[cls]));
      }
  JFC_B(cudaMemcpyAsync(&d_bs->km, &km, sizeof(km), cudaMemcpyHostToDevice, s));
  JFC_B(launch_kmeans(d_list, &d_bs->km, pixfmt, std::max(nf, nb), m.kmeans_iters, s));

  // 4. while the device iterates: n-link tables (data-dependent sigma) and,
  // when lambda_t changed, the t-link tables over the quantised probability
  std::vector<int> lxy = nlink_table(pixfmt, scale_xy, sigma2);
  std::vector<int> lz = G->dims == 3 ? nlink_table(pixfmt, scale_z, sigma2) : std::vector<int>();
  int* d_lxy = nullptr;
  int* d_lz = nullptr;
  JFC_B(cudaMallocAsync((void**)&d_lxy, sizeof(int) * lxy.size(), s));
  temps.push_back(d_lxy);
  JFC_B(cudaMemcpyAsync(d_lxy, lxy.data(), sizeof(int) * lxy.size(), cudaMemcpyHostToDevice, s));
  if (!lz.empty()) {
    JFC_B(cudaMallocAsync((void**)&d_lz, sizeof(int) * lz.size(), s));
    temps.push_back(d_lz);
    JFC_B(cudaMemcpyAsync(d_lz, lz.data(), sizeof(int) * lz.size(), cudaMemcpyHostToDevice, s));
  }
  if (M.lut_lambda_t != m.lambda_t) {
    std::vector<int> ls(JFC_TQ + 1), lt(JFC_TQ + 1);
    for (int q = 0; q <= JFC_TQ; ++q) {
      const double pb = ((double)q + 0.5) / (double)(JFC_TQ + 1);
      const double pf = ((double)JFC_TQ + 0.5 - (double)q) / (double)(JFC_TQ + 1);
      ls[q] = (int)std::floor((double)m.lambda_t * -std::log(pb) + 0.5);
      lt[q] = (int)std::floor((double)m.lambda_t * -std::log(pf) + 0.5);
    }
    M.lut_lambda_t = -1;
    JFC_B(cudaMemcpyAsync(M.d_lut_s, ls.data(), sizeof(int) * ls.size(), cudaMemcpyHostToDevice, s));
    JFC_B(cudaMemcpyAsync(M.d_lut_t, lt.data(), sizeof(int) * lt.size(), cudaMemcpyHostToDevice, s));
    M.lut_lambda_t = m.lambda_t;
  }
  JFC_B(cudaMemcpyAsync(km.mu, d_bs->km.mu, sizeof(km.mu), cudaMemcpyDeviceToHost, s));
  JFC_B(cudaStreamSynchronize(s));
  const int (&mu)[2][JFC_MAX_K * 3] = km.mu;
  const int k[2] = {km.k[0], km.k[1]};

  BuildModelDev bm{};
  bm.pixfmt = pixfmt; bm.channels = C; bm.kf = k[0]; bm.kb = k[1]; bm.seed_cap = m.seed_cap;
  std::memcpy(bm.mu_f, mu[0], sizeof(bm.mu_f));
  std::memcpy(bm.mu_b, mu[1], sizeof(bm.mu_b));
  JFC_B(launch_build_graph(G->g, M.d_img, M.d_seeds, bm, d_lxy, d_lz ? d_lz : d_lxy, M.d_lut_s, M.d_lut_t,
                           &d_bs->sink, s));
  JFC_B(cudaMemcpyAsync(&hbs.sink, &d_bs->sink, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  JFC_B(cudaStreamSynchronize(s));
#undef JFC_B
  cleanup();
  M.m = bm;
  M.valid = true;
  G->sink_total = (long long)hbs.sink;
  G->state = 1;
  return JFC_OK;
}

int set_core(jfc_graph* G, const int32_t* e, const int32_t* const* ncap, int64_t offset, cudaMemcpyKind kind) {
  if (!G || !e || !ncap) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  for (int k = 0; k < G->conn; ++k)
    if (!ncap[k]) return set_error(JFC_ERR_INVALID_ARG, "null capacity array");
  cudaStream_t s = G->ctx->stream;
  JFC_CUDA(cudaMemsetAsync(G->d_state, 0, G->state_bytes, s));
  JFC_CUDA(copy_plane(G->g.e, e, 4, G, false, kind, s));
  for (int k = 0; k < G->conn; ++k) JFC_CUDA(copy_plane(G->g.r[k], ncap[k], 4, G, false, kind, s));
  int* d_bad = nullptr;
  JFC_CUDA(cudaMallocAsync((void**)&d_bad, sizeof(int), s));
  JFC_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
  cudaError_t err = launch_fix_boundary(G->g, G->conn, d_bad, s);
  int bad = 0;
  if (err == cudaSuccess) err = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  cudaFreeAsync(d_bad, s);
  if (err != cudaSuccess) return cuda_status(err, "graph set");
  if (bad) return set_error(JFC_ERR_INVALID_ARG, "negative n-link capacity");
  int rc = ensure_tileset(G);
  if (rc) return rc;
  JFC_CUDA(launch_grid_sums(G->ts, s));
  long long sums[2];
  JFC_CUDA(cudaMemcpyAsync(sums, G->ts.d_grid_sum, sizeof(sums), cudaMemcpyDeviceToHost, s));
  JFC_CUDA(cudaStreamSynchronize(s));
  // sum ct = sum min(cs, ct) + sum max(-e0, 0)
  G->sink_total = (long long)offset - sums[0];
  G->model.valid = false;
  G->state = 1;
  return JFC_OK;
}

extern "C" {

void jfc_default_params(jfc_params* out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  fill_defaults(*out);
  out->use_graph = 1;
}

void jfc_default_model(jfc_model* out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  model_defaults(*out);
}

const char* jfc_strerror(int status) {
  switch (status) {
    case JFC_OK: return "ok";
    case JFC_ERR_INVALID_ARG: return "invalid argument";
    case JFC_ERR_NO_SEEDS: return "no labels: both seed classes are required";
    case JFC_ERR_OOM: return "out of device memory / over HBM budget";
    case JFC_ERR_NOT_CONVERGED: return "iteration budget exhausted before convergence";
    case JFC_ERR_CUDA: return "CUDA error";
    case JFC_ERR_NO_DEVICE: return "no CUDA device";
    case JFC_ERR_STATE: return "call out of order";
    case JFC_ERR_CANCELLED: return "request cancelled";
    case JFC_ERR_BUSY: return "busy";
    case JFC_ERR_IO: return "data file I/O error";
    default: return "unknown status";
  }
}

int jfc_create(int device, const jfc_params* params, jfc_ctx** out) {
  if (!out) return set_error(JFC_ERR_INVALID_ARG, "null out");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return set_error(JFC_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= n) return set_error(JFC_ERR_INVALID_ARG, "bad device index");
  JFC_CUDA(cudaSetDevice(device));
  jfc_ctx* c = new jfc_ctx();
  c->device = device;
  if (params) c->params = *params;
  else jfc_default_params(&c->params);
  fill_defaults(c->params);
  {
    // stream-ordered temporaries (capacity build, edits) come from the
    // device's default pool: keep up to 1 GiB of freed blocks mapped instead
    // of returning them at every synchronisation
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = 1ull << 30, cur = 0;
      if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur) == cudaSuccess && cur < keep)
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return cuda_status(e, "cudaStreamCreate"); }
  c->stream = c->own_stream;
  *out = c;
  return JFC_OK;
}

void jfc_destroy(jfc_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  if (c->h_pin) cudaFreeHost(c->h_pin);
  delete c;
}

int jfc_set_stream(jfc_ctx* c, void* stream) {
  if (!c) return set_error(JFC_ERR_INVALID_ARG, "null context");
  JFC_CUDA(cudaSetDevice(c->device));
  JFC_CUDA(cudaStreamSynchronize(c->stream));
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return JFC_OK;
}

int jfc_set_params(jfc_ctx* c, const jfc_params* params) {
  if (!c || !params) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (params->tile_rows && params->tile_rows != 8 && params->tile_rows != 16)
    return set_error(JFC_ERR_INVALID_ARG, "tile_rows must be 8 or 16");
  // tile depth 4 with tile_rows 8 falls back to the default depth (2)
  if (params->tile_depth && params->tile_depth != 1 && params->tile_depth != 2 && params->tile_depth != 4)
    return set_error(JFC_ERR_INVALID_ARG, "tile_depth must be 1, 2 or 4");
  c->params = *params;
  fill_defaults(c->params);
  return JFC_OK;
}

int jfc_get_params(jfc_ctx* c, jfc_params* out) {
  if (!c || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  *out = c->params;
  return JFC_OK;
}

size_t jfc_graph_bytes(int dims, int w, int h, int d) {
  if (dims == 2) d = 1;
  return state_bytes(dims, w, h, d);
}

int jfc_graph_create_grid(jfc_ctx* c, int dims, int w, int h, int d, int conn, jfc_graph** out) {
  if (!c || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (dims == 2) d = 1;
  if ((dims != 2 && dims != 3) || (dims == 2 && conn != 4) || (dims == 3 && conn != 6))
    return set_error(JFC_ERR_INVALID_ARG, "supported: dims 2 / conn 4, dims 3 / conn 6");
  if (w < 1 || h < 1 || d < 1) return set_error(JFC_ERR_INVALID_ARG, "empty grid");
  if ((long long)w * h * d > (1ll << 32) - 1) return set_error(JFC_ERR_INVALID_ARG, "grid larger than 2^32 nodes");
  JFC_CUDA(cudaSetDevice(c->device));
  jfc_graph* G = new jfc_graph();
  G->ctx = c;
  G->device = c->device;
  G->dims = dims; G->W = w; G->H = h; G->D = d; G->conn = conn;
  int pitch, Hp, Dp;
  grid_layout(dims, w, h, d, pitch, Hp, Dp);
  const size_t plane = (size_t)pitch * Hp * Dp;
  G->state_bytes = state_bytes(dims, w, h, d);
  // stream-ordered allocation on the context's stream (its release never
  // synchronises the device, see graph_release), zeroed there, ordered
  // before every later use of it
  cudaError_t e = cudaMallocAsync(&G->d_state, G->state_bytes, c->stream);
  if (e != cudaSuccess) { delete G; return cuda_status(e, "graph allocation"); }
  e = cudaMemsetAsync(G->d_state, 0, G->state_bytes, c->stream);
  if (e != cudaSuccess) { cudaFreeAsync(G->d_state, c->stream); delete G; return cuda_status(e, "graph clear"); }
  char* p = (char*)G->d_state;
  GridDev& g = G->g;
  std::memset(&g, 0, sizeof(g));
  g.dims = dims; g.W = w; g.H = h; g.D = d;
  g.pitch = pitch; g.Hp = Hp; g.Dp = Dp;
  g.plane = (long long)plane;
  const size_t pb = align256(plane * 4);
  g.e = (int*)p; p += pb;
  g.h = (int*)p; p += pb;
  for (int k = 0; k < conn; ++k) { g.r[k] = (int*)p; p += pb; }
  for (int k = conn; k < 6; ++k) g.r[k] = g.r[0];
  g.label = (uint8_t*)p;
  *out = G;
  return JFC_OK;
}

void jfc_graph_destroy(jfc_graph* G) {
  if (!G) return;
  // the context may already be gone: use only what the graph owns; nothing
  // may still run on the graph's memory when it goes back to the pool
  cudaSetDevice(G->device);
  cudaDeviceSynchronize();
  tileset_free(G->ts);
  if (G->d_state) cudaFree(G->d_state);
  if (G->model.d_img) cudaFree(G->model.d_img);
  if (G->model.d_seeds) cudaFree(G->model.d_seeds);
  if (G->model.d_lut_s) cudaFree(G->model.d_lut_s);
  if (G->model.d_lut_t) cudaFree(G->model.d_lut_t);
  delete G;
}

}  // extern "C"

void graph_release(jfc_graph* G, cudaStream_t s) {
  if (!G) return;
  tileset_free(G->ts);
  if (G->d_state) cudaFreeAsync(G->d_state, s);
  if (G->model.d_img) cudaFreeAsync(G->model.d_img, s);
  if (G->model.d_seeds) cudaFreeAsync(G->model.d_seeds, s);
  if (G->model.d_lut_s) cudaFreeAsync(G->model.d_lut_s, s);
  if (G->model.d_lut_t) cudaFreeAsync(G->model.d_lut_t, s);
  delete G;
}

extern "C" {

int jfc_graph_build_from_image(jfc_graph* g, const void* img, int pixfmt, const uint8_t* seeds,
                               const jfc_model* model) {
  if (!g) return set_error(JFC_ERR_INVALID_ARG, "null graph");
  JFC_CUDA(cudaSetDevice(g->ctx->device));
  return build_core(g, img, pixfmt, seeds, model, cudaMemcpyHostToDevice);
}

int jfc_graph_build_from_device(jfc_graph* g, const void* d_img, int pixfmt, const uint8_t* d_seeds,
                                const jfc_model* model) {
  if (!g) return set_error(JFC_ERR_INVALID_ARG, "null graph");
  JFC_CUDA(cudaSetDevice(g->ctx->device));
  return build_core(g, d_img, pixfmt, d_seeds, model, cudaMemcpyDeviceToDevice);
}

int jfc_graph_set(jfc_graph* g, const int32_t* excess, const int32_t* const* ncap, int64_t flow_offset) {
  if (!g) return set_error(JFC_ERR_INVALID_ARG, "null graph");
  JFC_CUDA(cudaSetDevice(g->ctx->device));
  return set_core(g, excess, ncap, flow_offset, cudaMemcpyHostToDevice);
}

int jfc_graph_set_device(jfc_graph* g, const int32_t* d_excess, const int32_t* const* d_ncap,
                         int64_t flow_offset) {
  if (!g) return set_error(JFC_ERR_INVALID_ARG, "null graph");
  JFC_CUDA(cudaSetDevice(g->ctx->device));
  return set_core(g, d_excess, d_ncap, flow_offset, cudaMemcpyDeviceToDevice);
}

int jfc_graph_get_state(jfc_graph* G, int32_t* excess, int32_t* const* ncap, int32_t* height) {
  if (!G) return set_error(JFC_ERR_INVALID_ARG, "null graph");
  if (G->state == 0) return set_error(JFC_ERR_STATE, "graph is empty");
  JFC_CUDA(cudaSetDevice(G->ctx->device));
  cudaStream_t s = G->ctx->stream;
  if (excess) JFC_CUDA(copy_plane(G->g.e, excess, 4, G, true, cudaMemcpyDeviceToHost, s));
  if (height) JFC_CUDA(copy_plane(G->g.h, height, 4, G, true, cudaMemcpyDeviceToHost, s));
  if (ncap)
    for (int k = 0; k < G->conn; ++k)
      if (ncap[k]) JFC_CUDA(copy_plane(G->g.r[k], ncap[k], 4, G, true, cudaMemcpyDeviceToHost, s));
  JFC_CUDA(cudaStreamSynchronize(s));
  return JFC_OK;
}

int jfc_solve(jfc_graph* G, jfc_stats* stats) {
  if (!G) return set_error(JFC_ERR_INVALID_ARG, "null graph");
  if (G->state == 0) return set_error(JFC_ERR_STATE, "no graph loaded");
  JFC_CUDA(cudaSetDevice(G->ctx->device));
  int rc = ensure_tileset(G);
  if (rc) return rc;
  std::vector<GridResult> res;
  jfc_stats st;
  rc = engine_solve(G->ctx, G->ts, G->ctx->params, res, st, &G->g);
  if (rc && rc != JFC_ERR_NOT_CONVERGED) return rc;
  G->flow = G->sink_total + res[0].neg_sum;
  G->source_nodes = res[0].labels;
  st.flow = G->flow;
  st.source_nodes = G->source_nodes;
  st.status = rc;
  G->last = st;
  if (stats) *stats = st;
  G->state = rc ? 1 : 2;
  return rc;
}

int jfc_get_flow(jfc_graph* G, int64_t* flow) {
  if (!G || !flow) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (G->state != 2) return set_error(JFC_ERR_STATE, "not solved");
  *flow = G->flow;
  return JFC_OK;
}

int jfc_read_labels(jfc_graph* G, uint8_t* out) {
  if (!G || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (G->state != 2) return set_error(JFC_ERR_STATE, "not solved");
  JFC_CUDA(cudaSetDevice(G->ctx->device));
  cudaStream_t s = G->ctx->stream;
  JFC_CUDA(copy_plane(G->g.label, out, 1, G, true, cudaMemcpyDeviceToHost, s));
  JFC_CUDA(cudaStreamSynchronize(s));
  return JFC_OK;
}

int jfc_read_labels_device(jfc_graph* G, uint8_t* d_out) {
  if (!G || !d_out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (G->state != 2) return set_error(JFC_ERR_STATE, "not solved");
  JFC_CUDA(cudaSetDevice(G->ctx->device));
  cudaStream_t s = G->ctx->stream;
  JFC_CUDA(copy_plane(G->g.label, d_out, 1, G, true, cudaMemcpyDeviceToDevice, s));
  JFC_CUDA(cudaStreamSynchronize(s));
  return JFC_OK;
}

int jfc_edit_tlinks(jfc_graph* G, const uint32_t* idx, const int32_t* dcs, const int32_t* dct, size_t n) {
  if (!G || (n && (!idx || !dcs || !dct))) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (G->state == 0) return set_error(JFC_ERR_STATE, "no graph loaded");
  const unsigned long long N = (unsigned long long)G->W * G->H * G->D;
  for (size_t j = 0; j < n; ++j)
    if (idx[j] >= N) return set_error(JFC_ERR_INVALID_ARG, "edit index out of range");
  if (n == 0) return JFC_OK;
  JFC_CUDA(cudaSetDevice(G->ctx->device));
  cudaStream_t s = G->ctx->stream;
  char* buf = nullptr;
  const size_t bytes = align256(n * 4) * 3 + 256;
  JFC_CUDA(cudaMallocAsync((void**)&buf, bytes, s));
  uint32_t* d_idx = (uint32_t*)buf;
  int32_t* d_dcs = (int32_t*)(buf + align256(n * 4));
  int32_t* d_dct = (int32_t*)(buf + 2 * align256(n * 4));
  long long* d_ds = (long long*)(buf + 3 * align256(n * 4));
  cudaError_t e = cudaMemcpyAsync(d_idx, idx, n * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_dcs, dcs, n * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_dct, dct, n * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_ds, 0, sizeof(long long), s);
  if (e == cudaSuccess) e = launch_edit_tlinks(G->g, d_idx, d_dcs, d_dct, n, d_ds, s);
  long long ds = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ds, d_ds, sizeof(ds), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(buf, s);
  if (e != cudaSuccess) return cuda_status(e, "edit t-links");
  G->sink_total += ds;
  G->state = 1;
  return JFC_OK;
}

int jfc_graph_compute_tag(jfc_graph* G, const uint8_t* seeds, uint8_t* tag) {
  if (!G || !tag) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (G->state != 2) return set_error(JFC_ERR_STATE, "not solved");
  if (!seeds && !G->model.valid) return set_error(JFC_ERR_STATE, "no seeds: graph was not built from an image");
  JFC_CUDA(cudaSetDevice(G->ctx->device));
  int rc = ensure_tileset(G);
  if (rc) return rc;
  cudaStream_t s = G->ctx->stream;
  const size_t n = (size_t)G->W * G->H * G->D;
  uint8_t* d_seeds = G->model.valid && !seeds ? G->model.d_seeds : nullptr;
  uint8_t* d_tmp = nullptr;
  if (seeds) {
    JFC_CUDA(cudaMallocAsync((void**)&d_tmp, n, s));
    d_seeds = d_tmp;
  }
  TileSet& ts = G->ts;
  DevCounters hc;
  cudaError_t e = seeds ? cudaMemcpyAsync(d_tmp, seeds, n, cudaMemcpyHostToDevice, s) : cudaSuccess;
  if (e == cudaSuccess) e = cudaMemsetAsync(ts.d_flag_bfs[0], 0, sizeof(int) * (size_t)ts.ntiles, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(ts.d_flag_bfs[1], 0, sizeof(int) * (size_t)ts.ntiles, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(ts.d_ctr->ticket, 0, sizeof(ts.d_ctr->ticket), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(ts.d_ctr->qn_bfs, 0, sizeof(ts.d_ctr->qn_bfs), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(&ts.d_ctr->bfs_status, 0, sizeof(int), s);
  if (e == cudaSuccess) e = launch_tag(ts, d_seeds, G->ctx->params.max_bfs_passes, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hc, ts.d_ctr, sizeof(hc), cudaMemcpyDeviceToHost, s);
  // tags leave in bit 1 of the label plane; the plane is restored afterwards
  if (e == cudaSuccess) e = copy_plane(G->g.label, tag, 1, G, true, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = launch_and_bytes(G->g.label, G->g.plane, 1, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (d_tmp) cudaFreeAsync(d_tmp, s);
  if (e != cudaSuccess) return cuda_status(e, "tag");
  if (hc.error) return set_error(JFC_ERR_CUDA, "a device-side wait timed out in a persistent kernel (grid barrier, worklist or tile staging)");
  if (hc.bfs_status == 2) return set_error(JFC_ERR_NOT_CONVERGED, "BFS pass budget exhausted");
  for (size_t i = 0; i < n; ++i) tag[i] = (tag[i] >> 1) & 1u;
  return JFC_OK;
}

int jfc_stroke_to_seeds(int device, void* stream, const jfc_view* view, int w, int h, int d,
                        const float* d_volume, const float* d_tf_rgba, int tf_size, const uint8_t* d_mask,
                        uint8_t label, uint8_t* d_seeds) {
  if (!view || !d_volume || !d_tf_rgba || !d_mask || !d_seeds) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (w < 2 || h < 2 || d < 2 || tf_size < 1 || view->samples < 3 || view->image_w < 1 || view->image_h < 1 ||
      !(view->box[0] > 0 && view->box[1] > 0 && view->box[2] > 0) || label > JFC_SEED_BG)
    return set_error(JFC_ERR_INVALID_ARG, "bad volume, view or label");
  JFC_CUDA(cudaSetDevice(device));
  cudaStream_t s = (cudaStream_t)stream;
  JFC_CUDA(launch_stroke_seeds(*view, w, h, d, d_volume, d_tf_rgba, tf_size, d_mask, label, d_seeds, s));
  JFC_CUDA(cudaStreamSynchronize(s));
  return JFC_OK;
}

int jfc_energy_device(int device, void* stream, int dims, int w, int h, int d, const int32_t* d_excess,
                      const int32_t* const* d_ncap, const uint8_t* d_labels, int64_t* data, int64_t* smooth) {
  if (!d_excess || !d_ncap || !d_labels || !data || !smooth) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (dims == 2) d = 1;
  if ((dims != 2 && dims != 3) || w < 1 || h < 1 || d < 1) return set_error(JFC_ERR_INVALID_ARG, "bad grid shape");
  for (int k = 0; k < (dims == 3 ? 6 : 4); ++k)
    if (!d_ncap[k]) return set_error(JFC_ERR_INVALID_ARG, "null capacity array");
  JFC_CUDA(cudaSetDevice(device));
  cudaStream_t s = (cudaStream_t)stream;
  unsigned long long* d_out = nullptr;
  JFC_CUDA(cudaMallocAsync((void**)&d_out, 2 * sizeof(unsigned long long), s));
  unsigned long long h_out[2] = {0, 0};
  cudaError_t e = cudaMemsetAsync(d_out, 0, sizeof(h_out), s);
  if (e == cudaSuccess) e = launch_energy(dims, w, h, d, d_excess, d_ncap, d_labels, d_out, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_out, d_out, sizeof(h_out), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(d_out, s);
  if (e != cudaSuccess) return cuda_status(e, "energy");
  *data = (int64_t)h_out[0];
  *smooth = (int64_t)h_out[1];
  return JFC_OK;
}

int jfc_graph_edit_seeds(jfc_graph* G, const uint32_t* idx, const uint8_t* new_seed, size_t n) {
  if (!G || (n && (!idx || !new_seed))) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (!G->model.valid) return set_error(JFC_ERR_STATE, "graph was not built from an image");
  const unsigned long long N = (unsigned long long)G->W * G->H * G->D;
  for (size_t j = 0; j < n; ++j)
    if (idx[j] >= N || new_seed[j] > 2) return set_error(JFC_ERR_INVALID_ARG, "bad edit");
  if (n == 0) return JFC_OK;
  if (n > (size_t)0x7fffffff) return set_error(JFC_ERR_INVALID_ARG, "edit list too long");
  // duplicates are resolved on the device (the last entry of a node wins)
  const size_t m = n;
  JFC_CUDA(cudaSetDevice(G->ctx->device));
  cudaStream_t s = G->ctx->stream;
  char* buf = nullptr;
  JFC_CUDA(cudaMallocAsync((void**)&buf, align256(m * 4) + align256(m) + 256, s));
  uint32_t* d_idx = (uint32_t*)buf;
  uint8_t* d_new = (uint8_t*)(buf + align256(m * 4));
  long long* d_ds = (long long*)(buf + align256(m * 4) + align256(m));
  cudaError_t e = cudaMemcpyAsync(d_idx, idx, m * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_new, new_seed, m, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_ds, 0, sizeof(long long), s);
  if (e == cudaSuccess)
    e = launch_edit_seeds(G->g, G->model.d_img, G->model.d_seeds, G->model.m, G->model.d_lut_s,
                          G->model.d_lut_t, d_idx, d_new, m, d_ds, s);
  long long ds = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ds, d_ds, sizeof(ds), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(buf, s);
  if (e != cudaSuccess) return cuda_status(e, "edit seeds");
  G->sink_total += ds;
  G->state = 1;
  return JFC_OK;
}

}  // extern "C"
