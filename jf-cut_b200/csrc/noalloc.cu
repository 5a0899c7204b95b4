// noalloc.cu — a 2D solve that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they need a cut:
// real-time frame loops that must not stall on the allocator (a cudaMalloc
// can synchronise the device and take milliseconds), and hosts that hand this
// library a fixed memory budget up front and forbid allocations after it.
// jfc_solve_grid2d_noalloc serves them: the whole working set of the solve
// (residual graph, heights, labels, tile tables, work queues, counters) lives
// in one file-scope device array of fixed size, so the call itself performs no
// cudaMalloc / cudaFree / cudaMallocHost and uses no allocating library
// routine.  The caller passes device inputs and outputs.  The call reads a few
// counters back between relabel cycles, so it synchronises `stream` before it
// returns.
//
// Limits and sharing:
//  * grids whose padded size (width rounded up to 32, height rounded up to
//    16) is at most kMaxNodes = 524,288 nodes — e.g. 1024 x 512 or the
//    600 x 450 / 640 x 480 images that ship with the reference; larger grids
//    are rejected with JFC_ERR_INVALID_ARG;
//  * the array (about 13.2 MB) is held by every GPU that loads the library,
//    until the process exits;
//  * every call shares the array and it keeps the last call's contents (the
//    solve clears what must start at zero); calls that overlap on the GPU —
//    on two streams, or from two threads — race and corrupt each other;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, once per device, with that device current); make
//    that first call before any stream capture begins;
//  * the caller's current device is restored before the call returns.
#include <cstring>
#include <mutex>

#include "engine.h"

namespace {

constexpr int kMaxNodes = 1 << 19;                 // padded nodes
constexpr int kMaxTiles = kMaxNodes / (32 * 8);    // tiles at the smallest tile height
constexpr size_t al(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kPlane = al(sizeof(int) * (size_t)kMaxNodes);
constexpr size_t kTileI = al(sizeof(int) * (size_t)kMaxTiles);
// layout of the scratch array
constexpr size_t kOffE = 0;
constexpr size_t kOffH = kOffE + kPlane;
constexpr size_t kOffR = kOffH + kPlane;            // 4 residual planes
constexpr size_t kOffLabel = kOffR + 4 * kPlane;
constexpr size_t kOffDesc = kOffLabel + al(kMaxNodes);
constexpr size_t kOffInfo = kOffDesc + al(sizeof(GridDev));
constexpr size_t kOffFlagPr = kOffInfo + al(sizeof(int4) * (size_t)kMaxTiles);
constexpr size_t kOffQPr = kOffFlagPr + kTileI;     // 4 queues
constexpr size_t kOffFlagBfs = kOffQPr + 4 * kTileI; // 2 flag arrays
constexpr size_t kOffQBfs = kOffFlagBfs + 2 * kTileI; // 2 frontiers
constexpr size_t kOffAct = kOffQBfs + 2 * kTileI;
constexpr size_t kOffGact = kOffAct + al(kMaxTiles);
constexpr size_t kOffSum = kOffGact + 256;
constexpr size_t kOffCtr = kOffSum + 256;
constexpr size_t kOffBad = kOffCtr + al(sizeof(DevCounters));
constexpr size_t kBytes = kOffBad + 256;

std::mutex g_mu;
void* g_addr[128] = {nullptr};

// Restores the calling thread's current device when the call returns.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() { if (cudaGetDevice(&prev) != cudaSuccess) prev = -1; }
  ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

// tile t of a single grid: {grid 0, tx, ty, tz 0}
__global__ void k_na_tile_info(int4* info, int tiles_x, int ntiles) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x)
    info[t] = make_int4(0, t % tiles_x, t / tiles_x, 0);
}

}  // namespace

// The working set of jfc_solve_grid2d_noalloc.  In host code this name is a
// host-side stand-in, not a device address: kernels get the address from
// cudaGetSymbolAddress (na_scratch below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kBytes];

namespace {

int na_scratch(int device, char** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (device < 0 || device >= 128) return set_error(JFC_ERR_INVALID_ARG, "bad device index");
  if (!g_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return cuda_status(e, "cudaGetSymbolAddress(no-allocation scratch)");
    g_addr[device] = p;
  }
  *out = (char*)g_addr[device];
  return JFC_OK;
}

cudaError_t na_copy(void* padded, const void* dense, size_t elem, int w, int h, int pitch, int Hp, bool to_dense,
                    cudaStream_t s) {
  cudaMemcpy3DParms p{};
  cudaPitchedPtr pad = make_cudaPitchedPtr(padded, (size_t)pitch * elem, (size_t)pitch, (size_t)Hp);
  cudaPitchedPtr den = make_cudaPitchedPtr(const_cast<void*>(dense), (size_t)w * elem, (size_t)w, (size_t)h);
  p.srcPtr = to_dense ? pad : den;
  p.dstPtr = to_dense ? den : pad;
  p.extent = make_cudaExtent((size_t)w * elem, (size_t)h, 1);
  p.kind = cudaMemcpyDeviceToDevice;
  return cudaMemcpy3DAsync(&p, s);
}

// Read back the control block into caller-stack memory (no pinned buffer).
int na_read(void* host, const void* dev, size_t bytes, cudaStream_t s) {
  JFC_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
  JFC_CUDA(cudaStreamSynchronize(s));
  return JFC_OK;
}

int na_bfs(TileSet& ts, const jfc_params& p, bool cut, cudaStream_t s, int* active, int* cut_bad) {
  JFC_CUDA(cudaMemsetAsync(ts.d_flag_bfs[0], 0, sizeof(int) * (size_t)ts.ntiles, s));
  JFC_CUDA(cudaMemsetAsync(ts.d_flag_bfs[1], 0, sizeof(int) * (size_t)ts.ntiles, s));
  if (!cut) JFC_CUDA(cudaMemsetAsync(ts.d_grid_active, 0, sizeof(int), s));
  JFC_CUDA(cudaMemsetAsync(ts.d_ctr->ticket, 0, sizeof(ts.d_ctr->ticket), s));
  JFC_CUDA(cudaMemsetAsync(ts.d_ctr->qn_bfs, 0, sizeof(ts.d_ctr->qn_bfs), s));
  JFC_CUDA(cudaMemsetAsync(&ts.d_ctr->bfs_status, 0, sizeof(int), s));
  if (cut) JFC_CUDA(cudaMemsetAsync(&ts.d_ctr->cut_bad, 0, sizeof(int), s));
  JFC_CUDA(launch_bfs(ts, cut, p.max_bfs_passes, s));
  DevCounters hc;
  int rc = na_read(&hc, ts.d_ctr, sizeof(hc), s);
  if (rc) return rc;
  if (hc.error) return set_error(JFC_ERR_CUDA, "a device-side wait timed out in a persistent kernel (grid barrier, worklist or tile staging)");
  if (hc.bfs_status == 2) return set_error(JFC_ERR_NOT_CONVERGED, "BFS pass budget exhausted");
  if (!cut) {
    rc = na_read(active, ts.d_grid_active, sizeof(int), s);
    if (rc) return rc;
  } else {
    *cut_bad = hc.cut_bad;
  }
  return JFC_OK;
}

}  // namespace

extern "C" int jfc_solve_grid2d_noalloc(int device, void* stream, const jfc_params* params, int w, int h,
                                        const int32_t* d_excess, const int32_t* const* d_ncap,
                                        int64_t flow_offset, uint8_t* d_labels, int64_t* flow) {
  if (!d_excess || !d_ncap || !d_labels || !flow) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  for (int k = 0; k < 4; ++k)
    if (!d_ncap[k]) return set_error(JFC_ERR_INVALID_ARG, "null capacity array");
  if (w < 1 || h < 1) return set_error(JFC_ERR_INVALID_ARG, "empty grid");
  const int pitch = (w + JFC_TW - 1) / JFC_TW * JFC_TW;
  const int Hp = (h + JFC_PAD_Y2 - 1) / JFC_PAD_Y2 * JFC_PAD_Y2;
  if ((long long)pitch * Hp > kMaxNodes)
    return set_error(JFC_ERR_INVALID_ARG,
                     "grid exceeds the no-allocation limit of 524288 nodes (width padded to 32, height to 16)");
  jfc_params p{};
  if (params) p = *params;
  fill_defaults(p);
  DeviceGuard restore;
  JFC_CUDA(cudaSetDevice(device));
  char* base = nullptr;
  int rc = na_scratch(device, &base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t plane = (size_t)pitch * Hp;

  GridDev g;
  std::memset(&g, 0, sizeof(g));
  g.dims = 2; g.W = w; g.H = h; g.D = 1;
  g.pitch = pitch; g.Hp = Hp; g.Dp = 1;
  g.plane = (long long)plane;
  g.e = (int*)(base + kOffE);
  g.h = (int*)(base + kOffH);
  for (int k = 0; k < 4; ++k) g.r[k] = (int*)(base + kOffR + k * kPlane);
  g.r[4] = g.r[5] = g.r[0];
  g.label = (uint8_t*)(base + kOffLabel);
  const int TR = p.tile_rows;
  g.tiles_x = pitch / JFC_TW;
  g.tiles_y = Hp / TR;
  g.tiles_z = 1;
  g.tile_base = 0;

  TileSet ts;
  ts.dims = 2; ts.TR = TR; ts.TY = TR; ts.TZ = 1;
  ts.ngrids = 1;
  ts.ntiles = g.tiles_x * g.tiles_y;
  int npar0 = 0;
  for (int ty = 0; ty < g.tiles_y; ++ty) npar0 += (g.tiles_x + 1 - (ty & 1)) / 2;
  ts.nlist[0] = npar0;
  ts.nlist[1] = ts.ntiles - npar0;
  ts.d_desc = (GridDev*)(base + kOffDesc);
  ts.d_info = (int4*)(base + kOffInfo);
  ts.d_flag_pr = (int*)(base + kOffFlagPr);
  for (int q = 0; q < 4; ++q) ts.d_q_pr[q >> 1][q & 1] = (int*)(base + kOffQPr + q * kTileI);
  ts.d_flag_bfs[0] = (int*)(base + kOffFlagBfs);
  ts.d_flag_bfs[1] = (int*)(base + kOffFlagBfs + kTileI);
  ts.d_q_bfs[0] = (int*)(base + kOffQBfs);
  ts.d_q_bfs[1] = (int*)(base + kOffQBfs + kTileI);
  ts.d_act = (uint8_t*)(base + kOffAct);
  ts.d_grid_active = (int*)(base + kOffGact);
  ts.d_grid_sum = (long long*)(base + kOffSum);
  ts.d_ctr = (DevCounters*)(base + kOffCtr);
  int* d_bad = (int*)(base + kOffBad);

  // ---- stage the graph: clear the planes in use, copy the caller's arrays in,
  //      zero arcs leaving the grid, clear the tables the solve reads
  for (int k = 0; k < 6; ++k) JFC_CUDA(cudaMemsetAsync(base + kOffE + k * kPlane, 0, plane * sizeof(int), s));
  JFC_CUDA(cudaMemsetAsync(g.label, 0, plane, s));
  JFC_CUDA(na_copy(g.e, d_excess, 4, w, h, pitch, Hp, false, s));
  for (int k = 0; k < 4; ++k) JFC_CUDA(na_copy(g.r[k], d_ncap[k], 4, w, h, pitch, Hp, false, s));
  JFC_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
  JFC_CUDA(launch_fix_boundary(g, 4, d_bad, s));
  JFC_CUDA(cudaMemsetAsync(base + kOffFlagPr, 0, kOffBad - kOffFlagPr, s));
  JFC_CUDA(cudaMemcpyAsync(ts.d_desc, &g, sizeof(g), cudaMemcpyHostToDevice, s));
  jfc_note_launch();
  k_na_tile_info<<<(ts.ntiles + 255) / 256, 256, 0, s>>>(ts.d_info, g.tiles_x, ts.ntiles);
  JFC_CUDA(cudaGetLastError());
  int bad = 0;
  rc = na_read(&bad, d_bad, sizeof(int), s);
  if (rc) return rc;
  if (bad) return set_error(JFC_ERR_INVALID_ARG, "negative n-link capacity");
  long long sums[2];
  JFC_CUDA(launch_grid_sums(ts, s));
  rc = na_read(sums, ts.d_grid_sum, sizeof(sums), s);
  if (rc) return rc;
  const long long sink_total = (long long)flow_offset - sums[0];  // sum ct

  // ---- solve: global relabel, push-relabel phases, device-side active count
  JFC_CUDA(launch_clear_counters(ts, s));
  if (p.spin_limit > 0) JFC_CUDA(launch_set_limits(ts, (unsigned long long)p.spin_limit, 0, s));
  int active = 0, sweeps = 0;
  rc = na_bfs(ts, p, false, s, &active, nullptr);
  if (rc) return rc;
  while (active > 0) {
    if (sweeps >= p.max_sweeps) return set_error(JFC_ERR_NOT_CONVERGED, "sweep budget exhausted");
    JFC_CUDA(cudaMemsetAsync(ts.d_ctr->ticket, 0, sizeof(ts.d_ctr->ticket), s));
    JFC_CUDA(launch_pr_phase(ts, interval_for(p, 2), p.local_iters, s));
    rc = na_bfs(ts, p, false, s, &active, nullptr);
    if (rc) return rc;
    int sw = 0;
    rc = na_read(&sw, &ts.d_ctr->sweeps_done, sizeof(int), s);
    if (rc) return rc;
    sweeps += sw > 0 ? sw : 1;
  }
  int cut_bad = 0;
  rc = na_bfs(ts, p, true, s, nullptr, &cut_bad);
  if (rc) return rc;
  if (cut_bad) return set_error(JFC_ERR_NOT_CONVERGED, "cut BFS reached a deficit node");
  JFC_CUDA(launch_grid_sums(ts, s));
  rc = na_read(sums, ts.d_grid_sum, sizeof(sums), s);
  if (rc) return rc;
  JFC_CUDA(na_copy(g.label, d_labels, 1, w, h, pitch, Hp, true, s));
  JFC_CUDA(cudaStreamSynchronize(s));
  *flow = sink_total + sums[0];
  return JFC_OK;
}
