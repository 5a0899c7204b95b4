// kernels_fast.cu — the reference's Fast-Cut variant (wave pushes along lines),
// kept as an in-framework comparison with the block-wise push-relabel.
//
// Reference: graphcut_push_relabel_fast.cl (graphcut_fast_relabel,
// graphcut_fast_push_x / _y / _z) driven by QGCWidget::relabelPushFast
// (QGCWidget.cpp:2156-2206): one relabel of every node in checkerboard parity
// (h = 1 + min over residual arcs, for nodes without a deficit), then one
// thread per line segment sweeps forward and backward pushing excess along
// admissible arcs, segments of alternating parity in separate launches so
// neighbouring segments never run at once; the last push of a segment lands
// in the first node of the next one.
//
// Here: the same steps on the padded SoA planes, one launch per step and
// parity; the exact global relabel and convergence test of the block solver
// run between groups of iterations (the schedule is the engine's).
#include "jfc_internal.h"

namespace {

constexpr int kSeg = 32;   // nodes per line segment of one thread

// h = 1 + min over residual arcs for nodes of one parity without a deficit
template <int DIMS>
__global__ void __launch_bounds__(256) k_fast_relabel(GridDev g, int parity) {
  const long long total = g.plane;
  const long long slab = (long long)g.pitch * g.Hp;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < total;
       n += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(n % g.pitch);
    const long long yz = n / g.pitch;
    const int y = (int)(yz % g.Hp), z = (int)(yz / g.Hp);
    if (((x + y + z) & 1) != parity) continue;
    if (x >= g.W || y >= g.H || z >= g.D) continue;
    if (g.e[n] < 0) continue;
    const int h0 = g.h[n];
    if (h0 >= JFC_INF) continue;
    int m = JFC_INF;
    // channel order 2D: +x, +y, -y, -x; 3D: +x, +y, +z, -z, -y, -x
    if (g.r[0][n] > 0) m = min(m, g.h[n + 1] + 1);
    if (g.r[1][n] > 0) m = min(m, g.h[n + g.pitch] + 1);
    if constexpr (DIMS == 2) {
      if (g.r[2][n] > 0) m = min(m, g.h[n - g.pitch] + 1);
      if (g.r[3][n] > 0) m = min(m, g.h[n - 1] + 1);
    } else {
      if (g.r[2][n] > 0) m = min(m, g.h[n + slab] + 1);
      if (g.r[3][n] > 0) m = min(m, g.h[n - slab] + 1);
      if (g.r[4][n] > 0) m = min(m, g.h[n - g.pitch] + 1);
      if (g.r[5][n] > 0) m = min(m, g.h[n - 1] + 1);
    }
    m = min(m, JFC_INF);
    if (m != h0) g.h[n] = m;
  }
}

// One thread per segment of kSeg nodes along `axis` (0 x, 1 y, 2 z); segments
// whose index has the given parity.  Forward sweep, then backward sweep; a
// push across the segment end goes into the neighbouring segment (other
// parity, not running).
template <int DIMS, int AXIS>
__global__ void __launch_bounds__(256) k_fast_push(GridDev g, int parity, int* moved) {
  const int len = AXIS == 0 ? g.W : AXIS == 1 ? g.H : g.D;
  const int nseg = (len + kSeg - 1) / kSeg;
  // lines: all (other two coordinates) combinations
  const int o1 = AXIS == 0 ? g.H : g.W;                   // first other extent
  const int o2 = DIMS == 3 ? (AXIS == 2 ? g.H : g.D) : 1; // second other extent
  const long long stride = AXIS == 0 ? 1 : AXIS == 1 ? g.pitch : (long long)g.pitch * g.Hp;
  const int kf = AXIS == 0 ? 0 : 1;                            // +axis arc slot
  const int kb = DIMS == 2 ? (AXIS == 0 ? 3 : 2) : (AXIS == 0 ? 5 : AXIS == 1 ? 4 : 3);   // -axis
  const int kz = 2;                                            // +z slot (3D)
  const int slot_f = AXIS == 2 ? kz : kf;
  const long long lines = (long long)o1 * o2;
  const long long work = lines * ((nseg + 1 - parity) / 2);
  bool any = false;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < work;
       w += (long long)gridDim.x * blockDim.x) {
    const long long line = w % lines;
    const int seg = (int)(w / lines) * 2 + parity;
    if (seg >= nseg) continue;
    const int a = (int)(line % o1), b = (int)(line / o1);
    int x, y, z;
    if (AXIS == 0) { x = 0; y = a; z = b; }
    else if (AXIS == 1) { x = a; y = 0; z = b; }
    else { x = a; y = b; z = 0; }
    const long long base = (long long)x + (long long)y * g.pitch + (long long)z * g.pitch * g.Hp;
    const int s0 = seg * kSeg;
    const int cnt = min(kSeg, len - s0);
    const long long n0 = base + (long long)s0 * stride;
    int e[kSeg], h[kSeg];
#pragma unroll
    for (int i = 0; i < kSeg; ++i)
      if (i < cnt) { e[i] = g.e[n0 + i * stride]; h[i] = g.h[n0 + i * stride]; }
    int e_in[kSeg];
#pragma unroll
    for (int i = 0; i < kSeg; ++i) e_in[i] = e[i];
    // forward: node i pushes to i+1 (the last one into the next segment)
#pragma unroll
    for (int i = 0; i < kSeg; ++i) {
      if (i >= cnt) break;
      const long long n = n0 + i * stride;
      if (e[i] <= 0) continue;
      const bool last = i == cnt - 1;
      if (last && s0 + cnt >= len) continue;
      const int hn = last ? g.h[n + stride] : h[i + (i + 1 < kSeg ? 1 : 0)];
      if (h[i] - hn != 1) continue;
      const int c = g.r[slot_f][n];
      const int d = min(c, e[i]);
      if (d <= 0) continue;
      g.r[slot_f][n] = c - d;
      g.r[kb][n + stride] += d;
      e[i] -= d;
      if (last) atomicAdd(g.e + n + stride, d);
      else e[i + (i + 1 < kSeg ? 1 : 0)] += d;
      any = true;
    }
    // backward: node i pushes to i-1 (the first one into the previous segment)
#pragma unroll
    for (int i = kSeg - 1; i >= 0; --i) {
      if (i >= cnt) continue;
      const long long n = n0 + i * stride;
      if (e[i] <= 0) continue;
      const bool first = i == 0;
      if (first && s0 == 0) continue;
      const int hn = first ? g.h[n - stride] : h[i > 0 ? i - 1 : 0];
      if (h[i] - hn != 1) continue;
      const int c = g.r[kb][n];
      const int d = min(c, e[i]);
      if (d <= 0) continue;
      g.r[kb][n] = c - d;
      g.r[slot_f][n - stride] += d;
      e[i] -= d;
      if (first) atomicAdd(g.e + n - stride, d);
      else e[i > 0 ? i - 1 : 0] += d;
      any = true;
    }
#pragma unroll
    for (int i = 0; i < kSeg; ++i)
      if (i < cnt && e[i] != e_in[i]) atomicAdd(g.e + n0 + i * stride, e[i] - e_in[i]);
  }
  if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) atomicOr(moved, 1);
}

int blocks_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

// One Fast-Cut iteration: relabel (two parities), then the line pushes along
// x, y (and z), each in two parities.  *moved is raised when anything moved.
cudaError_t launch_fast_iteration(const GridDev& g, int* moved, cudaStream_t s) {
  const int nb = blocks_for(g.plane);
  for (int par = 0; par < 2; ++par) {
    jfc_note_launch();
    if (g.dims == 2) k_fast_relabel<2><<<nb, 256, 0, s>>>(g, par);
    else k_fast_relabel<3><<<nb, 256, 0, s>>>(g, par);
  }
  const int axes = g.dims == 3 ? 3 : 2;
  for (int ax = 0; ax < axes; ++ax) {
    const long long len = ax == 0 ? g.W : ax == 1 ? g.H : g.D;
    const long long lines = ax == 0 ? (long long)g.H * g.D : ax == 1 ? (long long)g.W * g.D : (long long)g.W * g.H;
    const int pb = blocks_for(lines * ((len + kSeg - 1) / kSeg + 1) / 2);
    for (int par = 0; par < 2; ++par) {
      jfc_note_launch();
      if (g.dims == 2) {
        if (ax == 0) k_fast_push<2, 0><<<pb, 256, 0, s>>>(g, par, moved);
        else k_fast_push<2, 1><<<pb, 256, 0, s>>>(g, par, moved);
      } else {
        if (ax == 0) k_fast_push<3, 0><<<pb, 256, 0, s>>>(g, par, moved);
        else if (ax == 1) k_fast_push<3, 1><<<pb, 256, 0, s>>>(g, par, moved);
        else k_fast_push<3, 2><<<pb, 256, 0, s>>>(g, par, moved);
      }
    }
  }
  return cudaGetLastError();
}
