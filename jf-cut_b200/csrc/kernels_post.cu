// kernels_post.cu — checks and post-processing on a finished cut.
//
// Energy of a labelling (the reference's energy check after a solve,
// QGCWidget.cpp:2452-2520): data = sum over background nodes of max(e, 0) +
// sum over object nodes of max(-e, 0); smooth = sum of the capacities of arcs
// leaving an object node towards a background node.  On a graph in
// net-excess form, data + smooth of the canonical cut equals the max-flow:
// an independent certificate computed from the original capacities.
#include "jfc_internal.h"

namespace {

constexpr unsigned FULL = 0xffffffffu;

struct Caps {
  const int32_t* c[6];
};

__global__ void __launch_bounds__(256) k_energy(int dims, int w, int h, int d, const int32_t* __restrict__ e,
                                                Caps caps, const uint8_t* __restrict__ lab,
                                                unsigned long long* out) {
  const long long n = (long long)w * h * d;
  const long long plane = (long long)w * h;
  long long data = 0, smooth = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int ei = e[i];
    if (lab[i]) {
      if (ei < 0) data -= ei;
      const int x = (int)(i % w);
      const long long yz = i / w;
      const int y = (int)(yz % h), z = (int)(yz / h);
      // channel order 2D: +x, +y, -y, -x; 3D: +x, +y, +z, -z, -y, -x
      const bool ok[6] = {x < w - 1, y < h - 1, dims == 3 ? z < d - 1 : y > 0, dims == 3 ? z > 0 : x > 0,
                          y > 0, x > 0};
      const long long off[6] = {1, w, dims == 3 ? plane : -(long long)w, dims == 3 ? -plane : -1, -(long long)w, -1};
      const int K = dims == 3 ? 6 : 4;
      for (int k = 0; k < K; ++k)
        if (ok[k] && !lab[i + off[k]]) smooth += caps.c[k][i];
    } else if (ei > 0) {
      data += ei;
    }
  }
  for (int o = 16; o; o >>= 1) {
    data += __shfl_xor_sync(FULL, data, o);
    smooth += __shfl_xor_sync(FULL, smooth, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (data) atomicAdd(out, (unsigned long long)data);
    if (smooth) atomicAdd(out + 1, (unsigned long long)smooth);
  }
}

}  // namespace

namespace {
__global__ void k_and_bytes(uint8_t* p, long long n, uint8_t keep) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] &= keep;
}
}  // namespace

cudaError_t launch_and_bytes(uint8_t* p, long long n, uint8_t keep, cudaStream_t s) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  jfc_note_launch();
  k_and_bytes<<<(unsigned)blocks, 256, 0, s>>>(p, n, keep);
  return cudaGetLastError();
}

cudaError_t launch_energy(int dims, int w, int h, int d, const int32_t* e, const int32_t* const* caps,
                          const uint8_t* lab, unsigned long long* out, cudaStream_t s) {
  Caps c{};
  for (int k = 0; k < (dims == 3 ? 6 : 4); ++k) c.c[k] = caps[k];
  const long long n = (long long)w * h * d;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  jfc_note_launch();
  k_energy<<<(unsigned)blocks, 256, 0, s>>>(dims, w, h, dims == 3 ? d : 1, e, c, lab, out);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ strokes
// Stroke-to-seed mapping of a volume (graphcut_compute_visibility,
// graphcut_render_ray_casting.cl:275-346), compute only: for every stroke pixel
// a ray through the inverse view-projection is intersected with the volume's
// bounding box and marched with the reference's non-uniform steps; samples
// are trilinear (texel centres at i + 0.5, clamp to edge), classified by the
// transfer function (linear, clamp to edge) after the intensity window, and
// composited front to back with early termination; every sample more opaque
// than `alpha` marks the 8 voxels around it with the stroke's label.
namespace {

struct ViewDev {
  float m[16];
  float box[3];
  int iw, ih, samples;
  float ratio, step_scale, wmin, wmax, alpha;
};

__device__ __forceinline__ float tex3(const float* v, int w, int h, int d, float x, float y, float z) {
  x -= 0.5f; y -= 0.5f; z -= 0.5f;
  const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  const float ax = x - fx, ay = y - fy, az = z - fz;
  const int x0 = min(max((int)fx, 0), w - 1), x1 = min(max((int)fx + 1, 0), w - 1);
  const int y0 = min(max((int)fy, 0), h - 1), y1 = min(max((int)fy + 1, 0), h - 1);
  const int z0 = min(max((int)fz, 0), d - 1), z1 = min(max((int)fz + 1, 0), d - 1);
  auto at = [&](int xx, int yy, int zz) { return v[(long long)xx + (long long)w * (yy + (long long)h * zz)]; };
  const float c00 = at(x0, y0, z0) * (1.f - ax) + at(x1, y0, z0) * ax;
  const float c10 = at(x0, y1, z0) * (1.f - ax) + at(x1, y1, z0) * ax;
  const float c01 = at(x0, y0, z1) * (1.f - ax) + at(x1, y0, z1) * ax;
  const float c11 = at(x0, y1, z1) * (1.f - ax) + at(x1, y1, z1) * ax;
  const float c0 = c00 * (1.f - ay) + c10 * ay, c1 = c01 * (1.f - ay) + c11 * ay;
  return c0 * (1.f - az) + c1 * az;
}

__device__ __forceinline__ float4 tex1(const float4* tf, int n, float u) {
  float x = u * n - 0.5f;
  const float fx = floorf(x), a = x - fx;
  const int i0 = min(max((int)fx, 0), n - 1), i1 = min(max((int)fx + 1, 0), n - 1);
  const float4 p = tf[i0], q = tf[i1];
  return make_float4(p.x * (1.f - a) + q.x * a, p.y * (1.f - a) + q.y * a, p.z * (1.f - a) + q.z * a,
                     p.w * (1.f - a) + q.w * a);
}

__global__ void __launch_bounds__(256) k_stroke_seeds(ViewDev vw, int w, int h, int d, const float* __restrict__ vol,
                                                      const float4* __restrict__ tf, int ntf,
                                                      const uint8_t* __restrict__ mask, uint8_t label,
                                                      uint8_t* __restrict__ seeds) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = blockIdx.y;
  if (px >= vw.iw || py >= vw.ih || !mask[px + (long long)py * vw.iw]) return;
  const float u = (px + 0.5f) / vw.iw * 2.0f - 1.0f, v = (py + 0.5f) / vw.ih * 2.0f - 1.0f;
  const float* m = vw.m;
  // back-projection of (u, v, z, 1) with the column-major inverse view-projection
  auto bp = [&](float z, float* o) {
    for (int r = 0; r < 4; ++r) o[r] = u * m[r] + v * m[4 + r] + z * m[8 + r] + m[12 + r];
  };
  float a[4], b[4];
  bp(-1.0f, a);
  bp(0.0f, b);
  const float ox = a[0] / a[3], oy = a[1] / a[3], oz = a[2] / a[3];
  float dx = b[0] / b[3] - ox, dy = b[1] / b[3] - oy, dz = b[2] / b[3] - oz;
  const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
  dx *= inv; dy *= inv; dz *= inv;
  // slab intersection with [-box, box]
  const float ix = 1.0f / dx, iy = 1.0f / dy, iz = 1.0f / dz;
  const float bx0 = ix * (-vw.box[0] - ox), bx1 = ix * (vw.box[0] - ox);
  const float by0 = iy * (-vw.box[1] - oy), by1 = iy * (vw.box[1] - oy);
  const float bz0 = iz * (-vw.box[2] - oz), bz1 = iz * (vw.box[2] - oz);
  float tnear = fmaxf(fmaxf(fminf(bx0, bx1), fminf(by0, by1)), fminf(bz0, bz1));
  const float tfar = fminf(fminf(fmaxf(bx0, bx1), fmaxf(by0, by1)), fmaxf(bz0, bz1));
  if (!(tnear < tfar)) return;
  tnear = fmaxf(tnear, 0.0f);
  const float mx = w - 1.0f, my = h - 1.0f, mz = d - 1.0f;
  const float sx = mx * 0.5f / vw.box[0], sy = my * 0.5f / vw.box[1], sz = mz * 0.5f / vw.box[2];
  float qx = (ox + dx * tnear) * sx + mx * 0.5f, qy = (oy + dy * tnear) * sy + my * 0.5f,
        qz = (oz + dz * tnear) * sz + mz * 0.5f;
  const float ddx = dx * sx, ddy = dy * sy, ddz = dz * sz;
  float step = (tfar - tnear) / (vw.samples - 1) * vw.ratio;
  const float delta = ((tfar - tnear) / (vw.samples - 1) - step) / (vw.samples - 2);
  float acc = 0.0f;
  for (int i = 0; i < vw.samples; ++i) {
    const float s = tex3(vol, w, h, d, qx, qy, qz);
    const float4 c = tex1(tf, ntf, fminf(fmaxf(s, vw.wmin), vw.wmax));
    acc += c.w * vw.step_scale * step * expf(-acc);
    if (acc >= 1.0f) break;
    if (c.w > vw.alpha) {
      // the 8 voxels around the sample (floor / floor + 1, clamped)
      const int x0 = (int)fminf(fmaxf(floorf(qx), 0.f), mx), x1 = (int)fminf(fmaxf(floorf(qx) + 1.f, 0.f), mx);
      const int y0 = (int)fminf(fmaxf(floorf(qy), 0.f), my), y1 = (int)fminf(fmaxf(floorf(qy) + 1.f, 0.f), my);
      const int z0 = (int)fminf(fmaxf(floorf(qz), 0.f), mz), z1 = (int)fminf(fmaxf(floorf(qz) + 1.f, 0.f), mz);
      const int xs[2] = {x0, x1}, ys[2] = {y0, y1}, zs[2] = {z0, z1};
      for (int k = 0; k < 8; ++k)
        seeds[xs[k & 1] + (long long)w * (ys[(k >> 1) & 1] + (long long)h * zs[k >> 2])] = label;
    }
    qx += ddx * step; qy += ddy * step; qz += ddz * step;
    step += delta;
  }
}

}  // namespace

cudaError_t launch_stroke_seeds(const jfc_view& v, int w, int h, int d, const float* vol, const float* tf, int ntf,
                                const uint8_t* mask, uint8_t label, uint8_t* seeds, cudaStream_t s) {
  ViewDev vw;
  for (int i = 0; i < 16; ++i) vw.m[i] = v.inverse_mvp[i];
  for (int i = 0; i < 3; ++i) vw.box[i] = v.box[i];
  vw.iw = v.image_w; vw.ih = v.image_h; vw.samples = v.samples;
  vw.ratio = v.sample_ratio; vw.step_scale = v.sample_step_scale;
  vw.wmin = v.window_level - v.window_width / 2; vw.wmax = v.window_level + v.window_width / 2;
  vw.alpha = v.alpha;
  jfc_note_launch();
  k_stroke_seeds<<<dim3((v.image_w + 255) / 256, v.image_h), 256, 0, s>>>(vw, w, h, d, vol, (const float4*)tf, ntf,
                                                                         mask, label, seeds);
  return cudaGetLastError();
}
