// kernels_build.cu — capacity build: contrast n-links, k-means colour models,
// net-excess t-links, warm seed edits.
//
// Reference: graphcut_compute_capacity_bk/_lazy (graphcut_compute_capacity.cl:21-254),
// graphcut_kmeans (graphcut_kmeans.cl:21-159) with the host loop
// QGCWidget::kmeans (QGCWidget.cpp:1997-2107), graphcut_compute_excessflow_lazy
// (graphcut_compute_excessflow.cl:47-77, 109-139).
// The reference evaluates exp / log in float on the device; here every
// floating-point step happens once on the host in double into int32 lookup
// tables (n-link weight per contrast index, t-link cost per quantised
// probability), and the device only does integer arithmetic and table
// gathers, so the device build is bit-identical to the CPU restatement.
//   n-link  w = LUT[|dI|] (scalar) or LUT[||dI||^2] (RGB), symmetric
//   model   fixed-point (1/16) k-means over seed pixels, integer distances
//   t-link  q = floor(Q dF / (dF + dB)); cs = LUTs[q], ct = LUTt[q];
//           seeds: cs / ct = seed_cap; e = cs - ct; sink_total += ct
#include "jfc_internal.h"

namespace {

constexpr unsigned FULL = 0xffffffffu;

template <int PF>
__device__ __forceinline__ void feat(const void* __restrict__ img, long long i, int* f) {
  if constexpr (PF == JFC_PIX_GRAY8) {
    f[0] = ((const uint8_t*)img)[i];
  } else if constexpr (PF == JFC_PIX_RGB8) {
    const uint8_t* p = (const uint8_t*)img + 3 * i;
    f[0] = p[0]; f[1] = p[1]; f[2] = p[2];
  } else {
    f[0] = (int)((const int16_t*)img)[i] + 32768;
  }
}

template <int PF>
__device__ __forceinline__ unsigned pack_feat(const int* f) {
  if constexpr (PF == JFC_PIX_RGB8) return (unsigned)f[0] | ((unsigned)f[1] << 8) | ((unsigned)f[2] << 16);
  else return (unsigned)f[0];
}

// contrast-table index and squared difference of a neighbour pair
template <int PF>
__device__ __forceinline__ long long contrast_index(const int* a, const int* b) {
  if constexpr (PF == JFC_PIX_RGB8) {
    const int d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    return (long long)d0 * d0 + (long long)d1 * d1 + (long long)d2 * d2;
  } else {
    const int d = a[0] - b[0];
    return d < 0 ? -d : d;
  }
}
template <int PF>
__device__ __forceinline__ unsigned long long contrast_sq(const int* a, const int* b) {
  if constexpr (PF == JFC_PIX_RGB8) return (unsigned long long)contrast_index<PF>(a, b);
  else { const long long d = contrast_index<PF>(a, b); return (unsigned long long)(d * d); }
}

__device__ __forceinline__ void dense_xyz(const GridDev& g, long long i, int& x, int& y, int& z) {
  x = (int)(i % g.W);
  const long long yz = i / g.W;
  y = (int)(yz % g.H);
  z = (int)(yz / g.H);
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

template <int PF, int DIMS>
__global__ void k_contrast_sum(GridDev g, const void* __restrict__ img, unsigned long long* sum) {
  const long long n = (long long)g.W * g.H * g.D;
  const long long wh = (long long)g.W * g.H;
  unsigned long long acc = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    dense_xyz(g, i, x, y, z);
    int a[3], b[3];
    feat<PF>(img, i, a);
    if (x + 1 < g.W) { feat<PF>(img, i + 1, b); acc += contrast_sq<PF>(a, b); }
    if (y + 1 < g.H) { feat<PF>(img, i + g.W, b); acc += contrast_sq<PF>(a, b); }
    if (DIMS == 3 && z + 1 < g.D) { feat<PF>(img, i + wh, b); acc += contrast_sq<PF>(a, b); }
  }
  acc = warp_sum_u64(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(sum, acc);
}

// Seed statistics per class: count, per-channel min / max, and (fill) the
// packed features of the seed pixels (order is irrelevant: the k-means below
// is order-free).
template <int PF>
__global__ void k_seed_stats(GridDev g, const void* __restrict__ img, const uint8_t* __restrict__ seeds,
                             int* minmax, unsigned long long* count, uint32_t* list_f, uint32_t* list_b,
                             unsigned int* fill, int do_fill) {
  __shared__ int s_mm[2][3][2];
  __shared__ unsigned long long s_cnt[2];
  if (threadIdx.x < 12) ((int*)s_mm)[threadIdx.x] = (threadIdx.x & 1) ? -1 : 0x7fffffff;
  if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  constexpr int C = PF == JFC_PIX_RGB8 ? 3 : 1;
  const long long n = (long long)g.W * g.H * g.D;
  const int lane = threadIdx.x & 31;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long start = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long iters = (n + stride - 1) / stride;
  for (long long k = 0; k < iters; ++k) {
    const long long i = start + k * stride;
    const int s = (i < n) ? seeds[i] : 0;
    int f[3] = {0, 0, 0};
    if (s == 1 || s == 2) {
      feat<PF>(img, i, f);
      for (int c = 0; c < C; ++c) {
        atomicMin(&s_mm[s - 1][c][0], f[c]);
        atomicMax(&s_mm[s - 1][c][1], f[c]);
      }
    }
    for (int cls = 1; cls <= 2; ++cls) {
      const unsigned m = __ballot_sync(FULL, s == cls);
      if (!m) continue;
      unsigned base = 0;
      if (lane == 0) {
        atomicAdd(&s_cnt[cls - 1], (unsigned long long)__popc(m));
        if (do_fill) base = atomicAdd(&fill[cls - 1], (unsigned)__popc(m));
      }
      if (do_fill) {
        base = __shfl_sync(FULL, base, 0);
        if (s == cls) {
          const unsigned pos = base + __popc(m & ((1u << lane) - 1u));
          (cls == 1 ? list_f : list_b)[pos] = pack_feat<PF>(f);
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < 12) {
    const int v = ((int*)s_mm)[threadIdx.x];
    if (threadIdx.x & 1) { if (v >= 0) atomicMax(&minmax[threadIdx.x], v); }
    else if (v != 0x7fffffff) atomicMin(&minmax[threadIdx.x], v);
  }
  if (threadIdx.x < 2 && s_cnt[threadIdx.x]) atomicAdd(&count[threadIdx.x], s_cnt[threadIdx.x]);
}

struct MuParam {
  int mu[JFC_MAX_K * 3];
};

__device__ __forceinline__ void unpack_feat(unsigned v, int C, int* f) {
  if (C == 3) { f[0] = v & 255; f[1] = (v >> 8) & 255; f[2] = (v >> 16) & 255; }
  else f[0] = (int)v;
}

__device__ __forceinline__ long long fdist(const int* f, const int* mu, int C) {
  long long s = 0;
  for (int c = 0; c < C; ++c) {
    const long long t = 16ll * f[c] - mu[c];
    s += t * t;
  }
  return s;
}

__global__ void k_kmeans_assign(const uint32_t* __restrict__ list, unsigned n, int C, int k, MuParam mp,
                                unsigned long long* acc) {
  __shared__ unsigned long long s_acc[JFC_MAX_K * 4];
  for (int i = threadIdx.x; i < k * 4; i += blockDim.x) s_acc[i] = 0;
  __syncthreads();
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int f[3];
    unpack_feat(list[i], C, f);
    int best = 0;
    long long bd = fdist(f, mp.mu, C);
    for (int j = 1; j < k; ++j) {
      const long long d = fdist(f, mp.mu + 3 * j, C);
      if (d < bd) { bd = d; best = j; }
    }
    for (int c = 0; c < C; ++c) atomicAdd(&s_acc[best * 4 + c], (unsigned long long)f[c]);
    atomicAdd(&s_acc[best * 4 + 3], 1ull);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < k * 4; i += blockDim.x)
    if (s_acc[i]) atomicAdd(&acc[i], s_acc[i]);
}

template <int PF>
__device__ __forceinline__ void tlinks(const BuildModelDev& m, const int* __restrict__ lut_s,
                                       const int* __restrict__ lut_t, const int* f, int seed, int& cs,
                                       int& ct) {
  if (seed == JFC_SEED_FG) { cs = m.seed_cap; ct = 0; return; }
  if (seed == JFC_SEED_BG) { cs = 0; ct = m.seed_cap; return; }
  constexpr int C = PF == JFC_PIX_RGB8 ? 3 : 1;
  long long dF = fdist(f, m.mu_f, C), dB = fdist(f, m.mu_b, C);
  for (int j = 1; j < m.kf; ++j) dF = min(dF, fdist(f, m.mu_f + 3 * j, C));
  for (int j = 1; j < m.kb; ++j) dB = min(dB, fdist(f, m.mu_b + 3 * j, C));
  const unsigned long long s = (unsigned long long)dF + (unsigned long long)dB;
  const unsigned q = (s == 0) ? JFC_TQ / 2 : (unsigned)(((unsigned long long)JFC_TQ * (unsigned long long)dF) / s);
  cs = lut_s[q];
  ct = lut_t[q];
}

// One pass over the padded grid: n-links (both directions of every pair, from
// the contrast table), t-links, e = cs - ct, label = 0; padding is zeroed.
template <int PF, int DIMS>
__global__ void __launch_bounds__(256) k_build(GridDev g, const void* __restrict__ img,
                                               const uint8_t* __restrict__ seeds, BuildModelDev m,
                                               const int* __restrict__ lut_xy, const int* __restrict__ lut_z,
                                               const int* __restrict__ lut_s, const int* __restrict__ lut_t,
                                               unsigned long long* sink) {
  const int x = blockIdx.x * 32 + (threadIdx.x & 31);
  const int yz = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int y = yz % g.Hp, z = yz / g.Hp;
  unsigned long long acc = 0;
  if (z < g.Dp && x < g.pitch) {
    const long long p = (long long)x + (long long)g.pitch * (y + (long long)g.Hp * z);
    const bool real = x < g.W && y < g.H && z < g.D;
    if (!real) {
      g.e[p] = 0;
      for (int k = 0; k < (DIMS == 2 ? 4 : 6); ++k) g.r[k][p] = 0;
      g.label[p] = 0;
      g.h[p] = JFC_INF;
    } else {
      const long long wh = (long long)g.W * g.H;
      const long long i = (long long)x + (long long)g.W * y + wh * z;
      int a[3], b[3];
      feat<PF>(img, i, a);
      int w_xp = 0, w_yp = 0, w_ym = 0, w_xm = 0, w_zp = 0, w_zm = 0;
      if (x + 1 < g.W) { feat<PF>(img, i + 1, b); w_xp = lut_xy[contrast_index<PF>(a, b)]; }
      if (x > 0) { feat<PF>(img, i - 1, b); w_xm = lut_xy[contrast_index<PF>(a, b)]; }
      if (y + 1 < g.H) { feat<PF>(img, i + g.W, b); w_yp = lut_xy[contrast_index<PF>(a, b)]; }
      if (y > 0) { feat<PF>(img, i - g.W, b); w_ym = lut_xy[contrast_index<PF>(a, b)]; }
      if constexpr (DIMS == 3) {
        if (z + 1 < g.D) { feat<PF>(img, i + wh, b); w_zp = lut_z[contrast_index<PF>(a, b)]; }
        if (z > 0) { feat<PF>(img, i - wh, b); w_zm = lut_z[contrast_index<PF>(a, b)]; }
        g.r[0][p] = w_xp; g.r[1][p] = w_yp; g.r[2][p] = w_zp;
        g.r[3][p] = w_zm; g.r[4][p] = w_ym; g.r[5][p] = w_xm;
      } else {
        g.r[0][p] = w_xp; g.r[1][p] = w_yp; g.r[2][p] = w_ym; g.r[3][p] = w_xm;
      }
      int cs, ct;
      tlinks<PF>(m, lut_s, lut_t, a, seeds[i], cs, ct);
      g.e[p] = cs - ct;
      g.label[p] = 0;
      acc = (unsigned long long)ct;
    }
  }
  acc = warp_sum_u64(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(sink, acc);
}

// Warm stroke edit: re-seed nodes with the colour model fixed; the residual
// graph stays, only e moves by the change of cs - ct (indices unique).
// Duplicate indices in one edit list: the last entry of a node wins.  The
// height plane is scratch between solves (every solve starts with a global
// relabel that rewrites it), so it records the winning entry per node:
// mark -1 on every edited node, then atomicMax of the entry index.
__device__ __forceinline__ long long padded_of(const GridDev& g, long long i) {
  const int x = (int)(i % g.W);
  const long long yz = i / g.W;
  const int y = (int)(yz % g.H), z = (int)(yz / g.H);
  return (long long)x + (long long)g.pitch * (y + (long long)g.Hp * z);
}

__global__ void k_edit_mark(GridDev g, const uint32_t* __restrict__ idx, long long n, int last) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int* h = g.h + padded_of(g, idx[j]);
    if (last) atomicMax(h, (int)j);
    else *h = -1;
  }
}

template <int PF>
__global__ void k_edit_seeds(GridDev g, const void* __restrict__ img, uint8_t* __restrict__ seeds,
                             BuildModelDev m, const int* __restrict__ lut_s, const int* __restrict__ lut_t,
                             const uint32_t* __restrict__ idx, const uint8_t* __restrict__ nseed,
                             long long n, long long* dsink) {
  long long acc = 0;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const long long i = idx[j];
    if (g.h[padded_of(g, i)] != (int)j) continue;   // a later entry edits this node
    const int s1 = nseed[j], s0 = seeds[i];
    if (s0 == s1) continue;
    int f[3];
    feat<PF>(img, i, f);
    int cs0, ct0, cs1, ct1;
    tlinks<PF>(m, lut_s, lut_t, f, s0, cs0, ct0);
    tlinks<PF>(m, lut_s, lut_t, f, s1, cs1, ct1);
    int x, y, z;
    dense_xyz(g, i, x, y, z);
    const long long p = (long long)x + (long long)g.pitch * (y + (long long)g.Hp * z);
    atomicAdd(g.e + p, (cs1 - ct1) - (cs0 - ct0));
    acc += (long long)ct1 - ct0;
    seeds[i] = (uint8_t)s1;
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd((unsigned long long*)dsink, (unsigned long long)acc);
}

int flat_blocks(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

cudaError_t launch_contrast_sum(const GridDev& g, const void* d_img, int pixfmt,
                                unsigned long long* d_sum, cudaStream_t s) {
  const int nb = flat_blocks((long long)g.W * g.H * g.D);
  const bool d3 = g.dims == 3;
  jfc_note_launch();
  switch (pixfmt) {
    case JFC_PIX_GRAY8: d3 ? k_contrast_sum<JFC_PIX_GRAY8, 3><<<nb, 256, 0, s>>>(g, d_img, d_sum)
                           : k_contrast_sum<JFC_PIX_GRAY8, 2><<<nb, 256, 0, s>>>(g, d_img, d_sum); break;
    case JFC_PIX_RGB8: d3 ? k_contrast_sum<JFC_PIX_RGB8, 3><<<nb, 256, 0, s>>>(g, d_img, d_sum)
                          : k_contrast_sum<JFC_PIX_RGB8, 2><<<nb, 256, 0, s>>>(g, d_img, d_sum); break;
    case JFC_PIX_I16: d3 ? k_contrast_sum<JFC_PIX_I16, 3><<<nb, 256, 0, s>>>(g, d_img, d_sum)
                         : k_contrast_sum<JFC_PIX_I16, 2><<<nb, 256, 0, s>>>(g, d_img, d_sum); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_seed_stats(const GridDev& g, const void* d_img, int pixfmt, const uint8_t* d_seeds,
                              int* d_minmax, unsigned long long* d_count, uint32_t* d_list_f,
                              uint32_t* d_list_b, unsigned int* d_fill, bool fill, cudaStream_t s) {
  const int nb = flat_blocks((long long)g.W * g.H * g.D);
  switch (pixfmt) {
    case JFC_PIX_GRAY8:
      jfc_note_launch();
      k_seed_stats<JFC_PIX_GRAY8><<<nb, 256, 0, s>>>(g, d_img, d_seeds, d_minmax, d_count, d_list_f, d_list_b, d_fill, fill);
      break;
    case JFC_PIX_RGB8:
      jfc_note_launch();
      k_seed_stats<JFC_PIX_RGB8><<<nb, 256, 0, s>>>(g, d_img, d_seeds, d_minmax, d_count, d_list_f, d_list_b, d_fill, fill);
      break;
    case JFC_PIX_I16:
      jfc_note_launch();
      k_seed_stats<JFC_PIX_I16><<<nb, 256, 0, s>>>(g, d_img, d_seeds, d_minmax, d_count, d_list_f, d_list_b, d_fill, fill);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_kmeans_assign(const uint32_t* d_list, unsigned int n, int channels, int k,
                                 const int* mu, unsigned long long* d_acc, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  MuParam mp;
  for (int i = 0; i < JFC_MAX_K * 3; ++i) mp.mu[i] = (i < k * 3) ? mu[i] : 0;
  const int nb = flat_blocks((long long)n);
  jfc_note_launch();
  k_kmeans_assign<<<nb, 256, 0, s>>>(d_list, n, channels, k, mp, d_acc);
  return cudaGetLastError();
}

cudaError_t launch_build_graph(const GridDev& g, const void* d_img, const uint8_t* d_seeds,
                               const BuildModelDev& m, const int* d_lut_xy, const int* d_lut_z,
                               const int* d_lut_s, const int* d_lut_t, unsigned long long* d_sink,
                               cudaStream_t s) {
  dim3 grid((g.pitch + 31) / 32, (unsigned)((g.Hp * (long long)g.Dp + 7) / 8));
  const bool d3 = g.dims == 3;
  jfc_note_launch();
#define JFC_BUILD(PF)                                                                                   \
  (d3 ? k_build<PF, 3><<<grid, 256, 0, s>>>(g, d_img, d_seeds, m, d_lut_xy, d_lut_z, d_lut_s, d_lut_t, d_sink) \
      : k_build<PF, 2><<<grid, 256, 0, s>>>(g, d_img, d_seeds, m, d_lut_xy, d_lut_z, d_lut_s, d_lut_t, d_sink))
  switch (m.pixfmt) {
    case JFC_PIX_GRAY8: JFC_BUILD(JFC_PIX_GRAY8); break;
    case JFC_PIX_RGB8: JFC_BUILD(JFC_PIX_RGB8); break;
    case JFC_PIX_I16: JFC_BUILD(JFC_PIX_I16); break;
    default: return cudaErrorInvalidValue;
  }
#undef JFC_BUILD
  return cudaGetLastError();
}

cudaError_t launch_edit_seeds(const GridDev& g, const void* d_img, uint8_t* d_seeds, const BuildModelDev& m,
                              const int* d_lut_s, const int* d_lut_t, const uint32_t* d_idx,
                              const uint8_t* d_new, size_t n, long long* d_dsink, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int nb = flat_blocks((long long)n);
  jfc_note_launch(2);
  k_edit_mark<<<nb, 256, 0, s>>>(g, d_idx, (long long)n, 0);
  k_edit_mark<<<nb, 256, 0, s>>>(g, d_idx, (long long)n, 1);
  switch (m.pixfmt) {
    case JFC_PIX_GRAY8:
      jfc_note_launch();
      k_edit_seeds<JFC_PIX_GRAY8><<<nb, 256, 0, s>>>(g, d_img, d_seeds, m, d_lut_s, d_lut_t, d_idx, d_new, (long long)n, d_dsink);
      break;
    case JFC_PIX_RGB8:
      jfc_note_launch();
      k_edit_seeds<JFC_PIX_RGB8><<<nb, 256, 0, s>>>(g, d_img, d_seeds, m, d_lut_s, d_lut_t, d_idx, d_new, (long long)n, d_dsink);
      break;
    case JFC_PIX_I16:
      jfc_note_launch();
      k_edit_seeds<JFC_PIX_I16><<<nb, 256, 0, s>>>(g, d_img, d_seeds, m, d_lut_s, d_lut_t, d_idx, d_new, (long long)n, d_dsink);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
