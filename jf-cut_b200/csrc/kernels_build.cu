// kernels_build.cu — capacity build: contrast n-links, k-means colour models,
// net-excess t-links, warm seed edits.
//
// Reference: graphcut_compute_capacity_bk/_lazy (graphcut_compute_capacity.cl:21-254),
// graphcut_kmeans (graphcut_kmeans.cl:21-159) with the host loop
// QGCWidget::kmeans (QGCWidget.cpp:1997-2107) moved onto the device,
// graphcut_compute_excessflow_lazy (graphcut_compute_excessflow.cl:47-77, 109-139).
// The reference evaluates exp / log in float on the device; here every
// floating-point step happens once on the host in double into int32 lookup
// tables (n-link weight per contrast index, t-link cost per quantised
// probability), and the device only does integer arithmetic and table
// gathers, so the device build is bit-identical to the CPU restatement.
//   n-link  w = LUT[|dI|] (scalar) or LUT[||dI||^2] (RGB), symmetric
//   model   fixed-point (1/16) k-means over seed pixels, integer distances
//   t-link  q = floor(Q dF / (dF + dB)); cs = LUTs[q], ct = LUTt[q];
//           seeds: cs / ct = seed_cap; e = cs - ct; sink_total += ct
#include <algorithm>

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

// Sum, over one block, of a per-thread u64; thread 0 adds it to *dst.
__device__ __forceinline__ void block_sum_to(unsigned long long v, unsigned long long* dst) {
  __shared__ unsigned long long s_part[32];
  v = warp_sum_u64(v);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_part[w];
    if (t) atomicAdd(dst, t);
  }
}

// Sum of squared neighbour differences over every +x / +y (/ +z) pair.  One
// warp per image row at a time (rows stride over all warps of the grid).
template <int PF, int DIMS>
__global__ void __launch_bounds__(256) k_contrast_sum(GridDev g, const void* __restrict__ img,
                                                      unsigned long long* sum) {
  const long long rows = (long long)g.H * g.D;
  const long long wh = (long long)g.W * g.H;
  unsigned long long acc = 0;
  const int warps = (int)(blockDim.x >> 5);
  for (long long r = (long long)blockIdx.x * warps + (threadIdx.x >> 5); r < rows; r += (long long)gridDim.x * warps) {
    const int y = (int)(r % g.H), z = (int)(r / g.H);
    const long long row = r * g.W;
    for (int x = threadIdx.x & 31; x < g.W; x += 32) {
      const long long i = row + x;
      int a[3], b[3];
      feat<PF>(img, i, a);
      if (x + 1 < g.W) { feat<PF>(img, i + 1, b); acc += contrast_sq<PF>(a, b); }
      if (y + 1 < g.H) { feat<PF>(img, i + g.W, b); acc += contrast_sq<PF>(a, b); }
      if (DIMS == 3 && z + 1 < g.D) { feat<PF>(img, i + wh, b); acc += contrast_sq<PF>(a, b); }
    }
  }
  block_sum_to(acc, sum);
}

// Seed statistics per class: count, per-channel min / max, and (fill) the
// packed features of the seed pixels (order is irrelevant: the k-means below
// is order-free).  Each thread takes 16 seed bytes at a time with one vector
// load and skips them when all are unseeded (the common case); list slots
// are reserved once per warp from per-thread class counts.
__device__ __forceinline__ int count_bytes_eq(const uint4& v, unsigned pat) {
  return (__popc(__vcmpeq4(v.x, pat)) + __popc(__vcmpeq4(v.y, pat)) + __popc(__vcmpeq4(v.z, pat)) +
          __popc(__vcmpeq4(v.w, pat))) >> 3;
}

template <int PF>
__global__ void __launch_bounds__(256) k_seed_stats(GridDev g, const void* __restrict__ img,
                                                    const uint8_t* __restrict__ seeds, int* minmax,
                                                    unsigned long long* count, uint32_t* list_f,
                                                    uint32_t* list_b, unsigned int* fill, int do_fill) {
  __shared__ int s_mm[2][3][2];
  __shared__ unsigned long long s_cnt[2];
  if (threadIdx.x < 12) ((int*)s_mm)[threadIdx.x] = (threadIdx.x & 1) ? -1 : 0x7fffffff;
  if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  constexpr int C = PF == JFC_PIX_RGB8 ? 3 : 1;
  const long long n = (long long)g.W * g.H * g.D;
  const long long chunks = (n + 15) / 16;
  const int lane = threadIdx.x & 31;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long start = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long iters = (chunks + stride - 1) / stride;
  int mn[2][C], mx[2][C];
  for (int k = 0; k < 2; ++k)
    for (int c = 0; c < C; ++c) { mn[k][c] = 0x7fffffff; mx[k][c] = -1; }
  unsigned long long cnt[2] = {0, 0};
  for (long long it = 0; it < iters; ++it) {
    const long long ch = start + it * stride;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (ch < chunks) {
      const long long i0 = ch * 16;
      if (i0 + 16 <= n) {
        v = __ldg(reinterpret_cast<const uint4*>(seeds + i0));
      } else {
        unsigned long long lo = 0, hi = 0;
        for (int b = 0; b < 16 && i0 + b < n; ++b) {
          const unsigned long long t = (unsigned long long)seeds[i0 + b];
          if (b < 8) lo |= t << (8 * b);
          else hi |= t << (8 * (b - 8));
        }
        v = make_uint4((unsigned)lo, (unsigned)(lo >> 32), (unsigned)hi, (unsigned)(hi >> 32));
      }
    }
    const bool any = (v.x | v.y | v.z | v.w) != 0;
    if (!__any_sync(FULL, any)) continue;
    const int c1 = any ? count_bytes_eq(v, 0x01010101u) : 0;
    const int c2 = any ? count_bytes_eq(v, 0x02020202u) : 0;
    cnt[0] += c1;
    cnt[1] += c2;
    unsigned pos1 = 0, pos2 = 0;
    if (do_fill) {
      // exclusive warp scans of the per-thread counts, one reservation per class
      unsigned s1 = c1, s2 = c2;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned t1 = __shfl_up_sync(FULL, s1, o), t2 = __shfl_up_sync(FULL, s2, o);
        if (lane >= o) { s1 += t1; s2 += t2; }
      }
      unsigned b1 = 0, b2 = 0;
      if (lane == 31) {
        if (s1) b1 = atomicAdd(&fill[0], s1);
        if (s2) b2 = atomicAdd(&fill[1], s2);
      }
      b1 = __shfl_sync(FULL, b1, 31);
      b2 = __shfl_sync(FULL, b2, 31);
      pos1 = b1 + s1 - c1;
      pos2 = b2 + s2 - c2;
    }
    if (!any) continue;
#pragma unroll
    for (int b = 0; b < 16; ++b) {
      const unsigned w = b < 4 ? v.x : b < 8 ? v.y : b < 12 ? v.z : v.w;
      const int sd = (w >> (8 * (b & 3))) & 255;
      if (sd != 1 && sd != 2) continue;
      int f[3] = {0, 0, 0};
      feat<PF>(img, ch * 16 + b, f);
      if (sd == 1) {
#pragma unroll
        for (int c = 0; c < C; ++c) { mn[0][c] = min(mn[0][c], f[c]); mx[0][c] = max(mx[0][c], f[c]); }
        if (do_fill) list_f[pos1++] = pack_feat<PF>(f);
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c) { mn[1][c] = min(mn[1][c], f[c]); mx[1][c] = max(mx[1][c], f[c]); }
        if (do_fill) list_b[pos2++] = pack_feat<PF>(f);
      }
    }
  }
  for (int k = 0; k < 2; ++k)
    for (int c = 0; c < C; ++c) {
      const int lo = __reduce_min_sync(FULL, mn[k][c]), hi = __reduce_max_sync(FULL, mx[k][c]);
      if (lane == 0) {
        if (lo != 0x7fffffff) atomicMin(&s_mm[k][c][0], lo);
        if (hi >= 0) atomicMax(&s_mm[k][c][1], hi);
      }
    }
  for (int k = 0; k < 2; ++k) {
    const unsigned long long t = warp_sum_u64(cnt[k]);
    if (lane == 0 && t) atomicAdd(&s_cnt[k], t);
  }
  __syncthreads();
  if (threadIdx.x < 12) {
    const int v = ((int*)s_mm)[threadIdx.x];
    if (threadIdx.x & 1) { if (v >= 0) atomicMax(&minmax[threadIdx.x], v); }
    else if (v != 0x7fffffff) atomicMin(&minmax[threadIdx.x], v);
  }
  if (threadIdx.x < 2 && s_cnt[threadIdx.x]) atomicAdd(&count[threadIdx.x], s_cnt[threadIdx.x]);
}

__device__ __forceinline__ void unpack_feat(unsigned v, int C, int* f) {
  if (C == 3) { f[0] = v & 255; f[1] = (v >> 8) & 255; f[2] = (v >> 16) & 255; }
  else f[0] = (int)v;
}

// Squared distance of a feature (scaled by 16) to a fixed-point centre.  For
// 8-bit features every term is below 2^24 and the sum below 2^26, so 32-bit
// arithmetic is exact; 16-bit features need 64 bits.
template <int PF> struct Dist { using T = int; };
template <> struct Dist<JFC_PIX_I16> { using T = long long; };

template <int PF>
__device__ __forceinline__ typename Dist<PF>::T fdist(const int* f, const int* mu) {
  using T = typename Dist<PF>::T;
  constexpr int C = PF == JFC_PIX_RGB8 ? 3 : 1;
  T s = 0;
  for (int c = 0; c < C; ++c) {
    const T t = (T)16 * f[c] - mu[c];
    s += t * t;
  }
  return s;
}

// One k-means iteration over both classes' seed lists (classes that have
// stopped moving are skipped).  Sums are warp-aggregated per centre, then
// block-aggregated in shared memory; the last block to finish recomputes the
// centres (rounded mean, fixed point 1/16), clears the sums and records which
// classes moved.  A fixed number of launches is queued with no host round
// trip: once neither class moves every further launch returns at once.
template <int PF>
__global__ void __launch_bounds__(256) k_kmeans_step(const uint32_t* __restrict__ list, KmeansDev* km) {
  constexpr int C = PF == JFC_PIX_RGB8 ? 3 : 1;
  using T = typename Dist<PF>::T;
  __shared__ int s_mu[JFC_MAX_K * 3];
  __shared__ unsigned long long s_acc[JFC_MAX_K * 4];
  __shared__ int s_last, s_moved[2];
  const int live0 = km->live[0], live1 = km->live[1];
  if (!live0 && !live1) return;
  const int lane = threadIdx.x & 31;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long start = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (int cls = 0; cls < 2; ++cls) {
    if (!(cls ? live1 : live0)) continue;
    const int k = km->k[cls];
    const long long n = (long long)km->n[cls];
    const uint32_t* L = list + (cls ? km->n[0] : 0ull);
    for (int i = threadIdx.x; i < k * 3; i += blockDim.x) s_mu[i] = km->mu[cls][i];
    for (int i = threadIdx.x; i < k * 4; i += blockDim.x) s_acc[i] = 0;
    __syncthreads();
    const long long iters = (n + stride - 1) / stride;
    for (long long it = 0; it < iters; ++it) {
      const long long i = start + it * stride;
      int best = -1;
      int f[3] = {0, 0, 0};
      if (i < n) {
        unpack_feat(L[i], C, f);
        best = 0;
        T bd = fdist<PF>(f, s_mu);
        for (int j = 1; j < k; ++j) {
          const T d = fdist<PF>(f, s_mu + 3 * j);
          if (d < bd) { bd = d; best = j; }
        }
      }
      unsigned pending = __ballot_sync(FULL, best >= 0);
      while (pending) {
        const int leader = __ffs(pending) - 1;
        const int j = __shfl_sync(FULL, best, leader);
        const bool mine = best == j;
        const unsigned peers = __ballot_sync(FULL, mine);
        unsigned sum[C];
#pragma unroll
        for (int c = 0; c < C; ++c) sum[c] = __reduce_add_sync(FULL, mine ? (unsigned)f[c] : 0u);
        if (lane == leader) {
#pragma unroll
          for (int c = 0; c < C; ++c) atomicAdd(&s_acc[j * 4 + c], (unsigned long long)sum[c]);
          atomicAdd(&s_acc[j * 4 + 3], (unsigned long long)__popc(peers));
        }
        pending &= ~peers;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < k * 4; i += blockDim.x)
      if (s_acc[i]) atomicAdd(&km->acc[cls][i], s_acc[i]);
    __syncthreads();
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&km->done, 1u) == gridDim.x - 1;
  if (threadIdx.x < 2) s_moved[threadIdx.x] = 0;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int t = threadIdx.x; t < 2 * JFC_MAX_K * 3; t += blockDim.x) {
    const int cls = t / (JFC_MAX_K * 3), r = t % (JFC_MAX_K * 3), j = r / 3, c = r % 3;
    if (!(cls ? live1 : live0) || j >= km->k[cls] || c >= C) continue;
    const long long c4 = (long long)__ldcg(&km->acc[cls][j * 4 + 3]);
    if (c4 == 0) continue;
    const int v = (int)((16 * (long long)__ldcg(&km->acc[cls][j * 4 + c]) + c4 / 2) / c4);
    if (v != km->mu[cls][r]) { km->mu[cls][r] = v; s_moved[cls] = 1; }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 2 * JFC_MAX_K * 4; t += blockDim.x) (&km->acc[0][0])[t] = 0;
  if (threadIdx.x == 0 && live0) km->live[0] = s_moved[0];
  if (threadIdx.x == 1 && live1) km->live[1] = s_moved[1];
  if (threadIdx.x == 0) km->done = 0;
}

// t-link costs of one node.  q = floor(Q dF / (dF + dB)): for 8-bit features
// (dF + dB < 2^27) a float quotient lands within 1 of q and one exact integer
// step either way corrects it; 16-bit features divide in 64 bits.
template <int PF>
__device__ __forceinline__ void tlinks(const BuildModelDev& m, const int* __restrict__ lut_s,
                                       const int* __restrict__ lut_t, const int* f, int seed, int& cs,
                                       int& ct) {
  if (seed == JFC_SEED_FG) { cs = m.seed_cap; ct = 0; return; }
  if (seed == JFC_SEED_BG) { cs = 0; ct = m.seed_cap; return; }
  using T = typename Dist<PF>::T;
  T dF = fdist<PF>(f, m.mu_f), dB = fdist<PF>(f, m.mu_b);
  for (int j = 1; j < m.kf; ++j) dF = min(dF, fdist<PF>(f, m.mu_f + 3 * j));
  for (int j = 1; j < m.kb; ++j) dB = min(dB, fdist<PF>(f, m.mu_b + 3 * j));
  unsigned q;
  if constexpr (PF == JFC_PIX_I16) {
    const unsigned long long s = (unsigned long long)dF + (unsigned long long)dB;
    q = (s == 0) ? JFC_TQ / 2 : (unsigned)(((unsigned long long)JFC_TQ * (unsigned long long)dF) / s);
  } else {
    const unsigned s = (unsigned)dF + (unsigned)dB;
    if (s == 0) {
      q = JFC_TQ / 2;
    } else {
      q = (unsigned)(__fdividef((float)dF, (float)s) * (float)JFC_TQ);
      const unsigned long long num = (unsigned long long)JFC_TQ * (unsigned)dF;
      const unsigned long long qs = (unsigned long long)q * s;
      if (qs > num) --q;
      else if (qs + s <= num) ++q;
    }
  }
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
  // one warp per 32-node row segment; rows stride over gridDim.y so that the
  // sum of ct takes one atomic per block instead of one per warp
  const int x = blockIdx.x * 32 + (threadIdx.x & 31);
  const long long rows = (long long)g.Hp * g.Dp;
  unsigned long long acc = 0;
  for (long long yz = (long long)blockIdx.y * 8 + (threadIdx.x >> 5); yz < rows; yz += (long long)gridDim.y * 8) {
  const int y = (int)(yz % g.Hp), z = (int)(yz / g.Hp);
  if (x < g.pitch) {
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
      acc += (unsigned long long)ct;
    }
  }
  }
  __shared__ unsigned long long s_acc[8];
  acc = warp_sum_u64(acc);
  if ((threadIdx.x & 31) == 0) s_acc[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < 8; ++w) t += s_acc[w];
    if (t) atomicAdd(sink, t);
  }
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
  const int nb = (int)std::min<long long>(((long long)g.H * g.D + 7) / 8, 148 * 8);
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
  if (reinterpret_cast<uintptr_t>(d_seeds) & 15) return cudaErrorMisalignedAddress;   // 16-byte vector loads
  const int nb = flat_blocks(((long long)g.W * g.H * g.D + 15) / 16);
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

cudaError_t launch_kmeans(const uint32_t* d_list, KmeansDev* d_km, int pixfmt, unsigned long long nmax,
                          int iters, cudaStream_t s) {
  const int nb = (int)std::max<long long>(1, std::min<long long>(((long long)nmax + 255) / 256, 148 * 4));
  for (int it = 0; it < iters; ++it) {
    jfc_note_launch();
    switch (pixfmt) {
      case JFC_PIX_GRAY8: k_kmeans_step<JFC_PIX_GRAY8><<<nb, 256, 0, s>>>(d_list, d_km); break;
      case JFC_PIX_RGB8: k_kmeans_step<JFC_PIX_RGB8><<<nb, 256, 0, s>>>(d_list, d_km); break;
      case JFC_PIX_I16: k_kmeans_step<JFC_PIX_I16><<<nb, 256, 0, s>>>(d_list, d_km); break;
      default: return cudaErrorInvalidValue;
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_build_graph(const GridDev& g, const void* d_img, const uint8_t* d_seeds,
                               const BuildModelDev& m, const int* d_lut_xy, const int* d_lut_z,
                               const int* d_lut_s, const int* d_lut_t, unsigned long long* d_sink,
                               cudaStream_t s) {
  dim3 grid((g.pitch + 31) / 32, (unsigned)std::min<long long>((g.Hp * (long long)g.Dp + 7) / 8, 64));
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
