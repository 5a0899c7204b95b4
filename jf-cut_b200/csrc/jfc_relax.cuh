// jfc_relax.cuh — CTA tile geometry and the in-tile distance relaxation shared
// by the push-relabel visit (exact local relabel) and the global relabel.
#pragma once

#include "jfc_sync.cuh"

namespace jfc {

// One CTA per tile of 32 x TY (x TZ) nodes, one thread per node, one warp per
// tile row.  Heights live in a shared-memory box with a one-cell halo; a row
// of the box is HX_ wide and node x of the tile sits at column x + X0_ (the
// push-relabel visit uses a 40-wide box starting 4 columns left of the tile,
// the shape its tensor-copy staging lands in).
template <int DIMS, int TY_, int TZ_, int HX_ = 34, int X0_ = 1>
struct CtaTile {
  static constexpr int D = DIMS, TY = TY_, TZ = TZ_;
  static constexpr int R = TY * TZ;            // rows = warps
  static constexpr int NT = 32 * R;            // threads = nodes
  static constexpr int K = DIMS == 2 ? 4 : 6;  // arcs per node
  static constexpr int HX = HX_, X0 = X0_, HY = TY + 2, HZ = DIMS == 3 ? TZ + 2 : 1;
  static constexpr int HN = HX * HY * HZ;
  static constexpr int SY = HX, SZ = HX * HY; // box strides
  // arc slots (reference channel order)
  static constexpr int XP = 0, YP = 1;
  static constexpr int ZP = DIMS == 2 ? 0 : 2, ZM = DIMS == 2 ? 0 : 3;
  static constexpr int YM = DIMS == 2 ? 2 : 4, XM = DIMS == 2 ? 3 : 5;
  // halo cells: y faces (2 x TZ x 32), x faces (2 x R), z faces (2 x TY x 32)
  static constexpr int NHY = 2 * TZ * 32, NHX = 2 * R, NHZ = DIMS == 3 ? 2 * TY * 32 : 0;
  static constexpr int NHALO = NHY + NHX + NHZ;
  __device__ static constexpr int hidx(int x, int y, int z) {
    return ((DIMS == 3 ? (z + 1) * HY : 0) + (y + 1)) * HX + (x + X0);
  }
  // halo cell c -> (x, y, z) relative to the tile origin and its face
  // (0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+)
  __device__ static void halo_cell(int c, int& x, int& y, int& z, int& face) {
    if (c < NHY) {
      const int side = c / (TZ * 32), k = c % (TZ * 32);
      x = k & 31; z = k >> 5; y = side ? TY : -1; face = side ? 3 : 2;
    } else if (c < NHY + NHX) {
      const int k = c - NHY, side = k / R, row = k % R;
      x = side ? 32 : -1; y = row % TY; z = row / TY; face = side ? 1 : 0;
    } else {
      const int k = c - NHY - NHX, side = k / (TY * 32), m = k % (TY * 32);
      x = m & 31; y = m >> 5; z = side ? TZ : -1; face = side ? 5 : 4;
    }
  }
};

// Arc bits used by the relaxation: bit 0 +x, 1 +y, 2 -y, 3 -x, 4 +z, 5 -z.
constexpr unsigned A_XP = 1u, A_YP = 2u, A_YM = 4u, A_XM = 8u, A_ZP = 16u, A_ZM = 32u;

// One line of L nodes handled by L lanes (shuffle width L, lane p of its
// segment): min-plus closure h(p) = min(h(p), h(p+k) + k) along runs of
// residual arcs towards +d (bit fwd), then towards -d (bit bwd), by shuffle
// doubling; the halo values at both ends are folded into the end lanes
// first.  The arc runs come from two warp ballots of the arc bits (bits p ..
// p+k-1 of the segment set), so only the values move between lanes.
template <int L>
__device__ __forceinline__ bool line_scan(int* h, int i, int stride, unsigned a, int p, unsigned fwd,
                                          unsigned bwd) {
  const int lane = threadIdx.x & 31;
  const unsigned fm = __ballot_sync(FULL, (a & fwd) != 0u), bm = __ballot_sync(FULL, (a & bwd) != 0u);
  const int v = h[i];
  int vv = v;
  if (p == L - 1 && (a & fwd)) vv = min(vv, h[i + stride] + 1);
#pragma unroll
  for (int off = 1; off < L; off <<= 1) {
    const int nv = __shfl_down_sync(FULL, vv, off, L);
    if (p + off < L && ((~fm >> lane) & ((1u << off) - 1u)) == 0u) vv = min(vv, nv + off);
  }
  if (p == 0 && (a & bwd)) vv = min(vv, h[i - stride] + 1);
#pragma unroll
  for (int off = 1; off < L; off <<= 1) {
    const int nv = __shfl_up_sync(FULL, vv, off, L);
    if (p >= off && ((~bm >> (lane - off + 1)) & ((1u << off) - 1u)) == 0u) vv = min(vv, nv + off);
  }
  if (vv < v) {
    h[i] = vv;
    return true;
  }
  return false;
}

// In-tile relaxation h(u) = min(h(u), h(v) + 1) over residual arcs u -> v with
// the halo fixed, to the fixpoint: each iteration closes every row (32-lane
// scans), then every y column and z column (TY- / TZ-lane scans), so paths
// that turn a few times converge in a few iterations instead of one cell per
// step.  Monotone: reading a value another line just lowered is also valid.
// `arc` holds each node's arc bits (tile order).  All threads of the CTA call
// it; returns true when the fixpoint was reached within max_iter iterations.
// T: the tile geometry (CtaTile) the height box `h` is laid out in.
template <class T>
__device__ bool relax_cta_t(int* h, const uint8_t* arc, int max_iter) {
  constexpr int DIMS = T::D, TY = T::TY, TZ = T::TZ;
  const int t = threadIdx.x;
  for (int it = 0; it < max_iter; ++it) {
    bool ch = false;
    {  // rows: thread t = node t
      const int x = t & 31, row = t >> 5, y = row % TY, z = row / TY;
      ch |= line_scan<32>(h, T::hidx(x, y, z), 1, arc[t], x, A_XP, A_XM);
    }
    __syncthreads();
    {  // y columns: TY lanes per column
      const int c = t / TY, p = t % TY;
      const int x = c & 31, z = c >> 5;
      ch |= line_scan<TY>(h, T::hidx(x, p, z), T::SY, arc[(z * TY + p) * 32 + x], p, A_YP, A_YM);
    }
    if constexpr (DIMS == 3) {
      __syncthreads();
      const int c = t / TZ, p = t % TZ;
      const int x = c & 31, y = c >> 5;
      ch |= line_scan<TZ>(h, T::hidx(x, y, p), T::SZ, arc[(p * TY + y) * 32 + x], p, A_ZP, A_ZM);
    }
    if (!__syncthreads_or(ch)) return true;
  }
  return false;
}

template <int DIMS, int TY, int TZ>
__device__ bool relax_cta(int* h, const uint8_t* arc, int max_iter) {
  return relax_cta_t<CtaTile<DIMS, TY, TZ>>(h, arc, max_iter);
}

}  // namespace jfc
