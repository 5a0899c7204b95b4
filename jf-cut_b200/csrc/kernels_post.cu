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
