// synthetic.cpp — seeded synthetic inputs for the tests and both bench arms.
//
// INPUT GENERATION ONLY: the tests, __graft_entry__.smoke() and bench.py call
// these before any timed region to make the images, videos, volumes and
// strokes the workloads name; nothing on the solve path (libjfcut.so,
// jfcut.py) links or calls them.  They live beside the CPU checker so that
// bench.py's reference arm can build the same graph from the same bytes
// without loading the product library.
//
// The reference reads image / volume files and user brush strokes
// (QGCWidget.cpp:296-683, 2243-2287); the benchmark configurations here are
// synthetic, so these generators produce the named shapes with integer-only
// arithmetic (counter-based hashing, integer quadratic forms, Irwin-Hall
// noise), which makes every image bit-reproducible on any host.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <unordered_set>
#include <vector>


namespace {

constexpr int SYN_OK = 0, SYN_ERR_INVALID_ARG = 1;   // status codes
constexpr uint8_t SEED_FG = 1, SEED_BG = 2;           // seed bytes (0: none)

inline uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
inline uint64_t hash3(uint64_t seed, uint64_t a, uint64_t b) {
  return mix64(seed ^ mix64(a * 0x632be59bd9b4e019ull + mix64(b + 0x8cb92ba72f3d8dd7ull)));
}

// Approximately N(0, sigma) integer noise from one 64-bit hash (sum of four
// 16-bit uniforms, Irwin-Hall n = 4, scaled to unit variance).
inline int noise(uint64_t h, int sigma) {
  const long long s = (long long)(h & 0xffff) + ((h >> 16) & 0xffff) + ((h >> 32) & 0xffff) + (h >> 48);
  const long long num = (s - 131070) * (long long)sigma;
  const long long den = 37838;  // 65536 / sqrt(3)
  return (int)(num >= 0 ? (num + den / 2) / den : -((-num + den / 2) / den));
}

inline int clip255(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(mix64(seed ^ 0x5851f42d4c957f2dull)) {}
  uint64_t next() { s = mix64(s); return s; }
  int uni(int lo, int hi) { return lo + (int)(next() % (uint64_t)(hi - lo + 1)); }
};

// Rotations with integer cosine / sine: (p, q, r) with p^2 + q^2 = r^2.
const int kRot[][3] = {{1, 0, 1}, {0, 1, 1}, {3, 4, 5}, {4, 3, 5}, {5, 12, 13}, {12, 5, 13},
                       {8, 15, 17}, {15, 8, 17}, {7, 24, 25}, {24, 7, 25}, {20, 21, 29}, {21, 20, 29},
                       {-3, 4, 5}, {-4, 3, 5}, {-5, 12, 13}, {-12, 5, 13}, {-8, 15, 17}, {-15, 8, 17}};
const int kNRot = sizeof(kRot) / sizeof(kRot[0]);

struct Ellipse {
  long long cx, cy, a, b;
  int p, q, r;
  int col[3];
  int fg;
  bool inside(long long x, long long y) const {
    const long long dx = x - cx, dy = y - cy;
    const long long m = a > b ? a : b;
    if (dx > m || dx < -m || dy > m || dy < -m) return false;
    const long long u = dx * p + dy * q, v = -dx * q + dy * p;
    return b * b * u * u + a * a * v * v <= a * a * b * b * (long long)r * r;
  }
};

}  // namespace

extern "C" {

int syn_gray_ellipse(int w, int h, uint64_t seed, int noise_sigma, uint8_t* img, uint8_t* seeds) {
  if (w < 8 || h < 8 || !img || !seeds) return SYN_ERR_INVALID_ARG;
  const long long cx = w / 2, cy = h / 2, a = w / 4, b = h / 5;
  const size_t n = (size_t)w * h;
  std::vector<int> mask(n), tmp(n);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const long long dx = x - cx, dy = y - cy;
      mask[(size_t)y * w + x] = (b * b * dx * dx + a * a * dy * dy <= a * a * b * b) ? 255 : 0;
    }
  // Gaussian blur, sigma = 2 px: binomial kernel of order 16 (sum 65536), separable, clamped edges
  static const int kB[17] = {1, 16, 120, 560, 1820, 4368, 8008, 11440, 12870,
                             11440, 8008, 4368, 1820, 560, 120, 16, 1};
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      long long s = 0;
      for (int k = -8; k <= 8; ++k) s += (long long)kB[k + 8] * mask[(size_t)y * w + std::min(w - 1, std::max(0, x + k))];
      tmp[(size_t)y * w + x] = (int)((s + 32768) >> 16);
    }
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      long long s = 0;
      for (int k = -8; k <= 8; ++k) s += (long long)kB[k + 8] * tmp[(size_t)std::min(h - 1, std::max(0, y + k)) * w + x];
      const int blurred = (int)((s + 32768) >> 16);  // 0..255
      const int v = 80 + (90 * blurred + 127) / 255 + noise(hash3(seed, (uint64_t)y * w + x, 0), noise_sigma);
      img[(size_t)y * w + x] = (uint8_t)clip255(v);
    }
  std::memset(seeds, 0, n);
  for (long long x = cx - a / 2; x <= cx + a / 2; ++x) seeds[(size_t)cy * w + x] = SEED_FG;
  const int yb = h / 10;
  for (int x = w / 4; x < 3 * w / 4; ++x) seeds[(size_t)yb * w + x] = SEED_BG;
  return SYN_OK;
}

int syn_rgb_ellipses(int w, int h, uint64_t seed, int n_ellipses, int noise_sigma, int stroke_permille_x10,
                           uint8_t* img, uint8_t* seeds) {
  if (w < 8 || h < 8 || !img || !seeds || n_ellipses < 1 || n_ellipses > 256) return SYN_ERR_INVALID_ARG;
  Rng rng(seed);
  const int mside = std::min(w, h);
  int bgcol[3];
  for (int c = 0; c < 3; ++c) bgcol[c] = rng.uni(0, 255);
  std::vector<Ellipse> el(n_ellipses);
  for (int i = 0; i < n_ellipses; ++i) {
    Ellipse& E = el[i];
    E.cx = rng.uni(0, w - 1);
    E.cy = rng.uni(0, h - 1);
    E.a = rng.uni(std::max(2, mside / 20), std::max(3, mside / 4));
    E.b = rng.uni(std::max(2, mside / 20), std::max(3, mside / 4));
    const int* R = kRot[rng.uni(0, kNRot - 1)];
    E.p = R[0]; E.q = R[1]; E.r = R[2];
    for (int c = 0; c < 3; ++c) E.col[c] = rng.uni(0, 255);
    E.fg = (i % 2) == 0;
  }
  auto region = [&](long long x, long long y) -> int {
    for (int i = n_ellipses - 1; i >= 0; --i)
      if (el[i].inside(x, y)) return i;
    return -1;
  };
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y) {
    for (int x = 0; x < w; ++x) {
      const int rg = region(x, y);
      const int* col = rg >= 0 ? el[rg].col : bgcol;
      const size_t i = (size_t)y * w + x;
      for (int c = 0; c < 3; ++c)
        img[3 * i + c] = (uint8_t)clip255(col[c] + noise(hash3(seed, i, (uint64_t)c + 1), noise_sigma));
    }
  }
  // strokes: straight runs inside one region until the coverage target is met
  const size_t n = (size_t)w * h;
  std::memset(seeds, 0, n);
  const size_t target = std::max<size_t>(2, n * (size_t)stroke_permille_x10 / 10000);
  size_t marked = 0;
  static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {1, -1}, {-1, 1}};
  bool have[2] = {false, false};
  for (size_t tries = 0; (marked < target || !have[0] || !have[1]) && tries < target * 64 + 4096; ++tries) {
    long long x = rng.uni(0, w - 1), y = rng.uni(0, h - 1);
    const int rg = region(x, y);
    const bool fg = rg >= 0 && el[rg].fg;
    if (have[0] && have[1] && marked >= target) break;
    if (marked >= target && have[fg ? 0 : 1]) continue;
    const int lab = fg ? SEED_FG : SEED_BG;
    const int* d = dirs[rng.uni(0, 7)];
    const int len = rng.uni(16, 128);
    for (int s = 0; s < len; ++s) {
      if (x < 0 || y < 0 || x >= w || y >= h) break;
      const int r2 = region(x, y);
      if ((r2 >= 0 && el[r2].fg) != fg) break;
      uint8_t& sd = seeds[(size_t)y * w + x];
      if (!sd) { sd = (uint8_t)lab; ++marked; have[fg ? 0 : 1] = true; }
      x += d[0]; y += d[1];
    }
  }
  return SYN_OK;
}

int syn_rgb_video(int w, int h, int frames, uint64_t seed, uint8_t* img, uint8_t* seeds) {
  if (w < 32 || h < 32 || frames < 2 || !img || !seeds) return SYN_ERR_INVALID_ARG;
  Rng rng(seed);
  const int cell = 32;
  const int gw = w / cell + 2, gh = h / cell + 2;
  std::vector<int> lattice((size_t)gw * gh * 3);
  for (auto& v : lattice) v = rng.uni(0, 255);
  int objcol[3];
  for (int c = 0; c < 3; ++c) objcol[c] = rng.uni(0, 255);
  const long long a = w / 8, b = h / 6;
  const long long cy = h / 2, cx0 = w / 4;
  const size_t wh = (size_t)w * h;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < frames; ++z) {
    const long long cx = cx0 + 4ll * z;  // the object moves 4 px per frame
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        const size_t i = (size_t)z * wh + (size_t)y * w + x;
        const long long dx = x - cx, dy = y - cy;
        const bool in = b * b * dx * dx + a * a * dy * dy <= a * a * b * b;
        for (int c = 0; c < 3; ++c) {
          int base;
          if (in) {
            base = objcol[c];
          } else {
            // value noise: bilinear interpolation of a seeded lattice (integer weights)
            const int gx = x / cell, gy = y / cell, fx = x % cell, fy = y % cell;
            const int v00 = lattice[((size_t)gy * gw + gx) * 3 + c];
            const int v10 = lattice[((size_t)gy * gw + gx + 1) * 3 + c];
            const int v01 = lattice[((size_t)(gy + 1) * gw + gx) * 3 + c];
            const int v11 = lattice[((size_t)(gy + 1) * gw + gx + 1) * 3 + c];
            const int top = v00 * (cell - fx) + v10 * fx, bot = v01 * (cell - fx) + v11 * fx;
            base = (top * (cell - fy) + bot * fy + cell * cell / 2) / (cell * cell);
          }
          img[3 * i + c] = (uint8_t)clip255(base + noise(hash3(seed, i, (uint64_t)c + 7), 10));
        }
      }
  }
  std::memset(seeds, 0, wh * (size_t)frames);
  for (int z : {0, frames - 1}) {
    const long long cx = cx0 + 4ll * z;
    for (long long x = cx - a / 2; x <= cx + a / 2; ++x)
      if (x >= 0 && x < w) seeds[(size_t)z * wh + (size_t)cy * w + x] = SEED_FG;
    for (int x = w / 8; x < 7 * w / 8; ++x) {
      seeds[(size_t)z * wh + (size_t)(h / 12) * w + x] = SEED_BG;
      seeds[(size_t)z * wh + (size_t)(h - 1 - h / 12) * w + x] = SEED_BG;
    }
  }
  return SYN_OK;
}

int syn_i16_phantom(int w, int h, int d, uint64_t seed, int noise_sigma, int16_t* img, uint8_t* seeds) {
  if (w < 8 || h < 8 || d < 8 || !img || !seeds) return SYN_ERR_INVALID_ARG;
  const long long cx = w / 2, cy = h / 2, cz = d / 2;
  const long long R = std::min(std::min(w, h), d) / 4;
  const long long tr = std::max<long long>(2, R / 3);
  const long long tx = cx + R + tr + 2, ty = cy;  // tube along z beside the sphere
  const size_t wh = (size_t)w * h;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < d; ++z)
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        const size_t i = (size_t)z * wh + (size_t)y * w + x;
        const long long dx = x - cx, dy = y - cy, dz = z - cz;
        int v = 0;
        if (dx * dx + dy * dy + dz * dz <= R * R) v = 1000;
        else if ((x - tx) * (x - tx) + (y - ty) * (y - ty) <= tr * tr) v = 600;
        v += noise(hash3(seed, i, 11), noise_sigma);
        img[i] = (int16_t)std::max(-32768, std::min(32767, v));
      }
  std::memset(seeds, 0, wh * (size_t)d);
  const long long s = std::max<long long>(1, R / 4);
  for (long long z = cz - s; z <= cz + s; ++z)
    for (long long y = cy - s; y <= cy + s; ++y)
      for (long long x = cx - s; x <= cx + s; ++x) seeds[(size_t)z * wh + (size_t)y * w + x] = SEED_FG;
  for (long long z = 1; z <= 1 + s; ++z)
    for (long long y = 1; y <= 1 + s; ++y)
      for (long long x = 1; x <= 1 + s; ++x) seeds[(size_t)z * wh + (size_t)y * w + x] = SEED_BG;
  return SYN_OK;
}

int syn_stroke(int dims, int w, int h, int d, uint64_t seed, size_t n, uint8_t label, uint32_t* idx,
                     uint8_t* new_seed, size_t* n_out) {
  if (!idx || !new_seed || !n_out || w < 1 || h < 1) return SYN_ERR_INVALID_ARG;
  if (dims == 2) d = 1;
  Rng rng(seed);
  std::unordered_set<uint64_t> seen;
  seen.reserve(n * 2);
  long long x = rng.uni(0, w - 1), y = rng.uni(0, h - 1), z = rng.uni(0, d - 1);
  int dir = rng.uni(0, dims == 2 ? 3 : 5);
  static const int D6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  size_t k = 0;
  for (size_t step = 0; k < n && step < 8 * n + 64; ++step) {
    const uint64_t id = (uint64_t)x + (uint64_t)w * ((uint64_t)y + (uint64_t)h * (uint64_t)z);
    if (seen.insert(id).second) { idx[k] = (uint32_t)id; new_seed[k] = label; ++k; }
    if (rng.uni(0, 7) == 0) dir = rng.uni(0, dims == 2 ? 3 : 5);
    long long nx = x + D6[dir][0], ny = y + D6[dir][1], nz = z + D6[dir][2];
    if (nx < 0 || ny < 0 || nz < 0 || nx >= w || ny >= h || nz >= d) {
      dir = rng.uni(0, dims == 2 ? 3 : 5);
      continue;
    }
    x = nx; y = ny; z = nz;
  }
  *n_out = k;
  return SYN_OK;
}

}  // extern "C"
