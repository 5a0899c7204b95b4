// formats.cpp — the reference's on-disk formats, host side (no device work):
//
//   .dat  volume header, text "Key: values" lines
//         (QGCWidget::parseDataFile / saveDataFile, QGCWidget.cpp:296-683)
//   .raw  volume samples in the header's format and endianness
//   .ef / .c1 / .c2  a grid graph: int32 net excess; 2D ushort2 (+x, +y) and
//         ushort2 (-y, -x); 3D uchar4 (+x, +y, +z, pad) and uchar4 (-z, -y, -x,
//         pad)  (slotLoadGraphClicked / slotSaveGraphClicked,
//         QGCWidget.cpp:2631-2736; cl_node_2d / cl_node_3d, QGCSetting.h:31-44)
//   .cut  4 bytes per node {foreground seed, background seed, object, tag}
//         (cl_cut, QGCSetting.h:46-51; slotLoadCutClicked / slotSaveCutClicked,
//         QGCWidget.cpp:2971-2996)
//   .mfi  max-flow instance of the GridCut benchmark: "MFI" + packed header +
//         source / sink / per-direction neighbour capacities + mask
//         (src/QVisualizer/3rdParty/bench/mfi.cpp, QGCWidget::saveMFI,
//         QGCWidget.cpp:3339-3474; arc semantics as the benchmark builds its
//         graphs, benchmark/GridCut/bench-BK303.cpp)
//
// Graph arrays on this side of the ABI are dense (w*h*d, x fastest) int32 in
// the solver's channel order: 2D +x, +y, -y, -x; 3D +x, +y, +z, -z, -y, -x.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "engine.h"

namespace {

struct File {
  FILE* f = nullptr;
  explicit File(const char* path, const char* mode) { f = std::fopen(path, mode); }
  ~File() { if (f) std::fclose(f); }
};

int io_error(const std::string& what, const char* path) {
  return set_error(JFC_ERR_IO, what + ": " + (path ? path : "(null)"));
}

bool read_all(FILE* f, void* dst, size_t bytes) { return std::fread(dst, 1, bytes, f) == bytes; }
bool write_all(FILE* f, const void* src, size_t bytes) { return std::fwrite(src, 1, bytes, f) == bytes; }

size_t nodes_of(int dims, int w, int h, int d) { return (size_t)w * h * (dims == 3 ? d : 1); }

int check_shape(int dims, int w, int h, int d) {
  if ((dims != 2 && dims != 3) || w < 1 || h < 1 || (dims == 3 && d < 1))
    return set_error(JFC_ERR_INVALID_ARG, "bad grid shape");
  return JFC_OK;
}

// MFI packed header (3-byte magic "MFI" precedes it)
#pragma pack(push, 1)
struct MfiHeader {
  int32_t dimension, connectivity, width, height, depth;
  int64_t maxflow;
  int32_t symmetric_arcs;
  int8_t metadata[4096];
  int32_t active_count;
  int32_t type_terminal_cap, type_neighbor_cap;
};
#pragma pack(pop)
static_assert(sizeof(MfiHeader) == 4140, "MFI header layout");

// solver slot k <- MFI arc index (2D: LE 0, GE 1, EL 2, EG 3; 3D: LEE 0, GEE 1,
// ELE 2, EGE 3, EEL 4, EEG 5)
constexpr int kMfi2[4] = {1, 3, 2, 0};
constexpr int kMfi3[6] = {1, 3, 5, 4, 2, 0};

size_t type_size(int t) { return t == 0 ? 1 : t == 1 ? 2 : 4; }

uint32_t get_cap(const std::vector<uint8_t>& buf, int t, size_t i) {
  if (t == 0) return buf[i];
  if (t == 1) { uint16_t v; std::memcpy(&v, buf.data() + 2 * i, 2); return v; }
  uint32_t v;
  std::memcpy(&v, buf.data() + 4 * i, 4);
  return v;
}

void put_cap(std::vector<uint8_t>& buf, int t, size_t i, uint32_t v) {
  if (t == 0) buf[i] = (uint8_t)v;
  else if (t == 1) { const uint16_t x = (uint16_t)v; std::memcpy(buf.data() + 2 * i, &x, 2); }
  else std::memcpy(buf.data() + 4 * i, &v, 4);
}

const char* kFormats[] = {"UCHAR", "CHAR", "USHORT", "SHORT", "UINT", "INT", "FLOAT"};

}  // namespace

extern "C" {

int jfc_read_dat(const char* path, jfc_volume_info* out) {
  if (!path || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  std::ifstream in(path);
  if (!in) return io_error("cannot open", path);
  std::memset(out, 0, sizeof(*out));
  out->format = -1;
  out->thickness[0] = out->thickness[1] = out->thickness[2] = 1.0f;
  std::string line;
  bool have_res = false;
  while (std::getline(in, line)) {
    const size_t colon = line.find(':');
    if (colon == std::string::npos) continue;
    const std::string key = line.substr(0, colon);
    std::string val = line.substr(colon + 1);
    std::istringstream vs(val);
    if (key.find("Object File Name") != std::string::npos) {
      const size_t b = val.find_first_not_of(" \t\r"), e = val.find_last_not_of(" \t\r");
      if (b == std::string::npos) return set_error(JFC_ERR_INVALID_ARG, "empty object file name");
      const std::string name = val.substr(b, e - b + 1);
      if (name.size() >= sizeof(out->object_file)) return set_error(JFC_ERR_INVALID_ARG, "object file name too long");
      std::memcpy(out->object_file, name.c_str(), name.size() + 1);
    } else if (key.find("Resolution") != std::string::npos) {
      long long x = 0, y = 0, z = 0;
      vs >> x >> y >> z;
      if (x <= 1 || y <= 1 || z <= 0 || x > (1 << 30) || y > (1 << 30) || z > (1 << 30))
        return set_error(JFC_ERR_INVALID_ARG, "bad resolution");
      out->w = (int)x; out->h = (int)y; out->d = (int)z;
      have_res = true;
    } else if (key.find("Slice Thickness") != std::string::npos) {
      float x = 0, y = 0, z = 0;
      vs >> x >> y >> z;
      if (!(x > 0 && y > 0 && z > 0)) return set_error(JFC_ERR_INVALID_ARG, "bad slice thickness");
      out->thickness[0] = x; out->thickness[1] = y; out->thickness[2] = z;
    } else if (key.find("Format") != std::string::npos) {
      // longest names first: "UCHAR" contains "CHAR", "USHORT" contains "SHORT"
      if (val.find("UCHAR") != std::string::npos) out->format = JFC_FMT_UCHAR;
      else if (val.find("CHAR") != std::string::npos) out->format = JFC_FMT_CHAR;
      else if (val.find("USHORT") != std::string::npos) out->format = JFC_FMT_USHORT;
      else if (val.find("SHORT") != std::string::npos) out->format = JFC_FMT_SHORT;
      else if (val.find("UINT") != std::string::npos) out->format = JFC_FMT_UINT;
      else if (val.find("INT") != std::string::npos) out->format = JFC_FMT_INT;
      else if (val.find("FLOAT") != std::string::npos) out->format = JFC_FMT_FLOAT;
      else return set_error(JFC_ERR_INVALID_ARG, "unknown sample format");
    } else if (key.find("Endian") != std::string::npos) {
      if (val.find("BIG-ENDIAN") != std::string::npos) out->big_endian = 1;
      else if (val.find("LITTLE-ENDIAN") != std::string::npos) out->big_endian = 0;
      else return set_error(JFC_ERR_INVALID_ARG, "unknown endianness");
    } else if (key.find("Intensity Extremums") != std::string::npos) {
      vs >> out->intensity_min >> out->intensity_max;
    }
  }
  if (!have_res || out->format < 0 || !out->object_file[0])
    return set_error(JFC_ERR_INVALID_ARG, "header lacks object file name, resolution or format");
  return JFC_OK;
}

int jfc_write_dat(const char* path, const jfc_volume_info* in) {
  if (!path || !in) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (in->format < JFC_FMT_UCHAR || in->format > JFC_FMT_FLOAT || in->w < 1 || in->h < 1 || in->d < 1)
    return set_error(JFC_ERR_INVALID_ARG, "bad volume info");
  std::ofstream o(path);
  if (!o) return io_error("cannot create", path);
  o << "Object File Name: " << in->object_file << "\n";
  o << "Resolution: " << in->w << " " << in->h << " " << in->d << "\n";
  o << "Slice Thickness: " << in->thickness[0] << " " << in->thickness[1] << " " << in->thickness[2] << "\n";
  o << "Format: " << kFormats[in->format] << "\n";
  o << "Endian: " << (in->big_endian ? "BIG-ENDIAN" : "LITTLE-ENDIAN") << "\n";
  o << "Intensity Extremums: " << in->intensity_min << " " << in->intensity_max << "\n";
  return o.good() ? JFC_OK : io_error("write failed", path);
}

int jfc_read_raw(const char* path, const jfc_volume_info* info, float* out) {
  if (!path || !info || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  if (info->format < JFC_FMT_UCHAR || info->format > JFC_FMT_FLOAT) return set_error(JFC_ERR_INVALID_ARG, "bad format");
  const size_t n = (size_t)info->w * info->h * info->d;
  const size_t es = info->format <= JFC_FMT_CHAR ? 1 : info->format <= JFC_FMT_SHORT ? 2 : 4;
  File f(path, "rb");
  if (!f.f) return io_error("cannot open", path);
  std::vector<uint8_t> buf(n * es);
  if (!read_all(f.f, buf.data(), buf.size())) return io_error("short file", path);
  for (size_t i = 0; i < n; ++i) {
    uint8_t b[4] = {0, 0, 0, 0};
    for (size_t k = 0; k < es; ++k) b[k] = buf[i * es + (info->big_endian ? es - 1 - k : k)];
    float v = 0.f;
    switch (info->format) {
      case JFC_FMT_UCHAR: v = (float)b[0]; break;
      case JFC_FMT_CHAR: v = (float)(int8_t)b[0]; break;
      case JFC_FMT_USHORT: { uint16_t x; std::memcpy(&x, b, 2); v = (float)x; break; }
      case JFC_FMT_SHORT: { int16_t x; std::memcpy(&x, b, 2); v = (float)x; break; }
      case JFC_FMT_UINT: { uint32_t x; std::memcpy(&x, b, 4); v = (float)x; break; }
      case JFC_FMT_INT: { int32_t x; std::memcpy(&x, b, 4); v = (float)x; break; }
      default: std::memcpy(&v, b, 4); break;
    }
    out[i] = v;
  }
  return JFC_OK;
}

int jfc_load_graph_files(const char* base, int dims, int w, int h, int d, int32_t* excess, int32_t* const* ncap) {
  if (!base || !excess || !ncap) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  int rc = check_shape(dims, w, h, d);
  if (rc) return rc;
  const size_t n = nodes_of(dims, w, h, d);
  const int conn = dims == 2 ? 4 : 6;
  for (int k = 0; k < conn; ++k)
    if (!ncap[k]) return set_error(JFC_ERR_INVALID_ARG, "null capacity array");
  const std::string b(base);
  {
    File f((b + ".ef").c_str(), "rb");
    if (!f.f) return io_error("cannot open", (b + ".ef").c_str());
    if (!read_all(f.f, excess, n * 4)) return io_error("short file", (b + ".ef").c_str());
  }
  const size_t es = dims == 2 ? 2 : 1;   // ushort2 / uchar4 channels
  const size_t stride = dims == 2 ? 2 : 4;
  std::vector<uint8_t> c1(n * stride * es), c2(n * stride * es);
  for (int part = 0; part < 2; ++part) {
    const std::string p = b + (part ? ".c2" : ".c1");
    File f(p.c_str(), "rb");
    if (!f.f) return io_error("cannot open", p.c_str());
    if (!read_all(f.f, part ? c2.data() : c1.data(), c1.size())) return io_error("short file", p.c_str());
  }
  auto ch = [&](const std::vector<uint8_t>& c, size_t i, int j) -> int32_t {
    if (es == 1) return c[i * stride + j];
    uint16_t v;
    std::memcpy(&v, c.data() + 2 * (i * stride + j), 2);
    return v;
  };
  for (size_t i = 0; i < n; ++i) {
    if (dims == 2) {
      ncap[0][i] = ch(c1, i, 0);   // +x
      ncap[1][i] = ch(c1, i, 1);   // +y
      ncap[2][i] = ch(c2, i, 0);   // -y
      ncap[3][i] = ch(c2, i, 1);   // -x
    } else {
      ncap[0][i] = ch(c1, i, 0);   // +x
      ncap[1][i] = ch(c1, i, 1);   // +y
      ncap[2][i] = ch(c1, i, 2);   // +z
      ncap[3][i] = ch(c2, i, 0);   // -z
      ncap[4][i] = ch(c2, i, 1);   // -y
      ncap[5][i] = ch(c2, i, 2);   // -x
    }
  }
  return JFC_OK;
}

int jfc_save_graph_files(const char* base, int dims, int w, int h, int d, const int32_t* excess,
                         const int32_t* const* ncap) {
  if (!base || !excess || !ncap) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  int rc = check_shape(dims, w, h, d);
  if (rc) return rc;
  const size_t n = nodes_of(dims, w, h, d);
  const int conn = dims == 2 ? 4 : 6;
  const int32_t cap_max = dims == 2 ? 65535 : 255;
  for (int k = 0; k < conn; ++k) {
    if (!ncap[k]) return set_error(JFC_ERR_INVALID_ARG, "null capacity array");
    for (size_t i = 0; i < n; ++i)
      if (ncap[k][i] < 0 || ncap[k][i] > cap_max)
        return set_error(JFC_ERR_INVALID_ARG, dims == 2 ? "capacity does not fit ushort (.c1/.c2)"
                                                        : "capacity does not fit uchar (.c1/.c2)");
  }
  const size_t es = dims == 2 ? 2 : 1, stride = dims == 2 ? 2 : 4;
  std::vector<uint8_t> c1(n * stride * es, 0), c2(n * stride * es, 0);
  auto put = [&](std::vector<uint8_t>& c, size_t i, int j, int32_t v) {
    if (es == 1) c[i * stride + j] = (uint8_t)v;
    else { const uint16_t x = (uint16_t)v; std::memcpy(c.data() + 2 * (i * stride + j), &x, 2); }
  };
  for (size_t i = 0; i < n; ++i) {
    if (dims == 2) {
      put(c1, i, 0, ncap[0][i]); put(c1, i, 1, ncap[1][i]);
      put(c2, i, 0, ncap[2][i]); put(c2, i, 1, ncap[3][i]);
    } else {
      put(c1, i, 0, ncap[0][i]); put(c1, i, 1, ncap[1][i]); put(c1, i, 2, ncap[2][i]);
      put(c2, i, 0, ncap[3][i]); put(c2, i, 1, ncap[4][i]); put(c2, i, 2, ncap[5][i]);
    }
  }
  const std::string b(base);
  const std::pair<std::string, const void*> parts[3] = {{".ef", excess}, {".c1", c1.data()}, {".c2", c2.data()}};
  for (int p = 0; p < 3; ++p) {
    const std::string path = b + parts[p].first;
    File f(path.c_str(), "wb");
    if (!f.f) return io_error("cannot create", path.c_str());
    if (!write_all(f.f, parts[p].second, p == 0 ? n * 4 : c1.size())) return io_error("write failed", path.c_str());
  }
  return JFC_OK;
}

int jfc_read_cut(const char* path, size_t n, uint8_t* seeds, uint8_t* labels) {
  if (!path) return set_error(JFC_ERR_INVALID_ARG, "null path");
  File f(path, "rb");
  if (!f.f) return io_error("cannot open", path);
  std::vector<uint8_t> buf(n * 4);
  if (!read_all(f.f, buf.data(), buf.size())) return io_error("short file", path);
  for (size_t i = 0; i < n; ++i) {
    if (seeds) seeds[i] = buf[4 * i] ? JFC_SEED_FG : buf[4 * i + 1] ? JFC_SEED_BG : JFC_SEED_NONE;
    if (labels) labels[i] = buf[4 * i + 2] ? 1 : 0;
  }
  return JFC_OK;
}

int jfc_write_cut(const char* path, size_t n, const uint8_t* seeds, const uint8_t* labels) {
  if (!path) return set_error(JFC_ERR_INVALID_ARG, "null path");
  std::vector<uint8_t> buf(n * 4, 0);
  for (size_t i = 0; i < n; ++i) {
    if (seeds) {
      buf[4 * i] = seeds[i] == JFC_SEED_FG;
      buf[4 * i + 1] = seeds[i] == JFC_SEED_BG;
    }
    if (labels) buf[4 * i + 2] = labels[i] != 0;
  }
  File f(path, "wb");
  if (!f.f) return io_error("cannot create", path);
  if (!write_all(f.f, buf.data(), buf.size())) return io_error("write failed", path);
  return JFC_OK;
}

int jfc_read_mfi_info(const char* path, jfc_mfi_info* out) {
  if (!path || !out) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  File f(path, "rb");
  if (!f.f) return io_error("cannot open", path);
  char magic[3];
  MfiHeader hd;
  if (!read_all(f.f, magic, 3) || std::memcmp(magic, "MFI", 3) != 0) return io_error("not an MFI file", path);
  if (!read_all(f.f, &hd, sizeof(hd))) return io_error("short header", path);
  std::memset(out, 0, sizeof(*out));
  out->dims = hd.dimension;
  out->conn = hd.connectivity;
  out->w = hd.width;
  out->h = hd.height;
  out->d = hd.dimension == 2 ? 1 : hd.depth;
  out->maxflow = hd.maxflow;
  out->active_count = hd.active_count;
  out->type_terminal = hd.type_terminal_cap;
  out->type_neighbor = hd.type_neighbor_cap;
  if (!((out->dims == 2 && out->conn == 4) || (out->dims == 3 && out->conn == 6)))
    return set_error(JFC_ERR_INVALID_ARG, "MFI connectivity other than 2D/4 and 3D/6 is not supported");
  if (out->type_terminal < 0 || out->type_terminal > 2 || out->type_neighbor < 0 || out->type_neighbor > 2)
    return set_error(JFC_ERR_INVALID_ARG, "bad MFI capacity type");
  return check_shape(out->dims, out->w, out->h, out->d);
}

int jfc_load_mfi(const char* path, int32_t* excess, int32_t* const* ncap, int64_t* flow_offset, uint8_t* mask) {
  jfc_mfi_info info;
  int rc = jfc_read_mfi_info(path, &info);
  if (rc) return rc;
  if (!excess || !ncap || !flow_offset) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  for (int k = 0; k < info.conn; ++k)
    if (!ncap[k]) return set_error(JFC_ERR_INVALID_ARG, "null capacity array");
  const size_t n = nodes_of(info.dims, info.w, info.h, info.d);
  File f(path, "rb");
  if (!f.f) return io_error("cannot open", path);
  if (std::fseek(f.f, 3 + (long)sizeof(MfiHeader), SEEK_SET) != 0) return io_error("seek failed", path);
  const size_t ts = type_size(info.type_terminal), ns = type_size(info.type_neighbor);
  std::vector<uint8_t> src(n * ts), snk(n * ts), nb(n * ns);
  if (!read_all(f.f, src.data(), src.size()) || !read_all(f.f, snk.data(), snk.size()))
    return io_error("short file", path);
  long long off = 0;
  for (size_t i = 0; i < n; ++i) {
    const long long cs = get_cap(src, info.type_terminal, i), ct = get_cap(snk, info.type_terminal, i);
    const long long e = cs - ct;
    if (e > 0x7fffffffll || e < -0x7fffffffll) return set_error(JFC_ERR_INVALID_ARG, "terminal capacity exceeds int32");
    excess[i] = (int32_t)e;
    off += std::min(cs, ct);
  }
  const int* map = info.dims == 2 ? kMfi2 : kMfi3;
  for (int a = 0; a < info.conn; ++a) {
    if (!read_all(f.f, nb.data(), nb.size())) return io_error("short file", path);
    int k = 0;
    while (map[k] != a) ++k;
    for (size_t i = 0; i < n; ++i) {
      const uint32_t v = get_cap(nb, info.type_neighbor, i);
      if (v > 0x7fffffffu) return set_error(JFC_ERR_INVALID_ARG, "neighbour capacity exceeds int32");
      ncap[k][i] = (int32_t)v;
    }
  }
  if (mask && !read_all(f.f, mask, n)) return io_error("short file (mask)", path);
  *flow_offset = off;
  return JFC_OK;
}

int jfc_save_mfi(const char* path, int dims, int w, int h, int d, const int32_t* excess, const int32_t* const* ncap,
                 int64_t maxflow, const uint8_t* mask) {
  if (!path || !excess || !ncap) return set_error(JFC_ERR_INVALID_ARG, "null argument");
  int rc = check_shape(dims, w, h, d);
  if (rc) return rc;
  const int conn = dims == 2 ? 4 : 6;
  const size_t n = nodes_of(dims, w, h, d);
  // the reference's types (uint32 terminals; uint16 2D / uint8 3D neighbours),
  // widened to uint32 when a capacity does not fit
  int tn = dims == 2 ? 1 : 0;
  for (int k = 0; k < conn; ++k) {
    if (!ncap[k]) return set_error(JFC_ERR_INVALID_ARG, "null capacity array");
    for (size_t i = 0; i < n; ++i) {
      if (ncap[k][i] < 0) return set_error(JFC_ERR_INVALID_ARG, "negative capacity");
      if ((tn == 0 && ncap[k][i] > 255) || (tn == 1 && ncap[k][i] > 65535)) tn = 2;
    }
  }
  MfiHeader hd;
  std::memset(&hd, 0, sizeof(hd));
  hd.dimension = dims;
  hd.connectivity = conn;
  hd.width = w;
  hd.height = h;
  hd.depth = dims == 2 ? 1 : d;
  hd.maxflow = maxflow;
  hd.symmetric_arcs = 1;
  hd.type_terminal_cap = 2;
  hd.type_neighbor_cap = tn;
  std::vector<uint8_t> src(n * 4), snk(n * 4), nb(n * type_size(tn));
  int active = 0;
  for (size_t i = 0; i < n; ++i) {
    const int32_t e = excess[i];
    put_cap(src, 2, i, e >= 0 ? (uint32_t)e : 0u);
    put_cap(snk, 2, i, e >= 0 ? 0u : (uint32_t)(-(int64_t)e));
    active += e >= 0;
  }
  hd.active_count = active;
  File f(path, "wb");
  if (!f.f) return io_error("cannot create", path);
  if (!write_all(f.f, "MFI", 3) || !write_all(f.f, &hd, sizeof(hd)) || !write_all(f.f, src.data(), src.size()) ||
      !write_all(f.f, snk.data(), snk.size()))
    return io_error("write failed", path);
  const int* map = dims == 2 ? kMfi2 : kMfi3;
  for (int a = 0; a < conn; ++a) {
    int k = 0;
    while (map[k] != a) ++k;
    for (size_t i = 0; i < n; ++i) put_cap(nb, tn, i, (uint32_t)ncap[k][i]);
    if (!write_all(f.f, nb.data(), nb.size())) return io_error("write failed", path);
  }
  std::vector<uint8_t> m(n, 0);
  if (mask) std::memcpy(m.data(), mask, n);
  if (!write_all(f.f, m.data(), n)) return io_error("write failed", path);
  return JFC_OK;
}

}  // extern "C"
