// Surfel PLY import/export in the 3DGS ("INRIA") binary little-endian layout
// (first_attempt/crates/gs-io/src/ply/{header,layout,reader,writer}.rs):
// x y z | f_dc_0..2 | f_rest_0..N (channel-major) | opacity (logit) |
// scale_0..2 (log) | rot_0..3 (w first). The writer flattens surfels by
// writing log-scale −10 for the third axis. The reader locates properties by
// name (reordered or extra float properties are fine), accepts 0, 9, 24 or
// 45 f_rest values, and activates: sigmoid opacity, exp scales, normalised
// xyzw quaternion (identity when degenerate), coefficient-major SH.
// Host code only.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "gs_cuda.h"

namespace gs {
void set_error_message(const std::string& msg);
}

namespace {

constexpr float FLAT_LOG_SCALE = -10.0f;

gs_status fail_io(const std::string& m) {
  gs::set_error_message(m);
  return GS_ERR_IO;
}
gs_status fail_fmt(const std::string& m) {
  gs::set_error_message(m);
  return GS_ERR_FORMAT;
}

struct Prop {
  std::string name;
  int size = 0;        // bytes
  bool is_float = false;
  size_t offset = 0;   // within a row
};

struct Header {
  uint64_t count = 0;
  size_t stride = 0;
  bool has_list = false;
  std::vector<Prop> props;
  std::streamoff data_start = 0;
  const Prop* find(const std::string& n) const {
    for (const Prop& p : props)
      if (p.name == n) return &p;
    return nullptr;
  }
};

int type_size(const std::string& t, bool& is_float) {
  is_float = (t == "float" || t == "float32");
  if (t == "char" || t == "uchar" || t == "int8" || t == "uint8") return 1;
  if (t == "short" || t == "ushort" || t == "int16" || t == "uint16") return 2;
  if (t == "int" || t == "uint" || t == "int32" || t == "uint32" || is_float) return 4;
  if (t == "double" || t == "float64") return 8;
  return 0;
}

// Parses the header (ply/header.rs): magic, binary_little_endian 1.0, the
// vertex element and its properties; later elements are ignored.
gs_status parse_header(std::istream& in, Header& h) {
  std::string line;
  if (!std::getline(in, line) || line.rfind("ply", 0) != 0 || (line.size() > 3 && line[3] != '\r'))
    return fail_fmt("not a ply file (missing 'ply' magic)");
  bool in_vertex = false, seen_vertex = false;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream ls(line);
    std::string kw;
    ls >> kw;
    if (kw == "format") {
      std::string fmt, ver;
      ls >> fmt >> ver;
      if (fmt != "binary_little_endian" || ver != "1.0")
        return fail_fmt("unsupported ply format `" + fmt + " " + ver +
                        "` (only binary_little_endian 1.0 is supported)");
    } else if (kw == "comment" || kw == "obj_info" || kw.empty()) {
      continue;
    } else if (kw == "element") {
      std::string name;
      uint64_t n = 0;
      if (!(ls >> name >> n)) return fail_fmt("malformed ply header: bad element line: " + line);
      in_vertex = (name == "vertex");
      if (in_vertex) {
        if (seen_vertex) return fail_fmt("malformed ply header: two vertex elements");
        seen_vertex = true;
        h.count = n;
      }
    } else if (kw == "property") {
      std::string t;
      ls >> t;
      if (t == "list") {
        if (in_vertex) h.has_list = true;
        continue;
      }
      std::string name;
      if (!(ls >> name)) return fail_fmt("malformed ply header: bad property line: " + line);
      if (!in_vertex) continue;
      Prop p;
      p.name = name;
      p.size = type_size(t, p.is_float);
      if (p.size == 0) return fail_fmt("malformed ply header: unknown type `" + t + "`");
      p.offset = h.stride;
      h.stride += (size_t)p.size;
      h.props.push_back(p);
    } else if (kw == "end_header") {
      if (!seen_vertex) return fail_fmt("no `vertex` element in ply header");
      h.data_start = in.tellg();
      return GS_OK;
    } else {
      return fail_fmt("malformed ply header: unexpected line: " + line);
    }
  }
  return fail_fmt("malformed ply header: missing end_header");
}

struct Layout {
  size_t pos[3], dc[3], opacity, scale[3], rot[4];
  std::vector<size_t> rest;
};

// Splat layout (ply/layout.rs): every required property present and float.
gs_status splat_layout(const Header& h, Layout& L) {
  if (h.has_list) return fail_fmt("vertex element has a list property: not a splat ply");
  if (!h.find("f_dc_0")) return fail_fmt("point-cloud ply (no f_dc_*): no surfels to load");
  std::string missing;
  auto off = [&](const std::string& n, size_t& out) -> bool {
    const Prop* p = h.find(n);
    if (!p) {
      missing += (missing.empty() ? "" : ", ") + n;
      return true;
    }
    if (!p->is_float) return false;
    out = p->offset;
    return true;
  };
  const char* names_pos[3] = {"x", "y", "z"};
  for (int i = 0; i < 3; ++i)
    if (!off(names_pos[i], L.pos[i])) return fail_fmt(std::string("vertex property `") + names_pos[i] +
                                                      "` has unsupported type (expected float)");
  for (int i = 0; i < 3; ++i)
    if (!off("f_dc_" + std::to_string(i), L.dc[i]))
      return fail_fmt("vertex property `f_dc_" + std::to_string(i) + "` has unsupported type (expected float)");
  if (!off("opacity", L.opacity)) return fail_fmt("vertex property `opacity` has unsupported type (expected float)");
  for (int i = 0; i < 3; ++i)
    if (!off("scale_" + std::to_string(i), L.scale[i]))
      return fail_fmt("vertex property `scale_" + std::to_string(i) + "` has unsupported type (expected float)");
  for (int i = 0; i < 4; ++i)
    if (!off("rot_" + std::to_string(i), L.rot[i]))
      return fail_fmt("vertex property `rot_" + std::to_string(i) + "` has unsupported type (expected float)");
  if (!missing.empty()) {
    std::string all;
    for (const Prop& p : h.props) all += (all.empty() ? "" : ", ") + p.name;
    return fail_fmt("unknown vertex layout (missing " + missing + "); properties: " + all);
  }
  size_t rest_count = 0;
  for (const Prop& p : h.props)
    if (p.name.rfind("f_rest_", 0) == 0) ++rest_count;
  if (rest_count != 0 && rest_count != 9 && rest_count != 24 && rest_count != 45)
    return fail_fmt("f_rest count " + std::to_string(rest_count) +
                    " does not match any SH degree (expected 0, 9, 24, or 45)");
  L.rest.resize(rest_count);
  for (size_t i = 0; i < rest_count; ++i)
    if (!off("f_rest_" + std::to_string(i), L.rest[i]))
      return fail_fmt("vertex property `f_rest_" + std::to_string(i) + "` has unsupported type (expected float)");
  if (!missing.empty()) return fail_fmt("unknown vertex layout (missing " + missing + ")");
  return GS_OK;
}

gs_status open_splats(const char* path, std::ifstream& f, Header& h, Layout& L) {
  if (!path) return fail_io("null path");
  f.open(path, std::ios::binary);
  if (!f) return fail_io(std::string("cannot open ") + path);
  gs_status s = parse_header(f, h);
  if (s) return s;
  return splat_layout(h, L);
}

float rd(const unsigned char* row, size_t off) {
  float v;
  std::memcpy(&v, row + off, 4);
  return v;
}

float sigmoid(float x) { return 1.0f / (1.0f + std::exp(-x)); }

}  // namespace

extern "C" {

gs_status gs_ply_write(const char* path, uint32_t count, const float* positions4, const float* scales2,
                       const float* quats4, const float* opacities, const float* sh48) {
  if (!path || (count && (!positions4 || !scales2 || !quats4 || !opacities || !sh48)))
    return fail_io("gs_ply_write: null argument");
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return fail_io(std::string("cannot create ") + path);
  std::string hdr = "ply\nformat binary_little_endian 1.0\ncomment splattar_b200 surfel export (3DGS layout, third "
                    "axis flattened)\nelement vertex " + std::to_string(count) + "\n";
  for (const char* n : {"x", "y", "z"}) hdr += std::string("property float ") + n + "\n";
  for (int i = 0; i < 3; ++i) hdr += "property float f_dc_" + std::to_string(i) + "\n";
  for (int i = 0; i < 45; ++i) hdr += "property float f_rest_" + std::to_string(i) + "\n";
  hdr += "property float opacity\n";
  for (int i = 0; i < 3; ++i) hdr += "property float scale_" + std::to_string(i) + "\n";
  for (int i = 0; i < 4; ++i) hdr += "property float rot_" + std::to_string(i) + "\n";
  hdr += "end_header\n";
  bool ok = std::fwrite(hdr.data(), 1, hdr.size(), fp) == hdr.size();
  std::vector<float> row(62);
  for (uint32_t i = 0; ok && i < count; ++i) {
    size_t k = 0;
    for (int d = 0; d < 3; ++d) row[k++] = positions4[4 * (size_t)i + d];
    const float* sh = sh48 + 48 * (size_t)i;
    for (int c = 0; c < 3; ++c) row[k++] = sh[c];  // f_dc = coefficient 0
    for (int c = 0; c < 3; ++c)                    // f_rest channel-major over coefficients 1..15
      for (int j = 1; j < 16; ++j) row[k++] = sh[3 * j + c];
    const float o = std::fmin(std::fmax(opacities[i], 1e-6f), 1.0f - 1e-6f);
    row[k++] = std::log(o / (1.0f - o));
    row[k++] = std::log(std::fmax(scales2[2 * (size_t)i], 1e-9f));
    row[k++] = std::log(std::fmax(scales2[2 * (size_t)i + 1], 1e-9f));
    row[k++] = FLAT_LOG_SCALE;
    const float* q = quats4 + 4 * (size_t)i;  // xyzw in memory, w first on disk
    row[k++] = q[3]; row[k++] = q[0]; row[k++] = q[1]; row[k++] = q[2];
    ok = std::fwrite(row.data(), sizeof(float), k, fp) == k;
  }
  if (std::fclose(fp) != 0) ok = false;
  if (!ok) return fail_io(std::string("write failed: ") + path);
  return GS_OK;
}

gs_status gs_ply_info(const char* path, uint32_t* count, uint32_t* sh_coeffs) {
  if (!count || !sh_coeffs) return fail_io("gs_ply_info: null output");
  std::ifstream f;
  Header h;
  Layout L;
  gs_status s = open_splats(path, f, h, L);
  if (s) return s;
  if (h.count > 0xffffffffull) return fail_fmt("more than 2^32-1 vertices");
  *count = (uint32_t)h.count;
  *sh_coeffs = (uint32_t)(1 + L.rest.size() / 3);
  return GS_OK;
}

gs_status gs_ply_read(const char* path, uint32_t capacity, float* positions3, float* scales3, float* quats4,
                      float* opacities, float* sh, uint32_t* count) {
  if (!count || !positions3 || !scales3 || !quats4 || !opacities || !sh) return fail_io("gs_ply_read: null argument");
  std::ifstream f;
  Header h;
  Layout L;
  gs_status s = open_splats(path, f, h, L);
  if (s) return s;
  if (h.count > capacity) return fail_fmt("ply holds " + std::to_string(h.count) + " surfels, capacity " +
                                          std::to_string(capacity));
  const size_t rpc = L.rest.size() / 3, nc = 1 + rpc;
  std::vector<unsigned char> buf;
  const size_t chunk = std::max<size_t>(1, (8u << 20) / std::max<size_t>(h.stride, 1));
  uint64_t done = 0;
  while (done < h.count) {
    const size_t rows = (size_t)std::min<uint64_t>(chunk, h.count - done);
    buf.resize(rows * h.stride);
    f.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)buf.size());
    const size_t got = (size_t)f.gcount() / h.stride;
    for (size_t r = 0; r < got; ++r) {
      const unsigned char* row = buf.data() + r * h.stride;
      const size_t i = (size_t)(done + r);
      for (int d = 0; d < 3; ++d) positions3[3 * i + d] = rd(row, L.pos[d]);
      float* o = sh + nc * 3 * i;
      for (int c = 0; c < 3; ++c) o[c] = rd(row, L.dc[c]);
      for (size_t j = 0; j < rpc; ++j)
        for (int c = 0; c < 3; ++c) o[3 * (1 + j) + c] = rd(row, L.rest[c * rpc + j]);
      opacities[i] = sigmoid(rd(row, L.opacity));
      for (int d = 0; d < 3; ++d) scales3[3 * i + d] = std::exp(rd(row, L.scale[d]));
      const float w = rd(row, L.rot[0]), x = rd(row, L.rot[1]), y = rd(row, L.rot[2]), z = rd(row, L.rot[3]);
      const float n2 = x * x + y * y + z * z + w * w;
      float* q = quats4 + 4 * i;
      if (n2 > 1e-12f) {
        const float inv = 1.0f / std::sqrt(n2);
        q[0] = x * inv; q[1] = y * inv; q[2] = z * inv; q[3] = w * inv;
      } else {
        q[0] = q[1] = q[2] = 0.0f; q[3] = 1.0f;
      }
    }
    done += got;
    if (got < rows) {
      *count = (uint32_t)done;
      return fail_fmt("file ended early: expected " + std::to_string(h.count) + " vertices, payload holds " +
                      std::to_string(done));
    }
  }
  *count = (uint32_t)h.count;
  return GS_OK;
}

}  // extern "C"
