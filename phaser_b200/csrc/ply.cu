// PLY ingest (host): the vertex properties the registration reads, written
// straight into caller buffers (pinned host memory for an asynchronous upload).
//
// Reference behaviour: data::PlyHelper::readPlyFromFile
// (phaser_common/src/common/data/ply-helper.cc:26-64) requests, from element
// "vertex", x, y, z and the intensity field (both required: CHECK_GT at
// :36,41), then the reflectivity, ambient ("noise") and range fields
// (optional: a warning when absent), each converted to double by tinyply;
// PointCloud::parsePlyPointCloud (point-cloud.cc:329-348) narrows x, y, z and
// intensity to float.  Field names default to the reference's flag defaults
// (ply-helper.cc:8-22).  Here the header is parsed and ascii,
// binary_little_endian and binary_big_endian bodies are read; every scalar
// property type is accepted; list properties and other elements are skipped.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/phaser_gpu.h"

namespace {

enum PlyType { kI8, kU8, kI16, kU16, kI32, kU32, kF32, kF64, kBad };

PlyType ply_type(const std::string& t) {
  if (t == "char" || t == "int8") return kI8;
  if (t == "uchar" || t == "uint8") return kU8;
  if (t == "short" || t == "int16") return kI16;
  if (t == "ushort" || t == "uint16") return kU16;
  if (t == "int" || t == "int32") return kI32;
  if (t == "uint" || t == "uint32") return kU32;
  if (t == "float" || t == "float32") return kF32;
  if (t == "double" || t == "float64") return kF64;
  return kBad;
}

int type_size(PlyType t) {
  switch (t) {
    case kI8: case kU8: return 1;
    case kI16: case kU16: return 2;
    case kI32: case kU32: case kF32: return 4;
    case kF64: return 8;
    default: return 0;
  }
}

struct Prop {
  std::string name;
  PlyType type = kBad;
  bool is_list = false;
  PlyType count_type = kBad;
};

struct Element {
  std::string name;
  uint64_t count = 0;
  std::vector<Prop> props;
};

struct Header {
  int format = -1;  // 0 ascii, 1 binary little endian, 2 binary big endian
  std::vector<Element> elements;
};

// A header line quoted in an error message: printable ASCII only (a damaged
// file can put any byte there), at most 80 characters.
std::string quoted(const std::string& line) {
  std::string q;
  for (char ch : line) {
    if (q.size() >= 80) {
      q += "...";
      break;
    }
    const unsigned char u = (unsigned char)ch;
    q += (u >= 0x20 && u < 0x7f) ? ch : '?';
  }
  return q;
}

bool parse_header(std::istream& in, Header* h, std::string* err) {
  std::string line;
  if (!std::getline(in, line) || line.compare(0, 3, "ply") != 0) {
    *err = "not a PLY file";
    return false;
  }
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream ls(line);
    std::string key;
    ls >> key;
    if (key == "format") {
      std::string f;
      ls >> f;
      h->format = f == "ascii" ? 0 : f == "binary_little_endian" ? 1 : f == "binary_big_endian" ? 2 : -1;
    } else if (key == "element") {
      Element e;
      if (!(ls >> e.name >> e.count)) {
        *err = "bad element line: " + quoted(line);
        return false;
      }
      h->elements.push_back(e);
    } else if (key == "property") {
      if (h->elements.empty()) {
        *err = "property before element";
        return false;
      }
      Prop p;
      std::string t;
      ls >> t;
      if (t == "list") {
        std::string ct, it;
        ls >> ct >> it >> p.name;
        p.is_list = true;
        p.count_type = ply_type(ct);
        p.type = ply_type(it);
      } else {
        p.type = ply_type(t);
        ls >> p.name;
      }
      if (p.type == kBad || (p.is_list && p.count_type == kBad)) {
        *err = "unknown property type in: " + quoted(line);
        return false;
      }
      h->elements.back().props.push_back(p);
    } else if (key == "end_header") {
      if (h->format < 0) {
        *err = "missing or unknown format";
        return false;
      }
      return true;
    }
  }
  *err = "no end_header";
  return false;
}

bool host_is_little() {
  const uint16_t one = 1;
  unsigned char c;
  memcpy(&c, &one, 1);
  return c == 1;
}

double read_binary(const unsigned char* b, PlyType t, bool swap) {
  unsigned char v[8];
  const int n = type_size(t);
  for (int i = 0; i < n; ++i) v[i] = swap ? b[n - 1 - i] : b[i];
  switch (t) {
    case kI8: { int8_t x; memcpy(&x, v, 1); return x; }
    case kU8: { uint8_t x; memcpy(&x, v, 1); return x; }
    case kI16: { int16_t x; memcpy(&x, v, 2); return x; }
    case kU16: { uint16_t x; memcpy(&x, v, 2); return x; }
    case kI32: { int32_t x; memcpy(&x, v, 4); return x; }
    case kU32: { uint32_t x; memcpy(&x, v, 4); return x; }
    case kF32: { float x; memcpy(&x, v, 4); return x; }
    case kF64: { double x; memcpy(&x, v, 8); return x; }
    default: return 0.0;
  }
}

// Column of `rows` values of type T at `src` + r * stride (host byte order)
// into dst[r * dst_stride], narrowed as the reference does: to double, then
// to float.
template <typename T>
void decode_column_as(const unsigned char* src, uint64_t rows, int stride, float* dst, int dst_stride) {
  for (uint64_t r = 0; r < rows; ++r) {
    T v;
    memcpy(&v, src + r * stride, sizeof(T));
    dst[r * dst_stride] = (float)(double)v;
  }
}

void decode_column(const unsigned char* src, uint64_t rows, int stride, PlyType t, float* dst, int dst_stride) {
  switch (t) {
    case kI8: decode_column_as<int8_t>(src, rows, stride, dst, dst_stride); break;
    case kU8: decode_column_as<uint8_t>(src, rows, stride, dst, dst_stride); break;
    case kI16: decode_column_as<int16_t>(src, rows, stride, dst, dst_stride); break;
    case kU16: decode_column_as<uint16_t>(src, rows, stride, dst, dst_stride); break;
    case kI32: decode_column_as<int32_t>(src, rows, stride, dst, dst_stride); break;
    case kU32: decode_column_as<uint32_t>(src, rows, stride, dst, dst_stride); break;
    case kF32: decode_column_as<float>(src, rows, stride, dst, dst_stride); break;
    case kF64: decode_column_as<double>(src, rows, stride, dst, dst_stride); break;
    default: break;
  }
}

thread_local std::string g_ply_error;

// The seven requested fields: x, y, z, intensity (required), then
// reflectivity, ambient, range (optional).
constexpr int kFields = 7;

struct Layout {
  Header h;
  int vertex = -1;
  int col[kFields];
};

int open_layout(const char* path, const char* const* names_in, std::ifstream* in, Layout* L) {
  in->open(path, std::ios::binary);
  if (!in->is_open()) {
    g_ply_error = std::string("cannot open ") + path;
    return PHGPU_ERR_INVALID;
  }
  if (!parse_header(*in, &L->h, &g_ply_error)) return PHGPU_ERR_INVALID;
  for (size_t e = 0; e < L->h.elements.size(); ++e)
    if (L->h.elements[e].name == "vertex") {
      L->vertex = (int)e;
      break;
    }
  if (L->vertex < 0) {
    g_ply_error = "no vertex element";
    return PHGPU_ERR_INVALID;
  }
  const char* defaults[4] = {"intensity", "reflectivity", "noise", "range"};
  std::string names[kFields] = {"x", "y", "z", "", "", "", ""};
  for (int f = 0; f < 4; ++f) names[3 + f] = (names_in && names_in[f]) ? names_in[f] : defaults[f];
  const Element& ve = L->h.elements[L->vertex];
  for (int f = 0; f < kFields; ++f) {
    L->col[f] = -1;
    for (size_t p = 0; p < ve.props.size(); ++p)
      if (!ve.props[p].is_list && ve.props[p].name == names[f]) {
        L->col[f] = (int)p;
        break;
      }
  }
  for (int f = 0; f < 4; ++f)
    if (L->col[f] < 0) {
      g_ply_error = "vertex property missing: " + quoted(names[f]);
      return PHGPU_ERR_INVALID;
    }
  if (ve.count > 0xffffffffull) {
    g_ply_error = "too many vertices";
    return PHGPU_ERR_LIMIT;
  }
  return PHGPU_OK;
}

struct Sinks {
  float* xyzi;
  float* out[3];  // reflectivity, ambient, range
};

inline void emit(const Sinks& s, const int* col, const double* row, uint64_t i) {
  for (int c = 0; c < 4; ++c) s.xyzi[4 * i + c] = (float)row[col[c]];
  for (int f = 0; f < 3; ++f)
    if (s.out[f] && col[4 + f] >= 0) s.out[f][i] = (float)row[col[4 + f]];
}

// Skips one element instance of a binary body (lists read their counts).
bool skip_binary_row(std::istream& in, const Element& el, bool swap) {
  for (const Prop& pr : el.props) {
    unsigned char b[8];
    if (pr.is_list) {
      if (!in.read((char*)b, type_size(pr.count_type))) return false;
      const uint64_t cnt = (uint64_t)read_binary(b, pr.count_type, swap);
      in.seekg((std::streamoff)(cnt * type_size(pr.type)), std::ios::cur);
    } else {
      in.seekg(type_size(pr.type), std::ios::cur);
    }
  }
  return (bool)in;
}

int read_body(std::ifstream& in, const Layout& L, const Sinks& s) {
  const Header& h = L.h;
  const Element& ve = h.elements[L.vertex];
  const size_t np = ve.props.size();
  std::vector<double> row(np);
  if (h.format == 0) {
    for (int e = 0; e <= L.vertex; ++e) {
      const Element& el = h.elements[e];
      for (uint64_t i = 0; i < el.count; ++i) {
        for (size_t p = 0; p < el.props.size(); ++p) {
          const Prop& pr = el.props[p];
          double v = 0;
          if (!(in >> v)) {
            g_ply_error = "truncated ascii body";
            return PHGPU_ERR_INVALID;
          }
          if (pr.is_list)
            for (uint64_t k = 0; k < (uint64_t)v; ++k) {
              double skip;
              in >> skip;
            }
          else if (e == L.vertex)
            row[p] = v;
        }
        if (e == L.vertex) emit(s, L.col, row.data(), i);
      }
    }
    return PHGPU_OK;
  }
  const bool swap = (h.format == 2) == host_is_little();
  for (int e = 0; e < L.vertex; ++e)
    for (uint64_t i = 0; i < h.elements[e].count; ++i)
      if (!skip_binary_row(in, h.elements[e], swap)) {
        g_ply_error = "truncated binary body";
        return PHGPU_ERR_INVALID;
      }
  bool fixed = true;
  std::vector<int> offset(np);
  int stride = 0;
  for (size_t p = 0; p < np; ++p) {
    fixed = fixed && !ve.props[p].is_list;
    offset[p] = stride;
    stride += type_size(ve.props[p].type);
  }
  if (fixed) {
    // one read of the whole vertex block, then fixed-offset decoding: in host
    // byte order field by field with the type resolved once per chunk
    // (decode_column), otherwise value by value
    const uint64_t chunk_rows = 1u << 16;
    std::vector<unsigned char> buf(chunk_rows * stride);
    for (uint64_t i0 = 0; i0 < ve.count; i0 += chunk_rows) {
      const uint64_t rows = std::min<uint64_t>(chunk_rows, ve.count - i0);
      if (!in.read((char*)buf.data(), (std::streamsize)(rows * stride))) {
        g_ply_error = "truncated binary body";
        return PHGPU_ERR_INVALID;
      }
      if (!swap) {
        for (int f = 0; f < kFields; ++f) {
          const int p = L.col[f];
          if (p < 0 || (f >= 4 && !s.out[f - 4])) continue;
          float* dst = f < 4 ? s.xyzi + 4 * i0 + f : s.out[f - 4] + i0;
          decode_column(buf.data() + offset[p], rows, stride, ve.props[p].type, dst, f < 4 ? 4 : 1);
        }
        continue;
      }
      for (uint64_t r = 0; r < rows; ++r) {
        const unsigned char* b = buf.data() + r * stride;
        for (int f = 0; f < kFields; ++f)
          if (L.col[f] >= 0) row[L.col[f]] = read_binary(b + offset[L.col[f]], ve.props[L.col[f]].type, swap);
        emit(s, L.col, row.data(), i0 + r);
      }
    }
    return PHGPU_OK;
  }
  for (uint64_t i = 0; i < ve.count; ++i) {
    for (size_t p = 0; p < np; ++p) {
      const Prop& pr = ve.props[p];
      unsigned char b[8];
      if (pr.is_list) {
        if (!in.read((char*)b, type_size(pr.count_type))) break;
        const uint64_t cnt = (uint64_t)read_binary(b, pr.count_type, swap);
        in.seekg((std::streamoff)(cnt * type_size(pr.type)), std::ios::cur);
      } else if (in.read((char*)b, type_size(pr.type))) {
        row[p] = read_binary(b, pr.type, swap);
      }
    }
    if (!in) {
      g_ply_error = "truncated binary body";
      return PHGPU_ERR_INVALID;
    }
    emit(s, L.col, row.data(), i);
  }
  return PHGPU_OK;
}

}  // namespace

int phgpu_ply_info(const char* path, const char* const* field_names, uint32_t* n_points, uint32_t* present) {
  if (!path || !n_points) return PHGPU_ERR_INVALID;
  std::ifstream in;
  Layout L;
  const int rc = open_layout(path, field_names, &in, &L);
  if (rc != PHGPU_OK) return rc;
  *n_points = (uint32_t)L.h.elements[L.vertex].count;
  if (present)
    *present = (L.col[4] >= 0 ? PHGPU_PLY_REFLECTIVITY : 0u) | (L.col[5] >= 0 ? PHGPU_PLY_AMBIENT : 0u) |
               (L.col[6] >= 0 ? PHGPU_PLY_RANGE : 0u);
  return PHGPU_OK;
}

int phgpu_ply_read(const char* path, const char* const* field_names, float* xyzi, float* reflectivity,
                   float* ambient, float* range, uint32_t capacity, uint32_t* n_points) {
  if (!path || !xyzi || !n_points) return PHGPU_ERR_INVALID;
  std::ifstream in;
  Layout L;
  const int rc = open_layout(path, field_names, &in, &L);
  if (rc != PHGPU_OK) return rc;
  const uint64_t n = L.h.elements[L.vertex].count;
  if (n > capacity) {
    g_ply_error = "output capacity too small";
    return PHGPU_ERR_LIMIT;
  }
  *n_points = (uint32_t)n;
  return read_body(in, L, Sinks{xyzi, {reflectivity, ambient, range}});
}

const char* phgpu_ply_last_error(void) { return g_ply_error.c_str(); }
