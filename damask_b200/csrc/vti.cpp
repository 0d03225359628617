// Reader of the grid geometry files (VTK ImageData, .vti) that DAMASK_grid takes, behind a
// plain C-ABI: the native counterpart of the reference's C++ reader src/grid/VTI.cpp:45-445
// (C_VTI_new / C_VTI_readGeometry / C_VTI_readDatasetInt / C_VTI_readDatasetReal /
// C_VTI_delete, :417-445, which take Fortran descriptors; here pointers and sizes).
//
// Accepted: a VTKFile of type ImageData in little-endian byte order, optionally
// vtkZLibDataCompressor-compressed (header: number of blocks, block size, size of the last
// block, compressed block sizes), UInt32 or UInt64 header words; WholeExtent starting at 0
// giving the cells, Spacing x cells = size, Direction the identity; cell data arrays in binary
// (base64) format.  Errors mirror the reference's checks (VTI.cpp:45-330).
#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/damask_b200.h"

namespace dmk {
int record_error(int code, const std::string& msg);   // context.cu: the message of dmk_last_error
}

struct dmk_vti {
  int cells[3] = {0, 0, 0};
  double size[3] = {0, 0, 0}, origin[3] = {0, 0, 0};
  bool compressed = false;
  int word = 4;                                  // header word size: UInt32 or UInt64
  struct Array {
    std::string type, text;
    int components = 1;
  };
  std::map<std::string, Array> arrays;           // CellData arrays by Name
  std::vector<std::string> order;                // their order in the file
};

namespace {

using Attrs = std::map<std::string, std::string>;

// attributes of the start tag beginning at s[pos] == '<'; end: index after '>'
bool parse_tag(const std::string& s, size_t pos, std::string& name, Attrs& attrs, size_t& end, bool& self_closing) {
  size_t i = pos + 1;
  size_t j = i;
  while (j < s.size() && !isspace(static_cast<unsigned char>(s[j])) && s[j] != '>' && s[j] != '/') ++j;
  name = s.substr(i, j - i);
  attrs.clear();
  i = j;
  while (i < s.size()) {
    while (i < s.size() && isspace(static_cast<unsigned char>(s[i]))) ++i;
    if (i >= s.size()) return false;
    if (s[i] == '>') { self_closing = false; end = i + 1; return true; }
    if (s[i] == '/' && i + 1 < s.size() && s[i + 1] == '>') { self_closing = true; end = i + 2; return true; }
    size_t k = i;
    while (k < s.size() && s[k] != '=' && !isspace(static_cast<unsigned char>(s[k]))) ++k;
    const std::string key = s.substr(i, k - i);
    while (k < s.size() && s[k] != '"' && s[k] != '\'') ++k;
    if (k >= s.size()) return false;
    const char q = s[k];
    const size_t e = s.find(q, k + 1);
    if (e == std::string::npos) return false;
    attrs[key] = s.substr(k + 1, e - k - 1);
    i = e + 1;
  }
  return false;
}

// first start tag with the given name at or after pos
bool find_tag(const std::string& s, const std::string& tag, size_t from, size_t& at, Attrs& attrs, size_t& end,
              bool& self_closing) {
  for (size_t p = s.find('<', from); p != std::string::npos; p = s.find('<', p + 1)) {
    std::string name;
    if (s.compare(p + 1, tag.size(), tag) != 0) continue;
    if (!parse_tag(s, p, name, attrs, end, self_closing)) return false;
    if (name != tag) continue;
    at = p;
    return true;
  }
  return false;
}

std::vector<double> numbers(const std::string& text) {
  std::vector<double> v;
  std::istringstream in(text);
  double x;
  while (in >> x) v.push_back(x);
  return v;
}

int b64value(char c) {
  if (c >= 'A' && c <= 'Z') return c - 'A';
  if (c >= 'a' && c <= 'z') return c - 'a' + 26;
  if (c >= '0' && c <= '9') return c - '0' + 52;
  if (c == '+') return 62;
  if (c == '/') return 63;
  return -1;
}

// base64 text that may consist of several independently padded segments (header and payload
// are encoded separately and concatenated, padding included); whitespace is ignored
bool b64decode(const std::string& text, std::vector<uint8_t>& out) {
  out.clear();
  uint32_t acc = 0;
  int n = 0;
  for (char c : text) {
    if (isspace(static_cast<unsigned char>(c))) continue;
    if (c == '=') {                               // end of a segment: flush its partial group;
      if (n == 2) out.push_back(uint8_t(acc >> 4));          // a second '=' finds n == 0
      else if (n == 3) { out.push_back(uint8_t(acc >> 10)); out.push_back(uint8_t(acc >> 2)); }
      acc = 0;
      n = 0;
      continue;
    }
    const int v = b64value(c);
    if (v < 0) return false;
    acc = (acc << 6) | uint32_t(v);
    if (++n == 4) {
      out.push_back(uint8_t(acc >> 16));
      out.push_back(uint8_t(acc >> 8));
      out.push_back(uint8_t(acc));
      acc = 0;
      n = 0;
    }
  }
  if (n == 2) out.push_back(uint8_t(acc >> 4));
  else if (n == 3) { out.push_back(uint8_t(acc >> 10)); out.push_back(uint8_t(acc >> 2)); }
  return true;
}

uint64_t word_at(const std::vector<uint8_t>& b, size_t off, int word) {
  uint64_t v = 0;
  for (int k = word - 1; k >= 0; --k) v = (v << 8) | b[off + k];
  return v;
}

// raw bytes of a binary DataArray (VTI.cpp:200-330 for the block layout)
int decode(const dmk_vti& vti, const std::string& text, std::vector<uint8_t>& out, std::string& err) {
  std::vector<uint8_t> raw;
  if (!b64decode(text, raw)) { err = "invalid base64 data"; return -1; }
  const int w = vti.word;
  out.clear();
  if (vti.compressed) {
    if (raw.size() < size_t(3 * w)) { err = "header for compressed VTI too short"; return -1; }
    const uint64_t nblocks = word_at(raw, 0, w), bsize = word_at(raw, w, w), last = word_at(raw, 2 * w, w);
    const size_t hsize = size_t(3 + nblocks) * w;
    if (nblocks > raw.size() || raw.size() < hsize) { err = "missing header for compressed VTI"; return -1; }
    size_t off = hsize;
    for (uint64_t i = 0; i < nblocks; ++i) {
      const uint64_t cs = word_at(raw, size_t(3 + i) * w, w);
      if (off + cs > raw.size()) { err = "invalid VTI, defined size overflowing for block " + std::to_string(i); return -1; }
      const uint64_t want = (i + 1 == nblocks && last > 0) ? last : bsize;
      const size_t at = out.size();
      out.resize(at + want);
      uLongf dlen = uLongf(want);
      if (uncompress(out.data() + at, &dlen, raw.data() + off, uLong(cs)) != Z_OK || dlen != want) {
        err = "zlib inflate failed on block " + std::to_string(i);
        return -1;
      }
      off += cs;
    }
    return 0;
  }
  size_t off = 0;
  while (off + w <= raw.size()) {
    const uint64_t n = word_at(raw, off, w);
    off += w;
    if (n == 0) break;
    if (off + n > raw.size()) { err = "VTI uncompressed: data block exceeds payload"; return -1; }
    out.insert(out.end(), raw.begin() + long(off), raw.begin() + long(off + n));
    off += n;
  }
  return 0;
}

template <typename T>
int convert(const dmk_vti::Array& a, const std::vector<uint8_t>& b, T* out, int64_t n, std::string& err) {
  auto get = [&](int64_t i, auto tag) {
    using U = decltype(tag);
    U x;
    std::memcpy(&x, b.data() + size_t(i) * sizeof(U), sizeof(U));
    return static_cast<T>(x);
  };
  size_t es;
  const std::string& t = a.type;
  if (t == "Int8" || t == "UInt8") es = 1;
  else if (t == "Int16" || t == "UInt16") es = 2;
  else if (t == "Int32" || t == "UInt32" || t == "Float32") es = 4;
  else if (t == "Int64" || t == "UInt64" || t == "Float64") es = 8;
  else { err = "unknown VTK type '" + t + "'"; return -1; }
  if (b.size() != size_t(n) * es) {
    err = "DataArray has " + std::to_string(b.size() / es) + " values, " + std::to_string(n) + " expected";
    return -1;
  }
  for (int64_t i = 0; i < n; ++i) {
    if (t == "Int8") out[i] = get(i, int8_t());
    else if (t == "UInt8") out[i] = get(i, uint8_t());
    else if (t == "Int16") out[i] = get(i, int16_t());
    else if (t == "UInt16") out[i] = get(i, uint16_t());
    else if (t == "Int32") out[i] = get(i, int32_t());
    else if (t == "UInt32") out[i] = get(i, uint32_t());
    else if (t == "Int64") out[i] = get(i, int64_t());
    else if (t == "UInt64") out[i] = get(i, uint64_t());
    else if (t == "Float32") out[i] = get(i, float());
    else out[i] = get(i, double());
  }
  return 0;
}

int parse(const std::string& s, dmk_vti& vti, std::string& err) {
  size_t at, end;
  bool sc;
  Attrs a;
  if (!find_tag(s, "VTKFile", 0, at, a, end, sc)) { err = "missing <VTKFile> element"; return -1; }
  if (a["type"] != "ImageData") { err = "type is not ImageData (got '" + a["type"] + "')"; return -1; }
  if (a["byte_order"] != "LittleEndian") { err = "byte_order must be 'LittleEndian' (got '" + a["byte_order"] + "')"; return -1; }
  if (a.count("compressor")) {
    if (a["compressor"] != "vtkZLibDataCompressor") { err = "compressor is not vtkZLibDataCompressor (got '" + a["compressor"] + "')"; return -1; }
    vti.compressed = true;
  }
  vti.word = (a.count("header_type") && a["header_type"] == "UInt64") ? 8 : 4;
  if (!find_tag(s, "ImageData", end, at, a, end, sc)) { err = "missing ImageData element"; return -1; }
  if (a.count("Direction")) {
    const std::vector<double> d = numbers(a["Direction"]);
    const double id[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (d.size() != 9 || !std::equal(d.begin(), d.end(), id)) { err = "unsupported 'Direction' (got '" + a["Direction"] + "')"; return -1; }
  }
  const std::vector<double> ext = numbers(a["WholeExtent"]);
  if (ext.size() != 6 || ext[0] != 0 || ext[2] != 0 || ext[4] != 0) { err = "invalid 'WholeExtent' (got '" + a["WholeExtent"] + "')"; return -1; }
  const std::vector<double> sp = numbers(a["Spacing"]);
  if (sp.size() != 3) { err = "invalid 'Spacing'"; return -1; }
  const std::vector<double> org = a.count("Origin") ? numbers(a["Origin"]) : std::vector<double>{0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    vti.cells[i] = int(ext[2 * i + 1]);
    vti.size[i] = sp[i] * vti.cells[i];
    vti.origin[i] = org.size() == 3 ? org[i] : 0.0;
  }
  for (int i = 0; i < 3; ++i)
    if (!(vti.size[i] > 0.0)) { err = "one or more entries <= 0 for 'size'"; return -1; }
  for (int i = 0; i < 3; ++i)
    if (vti.cells[i] < 1) { err = "one or more entries < 1 for 'cells'"; return -1; }
  size_t cd_at, cd_end;
  if (!find_tag(s, "CellData", end, cd_at, a, cd_end, sc) || sc) return 0;
  const size_t cd_close = s.find("</CellData>", cd_end);
  size_t p = cd_end;
  while (find_tag(s, "DataArray", p, at, a, end, sc) && at < cd_close) {
    const std::string name = a["Name"];
    if (vti.arrays.count(name)) { err = "repeated label '" + name + "'"; return -1; }
    if (a["format"] != "binary") { err = "DataArray '" + name + "' is not binary"; return -1; }
    dmk_vti::Array arr;
    arr.type = a["type"];
    arr.components = a.count("NumberOfComponents") ? std::stoi(a["NumberOfComponents"]) : 1;
    if (!sc) {
      const size_t close = s.find("</DataArray>", end);
      if (close == std::string::npos) { err = "unterminated DataArray '" + name + "'"; return -1; }
      arr.text = s.substr(end, close - end);
      p = close + 12;
    } else {
      p = end;
    }
    vti.arrays[name] = arr;
    vti.order.push_back(name);
  }
  return 0;
}

int64_t cell_count(const dmk_vti* v) { return int64_t(v->cells[0]) * v->cells[1] * v->cells[2]; }

}  // namespace

extern "C" {

int dmk_vti_open(const char* path, dmk_vti** out) {
  if (!path || !out) return dmk::record_error(DMK_ERR_ARG, "null argument");
  *out = nullptr;
  std::ifstream in(path, std::ios::binary);
  if (!in) return dmk::record_error(DMK_ERR_ARG, std::string("cannot open ") + path);
  std::stringstream ss;
  ss << in.rdbuf();
  auto* v = new dmk_vti();
  std::string err;
  int rc;
  try {                                            // nothing is thrown across the C-ABI
    rc = parse(ss.str(), *v, err);
  } catch (const std::exception& e) {
    rc = -1;
    err = std::string("invalid VTI: ") + e.what();
  }
  if (rc) {
    delete v;
    return dmk::record_error(DMK_ERR_CONFIG, err);
  }
  *out = v;
  return 0;
}

int dmk_vti_geometry(const dmk_vti* v, int cells[3], double size[3], double origin[3]) {
  if (!v) return dmk::record_error(DMK_ERR_ARG, "null argument");
  for (int i = 0; i < 3; ++i) {
    if (cells) cells[i] = v->cells[i];
    if (size) size[i] = v->size[i];
    if (origin) origin[i] = v->origin[i];
  }
  return 0;
}

int dmk_vti_label(const dmk_vti* v, int index, char* out, int cap, int* components) {
  if (!v || !out || cap < 1) return dmk::record_error(DMK_ERR_ARG, "null argument");
  if (index < 0 || index >= int(v->order.size())) return int(v->order.size());
  const std::string& name = v->order[size_t(index)];
  std::strncpy(out, name.c_str(), size_t(cap) - 1);
  out[cap - 1] = '\0';
  if (components) *components = v->arrays.at(name).components;
  return int(v->order.size());
}

int dmk_vti_read_int(const dmk_vti* v, const char* label, int64_t* out, int64_t n) {
  if (!v || !label || !out) return dmk::record_error(DMK_ERR_ARG, "null argument");
  auto it = v->arrays.find(label);
  if (it == v->arrays.end()) return dmk::record_error(DMK_ERR_CONFIG, std::string("no DataArray with Name='") + label + "' found");
  if (n != cell_count(v) * it->second.components) return dmk::record_error(DMK_ERR_ARG, "output size does not match the cells");
  std::vector<uint8_t> b;
  std::string err;
  try {
    if (decode(*v, it->second.text, b, err) || convert<int64_t>(it->second, b, out, n, err))
      return dmk::record_error(DMK_ERR_CONFIG, err);
  } catch (const std::exception& e) {
    return dmk::record_error(DMK_ERR_CONFIG, std::string("invalid VTI data: ") + e.what());
  }
  return 0;
}

int dmk_vti_read_real(const dmk_vti* v, const char* label, double* out, int64_t n) {
  if (!v || !label || !out) return dmk::record_error(DMK_ERR_ARG, "null argument");
  auto it = v->arrays.find(label);
  if (it == v->arrays.end()) return dmk::record_error(DMK_ERR_CONFIG, std::string("no DataArray with Name='") + label + "' found");
  if (n != cell_count(v) * it->second.components) return dmk::record_error(DMK_ERR_ARG, "output size does not match the cells");
  std::vector<uint8_t> b;
  std::string err;
  try {
    if (decode(*v, it->second.text, b, err) || convert<double>(it->second, b, out, n, err))
      return dmk::record_error(DMK_ERR_CONFIG, err);
  } catch (const std::exception& e) {
    return dmk::record_error(DMK_ERR_CONFIG, std::string("invalid VTI data: ") + e.what());
  }
  return 0;
}

void dmk_vti_close(dmk_vti* v) { delete v; }

}  // extern "C"
