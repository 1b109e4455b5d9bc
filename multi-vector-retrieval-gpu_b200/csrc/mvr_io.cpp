// mvr_io.cpp -- see mvr_io.hpp.
#include "mvr_io.hpp"

#include <cstdio>
#include <cstring>
#include <memory>

namespace mvr {

namespace {
struct File {
  FILE *f = nullptr;
  explicit File(const std::string &p) { f = std::fopen(p.c_str(), "rb"); }
  ~File() { if (f) std::fclose(f); }
};

bool parse_header(const std::string &h, NpyArray &out, std::string &err) {
  auto find_val = [&](const char *key) -> std::string {
    const size_t k = h.find(key);
    if (k == std::string::npos) return "";
    size_t p = h.find(':', k);
    if (p == std::string::npos) return "";
    p++;
    while (p < h.size() && h[p] == ' ') p++;
    return h.substr(p);
  };
  std::string d = find_val("'descr'");
  if (d.size() < 3 || d[0] != '\'') { err = "npy: no descr"; return false; }
  out.descr = d.substr(1, d.find('\'', 1) - 1);
  std::string fo = find_val("'fortran_order'");
  if (fo.rfind("True", 0) == 0) { err = "npy: fortran order not supported"; return false; }
  std::string sh = find_val("'shape'");
  if (sh.empty() || sh[0] != '(') { err = "npy: no shape"; return false; }
  const size_t close = sh.find(')');
  std::string inner = sh.substr(1, close - 1);
  out.shape.clear();
  size_t p = 0;
  while (p < inner.size()) {
    while (p < inner.size() && (inner[p] == ' ' || inner[p] == ',')) p++;
    if (p >= inner.size()) break;
    size_t q = p;
    while (q < inner.size() && inner[q] >= '0' && inner[q] <= '9') q++;
    if (q == p) { err = "npy: bad shape"; return false; }
    out.shape.push_back(std::stoull(inner.substr(p, q - p)));
    p = q;
  }
  const char endian = out.descr[0];
  if (endian == '>') { err = "npy: big-endian data not supported"; return false; }
  out.word_size = std::stoul(out.descr.substr(2));
  return true;
}
}  // namespace

bool npy_load(const std::string &path, NpyArray &out, std::string &err) {
  File f(path);
  if (!f.f) { err = "cannot open " + path; return false; }
  unsigned char magic[8];
  if (std::fread(magic, 1, 8, f.f) != 8 || std::memcmp(magic, "\x93NUMPY", 6) != 0) {
    err = "not a .npy file: " + path;
    return false;
  }
  uint32_t hlen = 0;
  if (magic[6] == 1) {
    unsigned char b[2];
    if (std::fread(b, 1, 2, f.f) != 2) { err = "npy: truncated header " + path; return false; }
    hlen = b[0] | (b[1] << 8);
  } else {
    unsigned char b[4];
    if (std::fread(b, 1, 4, f.f) != 4) { err = "npy: truncated header " + path; return false; }
    hlen = b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24);
  }
  std::string h(hlen, '\0');
  if (std::fread(&h[0], 1, hlen, f.f) != hlen) { err = "npy: truncated header " + path; return false; }
  if (!parse_header(h, out, err)) { err += " in " + path; return false; }
  const uint64_t bytes = out.numel() * out.word_size;
  out.data.resize(bytes);
  if (bytes && std::fread(out.data.data(), 1, bytes, f.f) != bytes) {
    err = "npy: truncated payload " + path;
    return false;
  }
  return true;
}

bool ivf_load(const std::string &path, IvfCsr &out, std::string &err) {
  File f(path);
  if (!f.f) { err = "cannot open " + path; return false; }
  auto rd = [&](void *p, size_t n) { return std::fread(p, 1, n, f.f) == n; };
  if (!rd(&out.n_centroid, 4) || !rd(&out.n_ele, 8)) { err = "ivf: truncated header " + path; return false; }
  out.offset.resize(out.n_centroid);
  out.size.resize(out.n_centroid);
  out.ids.resize(out.n_ele);
  if (!rd(out.offset.data(), 8ull * out.n_centroid) || !rd(out.size.data(), 4ull * out.n_centroid) ||
      !rd(out.ids.data(), 4ull * out.n_ele)) {
    err = "ivf: truncated body " + path;
    return false;
  }
  for (uint32_t c = 0; c < out.n_centroid; c++)
    if (out.offset[c] + out.size[c] > out.n_ele) { err = "ivf: list out of range in " + path; return false; }
  return true;
}

}  // namespace mvr
