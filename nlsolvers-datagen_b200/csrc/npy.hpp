// Minimal .npy (format versions 1.0-3.0) reader/writer for '<f8' and '<c16'
// C-order arrays: the payloads the reference drivers exchange with the Python
// launchers (common/include/util.hpp:36-58 over the libnpy submodule, which
// is empty in the reference snapshot). Format per the NumPy NEP-1 / .npy spec.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace npy {

struct Array {
  std::string descr;            // "<f8" or "<c16"
  std::vector<uint64_t> shape;
  bool fortran = false;
  std::vector<unsigned char> data;
  uint64_t count() const {
    uint64_t n = 1;
    for (auto d : shape) n *= d;
    return n;
  }
};

inline std::string dict_value(const std::string &h, const std::string &key) {
  const std::string k = "'" + key + "'";
  size_t p = h.find(k);
  if (p == std::string::npos) throw std::runtime_error("npy header lacks " + key);
  p = h.find(':', p + k.size());
  if (p == std::string::npos) throw std::runtime_error("malformed npy header");
  ++p;
  while (p < h.size() && h[p] == ' ') ++p;
  if (h[p] == '\'') {
    size_t e = h.find('\'', p + 1);
    return h.substr(p + 1, e - p - 1);
  }
  if (h[p] == '(') {
    size_t e = h.find(')', p);
    return h.substr(p, e - p + 1);
  }
  size_t e = p;
  while (e < h.size() && h[e] != ',' && h[e] != '}') ++e;
  return h.substr(p, e - p);
}

inline Array load(const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open " + path);
  Array a;
  try {
    unsigned char magic[8];
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "\x93NUMPY", 6) != 0)
      throw std::runtime_error(path + ": not a .npy file");
    uint32_t hlen = 0;
    if (magic[6] == 1) {
      unsigned char b[2];
      if (std::fread(b, 1, 2, f) != 2) throw std::runtime_error(path + ": truncated header");
      hlen = b[0] | (b[1] << 8);
    } else {
      unsigned char b[4];
      if (std::fread(b, 1, 4, f) != 4) throw std::runtime_error(path + ": truncated header");
      hlen = b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24);
    }
    std::string h(hlen, ' ');
    if (std::fread(&h[0], 1, hlen, f) != hlen) throw std::runtime_error(path + ": truncated header");
    a.descr = dict_value(h, "descr");
    a.fortran = dict_value(h, "fortran_order").find("True") != std::string::npos;
    std::string sh = dict_value(h, "shape");
    for (size_t i = 0; i < sh.size();) {
      if (sh[i] >= '0' && sh[i] <= '9') {
        size_t e = i;
        while (e < sh.size() && sh[e] >= '0' && sh[e] <= '9') ++e;
        a.shape.push_back(std::stoull(sh.substr(i, e - i)));
        i = e;
      } else {
        ++i;
      }
    }
    size_t esz = 0;
    if (a.descr == "<f8" || a.descr == "f8" || a.descr == "=f8") {
      a.descr = "<f8";
      esz = 8;
    } else if (a.descr == "<c16" || a.descr == "c16" || a.descr == "=c16") {
      a.descr = "<c16";
      esz = 16;
    } else {
      throw std::runtime_error(path + ": unsupported dtype " + a.descr + " (need <f8 or <c16)");
    }
    const uint64_t bytes = a.count() * esz;
    a.data.resize(bytes);
    if (bytes && std::fread(a.data.data(), 1, bytes, f) != bytes)
      throw std::runtime_error(path + ": truncated data");
  } catch (...) {
    std::fclose(f);
    throw;
  }
  std::fclose(f);
  if (a.fortran && a.shape.size() > 1)
    throw std::runtime_error(path + ": Fortran-ordered arrays are not supported");
  return a;
}

inline void save(const std::string &path, const std::string &descr, const std::vector<uint64_t> &shape,
                 const void *data, uint64_t bytes) {
  std::string h = "{'descr': '" + descr + "', 'fortran_order': False, 'shape': (";
  for (size_t i = 0; i < shape.size(); ++i) {
    h += std::to_string(shape[i]);
    if (shape.size() == 1 || i + 1 < shape.size()) h += ",";
    if (i + 1 < shape.size()) h += " ";
  }
  h += "), }";
  // pad so that magic(6)+ver(2)+len(2)+header is a multiple of 64, ending in '\n'
  size_t total = 10 + h.size() + 1;
  size_t pad = (64 - total % 64) % 64;
  h.append(pad, ' ');
  h.push_back('\n');
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + path);
  const unsigned char pre[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
  const uint16_t hl = (uint16_t)h.size();
  const unsigned char lb[2] = {(unsigned char)(hl & 0xff), (unsigned char)(hl >> 8)};
  bool ok = std::fwrite(pre, 1, 8, f) == 8 && std::fwrite(lb, 1, 2, f) == 2 &&
            std::fwrite(h.data(), 1, h.size(), f) == h.size() &&
            (bytes == 0 || std::fwrite(data, 1, bytes, f) == bytes);
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) throw std::runtime_error("write failed: " + path);
}

}  // namespace npy
