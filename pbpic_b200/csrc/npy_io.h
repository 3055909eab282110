// Host-side reading and writing of NumPy .npy files (format version 1.0,
// little-endian, C order) for the dump/restart files of the B200 step, and a
// flat JSON object of numbers for the run parameters beside them. Only what
// the dump needs: dtypes <f4, <f8, <i4; shapes of rank 1 and 2.
#pragma once
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <map>
#include <string>
#include <vector>

namespace npyio {

// Write `bytes` of data with dtype `descr` and shape `shape`; false on I/O error.
inline bool write(const std::string& path, const char* descr, const std::vector<int64_t>& shape, const void* data,
                  size_t bytes) {
  std::string dict = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (";
  for (size_t i = 0; i < shape.size(); ++i) dict += std::to_string(shape[i]) + (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
  dict += "), }";
  // magic (6) + version (2) + header length (2) + dict + padding + '\n' is a multiple of 64
  size_t total = 10 + dict.size() + 1;
  const size_t pad = (64 - total % 64) % 64;
  dict.append(pad, ' ');
  dict += '\n';
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
  const uint16_t hl = (uint16_t)dict.size();
  bool ok = fwrite(magic, 1, 8, f) == 8 && fwrite(&hl, 2, 1, f) == 1 &&
            fwrite(dict.data(), 1, dict.size(), f) == dict.size() && (bytes == 0 || fwrite(data, 1, bytes, f) == bytes);
  ok = (fclose(f) == 0) && ok;
  return ok;
}

struct Array {
  std::string descr;
  std::vector<int64_t> shape;
  std::vector<unsigned char> data;
  int64_t count() const {
    int64_t n = 1;
    for (int64_t s : shape) n *= s;
    return n;
  }
};

// Read a file written by write(); returns an error message or "" on success.
inline std::string read(const std::string& path, Array* out) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return "cannot open " + path;
  unsigned char magic[8];
  uint16_t hl = 0;
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "\x93NUMPY", 6) != 0 || magic[6] != 1 || fread(&hl, 2, 1, f) != 1) {
    fclose(f);
    return path + ": not an .npy file of version 1";
  }
  std::string dict(hl, '\0');
  if (fread(&dict[0], 1, hl, f) != hl) {
    fclose(f);
    return path + ": truncated header";
  }
  auto field = [&](const char* key) -> std::string {
    const size_t k = dict.find(key);
    if (k == std::string::npos) return "";
    return dict.substr(k + strlen(key));
  };
  std::string d = field("'descr': '");
  out->descr = d.substr(0, d.find('\''));
  if (field("'fortran_order': ").rfind("False", 0) != 0) {
    fclose(f);
    return path + ": Fortran order is not supported";
  }
  std::string sh = field("'shape': (");
  sh = sh.substr(0, sh.find(')'));
  out->shape.clear();
  size_t pos = 0;
  while (pos < sh.size()) {
    while (pos < sh.size() && (sh[pos] == ' ' || sh[pos] == ',')) ++pos;
    if (pos >= sh.size()) break;
    out->shape.push_back(strtoll(sh.c_str() + pos, nullptr, 10));
    while (pos < sh.size() && sh[pos] != ',') ++pos;
  }
  const int64_t esize = (out->descr == "<f8") ? 8 : (out->descr == "<f4" || out->descr == "<i4") ? 4 : 0;
  if (esize == 0) {
    fclose(f);
    return path + ": unsupported dtype " + out->descr;
  }
  const size_t bytes = (size_t)(out->count() * esize);
  out->data.resize(bytes);
  const bool ok = bytes == 0 || fread(out->data.data(), 1, bytes, f) == bytes;
  fclose(f);
  return ok ? "" : path + ": truncated data";
}

// Values of a JSON object written by write_numbers (numbers only, no nesting).
inline bool write_numbers(const std::string& path, const std::vector<std::pair<std::string, double>>& kv) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return false;
  fprintf(f, "{\n");
  for (size_t i = 0; i < kv.size(); ++i)
    fprintf(f, "  \"%s\": %.17g%s\n", kv[i].first.c_str(), kv[i].second, i + 1 < kv.size() ? "," : "");
  fprintf(f, "}\n");
  return fclose(f) == 0;
}

inline bool read_numbers(const std::string& path, std::map<std::string, double>* out) {
  FILE* f = fopen(path.c_str(), "r");
  if (!f) return false;
  std::string s;
  char buf[4096];
  size_t m;
  while ((m = fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, m);
  fclose(f);
  size_t pos = 0;
  while ((pos = s.find('"', pos)) != std::string::npos) {
    const size_t e = s.find('"', pos + 1);
    if (e == std::string::npos) return false;
    const std::string key = s.substr(pos + 1, e - pos - 1);
    const size_t colon = s.find(':', e);
    if (colon == std::string::npos) return false;
    (*out)[key] = strtod(s.c_str() + colon + 1, nullptr);
    pos = s.find_first_of(",}", colon);
    if (pos == std::string::npos) break;
  }
  return true;
}

}  // namespace npyio
