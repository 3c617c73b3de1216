// cli_common.h -- helpers shared by the two command-line tools.
#pragma once

#include <cctype>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace cucm_cli {

// Size with an optional K/M/G suffix (parse_size, cucm_compress_v2.cu:1252-1286):
// leading blanks skipped, digits, optional blanks, first suffix letter only;
// anything unparsable is 0.
inline uint64_t parse_size(const std::string &s) {
  size_t i = 0;
  while (i < s.size() && std::isspace((unsigned char)s[i])) i++;
  size_t j = i;
  while (j < s.size() && std::isdigit((unsigned char)s[j])) j++;
  if (j == i) return 0;
  uint64_t v = std::stoull(s.substr(i, j - i));
  while (j < s.size() && std::isspace((unsigned char)s[j])) j++;
  if (j < s.size()) {
    switch (std::toupper((unsigned char)s[j])) {
      case 'K': v *= 1024ull; break;
      case 'M': v *= 1024ull * 1024ull; break;
      case 'G': v *= 1024ull * 1024ull * 1024ull; break;
      default: break;
    }
  }
  return v;
}

inline bool read_file(const char *path, std::vector<uint8_t> &buf) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  buf.resize(sz > 0 ? (size_t)sz : 0);
  bool ok = buf.empty() || std::fread(buf.data(), 1, buf.size(), f) == buf.size();
  std::fclose(f);
  return ok;
}

inline bool write_file(const char *path, const uint8_t *p, size_t n) {
  FILE *f = std::fopen(path, "wb");
  if (!f) return false;
  bool ok = n == 0 || std::fwrite(p, 1, n, f) == n;
  return std::fclose(f) == 0 && ok;
}

}  // namespace cucm_cli
