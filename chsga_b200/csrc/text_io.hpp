// Whole-file reads and a whitespace token scanner over the bytes, shared by
// the text readers of the alignment inputs and of graph ingest.
#pragma once

#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "common.hpp"

namespace chsga {

inline std::vector<char> slurp(const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "rb");
  require(f != nullptr, CHSGA_ERR_IO, "cannot open " + path + ": " + std::strerror(errno));
  std::vector<char> buf;
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz > 0) {
    buf.resize((size_t)sz);
    size_t got = std::fread(buf.data(), 1, buf.size(), f);
    std::fclose(f);
    require(got == buf.size(), CHSGA_ERR_IO, "short read of " + path);
  } else {
    std::fclose(f);
  }
  return buf;
}

// Whitespace-separated token scanner over an in-memory file.
struct Tok {
  const char* p;
  const char* e;
  std::string path;
  explicit Tok(const std::vector<char>& b, std::string pth)
      : p(b.data()), e(b.data() + b.size()), path(std::move(pth)) {}
  void skip() {
    while (p < e && std::isspace((unsigned char)*p)) ++p;
  }
  bool more() {
    skip();
    return p < e;
  }
  bool word(std::string& out) {
    skip();
    if (p >= e) return false;
    const char* s = p;
    while (p < e && !std::isspace((unsigned char)*p)) ++p;
    out.assign(s, p);
    return true;
  }
  // (the error messages are built only when a check fails: this runs once
  // per number of files with hundreds of millions of them)
  uint64_t u64(const char* what) {
    skip();
    if (!(p < e && *p >= '0' && *p <= '9')) fail(CHSGA_ERR_FORMAT, path + ": expected " + what);
    uint64_t v = 0;
    while (p < e && *p >= '0' && *p <= '9') {
      uint64_t d = (uint64_t)(*p - '0');
      if (v > (UINT64_MAX - d) / 10) fail(CHSGA_ERR_FORMAT, path + ": integer overflow");
      v = v * 10 + d;
      ++p;
    }
    if (!(p >= e || std::isspace((unsigned char)*p))) fail(CHSGA_ERR_FORMAT, path + ": malformed " + what);
    return v;
  }
  double real(const char* what) {
    skip();
    if (p >= e) fail(CHSGA_ERR_FORMAT, path + ": expected " + what);
    const char* s = p;
    while (p < e && !std::isspace((unsigned char)*p)) ++p;
    std::string t(s, p);
    char* end = nullptr;
    double v = std::strtod(t.c_str(), &end);
    if (!(end && *end == '\0')) fail(CHSGA_ERR_FORMAT, path + ": malformed " + what + " '" + t + "'");
    return v;
  }
};


}  // namespace chsga
