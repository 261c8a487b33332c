// Whole-file reads and a whitespace token scanner over the bytes, shared by
// the text readers of the alignment inputs and of graph ingest.
#pragma once

#include <omp.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unistd.h>
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
    // large files in slices on every thread (each slice its own pread)
    const int fd = fileno(f);
    const size_t n = buf.size();
    const int nt = n < (64u << 20) ? 1 : std::max(1, omp_get_max_threads());
    int short_read = 0;
#pragma omp parallel for num_threads(nt) schedule(static, 1) reduction(| : short_read)
    for (int t = 0; t < nt; ++t) {
      size_t a = n / nt * t, z = t + 1 == nt ? n : n / nt * (t + 1);
      while (a < z) {
        const ssize_t got = pread(fd, buf.data() + a, z - a, (off_t)a);
        if (got <= 0) {
          short_read = 1;
          break;
        }
        a += (size_t)got;
      }
    }
    std::fclose(f);
    require(!short_read, CHSGA_ERR_IO, "short read of " + path);
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


inline bool text_space(char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// Parses the first `count` whitespace-separated tokens of [b, e) with
// one(index, token begin, token end) -> bool, which stores token `index`,
// on every thread for large inputs (chunks cut at whitespace, tokens
// counted, then parsed in place). Returns false when there are fewer tokens
// or one() refuses one: the caller then scans sequentially, which reports
// the problem. *after is the end of the last parsed token.
template <typename F>
inline bool parse_tokens(const char* b, const char* e, uint64_t count, const char** after, F one) {
  *after = b;
  if (count == 0) return true;
  const size_t len = (size_t)(e - b);
  const int nt = len < (1u << 22) ? 1 : std::max(1, omp_get_max_threads());
  std::vector<const char*> cut(nt + 1);
  cut[0] = b;
  cut[nt] = e;
  for (int t = 1; t < nt; ++t) {
    const char* q = std::max(cut[t - 1], b + len / nt * t);
    while (q < e && !text_space(*q)) ++q;
    cut[t] = q;
  }
  std::vector<uint64_t> base(nt + 1, 0);
#pragma omp parallel for num_threads(nt) schedule(static, 1)
  for (int t = 0; t < nt; ++t) {
    uint64_t k = 0;
    bool in = false;
    for (const char* q = cut[t]; q < cut[t + 1]; ++q) {
      const bool sp = text_space(*q);
      k += (!sp && !in);
      in = !sp;
    }
    base[t + 1] = k;
  }
  for (int t = 0; t < nt; ++t) base[t + 1] += base[t];
  if (base[nt] < count) return false;
  int bad = 0;
  const char* last = b;
#pragma omp parallel for num_threads(nt) schedule(static, 1) reduction(| : bad)
  for (int t = 0; t < nt; ++t) {
    uint64_t k = base[t];
    const char* q = cut[t];
    const char* const z = cut[t + 1];
    while (k < count) {
      while (q < z && text_space(*q)) ++q;
      if (q >= z) break;
      const char* s0 = q;
      while (q < z && !text_space(*q)) ++q;
      if (!one(k, s0, q)) {
        bad = 1;
        break;
      }
      if (k == count - 1) last = q;
      ++k;
    }
  }
  if (bad) return false;
  *after = last;
  return true;
}

// A decimal integer of at most 19 digits.
inline bool token_u64(const char* s, const char* z, uint64_t& v) {
  if (z == s || z - s > 19) return false;
  v = 0;
  for (const char* q = s; q < z; ++q) {
    if (*q < '0' || *q > '9') return false;
    v = v * 10 + (uint64_t)(*q - '0');
  }
  return true;
}

// A number as strtod reads it ("1.0", the weight every writer emits, without
// a call).
inline bool token_real(const char* s, const char* z, double& v) {
  const size_t n = (size_t)(z - s);
  if (n == 3 && s[0] == '1' && s[1] == '.' && s[2] == '0') {
    v = 1.0;
    return true;
  }
  if (n == 0 || n > 63) return false;
  char tmp[64];
  std::memcpy(tmp, s, n);
  tmp[n] = '\0';
  char* end = nullptr;
  v = std::strtod(tmp, &end);
  return end == tmp + n;
}
// Decimal v followed by sep, appended to b.
inline void put_decimal(uint64_t v, char sep, std::vector<char>& b) {
  char tmp[24];
  int k = 0;
  do {
    tmp[k++] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  while (k) b.push_back(tmp[--k]);
  b.push_back(sep);
}

// Writes items [0, n) to f, item i formatted by put(i, buffer), on every
// thread in slices written in order. False on a short write.
template <typename F>
inline bool write_items(FILE* f, size_t n, size_t bytes_each, F put) {
  const int nt = n < (1u << 16) ? 1 : std::max(1, omp_get_max_threads());
  const size_t per = (n + (size_t)nt * 8 - 1) / ((size_t)nt * 8) + 1;  // slices of at most this many
  bool ok = true;
  // rounds of nt slices, so the buffers stay a few MB per thread
  for (size_t r0 = 0; r0 < n && ok; r0 += per * nt) {
    std::vector<std::vector<char>> part(nt);
#pragma omp parallel for num_threads(nt) schedule(static, 1)
    for (int t = 0; t < nt; ++t) {
      const size_t a = std::min(n, r0 + per * t), z = std::min(n, a + per);
      part[t].reserve((z - a) * bytes_each);
      for (size_t i = a; i < z; ++i) put(i, part[t]);
    }
    for (auto& b : part)
      if (!b.empty() && std::fwrite(b.data(), 1, b.size(), f) != b.size()) ok = false;
  }
  return ok;
}

}  // namespace chsga
