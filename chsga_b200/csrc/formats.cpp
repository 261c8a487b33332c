// File readers and writers for the alignment inputs. See host_graph.hpp for
// the layouts and the reference files each one follows.
#include <zlib.h>

#include <algorithm>
#include <array>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>

#include "host_graph.hpp"
#include "text_io.hpp"

namespace chsga {


HostCsr read_adj(const std::string& path) {
  std::vector<char> buf = slurp(path);
  Tok t(buf, path);
  std::string head;
  require(t.word(head), CHSGA_ERR_FORMAT, path + ": empty file");
  require(head == "AdjacencyGraph" || head == "WeightedAdjacencyGraph", CHSGA_ERR_FORMAT,
          path + ": unknown header '" + head + "'");
  HostCsr g;
  g.n = t.u64("vertex count");
  g.m = t.u64("edge count");
  require(g.n < (1ull << 32) && g.m < (1ull << 40), CHSGA_ERR_UNSUPPORTED,
          path + ": graph too large for 32-bit vertex ids");
  g.offset.resize(g.n + 1);
  g.target.resize(g.m);
  // the n offsets and m targets in one parallel pass; a malformed, missing
  // or out-of-range number sends the block to the sequential scanner, which
  // reports it
  const uint64_t n = g.n;
  const char* after = nullptr;
  const bool fast = parse_tokens(t.p, t.e, g.n + g.m, &after, [&](uint64_t k, const char* s, const char* z) {
    uint64_t v;
    if (!token_u64(s, z, v)) return false;
    if (k < n) {
      g.offset[k] = v;
      return true;
    }
    if (v >= n) return false;
    g.target[k - n] = (uint32_t)v;
    return true;
  });
  if (fast) {
    t.p = after;
  } else {
    for (uint64_t i = 0; i < g.n; ++i) g.offset[i] = t.u64("offset");
  }
  g.offset[g.n] = g.m;
  for (uint64_t i = 0; i < g.n; ++i)
    if (g.offset[i] > g.offset[i + 1])
      fail(CHSGA_ERR_FORMAT, path + ": offsets not non-decreasing at " + std::to_string(i));
  if (!fast)
    for (uint64_t i = 0; i < g.m; ++i) {
      uint64_t v = t.u64("edge target");
      if (v >= g.n) fail(CHSGA_ERR_FORMAT, path + ": edge target out of range");
      g.target[i] = (uint32_t)v;
    }
  if (t.more()) {
    // weights as csr_to_adj writes them ("1.0"); the DP multiplies them by
    // the integer insertion cost, so they must be non-negative integers.
    g.weight.resize(g.m);
    uint64_t not_one = 0;
    const bool wfast = parse_tokens(t.p, t.e, g.m, &after, [&](uint64_t k, const char* s, const char* z) {
      double w;
      if (!token_real(s, z, w) || !(w >= 0 && w == std::floor(w) && w < 4294967296.0)) return false;
      g.weight[k] = (uint32_t)w;
      return true;
    });
    if (!wfast) {
      for (uint64_t i = 0; i < g.m; ++i) {
        double w = t.real("edge weight");
        if (!(w >= 0 && w == std::floor(w) && w < 4294967296.0))
          fail(CHSGA_ERR_UNSUPPORTED, path + ": edge weights must be non-negative integers");
        g.weight[i] = (uint32_t)w;
      }
    }
#pragma omp parallel for reduction(+ : not_one) schedule(static)
    for (int64_t i = 0; i < (int64_t)g.m; ++i) not_one += g.weight[i] != 1;
    if (!not_one) g.weight.clear();
  } else {
    require(head == "AdjacencyGraph", CHSGA_ERR_FORMAT, path + ": missing weights");
  }
  return g;
}

void write_adj(const std::string& path, const HostCsr& g) {
  FILE* f = std::fopen(path.c_str(), "wb");
  require(f != nullptr, CHSGA_ERR_IO, "cannot write " + path);
  // "AdjacencyGraph", n, m, the offsets, the targets and a weight per edge
  // ("1.0" for unit weights), one per line, as csr_to_adj writes them
  std::vector<char> head;
  const char* h = "AdjacencyGraph\n";
  head.insert(head.end(), h, h + std::strlen(h));
  put_decimal(g.n, '\n', head);
  put_decimal(g.m, '\n', head);
  bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
  ok = ok && write_items(f, g.n, 10, [&](size_t i, std::vector<char>& b) { put_decimal(g.offset[i], '\n', b); });
  ok = ok && write_items(f, g.m, 10, [&](size_t i, std::vector<char>& b) { put_decimal(g.target[i], '\n', b); });
  ok = ok && write_items(f, g.m, 4, [&](size_t i, std::vector<char>& b) {
    if (g.weight.empty()) {
      b.insert(b.end(), {'1', '.', '0', '\n'});
    } else {
      put_decimal(g.weight[i], '.', b);
      b.push_back('0');
      b.push_back('\n');
    }
  });
  ok = (std::fclose(f) == 0) && ok;
  require(ok, CHSGA_ERR_IO, "write failed: " + path);
}

std::vector<char> read_labels(const std::string& path) {
  std::vector<char> buf = slurp(path);
  buf.erase(std::remove(buf.begin(), buf.end(), '\n'), buf.end());
  return buf;
}

void write_labels(const std::string& path, const std::vector<char>& labels) {
  FILE* f = std::fopen(path.c_str(), "wb");
  require(f != nullptr, CHSGA_ERR_IO, "cannot write " + path);
  if (!labels.empty()) std::fwrite(labels.data(), 1, labels.size(), f);
  require(std::fclose(f) == 0, CHSGA_ERR_IO, "write failed: " + path);
}

std::vector<uint64_t> read_label_offsets(const std::string& path) {
  std::vector<char> buf = slurp(path);
  Tok t(buf, path);
  std::vector<uint64_t> offs;
  // `ifs >> off` stops at the first token that is not an integer.
  while (t.more() && *t.p >= '0' && *t.p <= '9') offs.push_back(t.u64("label offset"));
  return offs;
}

void write_label_offsets(const std::string& path, const std::vector<uint64_t>& offs) {
  std::ofstream o(path);
  require(bool(o), CHSGA_ERR_IO, "cannot write " + path);
  // csr_to_adj.cpp:57-63 writes "o0 o1 ... " then the total and a newline.
  for (size_t i = 0; i + 1 < offs.size(); ++i) o << offs[i] << ' ';
  if (!offs.empty()) o << offs.back() << '\n';
  require(bool(o), CHSGA_ERR_IO, "write failed: " + path);
}

// Hierarchy file layout (little-endian, native on x86-64):
//   char[8] "CHSGAPCH", u32 version = 1, u32 flags = 0,
//   u64 n, m, rm, num_layers, num_cc,
//   u32 rank[n], u32 level[n], u32 layer_offset[num_layers+1],
//   u32 cc_offset[num_cc+1],
//   u64 up_offset[n+1], u32 up_v[m], u32 up_w[m],
//   u64 down_offset[n+1], u32 down_v[rm], u32 down_w[rm],
//   u64 FNV-1a of every preceding byte.
namespace {
constexpr char kPchMagic[8] = {'C', 'H', 'S', 'G', 'A', 'P', 'C', 'H'};
uint64_t fnv1a(const char* p, size_t n, uint64_t h = 1469598103934665603ull) {
  for (size_t i = 0; i < n; ++i) {
    h ^= (unsigned char)p[i];
    h *= 1099511628211ull;
  }
  return h;
}
}  // namespace

void write_pch(const std::string& path, const HostPch& p) {
  require(p.present, CHSGA_ERR_INVALID_ARG, "no hierarchy to write");
  std::vector<char> out;
  auto app = [&](const void* d, size_t n) {
    out.insert(out.end(), (const char*)d, (const char*)d + n);
  };
  auto app_vec = [&](const auto& v) { app(v.data(), v.size() * sizeof(v[0])); };
  app(kPchMagic, 8);
  uint32_t ver = 1, flags = 0;
  app(&ver, 4);
  app(&flags, 4);
  uint64_t hdr[5] = {p.n, p.m, p.rm, (uint64_t)p.layer_offset.size() - 1,
                     (uint64_t)p.cc_offset.size() - 1};
  app(hdr, sizeof(hdr));
  app_vec(p.rank);
  app_vec(p.level);
  app_vec(p.layer_offset);
  app_vec(p.cc_offset);
  app_vec(p.up_offset);
  app_vec(p.up_v);
  app_vec(p.up_w);
  app_vec(p.down_offset);
  app_vec(p.down_v);
  app_vec(p.down_w);
  uint64_t h = fnv1a(out.data(), out.size());
  app(&h, 8);
  FILE* f = std::fopen(path.c_str(), "wb");
  require(f != nullptr, CHSGA_ERR_IO, "cannot write " + path);
  size_t put = std::fwrite(out.data(), 1, out.size(), f);
  bool ok = (std::fclose(f) == 0) && put == out.size();
  require(ok, CHSGA_ERR_IO, "write failed: " + path);
}

void validate_pch(const HostPch& p, uint64_t S) {
  auto bad = [&](const std::string& m) { fail(CHSGA_ERR_FORMAT, "hierarchy: " + m); };
  if (p.n != S) bad("vertex count " + std::to_string(p.n) + " != string graph " + std::to_string(S));
  if (p.rank.size() != p.n || p.level.size() != p.n) bad("rank/level size");
  if (p.up_offset.size() != p.n + 1 || p.down_offset.size() != p.n + 1) bad("offset size");
  if (p.up_v.size() != p.m || p.up_w.size() != p.m) bad("up edge size");
  if (p.down_v.size() != p.rm || p.down_w.size() != p.rm) bad("down edge size");
  std::vector<uint8_t> seen(p.n, 0);
  for (uint64_t i = 0; i < p.n; ++i) {
    if (p.rank[i] >= p.n || seen[p.rank[i]]) bad("rank is not a permutation");
    seen[p.rank[i]] = 1;
  }
  if (p.layer_offset.empty() || p.layer_offset.front() != 0 || p.layer_offset.back() != p.n)
    bad("layer offsets must run from 0 to n");
  for (size_t i = 0; i + 1 < p.layer_offset.size(); ++i)
    if (p.layer_offset[i] > p.layer_offset[i + 1]) bad("layer offsets decrease");
  const uint64_t L = p.layer_offset.size() - 1;
  if (p.cc_offset.empty() || p.cc_offset.front() != 0 || p.cc_offset.back() != L)
    bad("cc offsets must run from 0 to the layer count");
  for (size_t i = 0; i + 1 < p.cc_offset.size(); ++i)
    if (p.cc_offset[i] > p.cc_offset[i + 1]) bad("cc offsets decrease");
  auto chk_csr = [&](const std::vector<uint64_t>& off, const std::vector<uint32_t>& v, uint64_t m,
                     const char* what) {
    if (off[0] != 0 || off[p.n] != m) bad(std::string(what) + " offsets do not span the edges");
    for (uint64_t i = 0; i < p.n; ++i)
      if (off[i] > off[i + 1]) bad(std::string(what) + " offsets decrease");
    for (uint64_t e = 0; e < m; ++e)
      if (v[e] >= p.n) bad(std::string(what) + " edge endpoint out of range");
  };
  chk_csr(p.up_offset, p.up_v, p.m, "up");
  chk_csr(p.down_offset, p.down_v, p.rm, "down");
}

HostPch read_pch(const std::string& path) {
  std::vector<char> buf = slurp(path);
  size_t pos = 0;
  auto take = [&](void* d, size_t n) {
    require(pos + n <= buf.size(), CHSGA_ERR_FORMAT, path + ": truncated hierarchy file");
    std::memcpy(d, buf.data() + pos, n);
    pos += n;
  };
  char magic[8];
  take(magic, 8);
  require(std::memcmp(magic, kPchMagic, 8) == 0, CHSGA_ERR_FORMAT,
          path + ": not a CHSGAPCH hierarchy file");
  uint32_t ver = 0, flags = 0;
  take(&ver, 4);
  take(&flags, 4);
  require(ver == 1, CHSGA_ERR_FORMAT, path + ": unsupported hierarchy version");
  uint64_t hdr[5];
  take(hdr, sizeof(hdr));
  HostPch p;
  p.present = true;
  p.n = hdr[0];
  p.m = hdr[1];
  p.rm = hdr[2];
  const uint64_t L = hdr[3], C = hdr[4];
  const uint64_t need = p.n * 8 + (L + 1) * 4 + (C + 1) * 4 + (p.n + 1) * 16 + p.m * 8 + p.rm * 8 + 8;
  require(p.n < (1ull << 32) && L <= p.n + 1 && C <= L + 1 && need <= buf.size(),
          CHSGA_ERR_FORMAT, path + ": hierarchy header inconsistent with file size");
  auto take_vec = [&](auto& v, uint64_t n) {
    v.resize(n);
    take(v.data(), n * sizeof(v[0]));
  };
  take_vec(p.rank, p.n);
  take_vec(p.level, p.n);
  take_vec(p.layer_offset, L + 1);
  take_vec(p.cc_offset, C + 1);
  take_vec(p.up_offset, p.n + 1);
  take_vec(p.up_v, p.m);
  take_vec(p.up_w, p.m);
  take_vec(p.down_offset, p.n + 1);
  take_vec(p.down_v, p.rm);
  take_vec(p.down_w, p.rm);
  uint64_t h = fnv1a(buf.data(), pos), stored = 0;
  take(&stored, 8);
  require(h == stored, CHSGA_ERR_FORMAT, path + ": hierarchy checksum mismatch");
  return p;
}

// FASTA/FASTQ reader with kseq's record rules (the reader behind
// src/load_reads.hpp:7-40): a record starts at '>' or '@'; sequence lines
// run until a line starting with '>', '+' or '@'; a FASTQ quality block ends
// once it is as long as the sequence; a malformed record ends the input.
// Bases are upper-cased and at most max_reads records are kept (0 = all).
HostReads read_reads(const std::string& path, uint64_t max_reads) {
  gzFile fp = gzopen(path.c_str(), "r");
  require(fp != nullptr, CHSGA_ERR_IO, "Cannot open reads file: " + path);
  std::vector<char> buf;
  // zlib sizes its buffers when gzdirect first looks at the input, so the
  // 1 MB decompression buffer is requested before that (a later gzbuffer
  // call is refused)
  if (gzbuffer(fp, 1 << 20) != 0) {
    gzclose(fp);
    require(false, CHSGA_ERR_IO, "Cannot set the read buffer for: " + path);
  }
  if (gzdirect(fp) == 0 || gzeof(fp)) {
    // gzip input (or an empty file): decompress in 1 MB pieces
    size_t used = 0;
    buf.resize(1 << 20);
    int got;
    while ((got = gzread(fp, buf.data() + used, (unsigned)(buf.size() - used))) > 0) {
      used += (size_t)got;
      if (used == buf.size()) buf.resize(buf.size() * 2);
    }
    buf.resize(used);
    gzclose(fp);
  } else {
    // plain text, which gzread would pass through unchanged
    gzclose(fp);
    buf = slurp(path);
  }
  // std::toupper in a program that sets no locale (the reference's): a..z
  // only, whatever locale the host process runs in
  static const auto upper = [] {
    std::array<char, 256> t{};
    for (int c = 0; c < 256; ++c) t[c] = (char)(c >= 'a' && c <= 'z' ? c - 'a' + 'A' : c);
    return t;
  }();
  HostReads r;
  if (max_reads == 0) r.data.reserve(buf.size());
  size_t i = 0, n = buf.size();
  auto line_end = [&](size_t s) {
    if (s >= n) return n;
    const void* q = std::memchr(buf.data() + s, '\n', n - s);
    return q ? (size_t)(static_cast<const char*>(q) - buf.data()) : n;
  };
  auto strip_cr = [&](size_t s, size_t e) { return (e > s && buf[e - 1] == '\r') ? e - 1 : e; };
  int last_char = 0;  // header char already consumed
  while (true) {
    if (last_char == 0) {
      while (i < n && buf[i] != '>' && buf[i] != '@') ++i;
      if (i >= n) break;
      ++i;
    }
    // header line (name + comment)
    i = line_end(i);
    if (i < n) ++i;
    // the sequence lines, appended to the reads' bytes
    const size_t start = r.data.size();
    int c = -1;
    while (i < n) {
      c = (unsigned char)buf[i++];
      if (c == '>' || c == '+' || c == '@') break;
      if (c == '\n') {
        c = -1;
        continue;
      }
      size_t s0 = i - 1, e = line_end(i);
      r.data.insert(r.data.end(), buf.data() + s0, buf.data() + strip_cr(s0, e));
      i = (e < n) ? e + 1 : e;
      c = -1;
    }
    const size_t slen = r.data.size() - start;
    if (c == '>' || c == '@') {
      last_char = c;
    } else {
      last_char = 0;
    }
    if (c == '+') {
      i = line_end(i);
      if (i >= n) {  // no quality string: kseq reports an error
        r.data.resize(start);
        break;
      }
      ++i;
      size_t ql = 0;
      while (i < n && ql < slen) {
        size_t e = line_end(i);
        ql += strip_cr(i, e) - i;
        i = (e < n) ? e + 1 : e;
      }
      if (ql != slen) {  // quality length mismatch ends the input
        r.data.resize(start);
        break;
      }
      last_char = 0;
    }
    for (size_t k = start; k < r.data.size(); ++k) r.data[k] = upper[(unsigned char)r.data[k]];
    r.offsets.push_back(r.data.size());
    if (max_reads != 0 && r.count() >= max_reads) break;
    if (c != '>' && c != '@' && c != '+' && i >= n) break;
  }
  require(r.count() > 0, CHSGA_ERR_IO, "No reads loaded from: " + path);
  return r;
}

void write_fasta(const std::string& path, const HostReads& r) {
  FILE* f = std::fopen(path.c_str(), "wb");
  require(f != nullptr, CHSGA_ERR_IO, "cannot write " + path);
  for (uint64_t i = 0; i < r.count(); ++i) {
    std::fprintf(f, ">read_%llu\n", (unsigned long long)i);
    std::fwrite(r.seq(i), 1, r.len(i), f);
    std::fputc('\n', f);
  }
  require(std::fclose(f) == 0, CHSGA_ERR_IO, "write failed: " + path);
}

std::string ckpt_row_path(const std::string& dir, int64_t row) {
  return dir + "/row_" + std::to_string(row) + ".bin";
}

void write_ckpt_row(const std::string& dir, int64_t row, const int32_t* data, uint64_t n) {
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);
  std::string p = ckpt_row_path(dir, row);
  std::ofstream ofs(p, std::ios::binary | std::ios::trunc);
  require(bool(ofs), CHSGA_ERR_IO, "checkpoint write failed: " + p);
  ofs.write(reinterpret_cast<const char*>(data), (std::streamsize)(n * sizeof(int32_t)));
  require(bool(ofs), CHSGA_ERR_IO, "checkpoint write incomplete: " + p);
}

void read_ckpt_row(const std::string& dir, int64_t row, int32_t* data, uint64_t n) {
  std::string p = ckpt_row_path(dir, row);
  std::ifstream ifs(p, std::ios::binary);
  require(bool(ifs), CHSGA_ERR_IO, "checkpoint read failed: " + p);
  ifs.read(reinterpret_cast<char*>(data), (std::streamsize)(n * sizeof(int32_t)));
  require(bool(ifs), CHSGA_ERR_IO, "checkpoint read incomplete: " + p);
}

}  // namespace chsga
