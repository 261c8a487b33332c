// Graph ingest: the reference's pipeline handlegraph_to_csr ->
// csr_to_adj (src/handlegraph_to_csr.cpp, src/csr_to_adj.cpp) in this
// library, so a variation graph becomes the five ConSGA input files.
//
// handlegraph_to_csr reads a vg PackedGraph through libbdsg, which is not
// available here; the same bidirected graph is read from GFA v1 text
// instead (S lines: numeric node id and sequence; L lines: from, from
// orientation, to, to orientation, overlap 0M or *; other lines ignored).
// What follows restates handlegraph_to_csr.cpp:44-127 and 164-247:
//  * nodes sorted by id; node i becomes string vertex 2i (forward) and
//    2i + 1 (reverse complement), "forward then flipped";
//  * the out-edges of an oriented handle are the handles its right side
//    links to: a link a(fa) -> b(fb) gives 2a+fa -> 2b+fb and its reverse
//    complement 2b+!fb -> 2a+!fa, each edge once, adjacency sorted;
//  * sequences as a PackedGraph stores them: upper-cased, any byte other
//    than A, C, G, T becomes N; the reverse complement maps A<->T, C<->G,
//    N->N;
//  * the char graph is build(): chars of a string chained, the last char of
//    string i linked to the first char of every out-neighbour of i.
// The CSR text files are handlegraph_to_csr's write_csr layout (n, m, the
// labels space-separated, n+1 offsets, m targets), which csr_to_adj turns
// into an AdjacencyGraph file, the concatenated labels and the label
// offsets (csr_to_adj.cpp:39-118).
#include <omp.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <parallel/algorithm>
#include <string>
#include <unordered_map>
#include <vector>

#include "host_graph.hpp"
#include "text_io.hpp"

namespace chsga {
extern thread_local std::string g_last_error;

namespace {

// A string-labeled CSR as handlegraph_to_csr's CSR_container holds it, the
// labels concatenated: label i is lab[lab_off[i] .. lab_off[i + 1]).
struct CsrText {
  std::string lab;
  std::vector<uint64_t> lab_off{0};
  std::vector<uint64_t> offsets{0};
  std::vector<uint64_t> adj;
  uint64_t n() const { return lab_off.size() - 1; }
  uint64_t len(uint64_t i) const { return lab_off[i + 1] - lab_off[i]; }
};

char packed_base(char c) {
  switch (c) {
    case 'A': case 'a': return 'A';
    case 'C': case 'c': return 'C';
    case 'G': case 'g': return 'G';
    case 'T': case 't': return 'T';
    default: return 'N';
  }
}

char complement(char c) {
  switch (c) {
    case 'A': return 'T';
    case 'C': return 'G';
    case 'G': return 'C';
    case 'T': return 'A';
    default: return 'N';
  }
}

// One tab-separated field of a GFA line, in the file's bytes.
struct Field {
  const char* p = nullptr;
  size_t n = 0;
  bool is(const char* s) const { return n == std::strlen(s) && std::memcmp(p, s, n) == 0; }
  std::string str() const { return std::string(p, n); }
};

// The first `maxf` fields of the line [b, e) (the last one ends at the next
// tab too); returns how many there are, up to maxf.
size_t split_tabs(const char* b, const char* e, Field* f, size_t maxf) {
  size_t k = 0;
  const char* a = b;
  while (k < maxf) {
    const char* t = static_cast<const char*>(std::memchr(a, '\t', (size_t)(e - a)));
    const char* end = t ? t : e;
    f[k++] = Field{a, (size_t)(end - a)};
    if (!t) break;
    a = t + 1;
  }
  return k;
}

uint64_t parse_id(const Field& s, const std::string& path, uint64_t line) {
  bool ok = s.n > 0 && s.n < 20;
  uint64_t v = 0;
  for (size_t i = 0; ok && i < s.n; ++i) {
    ok = s.p[i] >= '0' && s.p[i] <= '9';
    v = v * 10 + (uint64_t)(s.p[i] - '0');
  }
  if (!ok)
    fail(CHSGA_ERR_FORMAT,
         path + ":" + std::to_string(line) + ": segment names must be numeric node ids, got '" + s.str() + "'");
  return v;
}

CsrText gfa_to_string_csr(const std::string& path) {
  const std::vector<char> buf = slurp(path);
  struct Node {
    uint64_t id, off, len;  // sequence in seqs
  };
  struct Link {
    uint64_t a, b;
    bool ra, rb;  // reverse orientation
  };
  std::vector<Node> nodes;
  std::vector<Link> links;
  std::string seqs;
  const char* p = buf.data();
  const char* const e = p + buf.size();
  uint64_t ln = 0;
  Field f[6];
  while (p < e) {
    const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(e - p)));
    const char* le = nl ? nl : e;
    ++ln;
    if (le > p && le[-1] == '\r') --le;
    if (le > p && *p == 'S') {
      const size_t k = split_tabs(p, le, f, 3);
      if (k < 3)
        fail(CHSGA_ERR_FORMAT, path + ":" + std::to_string(ln) + ": S line needs a name and a sequence");
      if (f[2].is("*") || f[2].n == 0)
        fail(CHSGA_ERR_FORMAT, path + ":" + std::to_string(ln) + ": segment without a sequence");
      const uint64_t off = seqs.size();
      seqs.resize(off + f[2].n);
      for (size_t i = 0; i < f[2].n; ++i) seqs[off + i] = packed_base(f[2].p[i]);
      nodes.push_back({parse_id(f[1], path, ln), off, f[2].n});
    } else if (le > p && *p == 'L') {
      const size_t k = split_tabs(p, le, f, 6);
      if (k < 5) fail(CHSGA_ERR_FORMAT, path + ":" + std::to_string(ln) + ": L line needs 5 fields");
      if (!((f[2].is("+") || f[2].is("-")) && (f[4].is("+") || f[4].is("-"))))
        fail(CHSGA_ERR_FORMAT, path + ":" + std::to_string(ln) + ": link orientations must be + or -");
      if (!(k < 6 || f[5].is("*") || f[5].is("0M")))
        fail(CHSGA_ERR_UNSUPPORTED,
             path + ":" + std::to_string(ln) + ": overlapping links are not supported (blunt graphs only)");
      links.push_back({parse_id(f[1], path, ln), parse_id(f[3], path, ln), f[2].is("-"), f[4].is("-")});
    }
    p = nl ? nl + 1 : e;
  }
  require(!nodes.empty(), CHSGA_ERR_FORMAT, path + ": no segments");
  __gnu_parallel::sort(nodes.begin(), nodes.end(),
                       [](const Node& x, const Node& y) { return x.id < y.id; });
  for (uint64_t i = 1; i < nodes.size(); ++i)
    if (nodes[i].id == nodes[i - 1].id)
      fail(CHSGA_ERR_FORMAT, path + ": duplicate segment " + std::to_string(nodes[i].id));
  // node id -> position in id order: a table when the ids are dense enough
  const uint64_t max_id = nodes.back().id;
  const bool dense = max_id < 4 * (uint64_t)nodes.size() + 1024;
  std::vector<uint64_t> table;
  std::unordered_map<uint64_t, uint64_t> index;
  if (dense) {
    table.assign(max_id + 1, ~0ull);
    for (uint64_t i = 0; i < nodes.size(); ++i) table[nodes[i].id] = i;
  } else {
    index.reserve(nodes.size());
    for (uint64_t i = 0; i < nodes.size(); ++i) index.emplace(nodes[i].id, i);
  }
  auto handle = [&](uint64_t id, bool rev) {
    uint64_t i = ~0ull;
    if (dense) {
      if (id <= max_id) i = table[id];
    } else {
      auto it = index.find(id);
      if (it != index.end()) i = it->second;
    }
    if (i == ~0ull) fail(CHSGA_ERR_FORMAT, path + ": link to unknown segment " + std::to_string(id));
    return 2 * i + (rev ? 1 : 0);
  };
  CsrText s;
  const uint64_t V = 2 * nodes.size();
  s.lab.reserve(2 * seqs.size());
  s.lab_off.reserve(V + 1);
  for (const Node& nd : nodes) {
    s.lab.append(seqs, nd.off, nd.len);
    s.lab_off.push_back(s.lab.size());
    for (uint64_t i = nd.len; i-- > 0;) s.lab.push_back(complement(seqs[nd.off + i]));
    s.lab_off.push_back(s.lab.size());
  }
  // every link in both directions, then each handle's targets sorted, once
  std::vector<std::pair<uint64_t, uint64_t>> arcs;
  arcs.reserve(2 * links.size());
  for (const Link& l : links) {
    arcs.emplace_back(handle(l.a, l.ra), handle(l.b, l.rb));
    arcs.emplace_back(handle(l.b, !l.rb), handle(l.a, !l.ra));
  }
  __gnu_parallel::sort(arcs.begin(), arcs.end());
  arcs.erase(std::unique(arcs.begin(), arcs.end()), arcs.end());
  s.offsets.assign(V + 1, 0);
  s.adj.resize(arcs.size());
  for (size_t i = 0; i < arcs.size(); ++i) {
    ++s.offsets[arcs[i].first + 1];
    s.adj[i] = arcs[i].second;
  }
  for (uint64_t v = 0; v < V; ++v) s.offsets[v + 1] += s.offsets[v];
  return s;
}

// handlegraph_to_csr.cpp build(): one vertex per char.
CsrText expand_chars(const CsrText& s) {
  CsrText c;
  const uint64_t N = s.lab.size();
  c.lab = s.lab;
  c.lab_off.resize(N + 1);
  for (uint64_t i = 0; i <= N; ++i) c.lab_off[i] = i;
  c.offsets.resize(N + 1);
  c.offsets[0] = 0;
  c.adj.reserve(N + s.adj.size());
  uint64_t x = 0;
  for (uint64_t i = 0; i < s.n(); ++i) {
    const uint64_t L = s.len(i), f = s.lab_off[i];
    for (uint64_t j = 0; j < L; ++j) {
      if (j + 1 < L) {
        c.adj.push_back(f + j + 1);
      } else {
        for (uint64_t e = s.offsets[i]; e < s.offsets[i + 1]; ++e) c.adj.push_back(s.lab_off[s.adj[e]]);
      }
      c.offsets[++x] = c.adj.size();
    }
  }
  return c;
}

// Buffered writer of decimal integers and raw bytes.
struct TextOut {
  FILE* f;
  std::string path;
  std::vector<char> buf;
  explicit TextOut(const std::string& p) : f(std::fopen(p.c_str(), "wb")), path(p) {
    require(f != nullptr, CHSGA_ERR_IO, "cannot write " + path);
    buf.reserve(1 << 22);
  }
  void flush() {
    if (!buf.empty() && std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) {
      std::fclose(f);
      f = nullptr;
      fail(CHSGA_ERR_IO, "write failed: " + path);
    }
    buf.clear();
  }
  void room() {
    if (buf.size() > (1u << 22)) flush();
  }
  void num(uint64_t v, char sep) {
    char t[24];
    int k = 0;
    do {
      t[k++] = (char)('0' + v % 10);
      v /= 10;
    } while (v);
    while (k) buf.push_back(t[--k]);
    buf.push_back(sep);
    room();
  }
  void bytes(const char* p, size_t n, char sep) {
    buf.insert(buf.end(), p, p + n);
    buf.push_back(sep);
    room();
  }
  void put(char c) { buf.push_back(c); }
  void close() {
    flush();
    const bool ok = std::fclose(f) == 0;
    f = nullptr;
    require(ok, CHSGA_ERR_IO, "write failed: " + path);
  }
  ~TextOut() {
    if (f) std::fclose(f);
  }
};

// Text of items [0, n), each made by put(i, buffer), formatted on every
// thread in slices and written in order.
template <typename F>
void put_parallel(TextOut& o, size_t n, size_t bytes_each, F put) {
  const int nt = n < (1u << 16) ? 1 : std::max(1, omp_get_max_threads());
  std::vector<std::vector<char>> part(nt);
#pragma omp parallel for num_threads(nt) schedule(static, 1)
  for (int t = 0; t < nt; ++t) {
    const size_t a = n / nt * t, z = t + 1 == nt ? n : n / nt * (t + 1);
    part[t].reserve((z - a) * bytes_each);
    for (size_t i = a; i < z; ++i) put(i, part[t]);
  }
  o.flush();
  for (auto& b : part) {
    o.buf.swap(b);
    o.flush();
  }
}

void put_number(uint64_t v, char sep, std::vector<char>& b) {
  char tmp[24];
  int k = 0;
  do {
    tmp[k++] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  while (k) b.push_back(tmp[--k]);
  b.push_back(sep);
}

void write_csr_text(const std::string& path, const CsrText& s) {
  TextOut o(path);
  // write_csr (handlegraph_to_csr.cpp:130-161): every list ends with " \n"
  o.num(s.n(), '\n');
  o.num(s.adj.size(), '\n');
  put_parallel(o, s.n(), 4, [&](size_t i, std::vector<char>& b) {
    b.insert(b.end(), s.lab.data() + s.lab_off[i], s.lab.data() + s.lab_off[i + 1]);
    b.push_back(' ');
  });
  o.put('\n');
  put_parallel(o, s.offsets.size(), 10, [&](size_t i, std::vector<char>& b) { put_number(s.offsets[i], ' ', b); });
  o.put('\n');
  put_parallel(o, s.adj.size(), 10, [&](size_t i, std::vector<char>& b) { put_number(s.adj[i], ' ', b); });
  o.put('\n');
  o.close();
}

// The write_csr layout, sequentially (the checks name what is wrong).
CsrText read_csr_text_seq(const std::vector<char>& buf, const std::string& path) {
  Tok t(buf, path);
  const uint64_t n = t.u64("the vertex count (header n m)");
  const uint64_t m = t.u64("the edge count (header n m)");
  CsrText s;
  s.lab_off.reserve(n + 1);
  for (uint64_t i = 0; i < n; ++i) {
    t.skip();
    const char* b = t.p;
    while (t.p < t.e && !std::isspace((unsigned char)*t.p)) ++t.p;
    if (t.p == b) fail(CHSGA_ERR_FORMAT, path + ": failed to read label " + std::to_string(i));
    s.lab.append(b, t.p);
    s.lab_off.push_back(s.lab.size());
  }
  s.offsets.resize(n + 1);
  for (uint64_t i = 0; i <= n; ++i) {
    s.offsets[i] = t.u64("an offset");
    if (i > 0 && s.offsets[i] < s.offsets[i - 1])
      fail(CHSGA_ERR_FORMAT, path + ": offsets not non-decreasing at index " + std::to_string(i));
  }
  require(s.offsets[n] == m, CHSGA_ERR_FORMAT, path + ": final offset differs from the edge count");
  s.adj.resize(m);
  for (uint64_t e = 0; e < m; ++e) {
    s.adj[e] = t.u64("an adjacency entry");
    if (s.adj[e] >= n) fail(CHSGA_ERR_FORMAT, path + ": adjacency entry out of range");
  }
  return s;
}

// The same, the three lists parsed on every thread; any problem sends the
// file to the sequential reader, which reports it.
CsrText read_csr_text(const std::string& path) {
  const std::vector<char> buf = slurp(path);
  Tok t(buf, path);
  uint64_t n = 0, m = 0;
  t.skip();
  if (!(t.p < t.e && *t.p >= '0' && *t.p <= '9')) return read_csr_text_seq(buf, path);
  n = t.u64("the vertex count (header n m)");
  t.skip();
  if (!(t.p < t.e && *t.p >= '0' && *t.p <= '9')) return read_csr_text_seq(buf, path);
  m = t.u64("the edge count (header n m)");
  CsrText s;
  std::vector<const char*> lb(n);
  std::vector<uint32_t> ll(n);
  const char* after = nullptr;
  bool ok = parse_tokens(t.p, t.e, n, &after, [&](uint64_t k, const char* a, const char* z) {
    if (z - a >= (1ll << 32)) return false;
    lb[k] = a;
    ll[k] = (uint32_t)(z - a);
    return true;
  });
  if (!ok) return read_csr_text_seq(buf, path);
  s.lab_off.resize(n + 1);
  s.lab_off[0] = 0;
  for (uint64_t i = 0; i < n; ++i) s.lab_off[i + 1] = s.lab_off[i] + ll[i];
  s.lab.resize(s.lab_off[n]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) std::memcpy(&s.lab[s.lab_off[i]], lb[i], ll[i]);
  s.offsets.resize(n + 1);
  ok = parse_tokens(after, t.e, n + 1, &after, [&](uint64_t k, const char* a, const char* z) {
    return token_u64(a, z, s.offsets[k]);
  });
  if (!ok) return read_csr_text_seq(buf, path);
  for (uint64_t i = 1; i <= n; ++i)
    if (s.offsets[i] < s.offsets[i - 1]) return read_csr_text_seq(buf, path);
  if (s.offsets[n] != m) return read_csr_text_seq(buf, path);
  s.adj.resize(m);
  ok = parse_tokens(after, t.e, m, &after, [&](uint64_t k, const char* a, const char* z) {
    return token_u64(a, z, s.adj[k]) && s.adj[k] < n;
  });
  if (!ok) return read_csr_text_seq(buf, path);
  return s;
}

HostCsr to_host_csr(const CsrText& s) {
  HostCsr g;
  g.n = s.n();
  g.m = s.adj.size();
  g.offset = s.offsets;
  g.target.resize(g.m);
  for (uint64_t e = 0; e < g.m; ++e) {
    if (s.adj[e] >= (1ull << 32)) fail(CHSGA_ERR_UNSUPPORTED, "vertex ids above 2^32");
    g.target[e] = (uint32_t)s.adj[e];
  }
  return g;
}

// csr_to_adj on both CSR files: the string graph keeps its out-CSR, the
// labels are the concatenation of the string labels (equal to the char
// labels), the label offsets their prefix sums.
chsga_host_graph* host_graph_from(const CsrText& str, const CsrText& chr) {
  auto g = std::make_unique<chsga_host_graph>();
  g->string_graph = to_host_csr(str);
  g->char_graph = to_host_csr(chr);
  g->labels.assign(str.lab.begin(), str.lab.end());
  g->label_offsets = str.lab_off;
  require(g->labels.size() == chr.n(), CHSGA_ERR_FORMAT,
          "the char CSR does not have one vertex per char of the string CSR");
  for (uint64_t i = 0; i < chr.n(); ++i)
    if (!(chr.len(i) == 1 && chr.lab[chr.lab_off[i]] == g->labels[i]))
      fail(CHSGA_ERR_FORMAT, "char CSR label " + std::to_string(i) + " differs from the string labels");
  return g.release();
}

template <typename F>
chsga_status guarded_ingest(F&& f) {
  try {
    f();
    return CHSGA_OK;
  } catch (const ChsgaError& e) {
    g_last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    g_last_error = "host out of memory";
    return CHSGA_ERR_OOM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return CHSGA_ERR_INTERNAL;
  }
}

}  // namespace
}  // namespace chsga

using namespace chsga;

extern "C" {

chsga_status chsga_gfa_to_csr_text(const char* gfa_path, const char* string_csr_out,
                                   const char* char_csr_out) {
  return guarded_ingest([&] {
    require(gfa_path && string_csr_out && char_csr_out, CHSGA_ERR_INVALID_ARG, "null argument");
    const CsrText s = gfa_to_string_csr(gfa_path);
    write_csr_text(string_csr_out, s);
    write_csr_text(char_csr_out, expand_chars(s));
  });
}

chsga_status chsga_graph_from_gfa(const char* gfa_path, chsga_host_graph** out) {
  return guarded_ingest([&] {
    require(gfa_path && out, CHSGA_ERR_INVALID_ARG, "null argument");
    const CsrText s = gfa_to_string_csr(gfa_path);
    *out = host_graph_from(s, expand_chars(s));
  });
}

chsga_status chsga_graph_from_csr_text(const char* string_csr, const char* char_csr,
                                       chsga_host_graph** out) {
  return guarded_ingest([&] {
    require(string_csr && char_csr && out, CHSGA_ERR_INVALID_ARG, "null argument");
    *out = host_graph_from(read_csr_text(string_csr), read_csr_text(char_csr));
  });
}

chsga_status chsga_csr_text_to_adj(const char* csr_path, const char* adj_out, const char* labels_out,
                                   const char* label_offsets_out) {
  return guarded_ingest([&] {
    require(csr_path && adj_out && labels_out && label_offsets_out, CHSGA_ERR_INVALID_ARG,
            "null argument");
    const CsrText s = read_csr_text(csr_path);
    write_adj(adj_out, to_host_csr(s));
    write_labels(labels_out, std::vector<char>(s.lab.begin(), s.lab.end()));
    write_label_offsets(label_offsets_out, s.lab_off);
  });
}

}  // extern "C"
