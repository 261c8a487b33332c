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
#include <algorithm>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "host_graph.hpp"

namespace chsga {
extern thread_local std::string g_last_error;

namespace {

// A string-labeled CSR as handlegraph_to_csr's CSR_container holds it.
struct CsrText {
  std::vector<std::string> labels;
  std::vector<uint64_t> offsets{0};
  std::vector<uint64_t> adj;
  uint64_t n() const { return labels.size(); }
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

std::vector<std::string> split_tabs(const std::string& line) {
  std::vector<std::string> f;
  size_t a = 0;
  while (true) {
    size_t b = line.find('\t', a);
    f.push_back(line.substr(a, b == std::string::npos ? std::string::npos : b - a));
    if (b == std::string::npos) break;
    a = b + 1;
  }
  return f;
}

uint64_t parse_id(const std::string& s, const std::string& path, uint64_t line) {
  require(!s.empty() && s.size() < 20 && std::all_of(s.begin(), s.end(), ::isdigit), CHSGA_ERR_FORMAT,
          path + ":" + std::to_string(line) + ": segment names must be numeric node ids, got '" + s + "'");
  return std::stoull(s);
}

CsrText gfa_to_string_csr(const std::string& path) {
  std::ifstream in(path);
  require(bool(in), CHSGA_ERR_IO, "cannot read " + path);
  std::vector<std::pair<uint64_t, std::string>> nodes;
  struct Link {
    uint64_t a, b;
    bool ra, rb;  // reverse orientation
  };
  std::vector<Link> links;
  std::string line;
  uint64_t ln = 0;
  while (std::getline(in, line)) {
    ++ln;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty()) continue;
    if (line[0] == 'S') {
      const auto f = split_tabs(line);
      require(f.size() >= 3, CHSGA_ERR_FORMAT, path + ":" + std::to_string(ln) + ": S line needs a name and a sequence");
      require(f[2] != "*" && !f[2].empty(), CHSGA_ERR_FORMAT,
              path + ":" + std::to_string(ln) + ": segment without a sequence");
      std::string seq(f[2]);
      for (char& c : seq) c = packed_base(c);
      nodes.push_back({parse_id(f[1], path, ln), std::move(seq)});
    } else if (line[0] == 'L') {
      const auto f = split_tabs(line);
      require(f.size() >= 5, CHSGA_ERR_FORMAT, path + ":" + std::to_string(ln) + ": L line needs 5 fields");
      require((f[2] == "+" || f[2] == "-") && (f[4] == "+" || f[4] == "-"), CHSGA_ERR_FORMAT,
              path + ":" + std::to_string(ln) + ": link orientations must be + or -");
      require(f.size() < 6 || f[5] == "*" || f[5] == "0M", CHSGA_ERR_UNSUPPORTED,
              path + ":" + std::to_string(ln) + ": overlapping links are not supported (blunt graphs only)");
      links.push_back({parse_id(f[1], path, ln), parse_id(f[3], path, ln), f[2] == "-", f[4] == "-"});
    }
  }
  require(!nodes.empty(), CHSGA_ERR_FORMAT, path + ": no segments");
  std::sort(nodes.begin(), nodes.end(),
            [](const auto& x, const auto& y) { return x.first < y.first; });
  std::unordered_map<uint64_t, uint64_t> index;
  index.reserve(nodes.size());
  for (uint64_t i = 0; i < nodes.size(); ++i) {
    require(index.emplace(nodes[i].first, i).second, CHSGA_ERR_FORMAT,
            path + ": duplicate segment " + std::to_string(nodes[i].first));
  }
  CsrText s;
  const uint64_t V = 2 * nodes.size();
  s.labels.resize(V);
  for (uint64_t i = 0; i < nodes.size(); ++i) {
    const std::string& seq = nodes[i].second;
    s.labels[2 * i] = seq;
    std::string rc(seq.rbegin(), seq.rend());
    for (char& c : rc) c = complement(c);
    s.labels[2 * i + 1] = std::move(rc);
  }
  std::vector<std::vector<uint64_t>> out(V);
  auto handle = [&](uint64_t id, bool rev) {
    auto it = index.find(id);
    require(it != index.end(), CHSGA_ERR_FORMAT, path + ": link to unknown segment " + std::to_string(id));
    return 2 * it->second + (rev ? 1 : 0);
  };
  for (const Link& l : links) {
    out[handle(l.a, l.ra)].push_back(handle(l.b, l.rb));
    out[handle(l.b, !l.rb)].push_back(handle(l.a, !l.ra));
  }
  s.offsets.assign(1, 0);
  for (uint64_t v = 0; v < V; ++v) {
    auto& o = out[v];
    std::sort(o.begin(), o.end());
    o.erase(std::unique(o.begin(), o.end()), o.end());
    s.adj.insert(s.adj.end(), o.begin(), o.end());
    s.offsets.push_back(s.adj.size());
  }
  return s;
}

// handlegraph_to_csr.cpp build(): one vertex per char.
CsrText expand_chars(const CsrText& s) {
  CsrText c;
  std::vector<uint64_t> first(s.n() + 1, 0);
  for (uint64_t i = 0; i < s.n(); ++i) first[i + 1] = first[i] + s.labels[i].size();
  c.labels.reserve(first.back());
  c.offsets.assign(1, 0);
  for (uint64_t i = 0; i < s.n(); ++i) {
    const std::string& lab = s.labels[i];
    for (uint64_t j = 0; j < lab.size(); ++j) {
      c.labels.emplace_back(1, lab[j]);
      if (j + 1 < lab.size()) {
        c.adj.push_back(first[i] + j + 1);
      } else {
        for (uint64_t e = s.offsets[i]; e < s.offsets[i + 1]; ++e) c.adj.push_back(first[s.adj[e]]);
      }
      c.offsets.push_back(c.adj.size());
    }
  }
  return c;
}

void write_csr_text(const std::string& path, const CsrText& s) {
  std::ofstream o(path);
  require(bool(o), CHSGA_ERR_IO, "cannot write " + path);
  // write_csr (handlegraph_to_csr.cpp:130-161): every list ends with " \n"
  o << s.n() << "\n" << s.adj.size() << "\n";
  for (const auto& l : s.labels) o << l << " ";
  o << "\n";
  for (uint64_t x : s.offsets) o << x << " ";
  o << "\n";
  for (uint64_t x : s.adj) o << x << " ";
  o << "\n";
  require(bool(o), CHSGA_ERR_IO, "write failed: " + path);
}

CsrText read_csr_text(const std::string& path) {
  std::ifstream in(path);
  require(bool(in), CHSGA_ERR_IO, "cannot read " + path);
  uint64_t n = 0, m = 0;
  require(bool(in >> n >> m), CHSGA_ERR_FORMAT, path + ": failed to read header (n m)");
  CsrText s;
  s.labels.resize(n);
  for (uint64_t i = 0; i < n; ++i)
    require(bool(in >> s.labels[i]), CHSGA_ERR_FORMAT, path + ": failed to read label " + std::to_string(i));
  s.offsets.resize(n + 1);
  for (uint64_t i = 0; i <= n; ++i) {
    require(bool(in >> s.offsets[i]), CHSGA_ERR_FORMAT, path + ": failed to read offset " + std::to_string(i));
    require(i == 0 || s.offsets[i] >= s.offsets[i - 1], CHSGA_ERR_FORMAT,
            path + ": offsets not non-decreasing at index " + std::to_string(i));
  }
  require(s.offsets[n] == m, CHSGA_ERR_FORMAT, path + ": final offset differs from the edge count");
  s.adj.resize(m);
  for (uint64_t e = 0; e < m; ++e) {
    require(bool(in >> s.adj[e]), CHSGA_ERR_FORMAT, path + ": failed to read adjacency entry " + std::to_string(e));
    require(s.adj[e] < n, CHSGA_ERR_FORMAT, path + ": adjacency entry out of range");
  }
  return s;
}

HostCsr to_host_csr(const CsrText& s) {
  HostCsr g;
  g.n = s.n();
  g.m = s.adj.size();
  g.offset = s.offsets;
  g.target.resize(g.m);
  for (uint64_t e = 0; e < g.m; ++e) {
    require(s.adj[e] < (1ull << 32), CHSGA_ERR_UNSUPPORTED, "vertex ids above 2^32");
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
  g->label_offsets.assign(1, 0);
  for (const auto& l : str.labels) {
    g->labels.insert(g->labels.end(), l.begin(), l.end());
    g->label_offsets.push_back(g->labels.size());
  }
  require(g->labels.size() == chr.n(), CHSGA_ERR_FORMAT,
          "the char CSR does not have one vertex per char of the string CSR");
  for (uint64_t i = 0; i < chr.n(); ++i)
    require(chr.labels[i].size() == 1 && chr.labels[i][0] == g->labels[i], CHSGA_ERR_FORMAT,
            "char CSR label " + std::to_string(i) + " differs from the string labels");
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
    std::vector<char> labels;
    std::vector<uint64_t> offs{0};
    for (const auto& l : s.labels) {
      labels.insert(labels.end(), l.begin(), l.end());
      offs.push_back(labels.size());
    }
    write_labels(labels_out, labels);
    write_label_offsets(label_offsets_out, offs);
  });
}

}  // extern "C"
