// Seeded synthetic inputs: a variant-bubble DAG over a random ACGT backbone,
// its char-graph expansion, and simulated reads. These stand in for the
// graphs and read sets the reference is run on (its datasets are not part of
// the reference repository).
#include <algorithm>
#include <cmath>

#include "host_graph.hpp"

namespace chsga {

namespace {

constexpr char kBases[4] = {'A', 'C', 'G', 'T'};

struct GraphBuilder {
  std::vector<char> labels;
  std::vector<uint64_t> offs{0};
  std::vector<std::pair<uint32_t, uint32_t>> edges;
  Rng& rng;
  uint32_t vmin, vmax;
  GraphBuilder(Rng& r, uint32_t a, uint32_t b) : rng(r), vmin(a), vmax(b) {}

  uint32_t add_vertex(const char* s, size_t n) {
    labels.insert(labels.end(), s, s + n);
    offs.push_back(labels.size());
    return (uint32_t)(offs.size() - 2);
  }
  // Splits `text` into vertices of [vmin, vmax] chars, chains them, and
  // connects every frontier vertex to the first one. Returns the last id.
  uint32_t add_path(const std::string& text, const std::vector<uint32_t>& frontier) {
    size_t pos = 0;
    uint32_t prev = UINT32_MAX;
    while (pos < text.size()) {
      size_t len = (size_t)rng.range(vmin, vmax);
      len = std::min(len, text.size() - pos);
      uint32_t id = add_vertex(text.data() + pos, len);
      if (prev == UINT32_MAX) {
        for (uint32_t f : frontier) edges.push_back({f, id});
      } else {
        edges.push_back({prev, id});
      }
      prev = id;
      pos += len;
    }
    return prev;
  }
  std::string random_text(size_t n) {
    std::string s(n, 'A');
    for (auto& c : s) c = kBases[rng.below(4)];
    return s;
  }
};

HostCsr csr_from_edges(uint64_t n, std::vector<std::pair<uint32_t, uint32_t>>& edges) {
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  HostCsr g;
  g.n = n;
  g.m = edges.size();
  g.offset.assign(n + 1, 0);
  g.target.resize(g.m);
  for (auto& e : edges) g.offset[e.first + 1]++;
  for (uint64_t i = 0; i < n; ++i) g.offset[i + 1] += g.offset[i];
  for (uint64_t i = 0; i < g.m; ++i) g.target[i] = edges[i].second;
  return g;
}

}  // namespace

// Char-graph expansion of a string graph, following build() in
// src/handlegraph_to_csr.cpp:165-247: every char is a vertex; consecutive
// chars of one string are chained; the last char of string i inherits i's
// out-edges, each mapped to the first char of the neighbour string, in the
// order of i's adjacency list.
HostCsr expand_char_graph(const HostCsr& sg, const std::vector<uint64_t>& offs) {
  HostCsr cg;
  const uint64_t N = offs[sg.n];
  cg.n = N;
  cg.offset.reserve(N + 1);
  cg.offset.push_back(0);
  cg.target.reserve(N + sg.m);
  for (uint64_t i = 0; i < sg.n; ++i) {
    const uint64_t s = offs[i], e = offs[i + 1];
    require(e > s, CHSGA_ERR_UNSUPPORTED, "empty string vertex label");
    for (uint64_t v = s; v < e; ++v) {
      if (v + 1 < e) {
        cg.target.push_back((uint32_t)(v + 1));
      } else {
        for (uint64_t k = sg.offset[i]; k < sg.offset[i + 1]; ++k)
          cg.target.push_back((uint32_t)offs[sg.target[k]]);
      }
      cg.offset.push_back(cg.target.size());
    }
  }
  cg.m = cg.target.size();
  return cg;
}

void generate_graph(const chsga_gen_graph_cfg& c, chsga_host_graph& out) {
  require(c.backbone_len >= 2, CHSGA_ERR_INVALID_ARG, "backbone_len must be >= 2");
  require(c.vlen_min >= 1 && c.vlen_max >= c.vlen_min, CHSGA_ERR_INVALID_ARG, "vertex length range");
  require(c.bubble_gap_mean >= 1.0, CHSGA_ERR_INVALID_ARG, "bubble_gap_mean must be >= 1");
  const double psum = c.p_snp + c.p_indel + c.p_alt;
  require(psum > 0.999 && psum < 1.001, CHSGA_ERR_INVALID_ARG, "bubble mixture must sum to 1");
  require(c.indel_min >= 1 && c.indel_max >= c.indel_min && c.alt_min >= 1 &&
              c.alt_max >= c.alt_min,
          CHSGA_ERR_INVALID_ARG, "allele length ranges");
  Rng rng(c.seed);
  GraphBuilder b(rng, c.vlen_min, c.vlen_max);
  const double p = 1.0 / c.bubble_gap_mean;
  const double lq = std::log1p(-std::min(p, 0.999999));
  auto gap = [&]() -> uint64_t {
    if (p >= 1.0) return 1;
    double u = rng.uniform();
    return 1 + (uint64_t)std::floor(std::log1p(-u) / lq);
  };
  std::vector<uint32_t> frontier;  // empty: first path has no in-edges
  uint64_t pos = 0;
  const uint64_t B = c.backbone_len;
  while (pos < B) {
    uint64_t g = std::min<uint64_t>(gap(), B - pos);
    uint32_t last = b.add_path(b.random_text(g), frontier);
    frontier.assign(1, last);
    pos += g;
    if (pos >= B - 1) break;  // keep a linear tail after the last bubble
    double u = rng.uniform();
    std::vector<uint32_t> nf;
    if (u < c.p_snp) {
      char ref = kBases[rng.below(4)];
      char alt = kBases[(std::find(kBases, kBases + 4, ref) - kBases + 1 + rng.below(3)) % 4];
      nf.push_back(b.add_path(std::string(1, ref), frontier));
      nf.push_back(b.add_path(std::string(1, alt), frontier));
      pos += 1;
    } else if (u < c.p_snp + c.p_indel) {
      uint64_t len = (uint64_t)rng.range(c.indel_min, c.indel_max);
      bool deletion = rng.below(2) == 0;
      if (deletion) len = std::min<uint64_t>(len, B - 1 - pos);
      if (len == 0) continue;
      nf.push_back(b.add_path(b.random_text(len), frontier));
      nf.insert(nf.end(), frontier.begin(), frontier.end());  // the empty allele
      if (deletion) pos += len;
    } else {
      uint64_t lr = std::min<uint64_t>((uint64_t)rng.range(c.alt_min, c.alt_max), B - 1 - pos);
      uint64_t la = (uint64_t)rng.range(c.alt_min, c.alt_max);
      if (lr == 0) continue;
      nf.push_back(b.add_path(b.random_text(lr), frontier));
      nf.push_back(b.add_path(b.random_text(la), frontier));
      pos += lr;
    }
    frontier = nf;
  }
  if (frontier.size() != 1) {
    uint32_t last = b.add_path(b.random_text(1), frontier);
    frontier.assign(1, last);
  }
  const uint64_t S = b.offs.size() - 1;
  out.labels = std::move(b.labels);
  out.label_offsets = std::move(b.offs);
  out.string_graph = csr_from_edges(S, b.edges);
  out.char_graph = expand_char_graph(out.string_graph, out.label_offsets);
  out.pch = HostPch{};
}

// Reads from random paths: the start is a uniformly random char of the
// graph; the walk continues to the end of its string vertex and then along
// uniformly chosen out-edges. Errors: substitution (a different base),
// insertion or deletion of 1..indel_len_max bases (50/50), N.
void generate_reads(const chsga_host_graph& g, const chsga_gen_reads_cfg& c, HostReads& out) {
  const uint64_t N = g.labels.size();
  const HostCsr& sg = g.string_graph;
  require(N > 0 && sg.n > 0, CHSGA_ERR_INVALID_ARG, "empty graph");
  require(c.len_min >= 1 && c.len_max >= c.len_min, CHSGA_ERR_INVALID_ARG, "read length range");
  require(c.indel_len_max >= 1 || c.indel_rate == 0, CHSGA_ERR_INVALID_ARG, "indel length");
  Rng rng(c.seed);
  std::vector<uint32_t> vertex_of(N);
  for (uint64_t s = 0; s < sg.n; ++s)
    for (uint64_t p = g.label_offsets[s]; p < g.label_offsets[s + 1]; ++p) vertex_of[p] = (uint32_t)s;
  std::string read, truth;
  for (uint64_t r = 0; r < c.count; ++r) {
    uint32_t L = c.len_min;
    if (c.len_max > c.len_min) {
      double lo = std::log((double)c.len_min), hi = std::log((double)c.len_max);
      L = (uint32_t)std::llround(std::exp(lo + (hi - lo) * rng.uniform()));
      L = std::min(std::max(L, c.len_min), c.len_max);
    }
    for (int attempt = 0;; ++attempt) {
      require(attempt < 1000, CHSGA_ERR_INVALID_ARG, "graph paths too short for the read length");
      uint64_t p = rng.below(N);
      uint32_t s = vertex_of[p];
      read.clear();
      bool ended = false;
      // true-sequence cursor
      auto next_base = [&](char& out_c) -> bool {
        while (p >= g.label_offsets[s + 1]) {
          uint64_t d = sg.offset[s + 1] - sg.offset[s];
          if (d == 0) return false;
          s = sg.target[sg.offset[s] + rng.below(d)];
          p = g.label_offsets[s];
        }
        out_c = g.labels[p++];
        return true;
      };
      char t;
      while (read.size() < L) {
        double u = rng.uniform();
        if (u < c.sub_rate) {
          if (!next_base(t)) { ended = true; break; }
          int k = (int)(std::find(kBases, kBases + 4, t) - kBases);
          read.push_back(kBases[(k + 1 + (int)rng.below(3)) % 4]);
        } else if (u < c.sub_rate + c.indel_rate) {
          uint32_t len = (uint32_t)rng.range(1, c.indel_len_max);
          if (rng.below(2) == 0) {
            for (uint32_t i = 0; i < len; ++i) read.push_back(kBases[rng.below(4)]);
          } else {
            for (uint32_t i = 0; i < len && !ended; ++i) ended = !next_base(t);
            if (ended) break;
          }
        } else if (u < c.sub_rate + c.indel_rate + c.n_rate) {
          if (!next_base(t)) { ended = true; break; }
          read.push_back('N');
        } else {
          if (!next_base(t)) { ended = true; break; }
          read.push_back(t);
        }
      }
      if (ended) continue;
      read.resize(L);
      out.add(read.data(), read.size());
      break;
    }
  }
}

}  // namespace chsga
