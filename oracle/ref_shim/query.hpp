// ORACLE STAND-IN — test infrastructure, not product code.
//
// The reference's alignment headers include "query.hpp" from the
// Parallel-Contraction-Hierarchy submodule and use parlaylib; neither is
// present (ext/ is empty). This header supplies, in project-written code, the
// small interface those headers use, so that the reference's own
// src/align.hpp, src/traceback.hpp, src/ConSGA.cpp and src/ConSGA_traceback.cpp
// compile unchanged from the reference tree:
//   parlay: sequence, parallel_for, blocked_for, num_workers, worker_id,
//           reduce, minm (mapped onto OpenMP)
//   PCH:    NodeId, EdgeId, EdgeTy, Graph, PchGraph, PchQuery (holding GC),
//           read_graph (AdjacencyGraph text), read_contracted_graph (the
//           project's CHSGAPCH hierarchy file).
// Assumption, not pinned by any reference file: PchQuery::GC is the
// rank-ordered hierarchy exactly as read from the file (align.hpp indexes it
// by rank through contracted_str_to_og, consistent with this).
#pragma once

#include <omp.h>

#include <algorithm>
#include <array>
#include <cctype>
#include <chrono>
#include <cmath>
#include <map>
#include <numeric>
#include <set>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <limits>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace parlay {

template <typename T>
using sequence = std::vector<T>;

inline size_t num_workers() { return (size_t)omp_get_max_threads(); }
inline size_t worker_id() { return (size_t)omp_get_thread_num(); }

template <typename F>
void parallel_for(size_t start, size_t end, F f) {
#pragma omp parallel for schedule(dynamic, 512)
  for (long long i = (long long)start; i < (long long)end; ++i) f((size_t)i);
}

template <typename F>
void blocked_for(size_t start, size_t end, size_t block, F f) {
  if (end <= start) return;
  const long long nb = (long long)((end - start + block - 1) / block);
#pragma omp parallel for schedule(dynamic, 1)
  for (long long b = 0; b < nb; ++b) {
    size_t s = start + (size_t)b * block;
    size_t e = std::min(end, s + block);
    f((size_t)b, s, e);
  }
}

template <typename T>
struct minm {
  T identity = std::numeric_limits<T>::max();
  T operator()(T a, T b) const { return a < b ? a : b; }
};

template <typename Seq, typename M>
auto reduce(const Seq& s, M m) {
  auto acc = m.identity;
  for (const auto& x : s) acc = m(acc, x);
  return acc;
}

}  // namespace parlay

using parlay::parallel_for;
using parlay::sequence;

using NodeId = uint32_t;
using EdgeId = uint64_t;
using EdgeTy = uint32_t;

struct Edge {
  NodeId v;
  EdgeTy w;
};

struct Graph {
  size_t n = 0, m = 0;
  sequence<EdgeId> offset;
  sequence<Edge> E;
};

struct PchGraph {
  size_t n = 0, m = 0, rm = 0;
  sequence<EdgeId> offset, in_offset;
  sequence<Edge> E, in_E;
  sequence<NodeId> rank, level, layerOffset, ccOffset;
};

struct PchQuery {
  PchGraph GC;
  PchQuery(PchGraph& gc, Graph& /*origin*/) : GC(gc) {}
};

namespace chsga_shim {
inline std::vector<char> slurp(const char* p) {
  std::ifstream f(p, std::ios::binary);
  if (!f) throw std::runtime_error(std::string("cannot open ") + p);
  return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}
}  // namespace chsga_shim

// AdjacencyGraph text: header, n, m, n offsets, m targets, optional m weights.
inline Graph read_graph(const char* path) {
  std::vector<char> b = chsga_shim::slurp(path);
  b.push_back('\0');
  char* s = b.data();
  char* end = nullptr;
  while (*s && std::isspace((unsigned char)*s)) ++s;
  while (*s && !std::isspace((unsigned char)*s)) ++s;  // header word
  Graph g;
  g.n = std::strtoull(s, &end, 10);
  s = end;
  g.m = std::strtoull(s, &end, 10);
  s = end;
  g.offset.resize(g.n + 1);
  for (size_t i = 0; i < g.n; ++i) {
    g.offset[i] = std::strtoull(s, &end, 10);
    s = end;
  }
  g.offset[g.n] = g.m;
  g.E.resize(g.m);
  for (size_t i = 0; i < g.m; ++i) {
    g.E[i].v = (NodeId)std::strtoull(s, &end, 10);
    g.E[i].w = 1;
    s = end;
  }
  for (size_t i = 0; i < g.m; ++i) {
    double w = std::strtod(s, &end);
    if (end == s) break;
    g.E[i].w = (EdgeTy)w;
    s = end;
  }
  return g;
}

// CHSGAPCH v1 hierarchy file (layout in the product's formats.cpp).
inline void read_contracted_graph(const char* path, PchGraph& g) {
  std::vector<char> b = chsga_shim::slurp(path);
  size_t pos = 0;
  auto take = [&](void* d, size_t n) {
    if (pos + n > b.size()) throw std::runtime_error("truncated hierarchy file");
    std::memcpy(d, b.data() + pos, n);
    pos += n;
  };
  char magic[8];
  take(magic, 8);
  if (std::memcmp(magic, "CHSGAPCH", 8) != 0) throw std::runtime_error("not a CHSGAPCH file");
  uint32_t ver, flags;
  take(&ver, 4);
  take(&flags, 4);
  uint64_t h[5];
  take(h, sizeof(h));
  g.n = h[0];
  g.m = h[1];
  g.rm = h[2];
  auto vec32 = [&](sequence<NodeId>& v, uint64_t n) {
    v.resize(n);
    take(v.data(), n * 4);
  };
  auto vec64 = [&](sequence<EdgeId>& v, uint64_t n) {
    v.resize(n);
    take(v.data(), n * 8);
  };
  vec32(g.rank, g.n);
  vec32(g.level, g.n);
  vec32(g.layerOffset, h[3] + 1);
  vec32(g.ccOffset, h[4] + 1);
  auto edges = [&](sequence<Edge>& E, uint64_t m) {
    std::vector<uint32_t> v(m), w(m);
    take(v.data(), m * 4);
    take(w.data(), m * 4);
    E.resize(m);
    for (uint64_t i = 0; i < m; ++i) E[i] = Edge{v[i], w[i]};
  };
  vec64(g.offset, g.n + 1);
  edges(g.E, g.m);
  vec64(g.in_offset, g.n + 1);
  edges(g.in_E, g.rm);
}
