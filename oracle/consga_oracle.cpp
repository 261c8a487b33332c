// CPU ORACLE — test infrastructure, not product code.
//
// A restatement, in plain C++17 + OpenMP, of CHSGA's ConSGA alignment DP
// (reference files src/align.hpp, src/traceback.hpp, src/ConSGA.cpp,
// src/ConSGA_traceback.cpp, src/ParSGAoverrides/csr_align.hpp). Only the
// tests, the smoke check and the CPU-baseline leg of the benchmark load it;
// the product (libchsga.so) never links or calls it.
//
// Pinning: the restatement is checked against the reference's own
// align.hpp / traceback.hpp compiled by oracle/Makefile into oracle/_ref
// (against a stand-in for the missing PCH/parlay interfaces), and against the
// reference's exact DP serial_align_CSR (src/ParSGAoverrides/csr_align.hpp:
// 270-383) on graphs where the hierarchy closure is exact.
//
// Parlay's parallel_for / blocked_for become `omp parallel for`; cas_update
// (csr_align.hpp:386-402) stays an atomic compare-and-swap min.
#include <omp.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using NodeId = uint32_t;
using LogScore = int32_t;
constexpr uint8_t BP_DELETE = 0, BP_MATCHSUB = 1, BP_INSERT = 2;  // traceback.hpp:168-170

struct Csr {  // out-CSR as read_graph leaves it
  uint64_t n = 0, m = 0;
  std::vector<uint64_t> off;
  std::vector<NodeId> v;
  std::vector<uint32_t> w;
};
struct InCsr {  // align.hpp:214-218
  std::vector<uint64_t> in_offset;
  std::vector<NodeId> in_u;
};
struct Pch {  // the fields of PchQuery::GC that align.hpp:279-345 reads
  uint64_t n = 0;
  std::vector<uint32_t> rank, level, layerOffset, ccOffset;
  std::vector<uint64_t> offset, in_offset;
  std::vector<uint32_t> E_v, E_w, inE_v, inE_w;
};
struct Graph {
  std::vector<char> labels;
  std::vector<uint64_t> label_offsets;
  InCsr in_char;
  Csr str;
  InCsr in_str;  // build_in_csr_from(origin_str_graph), traceback.hpp:102-118
  Pch gc;
  std::vector<NodeId> contracted_to_og;  // ConSGA.cpp:203-206
  size_t num_chars() const { return labels.size(); }
  NodeId first(NodeId c) const { return (NodeId)label_offsets[c]; }         // align.hpp:186-192
  NodeId last(NodeId c) const { return (NodeId)(label_offsets[c + 1] - 1); }  // align.hpp:195-201
};

std::string g_err;

std::vector<char> slurp(const std::string& p) {
  std::ifstream f(p, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + p);
  return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

// AdjacencyGraph text: header, n, m, n offsets, m targets, [m weights].
Csr read_adj(const std::string& p) {
  std::vector<char> b = slurp(p);
  b.push_back('\0');
  char* s = b.data();
  char* end = nullptr;
  while (*s && std::isspace((unsigned char)*s)) ++s;
  char* h = s;
  while (*s && !std::isspace((unsigned char)*s)) ++s;
  std::string head(h, s);
  if (head != "AdjacencyGraph" && head != "WeightedAdjacencyGraph")
    throw std::runtime_error(p + ": bad header");
  Csr g;
  g.n = std::strtoull(s, &end, 10);
  s = end;
  g.m = std::strtoull(s, &end, 10);
  s = end;
  g.off.resize(g.n + 1);
  for (uint64_t i = 0; i < g.n; ++i) {
    g.off[i] = std::strtoull(s, &end, 10);
    s = end;
  }
  g.off[g.n] = g.m;
  g.v.resize(g.m);
  for (uint64_t i = 0; i < g.m; ++i) {
    g.v[i] = (NodeId)std::strtoull(s, &end, 10);
    s = end;
  }
  g.w.assign(g.m, 1);
  for (uint64_t i = 0; i < g.m; ++i) {
    double w = std::strtod(s, &end);
    if (end == s) break;
    g.w[i] = (uint32_t)w;
    s = end;
  }
  return g;
}

// align.hpp:220-242: sources of each in-list in ascending u.
InCsr build_in_csr(const Csr& G) {
  InCsr in;
  in.in_offset.assign(G.n + 1, 0);
  for (uint64_t u = 0; u < G.n; ++u)
    for (uint64_t e = G.off[u]; e < G.off[u + 1]; ++e) ++in.in_offset[G.v[e] + 1];
  for (uint64_t v = 0; v < G.n; ++v) in.in_offset[v + 1] += in.in_offset[v];
  in.in_u.resize(in.in_offset[G.n]);
  std::vector<uint64_t> cur = in.in_offset;
  for (uint64_t u = 0; u < G.n; ++u)
    for (uint64_t e = G.off[u]; e < G.off[u + 1]; ++e) in.in_u[cur[G.v[e]]++] = (NodeId)u;
  return in;
}

// Hierarchy file "CHSGAPCH" v1 (layout documented in the product's formats.cpp).
Pch read_pch(const std::string& p) {
  std::vector<char> b = slurp(p);
  size_t pos = 0;
  auto take = [&](void* d, size_t n) {
    if (pos + n > b.size()) throw std::runtime_error(p + ": truncated");
    std::memcpy(d, b.data() + pos, n);
    pos += n;
  };
  char magic[8];
  take(magic, 8);
  if (std::memcmp(magic, "CHSGAPCH", 8) != 0) throw std::runtime_error(p + ": bad magic");
  uint32_t ver, flags;
  take(&ver, 4);
  take(&flags, 4);
  uint64_t h[5];
  take(h, sizeof(h));
  Pch g;
  g.n = h[0];
  auto vec = [&](auto& v, uint64_t n) {
    v.resize(n);
    take(v.data(), n * sizeof(v[0]));
  };
  vec(g.rank, g.n);
  vec(g.level, g.n);
  vec(g.layerOffset, h[3] + 1);
  vec(g.ccOffset, h[4] + 1);
  vec(g.offset, g.n + 1);
  vec(g.E_v, h[1]);
  vec(g.E_w, h[1]);
  vec(g.in_offset, g.n + 1);
  vec(g.inE_v, h[2]);
  vec(g.inE_w, h[2]);
  return g;
}

// csr_align.hpp:41-50: ALPHABET_SIZE 5 (mismatchN, this build by default)
// matches equal bytes only; ALPHABET_SIZE 4 (matchN, built with
// -DORACLE_MATCH_N) also matches an 'N' on either side.
#ifdef ORACLE_MATCH_N
inline LogScore match_sub(char a, char b) { return (a == 'N' || b == 'N' || a == b) ? 0 : 1; }
#else
inline LogScore match_sub(char a, char b) { return a == b ? 0 : 1; }
#endif

inline void cas_min(LogScore* t, LogScore nv) {  // csr_align.hpp:386-402
  LogScore prev = __atomic_load_n(t, __ATOMIC_RELAXED);
  while (nv < prev) {
    if (__atomic_compare_exchange_n(t, &prev, nv, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
  }
}

// align.hpp:205-210
void init_row(const Graph& G, LogScore* row, char b) {
  const int64_t N = (int64_t)G.num_chars();
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < N; ++v) row[v] = match_sub(G.labels[v], b);
}

// align.hpp:245-277
void fused_deletion_substitution(const Graph& G, LogScore* dst, const LogScore* src, char b) {
  const int64_t N = (int64_t)G.num_chars();
#pragma omp parallel for schedule(static, 4096)
  for (int64_t v = 0; v < N; ++v) {
    LogScore best = src[v] + 1;
    const LogScore delta = match_sub(G.labels[v], b);
    for (uint64_t ie = G.in_char.in_offset[v]; ie < G.in_char.in_offset[v + 1]; ++ie) {
      LogScore cand = src[G.in_char.in_u[ie]] + delta;
      if (cand < best) best = cand;
    }
    dst[v] = best;
  }
}

// align.hpp:279-345: per connected component, upward layers with an atomic
// min into T[first(v)] from T[last(u)] + w, then downward layers pulling
// T[last(v)] + w into T[first(u)].
void hierarchy_sweep(const Graph& G, LogScore* T) {
  const Pch& gc = G.gc;
  for (size_t cc = 0; cc + 1 < gc.ccOffset.size(); ++cc) {
    for (uint32_t layer = gc.ccOffset[cc]; layer < gc.ccOffset[cc + 1]; ++layer) {
      const int64_t lo = gc.layerOffset[layer], hi = gc.layerOffset[layer + 1];
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t u = lo; u < hi; ++u) {
        const NodeId uix = G.last(G.contracted_to_og[u]);
        for (uint64_t j = gc.offset[u]; j < gc.offset[u + 1]; ++j) {
          const NodeId vix = G.first(G.contracted_to_og[gc.E_v[j]]);
          cas_min(&T[vix], __atomic_load_n(&T[uix], __ATOMIC_RELAXED) + (LogScore)gc.E_w[j]);
        }
      }
    }
    for (uint32_t layer = gc.ccOffset[cc + 1]; layer-- > gc.ccOffset[cc];) {
      const int64_t lo = gc.layerOffset[layer], hi = gc.layerOffset[layer + 1];
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t u = lo; u < hi; ++u) {
        const NodeId uix = G.first(G.contracted_to_og[u]);
        LogScore t = T[uix];
        for (uint64_t j = gc.in_offset[u]; j < gc.in_offset[u + 1]; ++j) {
          const NodeId vix = G.last(G.contracted_to_og[gc.inE_v[j]]);
          LogScore cand = T[vix] + (LogScore)gc.inE_w[j];
          if (cand < t) t = cand;
        }
        T[uix] = t;
      }
    }
  }
}

// align.hpp:347-397
void insertion(const Graph& G, LogScore* T) {
  const int64_t S = (int64_t)G.str.n;
#pragma omp parallel for schedule(static, 1024)
  for (int64_t u = 0; u < S; ++u)
    for (NodeId v = G.first((NodeId)u); v < G.last((NodeId)u); ++v)
      if (T[v] + 1 < T[v + 1]) T[v + 1] = T[v] + 1;
  hierarchy_sweep(G, T);
#pragma omp parallel for schedule(static, 1024)
  for (int64_t u = 0; u < S; ++u) {
    NodeId v = G.first((NodeId)u), e = G.last((NodeId)u);
    while (v < e) {
      if (T[v] + 1 < T[v + 1]) {
        T[v + 1] = T[v] + 1;
        ++v;
      } else {
        break;
      }
    }
  }
}

// One DP row: align.hpp:436-461.
void dp_row(const Graph& G, LogScore* dst, const LogScore* src, char b) {
  fused_deletion_substitution(G, dst, src, b);
  insertion(G, dst);
}

LogScore row_min(const Graph& G, const LogScore* row, NodeId* arg) {
  // align.hpp:505-513 (value) / traceback.hpp:695-714 (vertex). The
  // reference's per-worker argmin breaks ties arbitrarily; here the smallest
  // index wins.
  LogScore best = std::numeric_limits<LogScore>::max();
  NodeId bv = 0;
  for (size_t v = 0; v < G.num_chars(); ++v)
    if (row[v] < best) {
      best = row[v];
      bv = (NodeId)v;
    }
  if (arg) *arg = bv;
  return best;
}

// traceback.hpp:251-290
void fused_del_sub_with_bp(const Graph& G, LogScore* dst, uint32_t* bp, const LogScore* src, char b) {
  const int64_t N = (int64_t)G.num_chars();
#pragma omp parallel for schedule(static, 4096)
  for (int64_t v = 0; v < N; ++v) {
    LogScore best = src[v] + 1;
    NodeId sv = (NodeId)v;
    uint8_t op = BP_DELETE;
    const LogScore delta = match_sub(G.labels[v], b);
    for (uint64_t ie = G.in_char.in_offset[v]; ie < G.in_char.in_offset[v + 1]; ++ie) {
      NodeId u = G.in_char.in_u[ie];
      LogScore cand = src[u] + delta;
      if (cand < best) {
        best = cand;
        sv = u;
        op = BP_MATCHSUB;
      }
    }
    dst[v] = best;
    bp[v] = (uint32_t(op) << 30) | (sv & 0x3FFFFFFFu);
  }
}

// traceback.hpp:306-337. The reference's parallel second loop lets any
// satisfying edge win; here edges are visited in ascending u and the last
// satisfying one wins.
void compute_insert_bp(const Graph& G, const LogScore* dp, uint32_t* bp) {
  for (NodeId u = 0; u < G.str.n; ++u)
    for (NodeId p = G.first(u); p < G.last(u); ++p)
      if (dp[p + 1] == dp[p] + 1) bp[p + 1] = (uint32_t(BP_INSERT) << 30) | p;
  for (NodeId u = 0; u < G.str.n; ++u) {
    const NodeId ul = G.last(u);
    for (uint64_t e = G.str.off[u]; e < G.str.off[u + 1]; ++e) {
      NodeId vf = G.first(G.str.v[e]);
      if (dp[vf] == dp[ul] + 1) bp[vf] = (uint32_t(BP_INSERT) << 30) | ul;
    }
  }
}

struct Op {
  int64_t row;
  uint32_t vertex;
  uint8_t op;
  uint8_t pad[3];
};

// traceback.hpp:483-586
int walk_from_scores(const Graph& G, const LogScore* all, int64_t len, NodeId best,
                     const char* read, std::vector<Op>& path) {
  const size_t N = G.num_chars();
  auto vertex_of = [&](NodeId p) {
    auto it = std::upper_bound(G.label_offsets.begin(), G.label_offsets.end() - 1, (uint64_t)p);
    return (NodeId)((it - G.label_offsets.begin()) - 1);
  };
  NodeId cur_v = best;
  int64_t cur_row = len - 1;
  while (cur_row > 0) {
    const LogScore* row = all + (size_t)cur_row * N;
    const LogScore* prow = all + (size_t)(cur_row - 1) * N;
    const LogScore s = row[cur_v];
    uint8_t op = 255;
    NodeId src = cur_v;
    const NodeId sv = vertex_of(cur_v);
    if (cur_v > G.first(sv) && row[cur_v - 1] + 1 == s) {
      op = BP_INSERT;
      src = cur_v - 1;
    }
    if (op == 255 && cur_v == G.first(sv)) {
      for (uint64_t ie = G.in_str.in_offset[sv]; ie < G.in_str.in_offset[sv + 1]; ++ie) {
        NodeId ul = G.last(G.in_str.in_u[ie]);
        if (row[ul] + 1 == s) {
          op = BP_INSERT;
          src = ul;
          break;
        }
      }
    }
    if (op == 255 && prow[cur_v] + 1 == s) {
      op = BP_DELETE;
      src = cur_v;
    }
    if (op == 255) {
      const LogScore delta = match_sub(G.labels[cur_v], read[cur_row]);
      for (uint64_t ie = G.in_char.in_offset[cur_v]; ie < G.in_char.in_offset[cur_v + 1]; ++ie) {
        NodeId u = G.in_char.in_u[ie];
        if (prow[u] + delta == s) {
          op = BP_MATCHSUB;
          src = u;
          break;
        }
      }
    }
    if (op == 255) {
      g_err = "score-matrix traceback: no valid predecessor at row " + std::to_string(cur_row) +
              " vertex " + std::to_string(cur_v);
      return 7;
    }
    path.push_back({cur_row, cur_v, op, {0, 0, 0}});
    cur_v = src;
    if (op != BP_INSERT) --cur_row;
  }
  path.push_back({0, cur_v, BP_MATCHSUB, {0, 0, 0}});
  std::reverse(path.begin(), path.end());
  return 0;
}

std::string row_path(const std::string& dir, int64_t row) {
  return dir + "/row_" + std::to_string(row) + ".bin";
}

// traceback.hpp:588-1031. fast_cap_bytes plays FAST_BP_MAX_BYTES.
int traceback(const Graph& G, const char* read, int64_t len, int64_t k, uint64_t fast_cap_bytes,
              const std::string& dir, bool cleanup, std::vector<Op>& path, LogScore* score_out,
              int* checkpointed) {
  const size_t N = G.num_chars();
  const uint64_t store = (uint64_t)len * N * sizeof(LogScore);
  path.clear();
  if (store <= fast_cap_bytes) {
    *checkpointed = 0;
    std::vector<LogScore> all((size_t)len * N);
    init_row(G, all.data(), read[0]);
    for (int64_t i = 1; i < len; ++i)
      dp_row(G, all.data() + (size_t)i * N, all.data() + (size_t)(i - 1) * N, read[i]);
    NodeId best;
    *score_out = row_min(G, all.data() + (size_t)(len - 1) * N, &best);
    return walk_from_scores(G, all.data(), len, best, read, path);
  }
  *checkpointed = 1;
  std::filesystem::create_directories(dir);
  auto save = [&](int64_t row, const LogScore* d) {
    std::ofstream o(row_path(dir, row), std::ios::binary | std::ios::trunc);
    o.write((const char*)d, (std::streamsize)(N * sizeof(LogScore)));
    if (!o) throw std::runtime_error("checkpoint write failed");
  };
  auto load = [&](int64_t row, LogScore* d) {
    std::ifstream f(row_path(dir, row), std::ios::binary);
    f.read((char*)d, (std::streamsize)(N * sizeof(LogScore)));
    if (!f) throw std::runtime_error("checkpoint read failed");
  };
  NodeId best = 0;
  {
    std::vector<LogScore> fwd(2 * N);
    LogScore* prev = fwd.data();
    LogScore* curr = fwd.data() + N;
    init_row(G, prev, read[0]);
    save(0, prev);
    for (int64_t i = 1; i < len; ++i) {
      dp_row(G, curr, prev, read[i]);
      std::swap(prev, curr);
      if (i % k == 0) save(i, prev);
    }
    *score_out = row_min(G, prev, &best);
  }
  const int64_t bp_rows = std::min<int64_t>(k, len);
  std::vector<uint32_t> bp((size_t)bp_rows * N);
  std::vector<LogScore> ck(N), a(N), b(N);
  NodeId cur_v = best;
  int64_t cur_row = len - 1;
  while (cur_row > 0) {
    int64_t seg_start = (cur_row % k == 0) ? (cur_row - k) : (cur_row / k * k);
    if (seg_start < 0) seg_start = 0;
    const int64_t seg_end = cur_row;
    load(seg_start, ck.data());
    // recompute_segment_with_bp, traceback.hpp:352-420
    std::copy(ck.begin(), ck.end(), a.begin());
    LogScore* prev = a.data();
    LogScore* curr = b.data();
    for (int64_t i = seg_start + 1; i <= seg_end; ++i) {
      uint32_t* bpr = bp.data() + (size_t)(i - seg_start - 1) * N;
      fused_del_sub_with_bp(G, curr, bpr, prev, read[i]);
      insertion(G, curr);
      compute_insert_bp(G, curr, bpr);
      std::swap(prev, curr);
    }
    // traceback_segment, traceback.hpp:434-464
    int64_t row = seg_end;
    NodeId v = cur_v;
    while (row > seg_start) {
      uint32_t enc = bp[(size_t)(row - seg_start - 1) * N + v];
      uint8_t op = (uint8_t)(enc >> 30);
      NodeId src = enc & 0x3FFFFFFFu;
      path.push_back({row, v, op, {0, 0, 0}});
      v = src;
      if (op != BP_INSERT) --row;
    }
    if (cleanup && seg_start > 0) std::filesystem::remove(row_path(dir, seg_start));
    cur_v = v;
    cur_row = seg_start;
  }
  path.push_back({0, cur_v, BP_MATCHSUB, {0, 0, 0}});
  if (cleanup) std::filesystem::remove(row_path(dir, 0));
  std::reverse(path.begin(), path.end());
  return 0;
}

template <typename F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    g_err = e.what();
    return 9;
  }
}

}  // namespace

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }

int oracle_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

// Loads the five ConSGA inputs the way src/ConSGA.cpp:154-211 does.
int oracle_load(const char* char_adj, const char* str_adj, const char* pch, const char* labels,
                const char* offsets, void** out) {
  return guarded([&] {
    auto* g = new Graph();
    std::vector<char> lb = slurp(labels);
    for (char c : lb)
      if (c != '\n') g->labels.push_back(c);
    {
      std::ifstream f(offsets);
      if (!f) throw std::runtime_error(std::string("cannot open ") + offsets);
      uint64_t o;
      while (f >> o) g->label_offsets.push_back(o);
    }
    Csr cg = read_adj(char_adj);
    g->in_char = build_in_csr(cg);
    g->str = read_adj(str_adj);
    g->in_str = build_in_csr(g->str);
    g->gc = read_pch(pch);
    g->contracted_to_og.resize(g->gc.n);
    for (uint64_t i = 0; i < g->gc.n; ++i) g->contracted_to_og[g->gc.rank[i]] = (NodeId)i;
    if (cg.n != g->labels.size() || g->label_offsets.size() != g->str.n + 1 || g->gc.n != g->str.n)
      throw std::runtime_error("inconsistent inputs");
    *out = g;
    return 0;
  });
}

void oracle_free(void* h) { delete (Graph*)h; }

uint64_t oracle_num_chars(void* h) { return ((Graph*)h)->num_chars(); }

// align_combo (align.hpp:470-531): min over the final row of each read.
int oracle_align_scores(void* h, const char* data, const uint64_t* offs, uint64_t n, int32_t* out) {
  return guarded([&] {
    const Graph& G = *(Graph*)h;
    const size_t N = G.num_chars();
    std::vector<LogScore> buf(2 * N);
    for (uint64_t r = 0; r < n; ++r) {
      const char* rd = data + offs[r];
      const int64_t len = (int64_t)(offs[r + 1] - offs[r]);
      LogScore* src = buf.data();
      LogScore* dst = buf.data() + N;
      init_row(G, src, len > 0 ? rd[0] : '\0');
      for (int64_t i = 1; i < len; ++i) {
        dp_row(G, dst, src, rd[i]);
        std::swap(src, dst);
      }
      out[r] = row_min(G, src, nullptr);
    }
    return 0;
  });
}

// Every final row of one read, len x N.
int oracle_align_rows(void* h, const char* rd, uint64_t len, int32_t* rows) {
  return guarded([&] {
    const Graph& G = *(Graph*)h;
    const size_t N = G.num_chars();
    init_row(G, rows, rd[0]);
    for (uint64_t i = 1; i < len; ++i) dp_row(G, rows + i * N, rows + (i - 1) * N, rd[i]);
    return 0;
  });
}

// align_read_with_traceback. ops are written to ops_out (capacity cap,
// 16-byte records matching chsga_op); *nops receives the path length.
int oracle_traceback(void* h, const char* rd, uint64_t len, int64_t k, uint64_t fast_cap_bytes,
                     const char* dir, int cleanup, void* ops_out, uint64_t cap, uint64_t* nops,
                     int32_t* score, int* checkpointed) {
  return guarded([&] {
    const Graph& G = *(Graph*)h;
    std::vector<Op> path;
    int rc = traceback(G, rd, (int64_t)len, k, fast_cap_bytes, dir ? dir : "/tmp/consga_oracle_ckpt",
                       cleanup != 0, path, score, checkpointed);
    *nops = path.size();
    if (rc == 0 && ops_out) std::memcpy(ops_out, path.data(), std::min<uint64_t>(cap, path.size()) * sizeof(Op));
    return rc;
  });
}

// Exact DP on the char graph (restating serial_align_CSR,
// csr_align.hpp:270-383, DAG branch): a single pass in char-id order
// relaxes T[v] from T[u] + 1 along every char edge. Exact when char ids are
// topologically ordered. A diagnostic, not the parity target.
int oracle_exact_scores(void* h, const char* data, const uint64_t* offs, uint64_t n, int32_t* out) {
  return guarded([&] {
    const Graph& G = *(Graph*)h;
    const size_t N = G.num_chars();
    std::vector<LogScore> a(N), b(N);
    for (uint64_t r = 0; r < n; ++r) {
      const char* rd = data + offs[r];
      const uint64_t len = offs[r + 1] - offs[r];
      for (size_t v = 0; v < N; ++v) a[v] = match_sub(G.labels[v], rd[0]);
      for (uint64_t i = 1; i < len; ++i) {
        for (size_t v = 0; v < N; ++v) {
          LogScore best = a[v] + 1;
          const LogScore d = match_sub(G.labels[v], rd[i]);
          for (uint64_t ie = G.in_char.in_offset[v]; ie < G.in_char.in_offset[v + 1]; ++ie)
            best = std::min(best, a[G.in_char.in_u[ie]] + d);
          b[v] = best;
        }
        for (size_t v = 0; v < N; ++v)
          for (uint64_t ie = G.in_char.in_offset[v]; ie < G.in_char.in_offset[v + 1]; ++ie)
            b[v] = std::min(b[v], b[G.in_char.in_u[ie]] + 1);
        std::swap(a, b);
      }
      out[r] = *std::min_element(a.begin(), a.end());
    }
    return 0;
  });
}

}  // extern "C"
