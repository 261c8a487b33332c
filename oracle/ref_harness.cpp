// ORACLE HARNESS — test infrastructure, not product code.
//
// C entry points around the reference's OWN alignment code: this file
// includes src/traceback.hpp (which includes src/align.hpp) from the
// reference tree, compiled by oracle/Makefile against the stand-ins in
// oracle/ref_shim/. Tests use it to pin the restatement in
// consga_oracle.cpp and the GPU path; the benchmark's reference arm times it.
// Built twice: with the reference's default fast-path cap (full score matrix,
// traceback.hpp:614-618) and with FAST_BP_MAX_BYTES_OVERRIDE=0, which forces
// the checkpointed path (traceback.hpp:845-1030).
#include "traceback.hpp"

#include <memory>
#include <sstream>

namespace {

struct RefInputs {
  std::vector<char> labels;
  std::vector<size_t> offsets;
  Graph char_graph;
  InCSR in_char;
  Graph str_graph;
  PchGraph pch;
  std::unique_ptr<PchQuery> query;
  sequence<NodeId> to_og;
  std::unique_ptr<VertexLabelMapper<true>> mapper;
};

std::string g_err;

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

int ref_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

// The loading steps of src/ConSGA.cpp:154-211.
int ref_load(const char* char_adj, const char* str_adj, const char* pch, const char* labels,
             const char* offsets, void** out) {
  try {
    auto* r = new RefInputs();
    {
      std::ifstream ifs(labels);
      char ch;
      while (ifs.get(ch))
        if (ch != '\n') r->labels.push_back(ch);
    }
    {
      std::ifstream ifs(offsets);
      size_t off;
      while (ifs >> off) r->offsets.push_back(off);
    }
    r->char_graph = read_graph(char_adj);
    r->in_char = build_in_csr_from(r->char_graph);
    r->str_graph = read_graph(str_adj);
    read_contracted_graph(pch, r->pch);
    r->query = std::make_unique<PchQuery>(r->pch, r->str_graph);
    r->to_og.resize(r->pch.n);
    for (size_t i = 0; i < r->pch.n; ++i) r->to_og[r->pch.rank[i]] = (NodeId)i;
    r->mapper = std::make_unique<VertexLabelMapper<true>>(r->offsets);
    *out = r;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 9;
  }
}

void ref_free(void* h) { delete (RefInputs*)h; }

// align_combo<int> (align.hpp:470-531). Its timing report goes to stdout.
int ref_align_scores(void* h, const char* data, const uint64_t* offs, uint64_t n, int32_t* out) {
  auto* r = (RefInputs*)h;
  std::vector<std::string> reads;
  for (uint64_t i = 0; i < n; ++i) reads.emplace_back(data + offs[i], offs[i + 1] - offs[i]);
  std::streambuf* old = std::cout.rdbuf();
  std::ostringstream sink;
  std::cout.rdbuf(sink.rdbuf());
  std::vector<int> s = align_combo(reads, r->labels, r->in_char, r->str_graph, r->to_og, 0, 1, 1,
                                   1, *r->query, *r->mapper);
  std::cout.rdbuf(old);
  for (uint64_t i = 0; i < n; ++i) out[i] = s[i];
  return 0;
}

// Every final row of one read, driving the reference's own row functions in
// the order align_read_combo uses them (align.hpp:421-462).
int ref_align_rows(void* h, const char* rd, uint64_t len, int32_t* rows) {
  auto* r = (RefInputs*)h;
  const size_t N = r->labels.size();
  init_func_parallel<int>(rows, r->labels, rd[0], N, 0, 1);
  for (uint64_t i = 1; i < len; ++i) {
    fused_deletion_substitution<int, VertexLabelMapper<false>>(rows + i * N, rows + (i - 1) * N,
                                                                r->labels, r->in_char, rd[i], 0, 1,
                                                                1, N);
    insertion_func_parallel<int, VertexLabelMapper<true>>(rows + i * N, r->str_graph, r->to_og, 1,
                                                           *r->query, *r->mapper);
  }
  return 0;
}

// Rows want[0] < want[1] < ... of one read, from the same row functions in
// the same order as ref_align_rows, keeping two rows in memory instead of
// len (for graphs whose full matrix does not fit host memory).
int ref_rows_at(void* h, const char* rd, uint64_t len, const uint64_t* want, uint64_t nwant,
                int32_t* out) {
  auto* r = (RefInputs*)h;
  const size_t N = r->labels.size();
  std::vector<int32_t> a(N), b(N);
  int32_t* prev = a.data();
  int32_t* cur = b.data();
  uint64_t w = 0;
  init_func_parallel<int>(prev, r->labels, rd[0], N, 0, 1);
  if (w < nwant && want[w] == 0) std::copy(prev, prev + N, out + (w++) * N);
  for (uint64_t i = 1; i < len && w < nwant; ++i) {
    fused_deletion_substitution<int, VertexLabelMapper<false>>(cur, prev, r->labels, r->in_char, rd[i],
                                                                0, 1, 1, N);
    insertion_func_parallel<int, VertexLabelMapper<true>>(cur, r->str_graph, r->to_og, 1, *r->query,
                                                           *r->mapper);
    if (want[w] == i) std::copy(cur, cur + N, out + (w++) * N);
    std::swap(prev, cur);
  }
  return w == nwant ? 0 : 1;
}

// align_read_with_traceback<int> (traceback.hpp:588-1031). ops: 16-byte
// records {int64 row, uint32 vertex, uint8 op, pad}.
int ref_traceback(void* h, const char* rd, uint64_t len, int64_t k, const char* dir, int cleanup,
                  void* ops_out, uint64_t cap, uint64_t* nops) {
  auto* r = (RefInputs*)h;
  try {
    CheckpointConfig cfg;
    cfg.k = k;
    cfg.dir = dir;
    cfg.cleanup = cleanup != 0;
    std::string read(rd, len);
    std::vector<AlignOp> path = align_read_with_traceback<int>(
        read, r->labels.size(), r->labels, r->in_char, r->str_graph, r->to_og, 0, 1, 1, 1,
        *r->query, *r->mapper, cfg);
    *nops = path.size();
    struct Rec {
      int64_t row;
      uint32_t vertex;
      uint8_t op;
      uint8_t pad[3];
    };
    Rec* o = (Rec*)ops_out;
    for (uint64_t i = 0; i < std::min<uint64_t>(cap, path.size()); ++i)
      o[i] = Rec{path[i].row, path[i].vertex, path[i].op, {0, 0, 0}};
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 7;
  }
}

// The reference's exact DP, serial_align_CSR (csr_align.hpp:270-383), over
// the char graph's out-CSR.
int ref_exact_scores(void* h, const char* data, const uint64_t* offs, uint64_t n, int32_t* out) {
  auto* r = (RefInputs*)h;
  std::vector<std::string> reads;
  for (uint64_t i = 0; i < n; ++i) reads.emplace_back(data + offs[i], offs[i + 1] - offs[i]);
  std::vector<int> off(r->char_graph.n + 1), edges(r->char_graph.m);
  for (size_t i = 0; i <= r->char_graph.n; ++i) off[i] = (int)r->char_graph.offset[i];
  for (size_t e = 0; e < r->char_graph.m; ++e) edges[e] = (int)r->char_graph.E[e].v;
  std::vector<double> times[NUM_OPERATIONS];
  std::vector<int> s = serial_align_CSR<int>(reads, (int)r->char_graph.n, r->labels, off, edges, 0,
                                             1, 1, 1, times);
  for (uint64_t i = 0; i < n; ++i) out[i] = s[i];
  return 0;
}

}  // extern "C"
