// extern "C" entry points that need no GPU: loading, generating and writing
// the alignment inputs, and building the contraction hierarchy.
#include <algorithm>
#include <cstring>
#include <memory>
#include <new>

#include "device_graph.hpp"
#include "host_graph.hpp"

namespace chsga {
HostPch build_pch(const HostCsr& g, const std::vector<uint64_t>& offs, const chsga_pch_opts& o);
void generate_graph(const chsga_gen_graph_cfg& c, chsga_host_graph& out);
void generate_reads(const chsga_host_graph& g, const chsga_gen_reads_cfg& c, HostReads& out);

thread_local std::string g_last_error;

template <typename F>
chsga_status guarded(F&& f) {
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

// Consistency checks shared by file loading and chsga_load_graph.
void validate_host_graph(const chsga_host_graph& g) {
  const uint64_t N = g.labels.size();
  require(N > 0, CHSGA_ERR_FORMAT, "labels file is empty");
  require(g.char_graph.n == N, CHSGA_ERR_FORMAT,
          "char graph has " + std::to_string(g.char_graph.n) + " vertices but labels has " +
              std::to_string(N) + " chars");
  const uint64_t S = g.string_graph.n;
  require(g.label_offsets.size() == S + 1, CHSGA_ERR_FORMAT,
          "label offsets has " + std::to_string(g.label_offsets.size()) + " entries, expected " +
              std::to_string(S + 1));
  require(g.label_offsets[0] == 0 && g.label_offsets[S] == N, CHSGA_ERR_FORMAT,
          "label offsets must run from 0 to the number of labels");
  for (uint64_t s = 0; s < S; ++s)
    if (g.label_offsets[s] >= g.label_offsets[s + 1])
      fail(CHSGA_ERR_UNSUPPORTED, "string vertex " + std::to_string(s) + " has an empty label");
  require(g.pch.present, CHSGA_ERR_FORMAT, "no hierarchy attached");
  validate_pch(g.pch, S);
}

}  // namespace chsga

using namespace chsga;

extern "C" {

const char* chsga_last_error_global(void) { return g_last_error.c_str(); }

chsga_status chsga_graph_read_files(const char* char_adj, const char* string_adj,
                                    const char* pch_file, const char* labels_file,
                                    const char* label_offsets_file, chsga_host_graph** out) {
  return guarded([&] {
    require(char_adj && string_adj && pch_file && labels_file && label_offsets_file && out,
            CHSGA_ERR_INVALID_ARG, "null argument");
    auto g = std::make_unique<chsga_host_graph>();
    g->labels = read_labels(labels_file);
    g->label_offsets = read_label_offsets(label_offsets_file);
    g->char_graph = read_adj(char_adj);
    g->string_graph = read_adj(string_adj);
    g->pch = read_pch(pch_file);
    validate_host_graph(*g);
    *out = g.release();
  });
}

chsga_status chsga_graph_view(const chsga_host_graph* g, chsga_graph_host* v) {
  return guarded([&] {
    require(g && v, CHSGA_ERR_INVALID_ARG, "null argument");
    std::memset(v, 0, sizeof(*v));
    v->num_chars = g->labels.size();
    v->labels = g->labels.data();
    auto csr = [](const HostCsr& c, chsga_csr& o) {
      o.n = c.n;
      o.m = c.m;
      o.offset = c.offset.data();
      o.target = c.target.data();
      o.weight = c.weight.empty() ? nullptr : c.weight.data();
    };
    csr(g->char_graph, v->char_graph);
    csr(g->string_graph, v->string_graph);
    v->label_offsets = g->label_offsets.data();
    const HostPch& p = g->pch;
    if (p.present) {
      v->pch.n = p.n;
      v->pch.m = p.m;
      v->pch.rm = p.rm;
      v->pch.num_layers = p.layer_offset.size() - 1;
      v->pch.num_cc = p.cc_offset.size() - 1;
      v->pch.rank = p.rank.data();
      v->pch.level = p.level.data();
      v->pch.layer_offset = p.layer_offset.data();
      v->pch.cc_offset = p.cc_offset.data();
      v->pch.up_offset = p.up_offset.data();
      v->pch.up_v = p.up_v.data();
      v->pch.up_w = p.up_w.data();
      v->pch.down_offset = p.down_offset.data();
      v->pch.down_v = p.down_v.data();
      v->pch.down_w = p.down_w.data();
    }
  });
}

void chsga_graph_free(chsga_host_graph* g) { delete g; }

chsga_status chsga_graph_write_files(const chsga_host_graph* g, const char* prefix) {
  return guarded([&] {
    require(g && prefix, CHSGA_ERR_INVALID_ARG, "null argument");
    std::string p(prefix);
    write_adj(p + ".char.adj", g->char_graph);
    write_adj(p + ".string.adj", g->string_graph);
    write_labels(p + ".char.labels", g->labels);
    write_label_offsets(p + ".string.label_offsets", g->label_offsets);
    if (g->pch.present) write_pch(p + ".string.out", g->pch);
  });
}

chsga_status chsga_gen_graph(const chsga_gen_graph_cfg* cfg, chsga_host_graph** out) {
  return guarded([&] {
    require(cfg && out, CHSGA_ERR_INVALID_ARG, "null argument");
    auto g = std::make_unique<chsga_host_graph>();
    generate_graph(*cfg, *g);
    *out = g.release();
  });
}

chsga_status chsga_build_pch(chsga_host_graph* g, const chsga_pch_opts* opts) {
  return guarded([&] {
    require(g != nullptr, CHSGA_ERR_INVALID_ARG, "null graph");
    chsga_pch_opts o{};
    o.max_pop_count = 500;
    o.sample_bound = 1.0;
    o.use_label_lengths = 1;
    if (opts) o = *opts;
    g->pch = build_pch(g->string_graph, g->label_offsets, o);
  });
}

chsga_status chsga_reads_load(const char* path, uint64_t max_reads, chsga_reads** out) {
  return guarded([&] {
    require(path && out, CHSGA_ERR_INVALID_ARG, "null argument");
    auto r = std::make_unique<chsga_reads>();
    r->r = read_reads(path, max_reads);
    *out = r.release();
  });
}

chsga_status chsga_reads_from_arrays(const char* data, const uint64_t* offsets, uint64_t n,
                                     chsga_reads** out) {
  return guarded([&] {
    require(offsets && out && (data || offsets[n] == 0), CHSGA_ERR_INVALID_ARG, "null argument");
    auto r = std::make_unique<chsga_reads>();
    for (uint64_t i = 0; i < n; ++i) {
      require(offsets[i] <= offsets[i + 1], CHSGA_ERR_INVALID_ARG, "read offsets decrease");
      r->r.add(data + offsets[i], offsets[i + 1] - offsets[i]);
    }
    *out = r.release();
  });
}

uint64_t chsga_reads_count(const chsga_reads* r) { return r ? r->r.count() : 0; }
const char* chsga_reads_data(const chsga_reads* r) { return r ? r->r.data.data() : nullptr; }
const uint64_t* chsga_reads_offsets(const chsga_reads* r) {
  return r ? r->r.offsets.data() : nullptr;
}

chsga_status chsga_reads_write_fasta(const chsga_reads* r, const char* path) {
  return guarded([&] {
    require(r && path, CHSGA_ERR_INVALID_ARG, "null argument");
    write_fasta(path, r->r);
  });
}

void chsga_reads_free(chsga_reads* r) { delete r; }

chsga_status chsga_gen_reads(const chsga_host_graph* g, const chsga_gen_reads_cfg* cfg,
                             chsga_reads** out) {
  return guarded([&] {
    require(g && cfg && out, CHSGA_ERR_INVALID_ARG, "null argument");
    auto r = std::make_unique<chsga_reads>();
    generate_reads(*g, *cfg, r->r);
    *out = r.release();
  });
}

chsga_status chsga_check_layout(const chsga_host_graph* g, uint32_t slots, uint32_t row_bits,
                                uint32_t top_vertices,
                                chsga_layout_stats* out) {
  return guarded([&] {
    require(g && out, CHSGA_ERR_INVALID_ARG, "null argument");
    require(row_bits == 16 || row_bits == 32, CHSGA_ERR_INVALID_ARG, "row_bits must be 16 or 32");
    validate_host_graph(*g);
    chsga_graph_host v{};
    require(chsga_graph_view(g, &v) == CHSGA_OK, CHSGA_ERR_INTERNAL, "graph view");
    HostLayout L = build_layout(v);
    std::memset(out, 0, sizeof(*out));
    out->num_levels = L.levels;
    require(top_vertices <= kTopMaxVertices, CHSGA_ERR_INVALID_ARG,
            "top_vertices above " + std::to_string(kTopMaxVertices));
    HostTop top = build_top(L, top_vertices ? top_vertices : kTopDefaultVertices, 1024);
    out->top_first_level = top.first_level;
    out->top_vertices = top.K;
    for (uint32_t d = 0; d < top.K0; ++d) {
      const uint32_t nu = L.up_off[d + 1] - L.up_off[d], nd = L.dn_off[d + 1] - L.dn_off[d];
      out->sweep_up_targets += nu > 0;
      out->sweep_up_edges += nu;
      out->sweep_down_targets += nd > 0;
      out->sweep_down_edges += nd;
    }
    if (slots >= 32) {
      HostRowTiles t = build_row_tiles(L, slots, row_bits / 8);
      validate_row_tiles(L, slots, row_bits / 8, t);
      out->tiled = t.ok ? 1 : 0;
      out->tiles = t.ntiles();
      out->long_tiles = t.long_tiles;
      out->slot_bytes = t.slot_bytes();
      out->slots_per_block = t.nslots;
      out->smem_bytes = t.ok ? row_tiled_smem(t, slots) : 0;
    }
  });
}

chsga_status chsga_graph_get_stats(const chsga_host_graph* g, chsga_graph_stats* s) {
  return guarded([&] {
    require(g && s, CHSGA_ERR_INVALID_ARG, "null argument");
    std::memset(s, 0, sizeof(*s));
    s->num_chars = g->labels.size();
    s->num_char_edges = g->char_graph.m;
    s->num_strings = g->string_graph.n;
    s->num_string_edges = g->string_graph.m;
    for (uint64_t i = 0; i + 1 < g->label_offsets.size(); ++i) {
      uint64_t l = g->label_offsets[i + 1] - g->label_offsets[i];
      s->max_label_len = std::max(s->max_label_len, l);
      s->single_char_strings += (l == 1);
    }
    if (g->pch.present) {
      s->pch_up_edges = g->pch.m;
      s->pch_down_edges = g->pch.rm;
      s->pch_layers = g->pch.layer_offset.size() - 1;
      s->pch_ccs = g->pch.cc_offset.size() - 1;
      uint32_t mx = 0;
      for (uint32_t l : g->pch.level) mx = std::max(mx, l);
      s->pch_levels = mx;
    }
  });
}

}  // extern "C"
