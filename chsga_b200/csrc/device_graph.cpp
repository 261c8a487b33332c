// Host-side construction of the device layout (see device_graph.hpp), with
// the structural checks the GPU path relies on.
#include <algorithm>
#include <numeric>

#include "device_graph.hpp"

namespace chsga {

namespace {
int base_code(unsigned char c) {
  switch (c) {
    case 'A': return 0;
    case 'C': return 1;
    case 'G': return 2;
    case 'T': return 3;
    default: return -1;
  }
}
}  // namespace

HostLayout build_layout(const chsga_graph_host& g) {
  HostLayout L;
  require(g.labels && g.label_offsets && g.char_graph.offset && g.string_graph.offset,
          CHSGA_ERR_INVALID_ARG, "graph arrays missing");
  const uint64_t N64 = g.num_chars, S64 = g.string_graph.n;
  require(N64 > 0 && S64 > 0, CHSGA_ERR_INVALID_ARG, "empty graph");
  require(N64 < (1ull << 31) && S64 < (1ull << 30), CHSGA_ERR_UNSUPPORTED,
          "graph too large: chars must be < 2^31 and string vertices < 2^30");
  require(g.char_graph.n == N64, CHSGA_ERR_FORMAT, "char graph size differs from label count");
  require(g.label_offsets[0] == 0 && g.label_offsets[S64] == N64, CHSGA_ERR_FORMAT,
          "label offsets must run from 0 to the number of labels");
  const uint32_t N = (uint32_t)N64, S = (uint32_t)S64;
  L.N = N;
  L.S = S;
  // Every per-element check below keeps the first offending element (a min
  // over the parallel loop), so errors name what a sequential pass would.
  constexpr uint64_t kNone = ~0ull;

  // --- labels: 2-bit code plus one "special" byte class --------------------
  // the special byte is the first label byte outside A/C/G/T
  uint64_t first_sp = kNone;
#pragma omp parallel for reduction(min : first_sp) schedule(static)
  for (int64_t c = 0; c < (int64_t)N; ++c)
    if (base_code((unsigned char)g.labels[c]) < 0) first_sp = std::min(first_sp, (uint64_t)c);
  if (first_sp != kNone) L.special = (unsigned char)g.labels[first_sp];
  L.lab2.assign((N + 15) / 16, 0);
  L.lab_sp.assign((N + 31) / 32, 0);
  L.lab4.assign((N + 7) / 8 + 3, 0);  // three spare words: the key window reads two words ahead
  uint64_t bad_sp = kNone;
  const int64_t words = (N + 31) / 32;
#pragma omp parallel for reduction(min : bad_sp) schedule(static)
  for (int64_t w = 0; w < words; ++w) {
    // chars [32w, 32w + 32): one lab_sp word, two lab2 words, four lab4 words
    const uint32_t c1 = std::min<uint32_t>(N, (uint32_t)(32 * w + 32));
    for (uint32_t c = (uint32_t)(32 * w); c < c1; ++c) {
      const unsigned char ch = (unsigned char)g.labels[c];
      int code = base_code(ch);
      uint32_t key;
      if (code < 0) {
        if ((int)ch != L.special) bad_sp = std::min(bad_sp, (uint64_t)c);
        L.lab_sp[c >> 5] |= 1u << (c & 31);
        code = 0;
        key = 4u;
      } else {
        key = (uint32_t)code;
      }
      L.lab2[c >> 4] |= (uint32_t)code << ((c & 15) * 2);
      L.lab4[c >> 3] |= key << ((c & 7) * 4);
    }
  }
  if (bad_sp != kNone)
    fail(CHSGA_ERR_UNSUPPORTED, std::string("labels use more than one byte outside A/C/G/T ('") +
                                    (char)L.special + "' and '" + (char)g.labels[bad_sp] + "')");

  // --- string vertices and the char graph -----------------------------------
  L.sv_off.resize(S + 1);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s <= (int64_t)S; ++s) L.sv_off[s] = (uint32_t)g.label_offsets[s];
  std::vector<uint32_t> vertex_of(N);
  uint64_t empty_s = kNone;
  uint32_t max_len = 0;
#pragma omp parallel for reduction(min : empty_s) reduction(max : max_len) schedule(static)
  for (int64_t s = 0; s < (int64_t)S; ++s) {
    if (L.sv_off[s] >= L.sv_off[s + 1]) {
      empty_s = std::min(empty_s, (uint64_t)s);
      continue;
    }
    max_len = std::max(max_len, L.sv_off[s + 1] - L.sv_off[s]);
    for (uint32_t c = L.sv_off[s]; c < L.sv_off[s + 1]; ++c) vertex_of[c] = (uint32_t)s;
  }
  if (empty_s != kNone)
    fail(CHSGA_ERR_UNSUPPORTED, "string vertex " + std::to_string(empty_s) + " has an empty label");
  require(max_len < (1u << 29), CHSGA_ERR_UNSUPPORTED, "string vertex labels must be shorter than 2^29 chars");
  L.max_len = max_len;
  const chsga_csr& cg = g.char_graph;
  // in-CSR with sources in ascending order, as build_in_csr (align.hpp:220-242):
  // counted and placed in parallel, then each target's sources sorted
  std::vector<uint64_t> ioff(N + 1, 0);
  uint64_t bad_t = 0;
#pragma omp parallel for reduction(+ : bad_t) schedule(dynamic, 1 << 14)
  for (int64_t u = 0; u < (int64_t)N; ++u)
    for (uint64_t e = cg.offset[u]; e < cg.offset[u + 1]; ++e) {
      if (cg.target[e] >= N) {
        ++bad_t;
        continue;
      }
      __atomic_fetch_add(&ioff[cg.target[e] + 1], 1ull, __ATOMIC_RELAXED);
    }
  require(bad_t == 0, CHSGA_ERR_FORMAT, "char edge target out of range");
  for (uint32_t v = 0; v < N; ++v) ioff[v + 1] += ioff[v];
  std::vector<uint32_t> isrc(ioff[N]);
  {
    std::vector<uint64_t> cur(ioff.begin(), ioff.end() - 1);
#pragma omp parallel for schedule(dynamic, 1 << 14)
    for (int64_t u = 0; u < (int64_t)N; ++u)
      for (uint64_t e = cg.offset[u]; e < cg.offset[u + 1]; ++e)
        isrc[__atomic_fetch_add(&cur[cg.target[e]], 1ull, __ATOMIC_RELAXED)] = (uint32_t)u;
#pragma omp parallel for schedule(dynamic, 1 << 14)
    for (int64_t v = 0; v < (int64_t)N; ++v)
      if (ioff[v + 1] - ioff[v] > 1) std::sort(isrc.begin() + ioff[v], isrc.begin() + ioff[v + 1]);
  }
  L.char_in_edges = ioff[N];
  L.vin_off.assign(S + 1, 0);
  uint64_t bad_chain = kNone;
#pragma omp parallel for reduction(min : bad_chain) schedule(static)
  for (int64_t s = 0; s < (int64_t)S; ++s) {
    const uint32_t f = L.sv_off[s], e = L.sv_off[s + 1];
    for (uint32_t c = f + 1; c < e; ++c)
      if (!(ioff[c + 1] - ioff[c] == 1 && isrc[ioff[c]] == c - 1)) {
        bad_chain = std::min(bad_chain, (uint64_t)c);
        break;
      }
    L.vin_off[s + 1] = (uint32_t)(ioff[f + 1] - ioff[f]);
  }
  if (bad_chain != kNone)
    fail(CHSGA_ERR_UNSUPPORTED,
         "char " + std::to_string(bad_chain) + " is not the chain successor of char " +
             std::to_string(bad_chain - 1) +
             ": the char graph must be the expansion of the string graph "
             "(every char after the first of a string has the single in-edge c-1 -> c)");
  for (uint32_t s = 0; s < S; ++s) L.vin_off[s + 1] += L.vin_off[s];
  L.vin_src.resize(L.vin_off[S]);
  L.vin_srcv.resize(L.vin_off[S]);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < (int64_t)S; ++s) {
    const uint32_t f = L.sv_off[s];
    for (uint64_t k = 0; k < ioff[f + 1] - ioff[f]; ++k) {
      uint32_t u = isrc[ioff[f] + k];
      L.vin_src[L.vin_off[s] + k] = u;
      L.vin_srcv[L.vin_off[s] + k] = vertex_of[u];
    }
  }

  // --- hierarchy order -------------------------------------------------------
  const chsga_pch& p = g.pch;
  require(p.n == S && p.rank && p.level && p.layer_offset && p.cc_offset && p.up_offset &&
              p.down_offset,
          CHSGA_ERR_FORMAT, "hierarchy missing or of the wrong size");
  std::vector<uint32_t> og(S);
  {
    std::vector<uint8_t> seen(S, 0);
    for (uint32_t s = 0; s < S; ++s) {
      require(p.rank[s] < S && !seen[p.rank[s]], CHSGA_ERR_FORMAT, "hierarchy rank is not a permutation");
      seen[p.rank[s]] = 1;
      og[p.rank[s]] = s;
    }
  }
  // layer and component of each rank, and the level checks
  std::vector<uint32_t> cc_of(S), layer_of(S);
  require(p.num_cc >= 1 && p.cc_offset[0] == 0 && p.cc_offset[p.num_cc] == p.num_layers &&
              p.layer_offset[0] == 0 && p.layer_offset[p.num_layers] == S,
          CHSGA_ERR_FORMAT, "hierarchy layer/component offsets do not cover the vertices");
  for (uint64_t cc = 0; cc < p.num_cc; ++cc) {
    uint32_t prev_level = 0;
    for (uint32_t l = p.cc_offset[cc]; l < p.cc_offset[cc + 1]; ++l) {
      require(p.layer_offset[l] <= p.layer_offset[l + 1], CHSGA_ERR_FORMAT, "layer offsets decrease");
      for (uint32_t r = p.layer_offset[l]; r < p.layer_offset[l + 1]; ++r) {
        cc_of[r] = (uint32_t)cc;
        layer_of[r] = l;
        require(p.level[r] == p.level[p.layer_offset[l]], CHSGA_ERR_UNSUPPORTED,
                "a hierarchy layer mixes levels");
      }
      if (p.layer_offset[l] < p.layer_offset[l + 1]) {
        uint32_t lv = p.level[p.layer_offset[l]];
        require(l == p.cc_offset[cc] || lv > prev_level, CHSGA_ERR_UNSUPPORTED,
                "hierarchy layers of a component must have increasing levels");
        prev_level = lv;
      }
    }
  }
  // ranks in (level, rank) order: a stable counting sort by level
  std::vector<uint32_t> order(S);
  {
    uint32_t max_level = 0;
    for (uint32_t r = 0; r < S; ++r) max_level = std::max(max_level, p.level[r]);
    require(max_level < (1u << 24), CHSGA_ERR_UNSUPPORTED, "hierarchy levels above 2^24");
    std::vector<uint32_t> at((size_t)max_level + 2, 0);
    for (uint32_t r = 0; r < S; ++r) ++at[p.level[r] + 1];
    for (size_t l = 1; l < at.size(); ++l) at[l] += at[l - 1];
    for (uint32_t r = 0; r < S; ++r) order[at[p.level[r]]++] = r;
  }
  std::vector<uint32_t> dev(S);
  for (uint32_t d = 0; d < S; ++d) dev[order[d]] = d;
  L.dv_first.resize(S);
  L.dv_len.resize(S);
  L.dv_s.resize(S);
#pragma omp parallel for schedule(static)
  for (int64_t d = 0; d < (int64_t)S; ++d) {
    uint32_t s = og[order[d]];
    L.dv_first[d] = L.sv_off[s];
    L.dv_len[d] = L.sv_off[s + 1] - L.sv_off[s];
    L.dv_s[d] = s;
  }
  L.sv_dev.resize(S);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < (int64_t)S; ++s) L.sv_dev[s] = dev[p.rank[s]];
  // a first char's in-edges come from last chars (the string expansion); the
  // row kernels read those sources' final scores from the per-vertex array
  uint64_t bad_vin = kNone;
#pragma omp parallel for reduction(min : bad_vin) schedule(static)
  for (int64_t k = 0; k < (int64_t)L.vin_src.size(); ++k)
    if (L.vin_src[k] + 1 != L.sv_off[L.vin_srcv[k] + 1]) bad_vin = std::min(bad_vin, (uint64_t)k);
  if (bad_vin != kNone)
    fail(CHSGA_ERR_UNSUPPORTED,
         "char " + std::to_string(L.vin_src[bad_vin]) +
             " has an edge to the first char of another string but is not the last char of "
             "its own string: the char graph must be the expansion of the string graph");
  auto bv_last = [&](uint32_t rank) { return 2 * dev[rank] + (L.dv_len[dev[rank]] > 1 ? 1 : 0); };
  // pull lists, by target in hierarchy order; each list in the order of its
  // sources' ranks and of their edges (two passes: count, then fill)
  L.up_off.assign(S + 1, 0);
  L.dn_off.assign(S + 1, 0);
  for (uint32_t u = 0; u < S; ++u) {
    for (uint64_t j = p.up_offset[u]; j < p.up_offset[u + 1]; ++j) {
      const uint32_t v = p.up_v[j];
      require(v < S, CHSGA_ERR_FORMAT, "hierarchy edge out of range");
      require(cc_of[v] == cc_of[u] && layer_of[v] > layer_of[u], CHSGA_ERR_UNSUPPORTED,
              "upward hierarchy edge does not climb to a later layer of its component");
      require(p.up_w[j] >= 1 && p.up_w[j] <= (1u << 30), CHSGA_ERR_UNSUPPORTED,
              "hierarchy weights must be in [1, 2^30]");
      ++L.up_off[dev[v] + 1];
    }
    for (uint64_t j = p.down_offset[u]; j < p.down_offset[u + 1]; ++j) {
      const uint32_t v = p.down_v[j];
      require(v < S, CHSGA_ERR_FORMAT, "hierarchy edge out of range");
      require(cc_of[v] == cc_of[u] && layer_of[v] > layer_of[u], CHSGA_ERR_UNSUPPORTED,
              "downward hierarchy edge does not come from a later layer of its component");
      require(p.down_w[j] >= 1 && p.down_w[j] <= (1u << 30), CHSGA_ERR_UNSUPPORTED,
              "hierarchy weights must be in [1, 2^30]");
    }
    L.dn_off[dev[u] + 1] += (uint32_t)(p.down_offset[u + 1] - p.down_offset[u]);
  }
  for (uint32_t d = 0; d < S; ++d) {
    L.up_off[d + 1] += L.up_off[d];
    L.dn_off[d + 1] += L.dn_off[d];
  }
  L.up_in.resize(L.up_off[S]);
  L.dn_in.resize(L.dn_off[S]);
  {
    std::vector<uint32_t> at(L.up_off.begin(), L.up_off.end() - 1);
    for (uint32_t u = 0; u < S; ++u)
      for (uint64_t j = p.up_offset[u]; j < p.up_offset[u + 1]; ++j)
        L.up_in[at[dev[p.up_v[j]]]++] = {(int32_t)bv_last(u), (int32_t)p.up_w[j]};
  }
#pragma omp parallel for schedule(static)
  for (int64_t u = 0; u < (int64_t)S; ++u) {
    uint32_t k = L.dn_off[dev[u]];
    for (uint64_t j = p.down_offset[u]; j < p.down_offset[u + 1]; ++j)
      L.dn_in[k++] = {(int32_t)bv_last(p.down_v[j]), (int32_t)p.down_w[j]};
  }
  L.dn_head.assign((size_t)4 * S, 0);
  // upward lists average about two edges: their head carries the first two
  // (8 words: begin, end, src0, w0, src1, w1, 0, 0)
  L.up_head.assign((size_t)8 * S, 0);
  L.fin.assign((size_t)4 * S, 0);
#pragma omp parallel for schedule(static)
  for (int64_t d = 0; d < (int64_t)S; ++d) {
    uint32_t* h = &L.dn_head[(size_t)4 * d];
    h[0] = L.dn_off[d];
    h[1] = L.dn_off[d + 1];
    if (L.dn_off[d + 1] > L.dn_off[d]) {
      h[2] = (uint32_t)L.dn_in[L.dn_off[d]].src;
      h[3] = (uint32_t)L.dn_in[L.dn_off[d]].w;
    }
    uint32_t* u8 = &L.up_head[(size_t)8 * d];
    u8[0] = L.up_off[d];
    u8[1] = L.up_off[d + 1];
    for (uint32_t j = 0; j < 2 && L.up_off[d] + j < L.up_off[d + 1]; ++j) {
      u8[2 + 2 * j] = (uint32_t)L.up_in[L.up_off[d] + j].src;
      u8[3 + 2 * j] = (uint32_t)L.up_in[L.up_off[d] + j].w;
    }
    L.fin[4 * d] = L.dv_first[d];
    L.fin[4 * d + 1] = L.dv_len[d];
    L.fin[4 * d + 2] = L.dv_s[d];
  }
  // levels in hierarchy order
  L.lvl_off.push_back(0);
  for (uint32_t d = 1; d < S; ++d)
    if (p.level[order[d]] != p.level[order[d - 1]]) L.lvl_off.push_back(d);
  L.lvl_off.push_back(S);
  L.levels = (uint32_t)L.lvl_off.size() - 1;
  L.lvl_up_edges.resize(L.levels);
  L.lvl_up_maxdeg.assign(L.levels, 0);
  for (uint32_t l = 0; l < L.levels; ++l) {
    L.lvl_up_edges[l] = L.up_off[L.lvl_off[l + 1]] - L.up_off[L.lvl_off[l]];
    for (uint32_t d = L.lvl_off[l]; d < L.lvl_off[l + 1]; ++d)
      L.lvl_up_maxdeg[l] = std::max(L.lvl_up_maxdeg[l], L.up_off[d + 1] - L.up_off[d]);
  }

  // --- string-graph in-CSR for the traceback walk (traceback.hpp:716) -------
  const chsga_csr& sg = g.string_graph;
  L.istr_off.assign(S + 1, 0);
  for (uint64_t u = 0; u < S; ++u)
    for (uint64_t e = sg.offset[u]; e < sg.offset[u + 1]; ++e) {
      require(sg.target[e] < S, CHSGA_ERR_FORMAT, "string edge target out of range");
      L.istr_off[sg.target[e] + 1]++;
    }
  for (uint32_t v = 0; v < S; ++v) L.istr_off[v + 1] += L.istr_off[v];
  L.istr_src.resize(L.istr_off[S]);
  {
    std::vector<uint32_t> cur(L.istr_off.begin(), L.istr_off.end() - 1);
    for (uint64_t u = 0; u < S; ++u)
      for (uint64_t e = sg.offset[u]; e < sg.offset[u + 1]; ++e) L.istr_src[cur[sg.target[e]]++] = (uint32_t)u;
  }
  return L;
}

size_t row_tiled_smem(const HostRowTiles& t, uint32_t R) {
  // slots, full and empty barriers, per-slot minima, spare
  return (size_t)t.nslots * t.slot_bytes() + (size_t)kTileSlotsMax * 16 + (size_t)R * 8 + 16;
}

HostRowTiles build_row_tiles(const HostLayout& L, uint32_t R, uint32_t sz) {
  HostRowTiles t;
  const uint32_t PC = R * sz;  // bytes per char slot-row (and per FL entry)
  require(R >= 32 && PC % 16 == 0, CHSGA_ERR_INTERNAL, "tiled rows need R >= 32");
  t.d_cap = std::max<uint32_t>(8192, 32 * PC);
  t.fl_cap = 2 * kTileMaxVerts * PC;
  t.desc_cap = (16 * kTileMaxVerts + 4 * kTileMaxEdges + 15) / 16 * 16;
  t.ext_cap = kTileMaxExt * PC;
  t.nslots = std::min<uint32_t>(kTileSlotsMax, kTileSmemBudget / t.slot_bytes());
  if (t.nslots < 2) return t;
  auto edges_of = [&](uint32_t s) { return L.vin_off[s + 1] - L.vin_off[s]; };
  auto n_ext = [&](uint32_t s0, uint32_t e1) {
    uint32_t x = 0;
    for (uint32_t v = s0; v < e1; ++v)
      for (uint32_t k = L.vin_off[v]; k < L.vin_off[v + 1]; ++k)
        x += (L.vin_srcv[k] < s0 || L.vin_srcv[k] >= e1) ? 1 : 0;
    return x;
  };
  uint32_t s = 0;
  while (s < L.S) {
    const uint32_t s0 = s, c0 = L.sv_off[s0];
    const bool lng = (uint64_t)(L.sv_off[s0 + 1] - c0) * PC > t.d_cap;
    uint32_t s1 = s0 + 1, ne = edges_of(s0);
    if (ne > kTileMaxEdges || n_ext(s0, s1) > kTileMaxExt) return HostRowTiles{};
    if (!lng) {
      while (s1 < L.S && s1 - s0 < kTileMaxVerts &&
             (uint64_t)(L.sv_off[s1 + 1] - c0) * PC <= t.d_cap &&
             ne + edges_of(s1) <= kTileMaxEdges && n_ext(s0, s1 + 1) <= kTileMaxExt) {
        ne += edges_of(s1);
        ++s1;
      }
    }
    const uint32_t off = (uint32_t)t.desc.size();
    std::vector<uint32_t> ext;
    uint32_t eb = 0;
    for (uint32_t v = s0; v < s1; ++v) {
      const uint32_t ec = edges_of(v);
      t.desc.push_back(L.sv_off[v]);
      t.desc.push_back(L.sv_off[v + 1] - L.sv_off[v]);
      t.desc.push_back(L.sv_dev[v]);
      t.desc.push_back((eb << 16) | ec);
      eb += ec;
    }
    for (uint32_t v = s0; v < s1; ++v)
      for (uint32_t k = L.vin_off[v]; k < L.vin_off[v + 1]; ++k) {
        const uint32_t su = L.vin_srcv[k];
        if (su >= s0 && su < s1) {
          t.desc.push_back(su - s0);
        } else {
          t.desc.push_back(0x80000000u | (uint32_t)ext.size());
          ext.push_back(su);
        }
      }
    while (t.desc.size() % 4) t.desc.push_back(0);
    const uint32_t bytes = (uint32_t)(t.desc.size() - off) * 4;
    const uint32_t ext_off = (uint32_t)t.desc.size();
    t.desc.insert(t.desc.end(), ext.begin(), ext.end());
    while (t.desc.size() % 4) t.desc.push_back(0);
    const uint32_t c1 = L.sv_off[s1];
    const int32_t r0[4] = {(int32_t)s0, (int32_t)s1, (int32_t)c0,
                           (int32_t)(lng ? (c1 | 0x80000000u) : c1)};
    const int32_t r1[4] = {(int32_t)off, (int32_t)bytes, (int32_t)ext.size(), (int32_t)ext_off};
    t.rec.insert(t.rec.end(), r0, r0 + 4);
    t.rec.insert(t.rec.end(), r1, r1 + 4);
    t.long_tiles += lng ? 1 : 0;
    s = s1;
  }
  t.ok = true;
  return t;
}

void validate_row_tiles(const HostLayout& L, uint32_t R, uint32_t sz, const HostRowTiles& t) {
  auto bad = [&](uint32_t tile, const std::string& m) {
    fail(CHSGA_ERR_INTERNAL, "row tile " + std::to_string(tile) + ": " + m);
  };
  if (!t.ok) return;
  const uint64_t PC = (uint64_t)R * sz;
  const uint64_t row_bytes = ((uint64_t)L.N + 32) * PC;      // score row allocation
  const uint64_t fl_bytes = 2 * ((uint64_t)L.S + 16) * PC;   // FL allocation
  if (t.slot_bytes() % 16 || t.d_cap % 16 || t.fl_cap % 16 || t.desc_cap % 16 || t.ext_cap % 16)
    bad(0, "slot regions must be multiples of 16 bytes");
  if (row_tiled_smem(t, R) + 16 > kSmemPerBlockMax) bad(0, "shared memory above the per-block limit");
  if (t.nslots < 2 || t.nslots > kTileSlotsMax) bad(0, "slot count");
  uint32_t next_s = 0;
  for (uint32_t i = 0; i < t.ntiles(); ++i) {
    const int32_t* r0 = &t.rec[8 * i];
    const int32_t* r1 = r0 + 4;
    const uint32_t s0 = (uint32_t)r0[0], s1 = (uint32_t)r0[1], c0 = (uint32_t)r0[2];
    const bool lng = r0[3] < 0;
    const uint32_t c1 = (uint32_t)r0[3] & 0x7fffffffu;
    if (s0 != next_s || s1 <= s0 || s1 > L.S) bad(i, "tiles must cover the vertices in order");
    next_s = s1;
    const uint32_t nv = s1 - s0;
    if (nv > kTileMaxVerts || (lng && nv != 1)) bad(i, "vertex count");
    if (c0 != L.sv_off[s0] || c1 != L.sv_off[s1]) bad(i, "char range");
    if (!lng) {
      const uint64_t db = (uint64_t)(c1 - c0) * PC;
      if (db > t.d_cap || (c0 * PC) % 16 || db % 16 || c0 * PC + db > row_bytes) bad(i, "score copy");
    }
    const uint64_t flo = 2 * (uint64_t)s0 * PC, flb = 2 * (uint64_t)nv * PC;
    if (flb > t.fl_cap || flo % 16 || flb % 16 || flo + flb > fl_bytes) bad(i, "FL copy");
    const uint32_t off = (uint32_t)r1[0], bytes = (uint32_t)r1[1], next = (uint32_t)r1[2],
                   eoff = (uint32_t)r1[3];
    if (off % 4 || bytes % 16 || bytes > t.desc_cap || (uint64_t)off * 4 + bytes > t.desc.size() * 4)
      bad(i, "descriptor copy");
    if (next > kTileMaxExt || (uint64_t)next * PC > t.ext_cap || eoff + next > t.desc.size())
      bad(i, "external list");
    uint32_t eb = 0, edges = 0;
    for (uint32_t j = 0; j < nv; ++j) {
      const uint32_t* vr = &t.desc[off + 4 * j];
      const uint32_t s = s0 + j;
      if (vr[0] != L.sv_off[s] || vr[1] != L.sv_off[s + 1] - L.sv_off[s] || vr[2] != L.sv_dev[s] ||
          (vr[3] >> 16) != eb || (vr[3] & 0xFFFFu) != L.vin_off[s + 1] - L.vin_off[s])
        bad(i, "vertex record " + std::to_string(j));
      eb += vr[3] & 0xFFFFu;
    }
    edges = eb;
    if (16ull * nv + 4ull * edges > bytes) bad(i, "descriptor shorter than its records");
    uint32_t q = 0;
    for (uint32_t j = 0; j < nv; ++j)
      for (uint32_t k = L.vin_off[s0 + j]; k < L.vin_off[s0 + j + 1]; ++k, ++q) {
        const uint32_t loc = t.desc[off + 4 * nv + q];
        const uint32_t su = L.vin_srcv[k];
        if (loc & 0x80000000u) {
          const uint32_t x = loc & 0x7fffffffu;
          if (x >= next || t.desc[eoff + x] != su || (2ull * su + 2) * PC > fl_bytes)
            bad(i, "external in-edge record");
        } else if (loc >= nv || s0 + loc != su) {
          bad(i, "internal in-edge record");
        }
      }
  }
  if (next_s != L.S) bad(t.ntiles(), "tiles do not reach the last vertex");
}

HostT1 build_t1(const HostLayout& L) {
  HostT1 t;
  const uint32_t N = L.N, S = L.S;
  t.heads.assign((size_t)(N + 7) / 8 + 1, 0);
  t.vrec.assign((size_t)4 * S, 0);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < (int64_t)S; ++s) {
    const uint32_t f = L.sv_off[s], k0 = L.vin_off[s], k1 = L.vin_off[s + 1];
    uint32_t* r = &t.vrec[4 * (size_t)s];
    r[0] = f;
    r[1] = L.sv_dev[s] | (k1 - k0 > 2 ? 0x80000000u : 0u);
    r[2] = k1 > k0 ? L.vin_srcv[k0] : 0xFFFFFFFFu;
    r[3] = k1 > k0 + 1 ? L.vin_srcv[k0 + 1] : 0xFFFFFFFFu;
  }
  // vertices start in increasing char order, so each head byte has one writer per bit
  for (uint32_t s = 0; s < S; ++s) t.heads[L.sv_off[s] >> 3] |= (uint8_t)(1u << (L.sv_off[s] & 7));
  uint32_t s = 0;
  while (s < S) {
    const uint32_t cb = L.sv_off[s];
    uint32_t e = s;
    while (e < S && e - s < kT1MaxVerts && ((L.sv_off[e + 1] - 1) >> 3) - (cb >> 3) + 1 <= kT1Chunks)
      ++e;
    if (e == s) return HostT1{};  // one vertex longer than a tile
    t.desc.insert(t.desc.end(), {cb, L.sv_off[e], s, e});
    s = e;
  }
  t.ok = true;
  return t;
}

HostTop build_top(const HostLayout& L, uint32_t max_vertices, uint32_t chunk_edges) {
  require(max_vertices < 32768 && chunk_edges >= 32 && chunk_edges % 32 == 0, CHSGA_ERR_INTERNAL,
          "top region limits");
  HostTop t;
  uint32_t first = L.levels;
  while (first > 0 && L.S - L.lvl_off[first - 1] <= max_vertices) --first;
  t.first_level = first;
  t.K0 = L.lvl_off[first];
  t.K = L.S - t.K0;
  t.upg_off.assign(t.K + 1, 0);
  const int32_t lo = (int32_t)(2 * t.K0);
  for (uint32_t j = 0; j < t.K; ++j) {
    const uint32_t d = t.K0 + j;
    for (uint32_t e = L.up_off[d]; e < L.up_off[d + 1]; ++e)
      if (L.up_in[e].src < lo) t.upg.push_back(L.up_in[e]);
    t.upg_off[j + 1] = (uint32_t)t.upg.size();
  }
  const EdgeW pad{(int32_t)(t.K << 16), 0};  // scratch target K, source 0
  // a run of small levels (<= kTopWarpLevelMax edges each) forms one warp
  // chunk: every level padded to whole rounds of 32 edges, count negative
  std::vector<EdgeW> warp;
  auto flush_warp = [&] {
    if (warp.empty()) return;
    t.chunks.push_back({(int32_t)t.sched.size(), -(int32_t)warp.size()});
    t.sched.insert(t.sched.end(), warp.begin(), warp.end());
    warp.clear();
  };
  auto emit_level = [&](uint32_t l, bool up) {
    std::vector<EdgeW> es;
    for (uint32_t d = L.lvl_off[l]; d < L.lvl_off[l + 1]; ++d) {
      const uint32_t j = d - t.K0;
      const auto& off = up ? L.up_off : L.dn_off;
      const auto& in = up ? L.up_in : L.dn_in;
      for (uint32_t e = off[d]; e < off[d + 1]; ++e) {
        if (in[e].src < lo) {
          require(up, CHSGA_ERR_INTERNAL, "downward edge into the top region from below");
          continue;  // applied by the grid-wide pull
        }
        es.push_back({(int32_t)((j << 16) | (uint32_t)(in[e].src - lo)), in[e].w});
      }
    }
    if (es.empty()) return;
    const size_t rounds = (es.size() + 31) / 32;
    if (es.size() <= kTopWarpLevelMax && 32 * rounds <= chunk_edges) {
      if (warp.size() + 32 * rounds > chunk_edges) flush_warp();
      warp.insert(warp.end(), es.begin(), es.end());
      warp.resize(warp.size() + (32 * rounds - es.size()), pad);
      return;
    }
    flush_warp();
    for (size_t i = 0; i < es.size(); i += chunk_edges) {
      const size_t n = std::min<size_t>(chunk_edges, es.size() - i);
      t.chunks.push_back({(int32_t)t.sched.size(), (int32_t)(n + (n & 1))});
      t.sched.insert(t.sched.end(), es.begin() + i, es.begin() + i + n);
      if (n & 1) t.sched.push_back(pad);
    }
  };
  for (uint32_t l = first; l < L.levels; ++l) emit_level(l, true);
  for (uint32_t l = L.levels; l-- > first;) emit_level(l, false);
  flush_warp();
  return t;
}

}  // namespace chsga
