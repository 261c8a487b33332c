// Device-side layout of one alignment graph and the host code that builds it.
//
// The DP of src/align.hpp touches, per read row:
//   every char c (fused_deletion_substitution, align.hpp:245-277) through the
//     char graph's in-CSR and the char labels;
//   every string vertex s through first(s) = off[s], last(s) = off[s+1]-1
//     (insertion_func_parallel, align.hpp:347-397);
//   the contraction hierarchy, layer by layer (align.hpp:279-345).
// The layout below serves those three access patterns:
//
//   chars (original order)      2-bit label codes + a 1-bit "special" map
//   string vertices (original)  sv_off[S+1] char offsets, sv_dev[S] position
//                               in the hierarchy order, vin_* = in-edges of
//                               the vertex's first char (every other char of
//                               a vertex has exactly the chain edge c-1 -> c)
//   hierarchy vertices          ordered by (level, rank): one contiguous range
//                               per level, all components merged (components
//                               share no edges, so their sweeps commute)
//   boundary array BV           per hierarchy vertex d: BV[2d] = score at
//                               first(og d), BV[2d+1] = score at last(og d);
//                               single-char vertices use BV[2d] for both
//   up_in / dn_in               pull form of the two sweeps: for target d the
//                               list of (BV index of the source's last char,
//                               weight); an upward edge u->v of GC.E becomes an
//                               entry of up_in[v], a downward in-edge of
//                               GC.in_E[u] an entry of dn_in[u]
//
// Pull instead of push: every hierarchy edge joins two different layers of
// one component (checked at load), so the push-with-atomic-min of the
// reference's upward sweep and this pull compute the same minima.
#pragma once

#include <cstdint>
#include <vector>

#include "common.hpp"

namespace chsga {

struct EdgeW {  // matches the device int2 layout
  int32_t src;
  int32_t w;
};

struct HostLayout {
  uint32_t N = 0, S = 0, levels = 0;
  uint32_t max_len = 0;  // longest string vertex label
  // label encoding: code 0..3 for A,C,G,T; `special` holds the one other
  // byte that may occur in the labels (usually 'N'), flagged in lab_sp
  int special = -1;
  std::vector<uint32_t> lab2;   // ceil(N/16) words
  std::vector<uint32_t> lab_sp; // ceil(N/32) words
  std::vector<uint32_t> lab4;   // ceil(N/8)+2 words: 4-bit label key per char (0..3 ACGT, 4 special)
  std::vector<uint32_t> sv_off, sv_dev, vin_off, vin_src, vin_srcv;
  std::vector<uint32_t> dv_first, dv_len, dv_s;  // by hierarchy order
  std::vector<uint32_t> up_off, dn_off;    // S+1, by hierarchy order
  std::vector<EdgeW> up_in, dn_in;
  std::vector<uint32_t> dn_head;  // 4 words per position: begin, end, first src, first w
  std::vector<uint32_t> up_head;  // 8 words per position: begin, end, src0, w0, src1, w1, 0, 0
  std::vector<uint32_t> fin;               // 4 words per position: first char, length, string vertex, 0
  std::vector<uint32_t> lvl_off;           // levels+1
  std::vector<uint32_t> lvl_up_edges;      // per level: number of up_in entries
  std::vector<uint32_t> lvl_up_maxdeg;     // per level: most up_in entries of one position
  std::vector<uint32_t> istr_off, istr_src;  // string-graph in-CSR (ascending source)
  uint64_t char_in_edges = 0;
};

// Top region of the hierarchy (levels >= first_level), swept inside one CTA
// per slot with the boundary values staged in shared memory. Edges from
// below the region (upg) are applied by a grid-wide pull first; the region's
// own edges run as a chunk schedule: upward levels low -> high, then
// downward levels high -> low, each chunk at most chunk_edges edges of one
// level, padded to an even count with a no-op edge into the scratch slot K.
// Consecutive levels of at most kTopWarpLevelMax edges share one warp chunk
// instead (count stored negated): each level padded with no-op edges to
// whole rounds of 32, the rounds run in order by one warp.
constexpr uint32_t kTopWarpLevelMax = 64;
// Region size limits in hierarchy vertices: the most a region's scores and
// chunk buffers leave room for in one CTA's shared memory, and the default.
// A region that holds the big levels (6 and 7 on the config-2 graph) sweeps
// them on one SM per slot; in grid launches they cost less, and 8000
// vertices measured fastest or within 1 % of it at every slot count.
constexpr uint32_t kTopMaxVertices = 23000;
constexpr uint32_t kTopDefaultVertices = 8000;
struct HostTop {
  uint32_t first_level = 0;  // level index where the top region starts
  uint32_t K0 = 0, K = 0;    // hierarchy positions [K0, K0+K)
  std::vector<uint32_t> upg_off;  // K+1
  std::vector<EdgeW> upg;         // global source index
  std::vector<EdgeW> sched;       // src = target << 16 | local source, w
  std::vector<std::pair<int32_t, int32_t>> chunks;  // {first edge, count (< 0: warp chunk)}
};

// Tiles of consecutive string vertices for the shared-memory-staged row
// kernel (one warp per vertex, R >= 32 slots). Per tile: two int4 records
// r0 = {s0, s1, c0, c1 | long << 31}, r1 = {descriptor word offset,
// descriptor bytes, external count, external list word offset}; descriptor
// = per vertex {first char, length, hierarchy position, first edge << 16 |
// edge count}, then one word per in-edge (source vertex - s0 inside the tile,
// else 0x80000000 | external index), padded to 16 bytes, then the external
// source vertices. Each slot of shared memory holds the tile's scores
// (d_cap), its per-vertex final first/last scores (fl_cap), the descriptor
// (desc_cap) and the external sources' last scores (ext_cap).
constexpr uint32_t kTileMaxVerts = 16, kTileMaxEdges = 48, kTileMaxExt = 4;
constexpr uint32_t kTileSlotsMax = 16, kTileSmemBudget = 200 * 1024;
constexpr uint32_t kSmemPerBlockMax = 232448;  // sm_100 opt-in maximum

struct HostRowTiles {
  bool ok = false;  // false: some vertex cannot fit a tile (use the direct kernel)
  uint32_t d_cap = 0, fl_cap = 0, desc_cap = 0, ext_cap = 0, nslots = 0;
  std::vector<int32_t> rec;   // 8 per tile
  std::vector<uint32_t> desc;
  uint32_t long_tiles = 0;
  uint32_t slot_bytes() const { return d_cap + fl_cap + desc_cap + ext_cap; }
  uint32_t ntiles() const { return (uint32_t)(rec.size() / 8); }
};

// Shared memory of the tiled row kernel for these tiles.
size_t row_tiled_smem(const HostRowTiles& t, uint32_t R);
HostRowTiles build_row_tiles(const HostLayout& L, uint32_t R, uint32_t score_bytes);
// Checks every bound and alignment the kernel relies on; throws on violation.
void validate_row_tiles(const HostLayout& L, uint32_t R, uint32_t score_bytes, const HostRowTiles& t);

// Tiles of the one-read row kernel (k_row_t1, 16-bit rows): runs of whole
// consecutive string vertices whose chars span at most kT1Chunks aligned
// chunks of 8 chars and that hold at most kT1MaxVerts vertices; a warp
// takes one tile, a lane one chunk.
//   desc   4 words per tile: first char, end char, first vertex, end vertex
//   heads  1 byte per chunk: bit i set when char 8q + i is the first char of
//          its string vertex
//   vrec   4 words per string vertex: first char, hierarchy position (bit 31
//          set when the first char has more than two in-edges), source
//          vertex of the first and of the second first-char in-edge
//          (0xFFFFFFFF when absent)
// ok is false when some vertex alone spans more than kT1Chunks chunks.
constexpr uint32_t kT1Chunks = 32, kT1MaxVerts = 64;
struct HostT1 {
  bool ok = false;
  std::vector<uint32_t> desc;
  std::vector<uint8_t> heads;
  std::vector<uint32_t> vrec;
  uint32_t ntiles() const { return (uint32_t)(desc.size() / 4); }
};
HostT1 build_t1(const HostLayout& L);

HostLayout build_layout(const chsga_graph_host& g);
HostTop build_top(const HostLayout& L, uint32_t max_vertices, uint32_t chunk_edges);

}  // namespace chsga
