// Host check of the top-region chunk schedule (device_graph.cpp::build_top).
//
// k_top runs a region's upward levels low -> high and downward levels
// high -> low as chunks of edges {target << 16 | source, weight}: a block
// chunk relaxes all its edges at once, a warp chunk relaxes rounds of 32
// edges in order. This program builds the layout and the schedule of
// generated graphs for several region sizes and chunk sizes and checks:
//   - within a block chunk, and within a round of a warp chunk, no edge reads
//     a score that another edge of the same chunk or round writes (so any
//     order of the concurrent relaxations gives one result);
//   - a warp chunk is whole rounds and no larger than a chunk buffer;
//   - applying the schedule (after the pull of the edges from below the
//     region) gives the same first scores as relaxing the region's edges
//     level by level, the way align.hpp's sweeps order them.
// Exit status 0 and "OK" on success.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <set>
#include <string>
#include <vector>

#include "chsga.h"
#include "device_graph.hpp"

using namespace chsga;

namespace {

int fails = 0;

void check(bool ok, const std::string& what) {
  if (!ok && fails++ < 20) std::printf("FAIL: %s\n", what.c_str());
}

std::vector<int64_t> apply_schedule(const HostLayout& L, const HostTop& t, std::vector<int64_t> bv,
                                    uint32_t chunk_edges) {
  const uint32_t K0 = t.K0, K = t.K;
  // edges from below the region (sources final, outside the region)
  for (uint32_t j = 0; j < K; ++j)
    for (uint32_t e = t.upg_off[j]; e < t.upg_off[j + 1]; ++e) {
      check(t.upg[e].src < (int32_t)(2 * K0), "upg source below the region");
      bv[2 * (K0 + j)] = std::min(bv[2 * (K0 + j)], bv[t.upg[e].src] + t.upg[e].w);
    }
  std::vector<int64_t> sm(2 * (size_t)K + 2, 0);
  for (uint32_t j = 0; j < K; ++j) {
    sm[2 * j] = bv[2 * (K0 + j)];
    sm[2 * j + 1] = bv[2 * (K0 + j) + 1];
  }
  auto relax_set = [&](size_t b, size_t n, const std::string& what) {
    std::set<uint32_t> targets;
    for (size_t i = b; i < b + n; ++i) targets.insert(2 * ((uint32_t)t.sched[i].src >> 16));
    for (size_t i = b; i < b + n; ++i) {
      const uint32_t x = (uint32_t)t.sched[i].src;
      const uint32_t tgt = x >> 16, src = x & 0xFFFF;
      check(tgt <= K && src < 2 * K + 2, what + ": index in range");
      // the scratch slot 2K is only ever written
      check(!targets.count(src) || src == 2 * K, what + ": a source is written in the same step");
    }
    for (size_t i = b; i < b + n; ++i) {
      const uint32_t x = (uint32_t)t.sched[i].src;
      sm[2 * (x >> 16)] = std::min(sm[2 * (x >> 16)], sm[x & 0xFFFF] + t.sched[i].w);
    }
  };
  for (size_t c = 0; c < t.chunks.size(); ++c) {
    const int32_t first = t.chunks[c].first, count = t.chunks[c].second;
    check(first % 2 == 0, "chunk starts 16-byte aligned");
    const uint32_t n = (uint32_t)(count < 0 ? -count : count);
    check(n <= chunk_edges && n > 0, "chunk fits a buffer");
    check((size_t)first + n <= t.sched.size(), "chunk inside the schedule");
    if (count >= 0) {
      check(n % 2 == 0, "block chunk even");
      relax_set(first, n, "block chunk");
    } else {
      check(n % 32 == 0, "warp chunk whole rounds");
      for (uint32_t r = 0; r < n; r += 32) relax_set(first + r, 32, "warp round");
    }
  }
  for (uint32_t j = 0; j < K; ++j) bv[2 * (K0 + j)] = sm[2 * j];
  return bv;
}

std::vector<int64_t> by_levels(const HostLayout& L, uint32_t first_level, std::vector<int64_t> bv) {
  for (uint32_t l = first_level; l < L.levels; ++l)
    for (uint32_t d = L.lvl_off[l]; d < L.lvl_off[l + 1]; ++d)
      for (uint32_t e = L.up_off[d]; e < L.up_off[d + 1]; ++e)
        bv[2 * d] = std::min(bv[2 * d], bv[L.up_in[e].src] + L.up_in[e].w);
  for (uint32_t l = L.levels; l-- > first_level;)
    for (uint32_t d = L.lvl_off[l]; d < L.lvl_off[l + 1]; ++d)
      for (uint32_t e = L.dn_off[d]; e < L.dn_off[d + 1]; ++e)
        bv[2 * d] = std::min(bv[2 * d], bv[L.dn_in[e].src] + L.dn_in[e].w);
  return bv;
}

}  // namespace

int main() {
  const uint64_t backbones[] = {30000, 200000};
  uint64_t checked = 0;
  for (uint64_t bb : backbones) {
    chsga_gen_graph_cfg cfg{bb, 7 + bb, 50.0, 0.7, 0.2, 0.1, 1, 20, 50, 300, 1, 32};
    chsga_host_graph* g = nullptr;
    if (chsga_gen_graph(&cfg, &g) != CHSGA_OK) return 2;
    chsga_pch_opts po{500, 1.0, 0, 1, 0x5EED, 0, 0, 0, 0};
    if (chsga_build_pch(g, &po) != CHSGA_OK) return 2;
    chsga_graph_host view{};
    chsga_graph_view(g, &view);
    const HostLayout L = build_layout(view);
    std::mt19937_64 rng(bb);
    std::vector<int64_t> bv(2 * (size_t)L.S);
    for (auto& x : bv) x = (int64_t)(rng() % 2000);
    for (uint32_t maxv : {300u, 2000u, 8000u, 23000u})
      for (uint32_t cap : {32u, 96u, 1024u, 4096u}) {
        const HostTop t = build_top(L, maxv, cap);
        if (t.K == 0) continue;
        const auto got = apply_schedule(L, t, bv, cap);
        const auto want = by_levels(L, t.first_level, bv);
        for (uint32_t j = 0; j < t.K; ++j)
          check(got[2 * (t.K0 + j)] == want[2 * (t.K0 + j)],
                "first score of region position " + std::to_string(j) + " (region " +
                    std::to_string(maxv) + ", chunks of " + std::to_string(cap) + ")");
        ++checked;
      }
    chsga_graph_free(g);
  }
  if (fails || checked == 0) {
    std::printf("FAILED (%d)\n", fails);
    return 1;
  }
  std::printf("OK %llu schedules\n", (unsigned long long)checked);
  return 0;
}
