// Witness searches of the hierarchy builder on a CUDA device.
//
// Every round of the builder (pch_build.cpp) runs, on one snapshot of the
// overlay graph, a bounded Dijkstra per in-arc of every remaining vertex
// (the score stage, build_pch.hpp:396-478) and one per selected vertex (the
// relevance of its out-arcs, build_pch.hpp:1012-1045). PchGpu runs those
// searches on the device, one thread per search, with the CPU search's
// exact semantics: pops in (distance, vertex) order, stale entries skipped
// without counting, at most `pop_limit` pops, no pop beyond the bound, the
// source never re-entered, and a vertex x passed through costing
// through[x] more. The overlay holds the round's remaining vertices only,
// renumbered 0..n-1 by the caller. Each task returns one 64-bit mask:
//   score task (u, s, w): bit j (j < out-degree of u) = the j-th out-arc
//     (u, b, wb) of u needs a shortcut, i.e. b != s and
//     dist_s(b) >= w + wb + through[u]; bit 62 = dist_s(u) >= w (the in-arc
//     is relevant); the search from s is bounded by w + through[u] + max wb;
//   relevance task (u): bit j = dist_u(b) >= wb, bounded by max wb.
// kPchOverflow marks a task the device could not finish within its
// per-thread tables (or a vertex of out-degree above 62): the caller runs
// that search on the CPU, so results never depend on the device's limits.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

namespace chsga {

constexpr uint64_t kPchOverflow = 1ull << 63;
constexpr uint32_t kPchMaskDegree = 62;

struct PchGpuImpl;

class PchGpu {
 public:
  // Throws if the device cannot be used.
  PchGpu(int device, uint32_t pop_limit);
  ~PchGpu();
  PchGpu(const PchGpu&) = delete;
  PchGpu& operator=(const PchGpu&) = delete;

  // The overlay of this round: out-arcs of vertex v are
  // arcs[off[v] .. off[v+1]), each target | weight << 32, in the builder's
  // order; through[v] is the extra cost of passing through v (len - 1, or 0
  // without label lengths).
  void set_overlay(const std::vector<uint32_t>& off, const std::vector<uint64_t>& arcs,
                   const std::vector<uint32_t>& through);
  // Score tasks (tu[i], ts[i], tw[i]) or, with ts empty, relevance tasks
  // (tu[i]); one mask per task into `masks`.
  void run(const std::vector<uint32_t>& tu, const std::vector<uint32_t>& ts,
           const std::vector<uint32_t>& tw, std::vector<uint64_t>& masks);

 private:
  std::unique_ptr<PchGpuImpl> p_;
};

}  // namespace chsga
