// Contraction hierarchy over the string graph, restating the build_pch tool
// (src/CHoverrides/build_pch.cpp:6-131, src/CHoverrides/build_pch.hpp):
//   preprocess       drop self loops and parallel edges      build_pch.hpp:181-228
//   witness search   bounded Dijkstra; passing through a
//                    vertex x costs len(x)-1 more (-v)       build_pch.hpp:230-394
//   score            edge difference formula                 build_pch.hpp:396-478
//   selection        vertices whose (score, degree, random
//                    priority) beats every neighbour         build_pch.hpp:536-571
//   contraction      shortcut a->b via u unless a strictly
//                    shorter path exists, weight
//                    w(a,u)+w(u,b)+len(u)-1; relevant arcs
//                    become hierarchy edges; neighbours get
//                    level max(level, level[u]+1)            build_pch.hpp:1012-1067
//   order            rank by (component, level, id)          build_pch.hpp:1132-1220
// The upstream builder runs on parlaylib with concurrent hash tables; this
// one computes the same quantities with per-round snapshots (OpenMP), so
// selection and contraction within a round see one consistent graph. With
// use_gpu the witness searches of each round run on a CUDA device
// (pch_gpu.cu) against the same snapshot; a search the device cannot finish
// within its tables is redone here, so the hierarchy is the same either way.
#include <omp.h>

#include <algorithm>
#include <parallel/algorithm>
#include <chrono>
#include <cstdio>
#include <limits>
#include <numeric>
#include <queue>

#include "host_graph.hpp"
#include "pch_gpu.hpp"

namespace chsga {

namespace {

struct Arc {
  uint32_t v;
  uint32_t w;
  uint32_t hop;
};

struct Shortcut {
  uint32_t a, b, w, hop;
};

constexpr uint64_t kInf = std::numeric_limits<uint64_t>::max();

class PchBuilder {
 public:
  PchBuilder(const HostCsr& g, const std::vector<uint64_t>& offs, const chsga_pch_opts& o)
      : opt_(o), n_(g.n) {
    use_len_ = o.use_label_lengths != 0;
    if (use_len_) {
      require(offs.size() == n_ + 1, CHSGA_ERR_INVALID_ARG, "label offsets size");
      len_.resize(n_);
      for (uint64_t i = 0; i < n_; ++i) len_[i] = offs[i + 1] - offs[i];
    }
    k_ = o.weight_bound ? o.weight_bound : kInf;
    pop_limit_ = o.max_pop_count ? o.max_pop_count : 500;
    // preprocess: sort (u, v, w), drop self loops and repeated (u, v). The
    // sort is by the whole tuple, so any sort gives the same order; every
    // vertex's out-arcs are a range of it, its in-arcs follow in that order.
    require(g.offset.size() == n_ + 1 && g.offset[0] == 0 && g.offset[n_] == g.m,
            CHSGA_ERR_INVALID_ARG, "string graph offsets");
    const int nthreads = opt_.threads > 0 ? opt_.threads : omp_get_max_threads();
    std::vector<std::tuple<uint32_t, uint32_t, uint32_t>> el(g.m);
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nthreads)
    for (int64_t u = 0; u < (int64_t)n_; ++u)
      for (uint64_t e = g.offset[u]; e < g.offset[u + 1]; ++e)
        el[e] = std::make_tuple((uint32_t)u, g.target[e], g.w(e));
    __gnu_parallel::sort(el.begin(), el.end());
    const size_t M = el.size();
    std::vector<uint8_t> keep(M);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t i = 0; i < (int64_t)M; ++i) {
      const auto& [u, v, w] = el[i];
      (void)w;
      keep[i] = u != v && !(i > 0 && std::get<0>(el[i - 1]) == u && std::get<1>(el[i - 1]) == v);
    }
    std::vector<uint64_t> ioff(n_ + 1, 0);
    for (size_t i = 0; i < M; ++i)
      if (keep[i]) ++ioff[std::get<1>(el[i]) + 1];
    for (uint64_t v = 0; v < n_; ++v) ioff[v + 1] += ioff[v];
    std::vector<Arc> in_flat(ioff[n_]);
    {
      std::vector<uint64_t> at(ioff.begin(), ioff.end() - 1);
      for (size_t i = 0; i < M; ++i)
        if (keep[i]) in_flat[at[std::get<1>(el[i])]++] = {std::get<0>(el[i]), std::get<2>(el[i]), 1};
    }
    out_.resize(n_);
    in_.resize(n_);
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nthreads)
    for (int64_t u = 0; u < (int64_t)n_; ++u) {
      // el[offset[u] .. offset[u+1]) are u's edges: the sort keeps the
      // per-source counts of the input CSR
      uint64_t k = 0;
      for (uint64_t i = g.offset[u]; i < g.offset[u + 1]; ++i) k += keep[i];
      out_[u].reserve(k);
      for (uint64_t i = g.offset[u]; i < g.offset[u + 1]; ++i)
        if (keep[i]) out_[u].push_back({std::get<1>(el[i]), std::get<2>(el[i]), 1});
      in_[u].assign(in_flat.begin() + ioff[u], in_flat.begin() + ioff[u + 1]);
    }
    base_edges_ = std::move(el);
  }

  HostPch build() {
    auto t0 = std::chrono::steady_clock::now();
    level_.assign(n_, 1);
    removed_nbr_.assign(n_, 0);
    contracted_.assign(n_, 0);
    ed_.assign(n_, 0.f);
    require(n_ < (1ull << 32), CHSGA_ERR_UNSUPPORTED, "hierarchy builder: too many vertices");
    prio_.resize(n_);
    std::iota(prio_.begin(), prio_.end(), 1u);
    {
      Rng rng(opt_.seed ? opt_.seed : 0x5eed);
      for (uint64_t i = n_; i > 1; --i) std::swap(prio_[i - 1], prio_[rng.below(i)]);
    }
    up_.resize(n_);
    down_.resize(n_);
    if (opt_.use_gpu) {
      require(n_ < (1ull << 32) - 1, CHSGA_ERR_UNSUPPORTED, "hierarchy builder: too many vertices");
      gpu_ = std::make_unique<PchGpu>(opt_.device, pop_limit_);
      cid_.assign(n_, kNoId);
    }
    claim_in_.assign(n_, kNoClaim);
    claim_out_.assign(n_, kNoClaim);
    std::vector<uint32_t> remaining(n_);
    std::iota(remaining.begin(), remaining.end(), 0);
    const int nthreads = opt_.threads > 0 ? opt_.threads : omp_get_max_threads();
    scratch_.resize(nthreads);
    tcuts_.resize(nthreads);
#pragma omp parallel num_threads(nthreads)
    scratch_[omp_get_thread_num()].init(n_);
    for (auto& s : scratch_)
      if (s.hkey.empty()) s.init(n_);
    uint32_t round = 0;
    while (!remaining.empty()) {
      ++round;
      const size_t R = remaining.size();
      // per-vertex results in flat arrays: in-/out-arc relevance by arc
      // offset, shortcuts in per-thread buffers ({thread, start, count})
      std::vector<uint64_t> toff(R + 1), ooff(R + 1), masks;
      toff[0] = ooff[0] = 0;
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int64_t i = 0; i < (int64_t)R; ++i) {
        toff[i + 1] = in_[remaining[i]].size();
        ooff[i + 1] = out_[remaining[i]].size();
      }
      for (size_t i = 0; i < R; ++i) {
        toff[i + 1] += toff[i];
        ooff[i + 1] += ooff[i];
      }
      std::vector<uint8_t> in_rel(toff[R]), out_rel(ooff[R]);
      std::vector<CutRef> cref(R);
      for (auto& b : tcuts_) b.clear();
      if (gpu_) {
        upload_overlay(remaining, nthreads);
        // one search per in-arc of every remaining vertex
        std::vector<uint32_t> tu(toff[R]), ts(toff[R]), tw(toff[R]);
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (size_t i = 0; i < R; ++i) {
          const uint32_t u = remaining[i];
          for (size_t k = 0; k < in_[u].size(); ++k) {
            tu[toff[i] + k] = (uint32_t)i;
            ts[toff[i] + k] = cid_[in_[u][k].v];
            tw[toff[i] + k] = in_[u][k].w;
          }
        }
        gpu_->run(tu, ts, tw, masks);
        if (opt_.print_detail) {
          size_t host = 0;
          for (uint64_t m : masks) host += (m & kPchOverflow) ? 1 : 0;
          std::printf("Device witness searches: %zu (redone on the host: %zu)\n", masks.size(), host);
          std::fflush(stdout);
        }
      }
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
      for (size_t i = 0; i < R; ++i) {
        const int tid = omp_get_thread_num();
        std::vector<Shortcut>& buf = tcuts_[tid];
        const size_t start = buf.size();
        score(remaining[i], buf, in_rel.data() + toff[i], scratch_[tid],
              gpu_ ? masks.data() + toff[i] : nullptr);
        cref[i] = {(uint32_t)tid, (uint32_t)(buf.size() - start), start};
      }
      double bound = upper_bound(remaining, round);
      std::vector<uint8_t> sel(R, 0);
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (size_t i = 0; i < R; ++i) sel[i] = eligible(remaining[i], bound) ? 1 : 0;
      std::vector<uint64_t> rel_of(R, kPchOverflow);
      if (gpu_) {
        // one search per selected vertex, same snapshot
        std::vector<uint32_t> tu, none;
        std::vector<size_t> at;
        for (size_t i = 0; i < R; ++i)
          if (sel[i]) {
            tu.push_back((uint32_t)i);
            at.push_back(i);
          }
        gpu_->run(tu, none, none, masks);
        for (size_t k = 0; k < at.size(); ++k) rel_of[at[k]] = masks[k];
      }
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
      for (size_t i = 0; i < R; ++i)
        if (sel[i])
          out_relevance(remaining[i], out_rel.data() + ooff[i], scratch_[omp_get_thread_num()],
                        rel_of[i]);
      // Contraction in waves. Contracting u changes only out_ of its
      // in-neighbours and in_ of its out-neighbours (selected vertices are
      // never adjacent, so no other selected vertex's lists) besides the
      // commutative level / removed-neighbour updates. Each pending vertex
      // claims the lists it changes with the smallest selection index; a
      // vertex holding all its claims runs in this wave, in parallel with
      // the others (their lists are disjoint), the rest wait for the next.
      // Every list therefore sees its changes in selection order, as in one
      // sequential pass, and the smallest pending index always runs.
      std::vector<uint32_t> pending;
      for (size_t i = 0; i < R; ++i)
        if (sel[i]) pending.push_back((uint32_t)i);
      const size_t ncontracted = pending.size();
      require(ncontracted > 0, CHSGA_ERR_INTERNAL, "hierarchy build made no progress");
      std::vector<uint8_t> runs;
      while (!pending.empty()) {
        const int64_t P = (int64_t)pending.size();
        auto claim = [](uint32_t* p, uint32_t k) {
          uint32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
          while (k < cur && !__atomic_compare_exchange_n(p, &cur, k, true, __ATOMIC_RELAXED,
                                                         __ATOMIC_RELAXED)) {
          }
        };
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads)
        for (int64_t q = 0; q < P; ++q) {
          const uint32_t i = pending[q], u = remaining[i];
          for (const Arc& a : in_[u]) claim(&claim_out_[a.v], i);
          for (const Arc& b : out_[u]) claim(&claim_in_[b.v], i);
        }
        runs.assign(P, 1);
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads)
        for (int64_t q = 0; q < P; ++q) {
          const uint32_t i = pending[q], u = remaining[i];
          bool own = true;
          for (const Arc& a : in_[u])
            own = own && __atomic_load_n(&claim_out_[a.v], __ATOMIC_RELAXED) == i;
          for (const Arc& b : out_[u])
            own = own && __atomic_load_n(&claim_in_[b.v], __ATOMIC_RELAXED) == i;
          runs[q] = own;
        }
        // clear the claims while every pending vertex's lists are intact
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads)
        for (int64_t q = 0; q < P; ++q) {
          const uint32_t u = remaining[pending[q]];
          for (const Arc& a : in_[u]) __atomic_store_n(&claim_out_[a.v], kNoClaim, __ATOMIC_RELAXED);
          for (const Arc& b : out_[u]) __atomic_store_n(&claim_in_[b.v], kNoClaim, __ATOMIC_RELAXED);
        }
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
        for (int64_t q = 0; q < P; ++q) {
          if (!runs[q]) continue;
          const uint32_t i = pending[q];
          contract(remaining[i], tcuts_[cref[i].thread].data() + cref[i].start, cref[i].count,
                   in_rel.data() + toff[i], out_rel.data() + ooff[i]);
        }
        std::vector<uint32_t> rest;
        for (int64_t q = 0; q < P; ++q)
          if (!runs[q]) rest.push_back(pending[q]);
        pending.swap(rest);
      }
      std::vector<uint32_t> next;
      next.reserve(R - ncontracted);
      for (uint32_t u : remaining)
        if (!contracted_[u]) next.push_back(u);
        else if (gpu_) cid_[u] = kNoId;
      if (opt_.print_detail)
        std::printf("Round %u\nContract %zu vertices\nOverlay vertices number: %zu\n", round,
                    ncontracted, R);
      remaining.swap(next);
    }
    HostPch p = order(nthreads);
    double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (opt_.print_detail)
      std::printf("G.n: %llu, G.m: %llu, G.rm: %llu, G.layer: %u, total_time: %f\n",
                  (unsigned long long)p.n, (unsigned long long)p.m, (unsigned long long)p.rm,
                  max_level_, sec);
    return p;
  }

 private:
  // Tentative distances of one search: a small open-addressing table
  // (entries of earlier searches told apart by a generation stamp) that
  // stays in cache, moved to arrays over all vertices when a search
  // outgrows it (allocated on the first such search).
  struct Scratch {
    static constexpr uint32_t kBits = 10, kCap = 1u << kBits, kMaxFill = 3 * kCap / 4;
    uint64_t n = 0;
    std::vector<uint32_t> hkey, hgen;
    std::vector<uint64_t> hdist;
    uint32_t gen = 0, fill = 0;
    bool big = false;  // this search lives in the arrays
    std::vector<uint64_t> dist;
    std::vector<uint32_t> stamp;
    uint32_t cur = 0;
    void init(uint64_t nv) {
      n = nv;
      hkey.assign(kCap, 0);
      hgen.assign(kCap, 0);
      hdist.assign(kCap, kInf);
    }
    void reset() {
      if (++gen == 0) {
        std::fill(hgen.begin(), hgen.end(), 0);
        gen = 1;
      }
      fill = 0;
      big = false;
    }
    uint32_t slot(uint32_t v) const {
      uint32_t h = (v * 0x9E3779B1u) >> (32 - kBits);
      while (hgen[h] == gen && hkey[h] != v) h = (h + 1) & (kCap - 1);
      return h;
    }
    uint64_t get(uint32_t v) const {
      if (big) return stamp[v] == cur ? dist[v] : kInf;
      const uint32_t h = slot(v);
      return hgen[h] == gen ? hdist[h] : kInf;
    }
    void set(uint32_t v, uint64_t d) {
      if (!big) {
        const uint32_t h = slot(v);
        if (hgen[h] == gen) {
          hdist[h] = d;
          return;
        }
        if (fill < kMaxFill) {
          hgen[h] = gen;
          hkey[h] = v;
          hdist[h] = d;
          ++fill;
          return;
        }
        spill();
      }
      stamp[v] = cur;
      dist[v] = d;
    }
    void spill() {
      if (dist.empty()) {
        dist.assign(n, kInf);
        stamp.assign(n, 0);
      }
      if (++cur == 0) {
        std::fill(stamp.begin(), stamp.end(), 0);
        cur = 1;
      }
      for (uint32_t h = 0; h < kCap; ++h)
        if (hgen[h] == gen) {
          stamp[hkey[h]] = cur;
          dist[hkey[h]] = hdist[h];
        }
      big = true;
    }
  };

  uint64_t through(uint32_t x) const { return use_len_ ? len_[x] - 1 : 0; }

  // Bounded Dijkstra from s over the current overlay (build_pch.hpp:230-394):
  // the first hop costs the arc weight, every later hop also pays len-1 of
  // the vertex it leaves; never re-enters s; at most pop_limit_ pops.
  void search(uint32_t s, uint64_t bound, Scratch& sc) const {
    sc.reset();
    using T = std::pair<uint64_t, uint32_t>;
    std::priority_queue<T, std::vector<T>, std::greater<T>> pq;
    for (const Arc& a : out_[s]) {
      if (a.w < sc.get(a.v)) {
        sc.set(a.v, a.w);
        pq.push({a.w, a.v});
      }
    }
    uint32_t pops = 0;
    while (!pq.empty() && pops < pop_limit_) {
      auto [d, x] = pq.top();
      if (d > bound) break;
      pq.pop();
      if (sc.get(x) < d) continue;
      ++pops;
      const uint64_t base = d + through(x);
      for (const Arc& a : out_[x]) {
        if (a.v == s) continue;
        uint64_t nd = base + a.w;
        if (nd < sc.get(a.v)) {
          sc.set(a.v, nd);
          pq.push({nd, a.v});
        }
      }
    }
  }

  // The overlay snapshot of this round for the device searches: the
  // remaining vertices renumbered by their index in `remaining` (cid_), as
  // every arc joins two remaining vertices.
  void upload_overlay(const std::vector<uint32_t>& remaining, int nthreads) {
    const size_t R = remaining.size();
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (size_t i = 0; i < R; ++i) cid_[remaining[i]] = (uint32_t)i;
    std::vector<uint32_t> off(R + 1, 0), thru(R);
    for (size_t i = 0; i < R; ++i) {
      require(off[i] + out_[remaining[i]].size() < (1ull << 32), CHSGA_ERR_UNSUPPORTED,
              "hierarchy builder: overlay above 2^32 arcs");
      off[i + 1] = off[i] + (uint32_t)out_[remaining[i]].size();
    }
    std::vector<uint64_t> arcs(off[R]);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (size_t i = 0; i < R; ++i) {
      const uint32_t u = remaining[i];
      thru[i] = (uint32_t)through(u);
      for (size_t j = 0; j < out_[u].size(); ++j)
        arcs[off[i] + j] = cid_[out_[u][j].v] | (uint64_t)out_[u][j].w << 32;
    }
    gpu_->set_overlay(off, arcs, thru);
  }

  // Shortcuts contracting u would need, relevance of u's in-arcs, and the
  // edge-difference score (build_pch.hpp:396-478, 1012-1045). masks, when
  // given, holds the device's answer for each in-arc (pch_gpu.hpp); an
  // in-arc whose search overflowed there is searched here.
  void score(uint32_t u, std::vector<Shortcut>& cuts, uint8_t* in_rel, Scratch& sc,
             const uint64_t* masks) {
    const auto& in = in_[u];
    const auto& out = out_[u];
    uint64_t max_out = 0;
    for (const Arc& b : out) max_out = std::max<uint64_t>(max_out, b.w);
    uint64_t added = 0, added_hop = 0;
    for (size_t i = 0; i < in.size(); ++i) {
      const Arc& a = in[i];
      const uint64_t m = masks ? masks[i] : kPchOverflow;
      const bool host = (m & kPchOverflow) != 0;
      if (host) {
        search(a.v, (uint64_t)a.w + through(u) + max_out, sc);
        in_rel[i] = sc.get(u) >= a.w ? 1 : 0;
      } else {
        in_rel[i] = (uint8_t)((m >> 62) & 1);
      }
      for (size_t j = 0; j < out.size(); ++j) {
        const Arc& b = out[j];
        if (b.v == a.v) continue;
        uint64_t total = (uint64_t)a.w + b.w + through(u);
        if (total <= k_ && (host ? sc.get(b.v) >= total : ((m >> j) & 1) != 0)) {
          require(total < (1ull << 32), CHSGA_ERR_UNSUPPORTED, "shortcut weight overflow");
          cuts.push_back({a.v, b.v, (uint32_t)total, a.hop + b.hop});
          ++added;
          added_hop += a.hop + b.hop;
        }
      }
    }
    if (in.empty() || out.empty()) {
      ed_[u] = 0.f;
      return;
    }
    const double removed_arc = 1.0 + (double)in.size() + (double)out.size();
    double removed_hop = 1.0;
    for (const Arc& a : in) removed_hop += a.hop;
    for (const Arc& b : out) removed_hop += b.hop;
    ed_[u] = (float)(1.0 + 500.0 * level_[u] +
                     1000.0 * ((double)added + 0.2 * removed_nbr_[u]) / removed_arc +
                     1000.0 * (double)added_hop / removed_hop + 10.0 * removed_arc);
  }

  // Relevance of u's out-arcs: kept unless a strictly shorter u->b path
  // exists (the device's mask when it finished the search).
  void out_relevance(uint32_t u, uint8_t* rel, Scratch& sc, uint64_t mask) {
    const auto& out = out_[u];
    if (!(mask & kPchOverflow)) {
      for (size_t i = 0; i < out.size(); ++i) rel[i] = (uint8_t)((mask >> i) & 1);
      return;
    }
    uint64_t max_out = 0;
    for (const Arc& b : out) max_out = std::max<uint64_t>(max_out, b.w);
    search(u, max_out, sc);
    for (size_t i = 0; i < out.size(); ++i) rel[i] = sc.get(out[i].v) >= out[i].w ? 1 : 0;
  }

  double upper_bound(const std::vector<uint32_t>& rem, uint32_t round) const {
    if (opt_.sample_bound >= 1.0 || opt_.sample_bound <= 0.0)
      return std::numeric_limits<double>::max();
    constexpr int kSamples = 150;  // EDGEDIFF_SAMPLES, build_pch.hpp:19
    Rng rng((opt_.seed ? opt_.seed : 0x5eed) + round);
    if (rem.size() < kSamples) return ed_[rem[rng.below(rem.size())]];
    std::vector<double> s(kSamples + 1);
    for (auto& x : s) x = ed_[rem[rng.below(rem.size())]];
    std::sort(s.begin(), s.end());
    return s[(size_t)(kSamples * opt_.sample_bound)];
  }

  bool eligible(uint32_t u, double bound) const {
    if (ed_[u] > bound) return false;
    const size_t du = in_[u].size() + out_[u].size();
    auto beats = [&](uint32_t v) {
      if (ed_[v] > bound) return false;
      if (ed_[v] != ed_[u]) return ed_[v] < ed_[u];
      const size_t dv = in_[v].size() + out_[v].size();
      if (dv != du) return dv < du;
      return prio_[v] < prio_[u];
    };
    for (const Arc& a : out_[u])
      if (beats(a.v)) return false;
    for (const Arc& a : in_[u])
      if (beats(a.v)) return false;
    return true;
  }

  static void erase_arc(std::vector<Arc>& v, uint32_t x) {
    for (size_t i = 0; i < v.size(); ++i)
      if (v[i].v == x) {
        v[i] = v.back();
        v.pop_back();
        return;
      }
  }

  void contract(uint32_t u, const Shortcut* cuts, size_t ncuts, const uint8_t* in_rel,
                const uint8_t* out_rel) {
    // level_[u] is final here (only neighbours of contracted vertices
    // change level, and u has none this round); a neighbour may be shared
    // with a vertex of the same wave, so its level and count are updated
    // atomically (max and sum do not depend on the order)
    const uint32_t lu = level_[u] + 1;
    auto raise = [&](uint32_t x) {
      uint32_t* p = &level_[x];
      uint32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
      while (cur < lu && !__atomic_compare_exchange_n(p, &cur, lu, true, __ATOMIC_RELAXED,
                                                      __ATOMIC_RELAXED)) {
      }
      __atomic_fetch_add(&removed_nbr_[x], 1u, __ATOMIC_RELAXED);
    };
    for (size_t i = 0; i < out_[u].size(); ++i) {
      const Arc& b = out_[u][i];
      if (out_rel[i]) {
        up_[u].push_back({b.v, b.w, b.hop});
        raise(b.v);
      }
      erase_arc(in_[b.v], u);
    }
    for (size_t i = 0; i < in_[u].size(); ++i) {
      const Arc& a = in_[u][i];
      if (in_rel[i]) {
        down_[u].push_back({a.v, a.w, a.hop});
        raise(a.v);
      }
      erase_arc(out_[a.v], u);
    }
    for (size_t c = 0; c < ncuts; ++c) {
      const Shortcut& s = cuts[c];
      bool found = false;
      for (Arc& x : out_[s.a])
        if (x.v == s.b) {
          found = true;
          if (s.w < x.w) {
            x.w = s.w;
            x.hop = s.hop;
            for (Arc& y : in_[s.b])
              if (y.v == s.a) {
                y.w = s.w;
                y.hop = s.hop;
              }
          }
          break;
        }
      if (!found) {
        out_[s.a].push_back({s.b, s.w, s.hop});
        in_[s.b].push_back({s.a, s.w, s.hop});
      }
    }
    out_[u].clear();
    out_[u].shrink_to_fit();
    in_[u].clear();
    in_[u].shrink_to_fit();
    contracted_[u] = 1;
  }

  HostPch order(int nthreads) {
    // connected components of the input graph, ignoring direction
    std::vector<uint32_t> parent(n_);
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](uint32_t x) {
      while (parent[x] != x) x = parent[x] = parent[parent[x]];
      return x;
    };
    for (auto& [u, v, w] : base_edges_) {
      (void)w;
      uint32_t a = find(u), b = find(v);
      if (a != b) parent[std::max(a, b)] = std::min(a, b);
    }
    std::vector<uint32_t> cc(n_);
    for (uint64_t i = 0; i < n_; ++i) cc[i] = find((uint32_t)i);
    std::vector<uint32_t> ord(n_);
    std::iota(ord.begin(), ord.end(), 0);
    // a strict total order (ids break every tie): any sort gives one result
    __gnu_parallel::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
      if (cc[a] != cc[b]) return cc[a] < cc[b];
      if (level_[a] != level_[b]) return level_[a] < level_[b];
      return a < b;
    });
    HostPch p;
    p.present = true;
    p.n = n_;
    p.rank.resize(n_);
    p.level.resize(n_);
    for (uint64_t r = 0; r < n_; ++r) {
      p.rank[ord[r]] = (uint32_t)r;
      p.level[r] = level_[ord[r]];
      max_level_ = std::max(max_level_, level_[ord[r]]);
    }
    for (uint64_t r = 0; r <= n_; ++r) {
      bool cut = r == 0 || r == n_ || cc[ord[r]] != cc[ord[r - 1]] ||
                 level_[ord[r]] != level_[ord[r - 1]];
      if (cut) p.layer_offset.push_back((uint32_t)r);
    }
    for (size_t l = 0; l < p.layer_offset.size(); ++l) {
      size_t L = p.layer_offset.size() - 1;
      bool cut = l == 0 || l == L || cc[ord[p.layer_offset[l]]] != cc[ord[p.layer_offset[l - 1]]];
      if (cut) p.cc_offset.push_back((uint32_t)l);
    }
    auto emit = [&](const std::vector<std::vector<Arc>>& lists, std::vector<uint64_t>& off,
                    std::vector<uint32_t>& vv, std::vector<uint32_t>& ww) {
      off.assign(n_ + 1, 0);
      for (uint64_t r = 0; r < n_; ++r) off[r + 1] = off[r] + lists[ord[r]].size();
      vv.resize(off[n_]);
      ww.resize(off[n_]);
#pragma omp parallel num_threads(nthreads)
      {
        std::vector<std::pair<uint32_t, uint32_t>> tmp;
#pragma omp for schedule(dynamic, 4096)
        for (int64_t r = 0; r < (int64_t)n_; ++r) {
          tmp.clear();
          for (const Arc& a : lists[ord[r]]) tmp.push_back({p.rank[a.v], a.w});
          std::sort(tmp.begin(), tmp.end());
          for (size_t i = 0; i < tmp.size(); ++i) {
            vv[off[r] + i] = tmp[i].first;
            ww[off[r] + i] = tmp[i].second;
          }
        }
      }
    };
    emit(up_, p.up_offset, p.up_v, p.up_w);
    emit(down_, p.down_offset, p.down_v, p.down_w);
    p.m = p.up_v.size();
    p.rm = p.down_v.size();
    return p;
  }

  chsga_pch_opts opt_;
  uint64_t n_;
  bool use_len_ = false;
  std::vector<uint64_t> len_;
  uint64_t k_ = kInf;
  uint32_t pop_limit_ = 500;
  std::vector<std::tuple<uint32_t, uint32_t, uint32_t>> base_edges_;
  std::vector<std::vector<Arc>> out_, in_, up_, down_;
  std::vector<uint32_t> level_, removed_nbr_;
  std::vector<uint8_t> contracted_;
  std::vector<float> ed_;
  std::vector<uint32_t> prio_;
  std::vector<Scratch> scratch_;
  struct CutRef {
    uint32_t thread, count;
    uint64_t start;
  };
  std::vector<std::vector<Shortcut>> tcuts_;  // per-thread shortcut buffers of a round
  // smallest selection index of a pending vertex that changes in_[x] /
  // out_[x] in the current contraction wave (kNoClaim between waves)
  static constexpr uint32_t kNoClaim = 0xFFFFFFFFu;
  std::vector<uint32_t> claim_in_, claim_out_;
  std::unique_ptr<PchGpu> gpu_;
  static constexpr uint32_t kNoId = 0xFFFFFFFFu;
  std::vector<uint32_t> cid_;  // device overlay id of each remaining vertex
  uint32_t max_level_ = 0;
};

}  // namespace

HostPch build_pch(const HostCsr& g, const std::vector<uint64_t>& offs, const chsga_pch_opts& o) {
  PchBuilder b(g, offs, o);
  return b.build();
}

}  // namespace chsga
