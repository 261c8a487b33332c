// Serving loop behind chsga_server_* (include/chsga.h). No reference
// counterpart: the reference aligns a fixed read set serially
// (src/align.hpp:488, src/ConSGA_traceback.cpp:160-225).
//
// Score requests: one engine thread drives a ScoreLane (engine.cu), a
// forked context whose batched engine runs continuously in CUDA-graph
// blocks of row-steps. Between blocks the thread admits waiting reads in
// arrival order while the lane has free result slots and its device arena
// has room for their bases (one arena block per admission round, released
// when its last read finishes), and harvests finished reads one block
// behind the device.
//
// Traceback requests: worker threads, each with a forked context sharing
// the graph, take requests in arrival order; the request at the head runs
// once its projected device footprint fits what the running ones leave of
// the budget (head-of-line: a large request is never overtaken forever).
#include <algorithm>
#include <chrono>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine_api.hpp"

namespace chsga {
extern thread_local std::string g_last_error;
namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

constexpr uint64_t kArenaAlign = 256;
constexpr uint64_t kNone = ~0ull;

uint64_t round_up(uint64_t n, uint64_t a) { return (n + a - 1) / a * a; }

// First-fit allocator over [0, bytes) with coalescing frees.
class ArenaAlloc {
 public:
  explicit ArenaAlloc(uint64_t bytes) : total_(bytes) {
    if (bytes) free_[0] = bytes;
  }
  uint64_t alloc(uint64_t n) {
    n = round_up(std::max<uint64_t>(n, 1), kArenaAlign);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      const uint64_t off = it->first, rest = it->second - n;
      free_.erase(it);
      if (rest) free_[off + n] = rest;
      used_ += n;
      return off;
    }
    return kNone;
  }
  void release(uint64_t off, uint64_t n) {
    n = round_up(std::max<uint64_t>(n, 1), kArenaAlign);
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  uint64_t used() const { return used_; }
  uint64_t total() const { return total_; }

 private:
  uint64_t total_, used_ = 0;
  std::map<uint64_t, uint64_t> free_;
};

struct Request {
  uint64_t ticket = 0;
  uint32_t mode = CHSGA_REQ_SCORE;
  std::string read;
  int64_t submit_ns = 0;
  uint64_t footprint = 0;  // traceback: projected device bytes
  float predicted_ms = 0;
};

struct Running {  // a score read on the lane
  uint64_t ticket;
  int64_t submit_ns;
  uint32_t len;
  uint64_t block;  // arena block holding its bases
};

struct Block {
  uint64_t bytes;
  uint32_t live;
};

double percentile_ms(std::vector<int64_t> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const size_t i = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
  return (double)v[i] / 1e6;
}

}  // namespace
}  // namespace chsga

using namespace chsga;

struct chsga_server {
  chsga_ctx* ctx = nullptr;
  chsga_server_opts o{};
  uint64_t num_chars = 0;
  int32_t empty_score = 1;
  std::unique_ptr<ScoreLane> lane;
  std::vector<chsga_ctx*> tb_ctx;
  std::thread engine;
  std::vector<std::thread> workers;

  std::mutex mu;
  std::mutex cm_mu;  // the cost model is not re-entrant
  std::condition_variable cv_engine, cv_tb, cv_done;
  std::deque<Request> pend_score, pend_tb;
  bool pend_dirty = false;  // score requests arrived since the last ordering
  std::deque<chsga_server_result> done;
  bool stop = false;
  chsga_status broken = CHSGA_OK;  // the score lane failed: score requests fail with this
  std::atomic<bool> inject_fail{false};  // chsga_server_selftest_fail: at the next block
  std::string err;
  uint64_t next_ticket = 1;
  uint64_t submitted = 0, finished = 0, failed = 0;
  uint64_t lane_running = 0;  // published to the lane, not yet harvested
  uint64_t tb_running = 0, tb_used = 0, tb_peak = 0;
  uint64_t cells = 0;
  int64_t first_submit = 0, last_done = 0;
  std::vector<int64_t> lat_score, lat_tb;

  // engine-thread state
  ArenaAlloc arena{0};
  std::vector<uint32_t> free_ids;
  std::vector<Running> running;
  std::unordered_map<uint64_t, Block> blocks;

  void finish(chsga_server_result&& r) {  // under mu
    if (r.status == CHSGA_OK) {
      const int64_t lat = r.done_ns - r.submit_ns;
      (r.mode == CHSGA_REQ_SCORE ? lat_score : lat_tb).push_back(lat);
      cells += (uint64_t)r.read_len * num_chars;
      last_done = std::max(last_done, r.done_ns);
    } else {
      ++failed;
    }
    ++finished;
    done.push_back(r);
    cv_done.notify_all();
  }

  void fail_score_requests(chsga_status st) {  // under mu
    broken = st;
    for (auto& q : pend_score) {
      chsga_server_result r{};
      r.ticket = q.ticket;
      r.status = st;
      r.mode = CHSGA_REQ_SCORE;
      r.submit_ns = q.submit_ns;
      r.done_ns = now_ns();
      finish(std::move(r));
    }
    pend_score.clear();
    for (auto& x : running) {
      if (x.ticket == 0) continue;
      chsga_server_result r{};
      r.ticket = x.ticket;
      r.status = st;
      r.mode = CHSGA_REQ_SCORE;
      r.submit_ns = x.submit_ns;
      r.done_ns = now_ns();
      finish(std::move(r));
      x.ticket = 0;
    }
    lane_running = 0;
  }

  // Takes waiting score reads (arrival order) into one arena block and
  // publishes them; returns how many.
  uint32_t admit_scores() {
    std::vector<Request> batch;
    {
      std::lock_guard<std::mutex> lk(mu);
      if (o.order == CHSGA_ORDER_LONGEST && pend_dirty) {
        std::stable_sort(pend_score.begin(), pend_score.end(), [](const Request& a, const Request& b) {
          return a.read.size() > b.read.size();
        });
        pend_dirty = false;
      }
      uint64_t bytes = 0;
      while (!pend_score.empty() && batch.size() < free_ids.size()) {
        const uint64_t b = round_up(pend_score.front().read.size(), 16);
        if (bytes + b > arena.total()) break;
        bytes += b;
        batch.push_back(std::move(pend_score.front()));
        pend_score.pop_front();
      }
      if (batch.empty()) return 0;
      // shrink to what the arena can hold now; the rest goes back in front
      uint64_t base = kNone;
      while (!batch.empty()) {
        base = arena.alloc(bytes);
        if (base != kNone) break;
        const uint64_t b = round_up(batch.back().read.size(), 16);
        bytes -= b;
        pend_score.push_front(std::move(batch.back()));
        batch.pop_back();
      }
      if (batch.empty()) return 0;
      blocks[base] = Block{bytes, (uint32_t)batch.size()};
      lane_running += batch.size();
      std::vector<LaneRead> pub(batch.size());
      uint64_t off = base;
      unsigned char* st = lane->staging();
      for (size_t i = 0; i < batch.size(); ++i) {
        const uint32_t id = free_ids.back();
        free_ids.pop_back();
        const uint32_t len = (uint32_t)batch[i].read.size();
        std::memcpy(st + off, batch[i].read.data(), len);
        pub[i] = LaneRead{off, len, id};
        running[id] = Running{batch[i].ticket, batch[i].submit_ns, len, base};
        off += round_up(len, 16);
      }
      // the lock is held across the host->device publication so close()
      // and stats see a consistent count; it is a handful of async calls
      lane->publish(base, base + bytes, pub.data(), (uint32_t)pub.size());
    }
    return (uint32_t)batch.size();
  }

  void collect(std::vector<LaneDone>& d) {
    if (d.empty()) return;
    std::lock_guard<std::mutex> lk(mu);
    for (const LaneDone& x : d) {
      Running& run = running[x.id];
      chsga_server_result r{};
      r.ticket = run.ticket;
      r.status = CHSGA_OK;
      r.score = x.score;
      r.vertex = x.vertex;
      r.read_len = run.len;
      r.mode = CHSGA_REQ_SCORE;
      r.submit_ns = run.submit_ns;
      // device times, mapped to the host clock; admission cannot precede
      // the submission that caused it
      r.start_ns = std::max(run.submit_ns, x.admit_ns);
      r.done_ns = std::max(r.start_ns, x.done_ns);
      auto it = blocks.find(run.block);
      if (it != blocks.end() && --it->second.live == 0) {
        arena.release(it->first, it->second.bytes);
        blocks.erase(it);
      }
      run.ticket = 0;
      free_ids.push_back(x.id);
      --lane_running;
      finish(std::move(r));
    }
    d.clear();
    cv_engine.notify_all();
  }

  void engine_loop() {
    std::vector<LaneDone> d;
    try {
      bind_device(*ctx);
      while (true) {
        {
          std::unique_lock<std::mutex> lk(mu);
          cv_engine.wait(lk, [&] { return stop || !pend_score.empty() || lane_running > 0; });
          if (stop && pend_score.empty() && lane_running == 0) break;
        }
        admit_scores();
        bool busy;
        {
          std::lock_guard<std::mutex> lk(mu);
          busy = lane_running > 0;
        }
        if (busy) {
          if (inject_fail.exchange(false)) lane->inject_wait_timeout();
          lane->step(d);
          collect(d);
        }
      }
      lane->drain(d);
      collect(d);
    } catch (const ChsgaError& e) {
      std::lock_guard<std::mutex> lk(mu);
      err = e.what();
      fail_score_requests(e.status);
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lk(mu);
      err = e.what();
      fail_score_requests(CHSGA_ERR_INTERNAL);
    }
  }

  void tb_loop(size_t w) {
    chsga_ctx* c = tb_ctx[w];
    const uint64_t budget = o.hbm_budget_bytes;
    while (true) {
      Request q;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_tb.wait(lk, [&] {
          return stop || (!pend_tb.empty() && tb_used + pend_tb.front().footprint <= budget);
        });
        if (pend_tb.empty() || tb_used + pend_tb.front().footprint > budget) {
          if (stop) break;
          continue;
        }
        q = std::move(pend_tb.front());
        pend_tb.pop_front();
        tb_used += q.footprint;
        tb_peak = std::max(tb_peak, tb_used);
        ++tb_running;
      }
      chsga_server_result r{};
      r.ticket = q.ticket;
      r.read_len = (uint32_t)q.read.size();
      r.mode = CHSGA_REQ_TRACEBACK;
      r.submit_ns = q.submit_ns;
      r.projected_bytes = q.footprint;
      r.predicted_ms = q.predicted_ms;
      r.start_ns = now_ns();
      chsga_tb_opts t{o.tb_k, nullptr, 0, o.tb_cap_bytes};
      const int64_t base = meter_reset();
      r.status = chsga_align_traceback(c, q.read.data(), (uint32_t)q.read.size(), &t, &r.tb);
      r.peak_bytes = meter_peak_since(base);
      r.score = r.tb.score;
      r.done_ns = now_ns();
      std::lock_guard<std::mutex> lk(mu);
      if (r.status != CHSGA_OK && err.empty()) err = chsga_last_error(c);
      tb_used -= q.footprint;
      --tb_running;
      finish(std::move(r));
      cv_tb.notify_all();
    }
  }
};

namespace {

template <typename F>
chsga_status guarded_srv(chsga_server* s, F&& f) {
  try {
    f();
    return CHSGA_OK;
  } catch (const ChsgaError& e) {
    if (s) {
      std::lock_guard<std::mutex> lk(s->mu);
      s->err = e.what();
    }
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

void stop_server(chsga_server* s) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_engine.notify_all();
  s->cv_tb.notify_all();
  if (s->engine.joinable()) s->engine.join();
  for (auto& t : s->workers)
    if (t.joinable()) t.join();
  s->workers.clear();
}

}  // namespace

extern "C" {

chsga_status chsga_server_open(chsga_ctx* ctx, const chsga_server_opts* opts, chsga_server** out) {
  return guarded_srv(nullptr, [&] {
    require(ctx && out, CHSGA_ERR_INVALID_ARG, "null argument");
    auto s = std::make_unique<chsga_server>();
    chsga_server_opts o = opts ? *opts : chsga_server_opts{};
    if (!o.slots) o.slots = 128;
    if (!o.steps_per_graph) o.steps_per_graph = 8;
    if (!o.queue_capacity) o.queue_capacity = 4096;
    if (!o.tb_workers) o.tb_workers = 2;
    if (!o.arena_bytes) o.arena_bytes = 64ull << 20;
    if (!o.tb_k) o.tb_k = 500;
    if (!o.row_bits) o.row_bits = 16;
    if (!o.max_pending) o.max_pending = 1u << 20;
    require(o.footprint <= CHSGA_FP_ANALYTIC, CHSGA_ERR_INVALID_ARG, "footprint must be CHSGA_FP_*");
    require(o.order <= CHSGA_ORDER_LONGEST, CHSGA_ERR_INVALID_ARG, "order must be CHSGA_ORDER_*");
    require(o.footprint != CHSGA_FP_MODEL || o.cost_model, CHSGA_ERR_INVALID_ARG,
            "CHSGA_FP_MODEL needs a cost model");
    require(o.tb_workers <= 16, CHSGA_ERR_INVALID_ARG, "at most 16 traceback workers");
    s->ctx = ctx;
    s->num_chars = graph_chars(*ctx);
    s->empty_score = empty_read_score(*ctx);
    if (!o.hbm_budget_bytes) o.hbm_budget_bytes = device_free_bytes(*ctx) / 2;
    s->o = o;
    s->lane = make_score_lane(*ctx, o.slots, o.steps_per_graph, o.queue_capacity, o.arena_bytes,
                              o.row_bits);
    s->arena = ArenaAlloc(o.arena_bytes);
    s->running.resize(o.queue_capacity);
    for (uint32_t i = o.queue_capacity; i-- > 0;) s->free_ids.push_back(i);
    try {
      for (uint32_t w = 0; w < o.tb_workers; ++w) s->tb_ctx.push_back(fork_context(*ctx));
    } catch (...) {
      for (auto* c : s->tb_ctx) chsga_close(c);
      throw;
    }
    chsga_server* p = s.get();
    p->engine = std::thread([p] { p->engine_loop(); });
    for (uint32_t w = 0; w < o.tb_workers; ++w) p->workers.emplace_back([p, w] { p->tb_loop(w); });
    *out = s.release();
  });
}

chsga_status chsga_server_selftest_fail(chsga_server* s) {
  return guarded_srv(s, [&] {
    require(s != nullptr, CHSGA_ERR_INVALID_ARG, "null argument");
    s->inject_fail = true;
    std::lock_guard<std::mutex> lk(s->mu);
    s->cv_engine.notify_all();
  });
}

chsga_status chsga_server_submit(chsga_server* s, const char* read, uint32_t len, uint32_t mode,
                                 uint64_t* ticket) {
  return guarded_srv(s, [&] {
    require(s && (read || len == 0), CHSGA_ERR_INVALID_ARG, "null argument");
    require(mode == CHSGA_REQ_SCORE || mode == CHSGA_REQ_TRACEBACK, CHSGA_ERR_INVALID_ARG,
            "mode must be CHSGA_REQ_SCORE or CHSGA_REQ_TRACEBACK");
    Request q;
    q.mode = mode;
    if (mode == CHSGA_REQ_SCORE) {
      require(!(s->o.row_bits == 16 && len > 65000), CHSGA_ERR_UNSUPPORTED,
              "score reads over 65000 bases need a server with row_bits = 32");
      require(round_up(len, 16) <= s->o.arena_bytes, CHSGA_ERR_INVALID_ARG,
              "read longer than the server's arena");
    } else {
      require(len > 0, CHSGA_ERR_INVALID_ARG, "traceback of an empty read");
      chsga_tb_opts t{s->o.tb_k, nullptr, 0, s->o.tb_cap_bytes};
      q.footprint = traceback_device_bytes(*s->tb_ctx[0], len, &t);
      if (s->o.cost_model) {
        float x[CHSGA_CM_FEATURES], y[CHSGA_CM_OUTPUTS];
        request_features(*s->tb_ctx[0], len, mode, 1, s->o.tb_k, s->o.tb_cap_bytes, x);
        std::lock_guard<std::mutex> lk(s->cm_mu);
        const chsga_status st = chsga_cm_predict(s->o.cost_model, x, 1, y);
        require(st == CHSGA_OK, st, "cost model prediction failed");
        q.predicted_ms = y[0];
        if (s->o.footprint == CHSGA_FP_MODEL) q.footprint = (uint64_t)std::max(0.f, y[1]);
      }
      if (s->o.footprint == CHSGA_FP_ANALYTIC) q.footprint = 4ull * len * s->num_chars;
      require(q.footprint <= s->o.hbm_budget_bytes, CHSGA_ERR_OOM,
              "traceback footprint " + std::to_string(q.footprint) + " bytes exceeds the budget");
    }
    q.read.assign(read ? read : "", len);
    std::lock_guard<std::mutex> lk(s->mu);
    require(!s->stop, CHSGA_ERR_INVALID_ARG, "server is closing");
    if (mode == CHSGA_REQ_SCORE && s->broken != CHSGA_OK)
      fail(s->broken, "score lane failed: " + s->err);
    const uint64_t pending = s->pend_score.size() + s->pend_tb.size();
    if (pending >= s->o.max_pending) fail(CHSGA_ERR_BUSY, "server queue full");
    q.ticket = s->next_ticket++;
    q.submit_ns = now_ns();
    if (s->submitted == 0) s->first_submit = q.submit_ns;
    ++s->submitted;
    if (ticket) *ticket = q.ticket;
    if (mode == CHSGA_REQ_SCORE && len == 0) {
      // row 0 against '\0', as chsga_align_scores
      chsga_server_result r{};
      r.ticket = q.ticket;
      r.score = s->empty_score;
      r.mode = CHSGA_REQ_SCORE;
      r.submit_ns = r.start_ns = r.done_ns = q.submit_ns;
      s->finish(std::move(r));
      return;
    }
    if (mode == CHSGA_REQ_SCORE) {
      s->pend_score.push_back(std::move(q));
      s->pend_dirty = true;
      s->cv_engine.notify_all();
    } else {
      s->pend_tb.push_back(std::move(q));
      s->cv_tb.notify_all();
    }
  });
}

chsga_status chsga_server_poll(chsga_server* s, chsga_server_result* out, uint32_t max,
                               uint32_t* n_out, int32_t wait_ms) {
  return guarded_srv(s, [&] {
    require(s && n_out && (out || max == 0), CHSGA_ERR_INVALID_ARG, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] { return !s->done.empty(); };
    if (!ready() && wait_ms != 0) {
      if (wait_ms < 0)
        s->cv_done.wait(lk, [&] { return ready() || s->finished == s->submitted; });
      else
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
    }
    uint32_t n = 0;
    while (n < max && !s->done.empty()) {
      out[n++] = s->done.front();
      s->done.pop_front();
    }
    *n_out = n;
  });
}

chsga_status chsga_server_stats_get(chsga_server* s, chsga_server_stats* out) {
  return guarded_srv(s, [&] {
    require(s && out, CHSGA_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    chsga_server_stats t{};
    t.submitted = s->submitted;
    t.completed = s->finished - s->failed;
    t.failed = s->failed;
    t.pending = s->pend_score.size() + s->pend_tb.size();
    t.running = s->lane_running + s->tb_running;
    t.cells = s->cells;
    t.wall_s = s->last_done > s->first_submit ? (double)(s->last_done - s->first_submit) / 1e9 : 0.0;
    t.gcups = t.wall_s > 0 ? (double)s->cells / t.wall_s / 1e9 : 0.0;
    std::vector<int64_t> all(s->lat_score);
    all.insert(all.end(), s->lat_tb.begin(), s->lat_tb.end());
    t.p50_ms = percentile_ms(all, 0.50);
    t.p99_ms = percentile_ms(all, 0.99);
    t.score_p50_ms = percentile_ms(s->lat_score, 0.50);
    t.score_p99_ms = percentile_ms(s->lat_score, 0.99);
    t.tb_p50_ms = percentile_ms(s->lat_tb, 0.50);
    t.tb_p99_ms = percentile_ms(s->lat_tb, 0.99);
    t.peak_tb_bytes = s->tb_peak;
    t.blocks = s->lane->blocks();
    t.gpu_launches = s->lane->blocks() * s->lane->kernels_per_block();
    *out = t;
  });
}

chsga_status chsga_server_drain(chsga_server* s) {
  return guarded_srv(s, [&] {
    require(s, CHSGA_ERR_INVALID_ARG, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->finished == s->submitted; });
  });
}

void chsga_server_close(chsga_server* s) {
  if (!s) return;
  chsga_server_drain(s);
  stop_server(s);
  s->lane.reset();
  for (auto* c : s->tb_ctx) chsga_close(c);
  for (auto& r : s->done) chsga_tb_result_free(&r.tb);
  delete s;
}

const char* chsga_server_last_error(chsga_server* s) {
  return s ? s->err.c_str() : g_last_error.c_str();
}

}  // extern "C"
