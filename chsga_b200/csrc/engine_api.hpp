// Internal interface between the device engine (engine.cu) and the serving
// loop (server.cpp). Not part of the C-ABI.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "common.hpp"

namespace chsga {

// A new context on the same device that shares `parent`'s loaded graph (no
// copy) and has its own streams and working buffers. Close it with
// chsga_close; the graph lives while any context holds it.
chsga_ctx* fork_context(chsga_ctx& parent);

// Device bytes a traceback of a read of `len` bases takes at its peak on a
// context of this graph (the full matrix, or the checkpointed path's row
// ring and largest recompute segment), excluding the context's fixed
// per-slot buffers.
uint64_t traceback_device_bytes(const chsga_ctx& c, uint32_t len, const chsga_tb_opts* o);

// Chars N and string vertices S of the context's graph.
uint64_t graph_chars(const chsga_ctx& c);
uint64_t graph_string_vertices(const chsga_ctx& c);
// Score a length-0 read gets (the reference scores row 0 against '\0').
int32_t empty_read_score(const chsga_ctx& c);
// Makes the context's device current on the calling thread.
void bind_device(const chsga_ctx& c);
// Free device memory now (cudaMemGetInfo) on the context's device.
uint64_t device_free_bytes(const chsga_ctx& c);
// Device bytes the library allocated on this thread: meter_reset starts a
// window (returns its base), meter_peak_since(base) is the window's peak
// above the base.
int64_t meter_reset();
uint64_t meter_peak_since(int64_t base);
// Cost-model features of one request (chsga_cm_features).
void request_features(const chsga_ctx& c, uint32_t len, uint32_t mode, uint32_t slots, int64_t k,
                      uint64_t cap_bytes, float* x);

// Queue entry of the score lane: bytes at `off` in the lane's arena.
struct LaneRead {
  uint64_t off;
  uint32_t len;
  uint32_t id;  // result slot, < capacity
};

// A finished read of the score lane; times are host steady-clock ns.
struct LaneDone {
  uint32_t id;
  int32_t score;
  uint32_t vertex;
  int64_t admit_ns, done_ns;
};

// The batched engine run continuously: a forked context whose R slots take
// reads from a device queue ring that the host refills between CUDA-graph
// blocks of row-steps. Every call comes from one host thread.
class ScoreLane {
 public:
  virtual ~ScoreLane() = default;
  virtual uint32_t capacity() const = 0;      // queue ring entries = result slots
  virtual uint64_t arena_bytes() const = 0;   // device bytes for read bases
  virtual unsigned char* staging() = 0;       // pinned host mirror of the arena
  // Copies arena bytes [lo, hi) from the mirror, appends the reads to the
  // queue ring and publishes them to the device (stream-ordered, before the
  // next block).
  virtual void publish(uint64_t lo, uint64_t hi, const LaneRead* reads, uint32_t n) = 0;
  // Launches one block of row-steps, then harvests the block launched
  // before it (one block behind the device); completions are appended.
  virtual void step(std::vector<LaneDone>& out) = 0;
  // Waits for every launched block and harvests them.
  virtual void drain(std::vector<LaneDone>& out) = 0;
  virtual uint64_t blocks() const = 0;        // blocks launched
  virtual uint32_t kernels_per_block() const = 0;
  // Self-test of the failure path: enqueues a bounded device-side wait that
  // cannot succeed against the lane's control block; the harvest of the
  // next block then fails with CHSGA_ERR_TIMEOUT, as for an expired wait.
  virtual void inject_wait_timeout() = 0;
};

// slots: 2..128 (power of two); capacity: power of two; row_bits 16 or 32.
std::unique_ptr<ScoreLane> make_score_lane(chsga_ctx& parent, uint32_t slots, uint32_t per_graph,
                                           uint32_t capacity, uint64_t arena_bytes,
                                           uint32_t row_bits);

}  // namespace chsga
