// Device context, graph upload and the orchestration of the row-step kernels
// (kernels.cuh) behind the C-ABI of include/chsga.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <set>
#include <type_traits>

#include "device_graph.hpp"
#include "engine_api.hpp"
#include "host_graph.hpp"
#include "kernels.cuh"
#include "persist.cuh"

namespace chsga {

extern thread_local std::string g_last_error;
void validate_host_graph(const chsga_host_graph& g);

#define CK(x)                                                                                \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess)                                                                   \
      fail(e_ == cudaErrorMemoryAllocation ? CHSGA_ERR_OOM : CHSGA_ERR_CUDA,                 \
           std::string(#x) + ": " + cudaGetErrorString(e_));                                 \
  } while (0)

// Device bytes held by DevArr allocations made on this thread, and their
// peak since the last meter_reset (the serving loop logs a traceback
// request's peak from it).
thread_local int64_t t_live_bytes = 0, t_peak_bytes = 0;

template <typename T>
struct DevArr {
  T* p = nullptr;
  size_t n = 0;
  DevArr() = default;
  DevArr(const DevArr&) = delete;
  DevArr& operator=(const DevArr&) = delete;
  ~DevArr() { release(); }
  void release() {
    if (p) {
      cudaFree(p);
      t_live_bytes -= (int64_t)(n * sizeof(T));
    }
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count <= n && p) return;
    release();
    if (count == 0) count = 1;
    CK(cudaMalloc((void**)&p, count * sizeof(T)));
    n = count;
    t_live_bytes += (int64_t)(count * sizeof(T));
    t_peak_bytes = std::max(t_peak_bytes, t_live_bytes);
  }
  void upload(const std::vector<T>& v, cudaStream_t s) {
    alloc(v.size());
    if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  }
};

template <typename T>
struct PinnedArr {
  T* p = nullptr;
  size_t n = 0;
  PinnedArr() = default;
  PinnedArr(const PinnedArr&) = delete;
  PinnedArr& operator=(const PinnedArr&) = delete;
  ~PinnedArr() {
    if (p) cudaFreeHost(p);
  }
  void alloc(size_t count) {
    if (count <= n && p) return;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    CK(cudaHostAlloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T), cudaHostAllocDefault));
    n = count;
  }
};

struct GraphDev {
  DevArr<uint32_t> lab2, lab_sp, lab4, sv_off, sv_dev, vin_off, vin_src, vin_srcv, dv_first, dv_len;
  DevArr<uint32_t> up_off, dn_off, istr_off, istr_src;
  DevArr<uint32_t> dv_s;
  DevArr<int2> up_in, dn_in;
  DevArr<uint4> dn_head, up_head, fin;
  DevArr<uint4> t1_desc, t1_vrec;  // tiles of the one-read row kernel (k_row_t1)
  DevArr<uint8_t> t1_heads;
  DevArr<uint32_t> delta_order;    // k_row_delta: runs of 32 string vertices by decreasing char count
};

struct TopDev {
  HostTop h;
  DevArr<uint32_t> upg_off;
  DevArr<int2> upg, sched, chunks;
  dev::TopPtrs ptrs{};
};

// Buffers of one slot configuration (R slots). Score rows and boundary
// arrays are raw bytes used as int32 or uint16 storage (see scores_with).
struct SlotBufs {
  int R = 0;
  DevArr<unsigned char> rows[2];
  DevArr<unsigned char> BV;
  DevArr<unsigned char> FL;  // final first/last score per vertex, char order
  DevArr<dev::SlotState> slots;
  DevArr<uint32_t> word;
  DevArr<unsigned long long> best;
  DevArr<dev::StepCtl> ctl;
  DevArr<dev::GridBar> bar;  // grid barrier of the persistent row-step kernel
};

// Row kernel choice: the DPX kernel for 16-bit rows (default), the direct
// kernel, or the shared-memory tile-staged kernel (CHSGA_ROW_KERNEL=direct |
// tiled, for comparisons).
enum class RowKernel { Auto, Direct, Tiled, Dpx, Stream, Delta };

struct RowTileDev {
  DevArr<int4> rec;
  DevArr<uint32_t> desc;
  dev::RowTiles rt{};
  bool ok = false;
};

constexpr uint32_t kRow16Max = 65000;  // longest read whose rows fit uint16  // 2 x int32 per vertex in shared memory
constexpr int kTopThreads = 1024;

}  // namespace chsga

namespace chsga {
// A graph on the device with its host-side layout. Contexts that work on the
// same graph (the traceback workers of a server) share one instance.
struct LoadedGraph {
  HostLayout L;
  GraphDev gd;
  dev::GraphPtrs gp{};
  std::unique_ptr<TopDev> top;
  dev::T1Ptrs t1{};  // ntiles = 0: some vertex is too long for k_row_t1
  size_t pitch = 0;  // traceback matrix row stride (elements), 16-byte aligned rows
  bool nul_label = false;
  bool n_label = false;  // some label byte is 'N'
};
}  // namespace chsga

struct chsga_ctx {
  int device = 0;
  cudaStream_t st = nullptr, side = nullptr;
  std::string err;
  uint64_t cap = 0;
  uint32_t flags = 0;
  bool loaded = false;
  std::shared_ptr<chsga::LoadedGraph> g;
  std::map<int, std::unique_ptr<chsga::SlotBufs>> bufs;
  std::map<int, std::unique_ptr<chsga::RowTileDev>> row_tiles;  // by R * 8 + sizeof(score)
  // top regions other than the graph's default, by their vertex limit
  std::map<uint32_t, std::unique_ptr<chsga::TopDev>> tops;
  const chsga::TopDev* top_sel = nullptr;  // this call's top region (nullptr: the default)
  int num_sms = 148;
  chsga::RowKernel row_kernel = chsga::RowKernel::Auto;
  // launch mode of the one-read path (chsga_align_scores): CHSGA_LAUNCH_*;
  // CUDA graphs, measured faster than the persistent kernel at one slot
  uint32_t plain_mode = CHSGA_LAUNCH_GRAPHS;
  // programmatic dependent launch between the kernels of a row-step
  // (CHSGA_PDL=0 turns it off; measured 1-4 % faster per row-step)
  bool pdl = true;
  // upward levels with the lane group's cooperative edge loads, 64+ slots (CHSGA_PULL_COOP)
  bool pull_coop = false;
  // upward levels in the form bounded by the level's largest edge list
  // (CHSGA_PULL_LEAN=0 runs the unbounded form everywhere)
  bool pull_lean = true;
  // resident blocks of k_row_delta on this device (0 until the first 128-slot buffers)
  uint32_t delta_grid = 0;
  chsga::DevArr<unsigned char> reads;
  chsga::DevArr<chsga::dev::ReadDesc> queue;
  uint32_t qmask = 0xFFFFFFFFu;                      // queue ring mask (serving), else linear
  chsga::DevArr<chsga::dev::CompletionRec> done_ring;  // serving: finished reads, in order
  chsga::DevArr<int32_t> res_score;
  chsga::DevArr<uint32_t> res_vertex;
  chsga::DevArr<unsigned long long> res_t0, res_t1;  // admission / completion, device ns
  std::vector<uint32_t> last_ids;  // caller index of each queued read of the last call
  chsga::PinnedArr<chsga::dev::StepCtl> h_ctl;
  chsga::PinnedArr<int32_t> h_ckpt;     // checkpoint rows of the checkpointed traceback (int32 rows)
  chsga::PinnedArr<uint16_t> h_ckpt16;  // the same for 16-bit rows
  chsga_profile prof{};
};

namespace chsga {

namespace {

using dev::Lanes;

unsigned nblocks(uint64_t items, unsigned tpb = 256) { return (unsigned)((items + tpb - 1) / tpb); }

void set_device(chsga_ctx& c) { CK(cudaSetDevice(c.device)); }

// 1 when the context scores with matchN (an 'N' matches every base).
int match_n(const chsga_ctx& c) { return (c.flags & CHSGA_FLAG_MATCH_N) ? 1 : 0; }

// Score of a length-0 read: row 0 against the byte '\0' (the reference
// reads read[0] of an empty string), 0 if some label matches it.
int32_t empty_score(const chsga_ctx& c) {
  return (c.g->nul_label || (match_n(c) && c.g->n_label)) ? 0 : 1;
}

void check_launch() { CK(cudaGetLastError()); }

// Runs f once for each (key, device) pair: kernel attributes such as the
// dynamic shared-memory limit are per device, and several threads (serving
// lane, traceback workers) may ask at once.
template <typename F>
void once_per_device(const void* key, int device, F&& f) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({key, device})) return;
  f();
  done.insert({key, device});
}

template <int R, typename ST>
SlotBufs& get_bufs(chsga_ctx& c, bool need_rows) {
  auto& b = c.bufs[R];
  if (!b) b = std::make_unique<SlotBufs>();
  b->R = R;
  const size_t N = c.g->L.N, S = c.g->L.S;
  if (need_rows) {
    // bulk tile copies may read up to 16 bytes past the last char; 128
    // 16-bit slots may hold delta rows instead (k_row_delta)
    size_t rb = (N + 32) * R * sizeof(ST);
    if (std::is_same_v<ST, uint16_t> && R == 128) rb = std::max(rb, dev::delta_row_bytes(N, S));
    b->rows[0].alloc(rb);
    b->rows[1].alloc(rb);
  }
  b->BV.alloc(2 * S * R * sizeof(ST));
  b->FL.alloc(2 * (S + 16) * R * sizeof(ST));
  b->slots.alloc(R);
  b->word.alloc(R);
  b->best.alloc(R);
  b->ctl.alloc(1);
  b->bar.alloc(1);
  // the large dynamic shared memory of these kernels, once per device
  once_per_device((const void*)dev::k_top<R, ST>, c.device, [] {
    CK(cudaFuncSetAttribute(dev::k_top<R, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)dev::top_smem_bytes(kTopMaxVertices)));
  });
  if constexpr (std::is_same_v<ST, uint16_t> && R == 128) {
    once_per_device((const void*)dev::k_row_delta, c.device, [] {
      CK(cudaFuncSetAttribute(dev::k_row_delta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)dev::delta_smem_bytes()));
    });
    if (!c.delta_grid) {
      int per_sm = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_row_delta, dev::kStreamWarps * 32,
                                                       dev::delta_smem_bytes()));
      c.delta_grid = (uint32_t)std::max(per_sm, 1) * (uint32_t)c.num_sms;
    }
  }
  if constexpr (std::is_same_v<ST, uint16_t> && R >= 64) {
    once_per_device((const void*)dev::k_row_stream<R, true>, c.device, [] {
      for (auto k : {dev::k_row_stream<R, true>, dev::k_row_stream<R, false>})
        CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dev::stream_smem_bytes(R)));
    });
  }
  return *b;
}

const TopDev& cur_top(const chsga_ctx& c) { return c.top_sel ? *c.top_sel : *c.g->top; }

// The top region of the hierarchy with at most K vertices (levels from the
// highest down, while they fit) and its chunk schedule, on the device.
std::unique_ptr<TopDev> make_top(const HostLayout& L, const GraphDev& d, uint32_t K, cudaStream_t s) {
  auto top = std::make_unique<TopDev>();
  const uint32_t cap = dev::top_chunk_for(
      (uint32_t)std::min<size_t>(K, L.S), dev::top_smem_bytes(kTopMaxVertices));
  top->h = build_top(L, K, cap);
  const HostTop& h = top->h;
  auto to2 = [](const std::vector<EdgeW>& v) {
    std::vector<int2> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = make_int2(v[i].src, v[i].w);
    return o;
  };
  top->upg_off.upload(h.upg_off, s);
  top->upg.upload(to2(h.upg), s);
  top->sched.upload(to2(h.sched), s);
  std::vector<int2> ch(h.chunks.size());
  for (size_t i = 0; i < ch.size(); ++i) ch[i] = make_int2(h.chunks[i].first, h.chunks[i].second);
  top->chunks.upload(ch, s);
  top->ptrs = dev::TopPtrs{h.K0, h.K, (uint32_t)h.chunks.size(), top->chunks.p, top->sched.p,
                           d.dv_len.p, cap};
  CK(cudaStreamSynchronize(s));
  return top;
}

// The top region for a vertex limit (0 = the graph's default), built once
// per context and limit.
const TopDev* top_for(chsga_ctx& c, uint32_t K) {
  if (K == 0 || K == kTopDefaultVertices) return nullptr;
  require(K <= kTopMaxVertices, CHSGA_ERR_INVALID_ARG,
          "top_vertices above " + std::to_string(kTopMaxVertices) + " do not fit shared memory");
  auto& t = c.tops[K];
  if (!t) t = make_top(c.g->L, c.g->gd, K, c.st);
  return t.get();
}

// Uploads reads (raw bytes) and their queue descriptors; ids are 0..n-1.
// With longest_first the queue admits reads in decreasing length (stable), so
// the slots of the batched engine drain on the short reads at the end.
void upload_reads(chsga_ctx& c, const char* const* reads, const uint32_t* lens, uint32_t n,
                  bool longest_first = false) {
  std::vector<unsigned char> bytes;
  std::vector<dev::ReadDesc> q(n);
  uint64_t total = 0;
  for (uint32_t i = 0; i < n; ++i) total += lens[i];
  bytes.resize(std::max<uint64_t>(total, 1));
  uint64_t off = 0;
  for (uint32_t i = 0; i < n; ++i) {
    require(reads[i] != nullptr || lens[i] == 0, CHSGA_ERR_INVALID_ARG, "null read");
    if (lens[i]) std::memcpy(bytes.data() + off, reads[i], lens[i]);
    q[i] = dev::ReadDesc{off, lens[i], (int32_t)i};
    off += lens[i];
  }
  if (longest_first)
    std::stable_sort(q.begin(), q.end(),
                     [](const dev::ReadDesc& a, const dev::ReadDesc& b) { return a.len > b.len; });
  c.reads.upload(bytes, c.st);
  c.queue.upload(q, c.st);
  c.res_score.alloc(n);
  c.res_vertex.alloc(n);
  c.res_t0.alloc(n);
  c.res_t1.alloc(n);
  CK(cudaStreamSynchronize(c.st));  // the staging vectors die with this frame
}

template <int R>
void reset_slots(chsga_ctx& c, SlotBufs& b, uint32_t q_count) {
  std::vector<dev::SlotState> s(R);
  for (auto& x : s) x = dev::SlotState{0, 0, 0, -1, 0};
  CK(cudaMemcpyAsync(b.slots.p, s.data(), sizeof(dev::SlotState) * R, cudaMemcpyHostToDevice, c.st));
  dev::StepCtl ctl{};
  ctl.q_count = q_count;
  CK(cudaMemcpyAsync(b.ctl.p, &ctl, sizeof(ctl), cudaMemcpyHostToDevice, c.st));
  CK(cudaMemsetAsync(b.bar.p, 0, sizeof(dev::GridBar), c.st));
  CK(cudaStreamSynchronize(c.st));  // host copies above are from stack memory
}

// Tiles of consecutive string vertices for k_row_tiled (R >= 32): per tile
// the char range, the FL range, a descriptor of vertex and in-edge records
// and the list of in-edge source vertices outside the tile (see
// kernels.cuh). Returns nullptr when some vertex cannot fit a tile (too many
// in-edges), in which case the direct kernel runs instead.
template <int R, typename ST>
const dev::RowTiles* row_tiles(chsga_ctx& c) {
  if constexpr (R < 32) {
    return nullptr;
  } else {
    auto& slot = c.row_tiles[R * 8 + (int)sizeof(ST)];
    if (slot) return slot->ok ? &slot->rt : nullptr;
    slot = std::make_unique<RowTileDev>();
    const HostRowTiles h = build_row_tiles(c.g->L, R, sizeof(ST));
    if (!h.ok) return nullptr;
    validate_row_tiles(c.g->L, R, sizeof(ST), h);
    std::vector<int4> rec(h.ntiles() * 2);
    std::memcpy(rec.data(), h.rec.data(), h.rec.size() * 4);
    slot->rec.upload(rec, c.st);
    slot->desc.upload(h.desc, c.st);
    CK(cudaStreamSynchronize(c.st));
    dev::RowTiles rt{};
    rt.rec = slot->rec.p;
    rt.desc = slot->desc.p;
    rt.ntiles = h.ntiles();
    rt.nslots = h.nslots;
    rt.d_cap = h.d_cap;
    rt.fl_cap = h.fl_cap;
    rt.desc_cap = h.desc_cap;
    rt.ext_cap = h.ext_cap;
    slot->rt = rt;
    slot->ok = true;
    const int smem = (int)row_tiled_smem(h, R);
    CK(cudaFuncSetAttribute(dev::k_row_tiled<R, true, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CK(cudaFuncSetAttribute(dev::k_row_tiled<R, false, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return &slot->rt;
  }
}

// The checked build (CHSGA_CHECKED): fails with CHSGA_ERR_INTERNAL, naming
// the check site and the index, when a kernel met a graph-derived index out
// of range (kernels.cuh, CHSGA_CHK), and clears the record. Every entry
// point that takes a context runs it after its own work, which has finished
// on the device by then. The regular build has no record and no check.
void check_indices() {
#ifdef CHSGA_CHECKED
  CK(cudaDeviceSynchronize());
  unsigned int flag = 0;
  unsigned long long first = 0;
  CK(cudaMemcpyFromSymbol(&flag, dev::g_chk_fail, sizeof(flag)));
  if (!flag) return;
  CK(cudaMemcpyFromSymbol(&first, dev::g_chk_first, sizeof(first)));
  const unsigned int zero = 0;
  const unsigned long long zero64 = 0;
  CK(cudaMemcpyToSymbol(dev::g_chk_fail, &zero, sizeof(zero)));
  CK(cudaMemcpyToSymbol(dev::g_chk_first, &zero64, sizeof(zero64)));
  fail(CHSGA_ERR_INTERNAL, "device index check failed at check site " + std::to_string(first >> 40) +
                               ", index " + std::to_string(first & 0xFFFFFFFFFFull));
#endif
}

// Fails with CHSGA_ERR_TIMEOUT if a kernel's bounded wait expired.
void require_step_ok(uint32_t error) {
  require(!(error & dev::ERR_ROW_DELTA), CHSGA_ERR_INTERNAL,
          "a 2-bit row delta fell outside -1..1 (code " + std::to_string(error) + ")");
  require(error == 0, CHSGA_ERR_TIMEOUT,
          "a bounded device-side wait expired (code " + std::to_string(error) + ")");
}

void check_device_error(chsga_ctx& c, SlotBufs& b) {
  dev::StepCtl fin{};
  CK(cudaMemcpyAsync(&fin, b.ctl.p, sizeof(fin), cudaMemcpyDeviceToHost, c.st));
  CK(cudaStreamSynchronize(c.st));
  require_step_ok(fin.error);
}

// Launches a kernel of the row-step chain. With programmatic dependent launch
// (chsga_ctx::pdl, on unless CHSGA_PDL=0) the launch may begin while the kernel before
// it on the stream drains; every chain kernel starts with
// griddepcontrol.wait (dev::pdl_wait), which holds it until that kernel has
// finished and its writes are visible, so results are the same either way.
template <typename... KArgs, typename... Args>
void chain_launch(const chsga_ctx& c, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem,
                  cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  if (c.pdl) {
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
  }
  CK(cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...));
}

template <int R>
void launch_advance(chsga_ctx& c, SlotBufs& b, int prime, cudaStream_t s) {
  chain_launch(c, dev::k_advance<R>, 1, 128, 0, s, b.slots.p, c.queue.p, c.reads.p, b.best.p, c.res_score.p,
               c.res_vertex.p, c.res_t0.p, c.res_t1.p, b.word.p, b.ctl.p, c.g->L.special, prime, c.qmask,
               c.done_ring.p, match_n(c));
}

// CUDA events between the kernel groups of one row-step (profiling mode).
struct StepEvents {
  cudaEvent_t e[6];
  StepEvents() {
    for (auto& x : e) CK(cudaEventCreate(&x));
  }
  ~StepEvents() {
    for (auto& x : e) cudaEventDestroy(x);
  }
  // accumulates the five group durations of the step just recorded
  void add(chsga_profile& p) {
    CK(cudaEventSynchronize(e[5]));
    float ms[5];
    for (int i = 0; i < 5; ++i) CK(cudaEventElapsedTime(&ms[i], e[i], e[i + 1]));
    p.row_ms += ms[0];
    p.sweep_up_ms += ms[1];
    p.top_ms += ms[2];
    p.sweep_down_ms += ms[3];
    p.other_ms += ms[4];
  }
};

// One row-step for every slot: D = previous rows, T = rows being computed,
// BVc = this step's boundary scores. DEFER (score-only): rows stay raw and
// BVp holds the previous step's swept boundary scores; otherwise every row
// is written final (rows that are kept for traceback).
// Per-read matrices of the batched traceback: every active slot's final row
// is copied there after the sweeps, before k_advance.
struct RowSink {
  uint16_t* const* mats;  // device array, one matrix per read id
  size_t pitch;
};

template <int R, bool DEFER, typename ST>
void row_step(chsga_ctx& c, SlotBufs& b, const ST* D, ST* T, cudaStream_t s,
              StepEvents* ev = nullptr, const RowSink* sink = nullptr) {
  ST* BVc = reinterpret_cast<ST*>(b.BV.p);
  const HostLayout& L = c.g->L;
  const TopDev& top = cur_top(c);
  constexpr int G = Lanes<R>::G;
  if (ev) CK(cudaEventRecord(ev->e[0], s));
  ST* FL = reinterpret_cast<ST*>(b.FL.p);
  bool done = false;
  bool delta_rows = false;  // the delta row kernel reads first scores from BV, so FL holds last scores only
  if constexpr (std::is_same_v<ST, uint16_t> && R == 1) {
    // one read: a warp per tile of whole vertices, a lane per 8 chars
    if (c.g->t1.ntiles && c.row_kernel == RowKernel::Auto) {
      chain_launch(c, dev::k_row_t1<DEFER>, (c.g->t1.ntiles + dev::kT1Warps - 1) / dev::kT1Warps,
                   dev::kT1Warps * 32, 0, s, c.g->gp, c.g->t1, D, T, BVc, FL, b.word.p, b.best.p, b.ctl.p);
      done = true;
    }
  }
  if constexpr (std::is_same_v<ST, uint16_t> && DEFER && R == 128) {
    // 2-bit delta rows (score-only; AUTO at 128 slots): every step of a run
    // uses this kernel, so the rows stay in its format from the first
    // admission on
    if (L.max_len <= 512 && (c.row_kernel == RowKernel::Delta || c.row_kernel == RowKernel::Auto)) {
      const uint32_t runs = (L.S + 31) / 32;
      constexpr unsigned tpb = dev::kStreamWarps * 32;
      // at most the resident blocks: every warp after its first run takes the next from the list
      const uint32_t all = (uint32_t)nblocks((uint64_t)runs * 32, tpb);
      const uint32_t grid = c.delta_grid ? std::min(all, c.delta_grid) : all;
      chain_launch(c, dev::k_row_delta, grid, tpb, dev::delta_smem_bytes(), s, c.g->gp, D, T, BVc, FL, b.word.p,
                   b.best.p, b.ctl.p, (const uint32_t*)c.g->gd.delta_order.p, runs);
      done = true;
      delta_rows = true;
    }
  }
  if constexpr (std::is_same_v<ST, uint16_t> && R >= 2) {
    // packed 16-bit DPX kernels; exact while F + (c - first) stays below 2^16
    if (!done && L.max_len <= 512 && c.row_kernel != RowKernel::Tiled && c.row_kernel != RowKernel::Direct) {
      if constexpr (R >= 64) {
        if (c.row_kernel != RowKernel::Dpx) {
          const uint64_t runs = ((uint64_t)L.S + 31) / 32;
          constexpr unsigned tpb = dev::kStreamWarps * 32;
          chain_launch(c, dev::k_row_stream<R, DEFER>, nblocks(runs * 32, tpb), tpb, dev::stream_smem_bytes(R), s,
                       c.g->gp, D, T, BVc, FL, b.word.p, b.best.p, b.ctl.p);
          done = true;
        }
      }
      if (!done) {
        chain_launch(c, dev::k_row_dpx<R, DEFER>, nblocks((uint64_t)L.S * dev::Pairs<R>::G), 256, 0, s,
                     c.g->gp, D, T, BVc, FL, b.word.p, b.best.p, b.ctl.p);
        done = true;
      }
    }
  }
  if constexpr (R >= 32) {
    if (!done && c.row_kernel == RowKernel::Tiled) {
      if (const dev::RowTiles* rt = row_tiles<R, ST>(c)) {
        chain_launch(c, dev::k_row_tiled<R, DEFER, ST>, c.num_sms, dev::kRowThreads,
                     dev::row_smem_bytes(dev::row_slot_bytes(*rt), rt->nslots, R), s, c.g->gp, *rt, D, T, BVc,
                     FL, b.word.p, b.best.p, b.ctl.p);
        done = true;
      }
    }
  }
  if (!done)
    chain_launch(c, dev::k_row_direct<R, DEFER, ST>, nblocks((uint64_t)L.S * G), 256, 0, s, c.g->gp, D, T,
                 BVc, FL, b.word.p, b.best.p, b.ctl.p);
  if (ev) CK(cudaEventRecord(ev->e[1], s));
  const uint32_t fl = top.h.first_level;
  for (uint32_t l = 0; l < fl; ++l) {
    if (L.lvl_up_edges[l] == 0) continue;
    const uint32_t lo = L.lvl_off[l], hi = L.lvl_off[l + 1];
    if constexpr (std::is_same_v<ST, uint16_t> && R >= 8) {
      // the two- or four-edge form where no target of the level has more
      const uint32_t md = c.pull_lean ? L.lvl_up_maxdeg[l] : ~0u;
      auto k = md <= 2 ? dev::k_pull_lv16<R, 2> : md <= 4 ? dev::k_pull_lv16<R, 4> : dev::k_pull_lv16<R, 0>;
      if constexpr (R >= 64) {
        if (c.pull_coop) k = dev::k_pull_lv16c<R>;
      }
      chain_launch(c, k, nblocks((uint64_t)(hi - lo) * (R / 8)), 256, 0, s, BVc, lo, hi, c.g->gd.up_head.p,
                   c.g->gd.up_in.p, c.g->gp.n_up, b.ctl.p);
    } else
      chain_launch(c, dev::k_pull_lv<R, ST>, nblocks((uint64_t)(hi - lo) * G), 256, 0, s, BVc, lo, hi,
                   c.g->gd.up_head.p, c.g->gd.up_in.p, c.g->gp.n_up, b.ctl.p);
  }
  if (ev) CK(cudaEventRecord(ev->e[2], s));
  if (top.h.K) {
    if (!top.h.upg.empty())
      chain_launch(c, dev::k_pull<R, ST>, nblocks((uint64_t)top.h.K * G), 256, 0, s, BVc, top.h.K0, L.S,
                   top.upg_off.p, top.upg.p, top.h.K0, b.ctl.p);
    chain_launch(c, dev::k_top<R, ST>, R, kTopThreads, dev::top_smem_bytes(top.h.K, top.ptrs.chunk_cap), s, BVc,
                 top.ptrs, b.word.p, b.ctl.p);
  }
  if (ev) CK(cudaEventRecord(ev->e[3], s));
  auto down = [&](uint32_t lo, uint32_t mid, uint32_t hi) {
    if constexpr (std::is_same_v<ST, uint16_t> && DEFER && R >= 8) {
      auto k = dev::k_down16<R, true>;
      if constexpr (R == 128) {
        if (delta_rows) k = dev::k_down16<R, false>;
      }
      chain_launch(c, k, nblocks((uint64_t)(hi - lo) * (R / 8)), 256, 0, s, c.g->gp, BVc, FL, lo, mid, hi,
                   b.word.p, b.best.p, b.ctl.p);
    } else
      chain_launch(c, dev::k_down<R, !DEFER, ST>, nblocks((uint64_t)(hi - lo) * G), 256, 0, s, c.g->gp, BVc, T,
                   FL, lo, mid, hi, b.word.p, b.best.p, b.ctl.p);
  };
  if (fl == 0) {
    down(0, 0, L.S);
  } else {
    for (int l = (int)fl - 1; l >= 0; --l) {
      const uint32_t lo = L.lvl_off[l], mid = L.lvl_off[l + 1];
      down(lo, mid, (l == (int)fl - 1) ? L.S : mid);
    }
  }
  if constexpr (std::is_same_v<ST, uint16_t> && !DEFER && R >= 2) {
    if (sink)
      chain_launch(c, dev::k_store_rows<R>, (L.N + 63) / 64, 256, 0, s, T, b.slots.p, sink->mats, sink->pitch,
                   L.N, b.ctl.p);
  }
  if (ev) CK(cudaEventRecord(ev->e[4], s));
  launch_advance<R>(c, b, 0, s);
  if (ev) CK(cudaEventRecord(ev->e[5], s));
}

uint32_t kernels_per_step(const chsga_ctx& c) {
  uint32_t k = 2;  // k_row + k_advance
  const TopDev& top = cur_top(c);
  const uint32_t fl = top.h.first_level;
  for (uint32_t l = 0; l < fl; ++l) k += c.g->L.lvl_up_edges[l] ? 1 : 0;
  if (top.h.K) k += 1 + (top.h.upg.empty() ? 0 : 1);
  k += fl == 0 ? 1 : fl;
  return k;
}

constexpr uint32_t kLaunchStream = CHSGA_LAUNCH_STREAM, kLaunchGraphs = CHSGA_LAUNCH_GRAPHS,
                   kLaunchPersistent = CHSGA_LAUNCH_PERSISTENT;

// Grid of the persistent row-step kernel (k_persist) for this context's
// configuration, 0 when it does not apply: 32-bit rows, a row kernel other
// than AUTO, string vertices too long for its row phase, more levels below
// the top region than its argument block holds, or fewer resident blocks
// than slots (block r sweeps slot r's top region).
template <int R, typename ST>
uint32_t persist_grid(chsga_ctx& c) {
  if constexpr (!std::is_same_v<ST, uint16_t>) {
    return 0;
  } else {
    const HostLayout& L = c.g->L;
    const TopDev& top = cur_top(c);
    if (c.row_kernel != RowKernel::Auto || top.h.first_level > (uint32_t)dev::kPersistMaxLevels) return 0;
    if (R == 1 ? c.g->t1.ntiles == 0 : L.max_len > 512) return 0;
    constexpr int TH = dev::PersistShape<R>::threads;
    const size_t smem_max = dev::top_smem_bytes(kTopMaxVertices);
    static_assert(dev::persist_row_smem<R>() <= dev::top_smem_bytes(kTopMaxVertices), "row phase smem");
    once_per_device((const void*)dev::k_persist<R>, c.device, [&] {
      CK(cudaFuncSetAttribute(dev::k_persist<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    });
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_persist<R>, TH, smem_max));
    const uint32_t grid = (uint32_t)std::max(per_sm, 0) * (uint32_t)c.num_sms;
    return grid >= (uint32_t)R ? grid : 0;
  }
}

// One cooperative launch of k_persist: `steps` row-steps of every slot
// (rows[0] holds the previous row at the first step; steps is even).
template <int R>
void launch_persist(chsga_ctx& c, SlotBufs& b, uint32_t grid, uint32_t steps, cudaStream_t s) {
  const HostLayout& L = c.g->L;
  const TopDev& top = cur_top(c);
  dev::PersistArgs a{};
  a.g = c.g->gp;
  a.t1 = c.g->t1;
  a.top = top.ptrs;
  a.upg_off = top.upg_off.p;
  a.upg = top.upg.p;
  a.has_upg = top.h.upg.empty() ? 0u : 1u;
  a.steps = steps;
  a.rows[0] = reinterpret_cast<uint16_t*>(b.rows[0].p);
  a.rows[1] = reinterpret_cast<uint16_t*>(b.rows[1].p);
  a.BV = reinterpret_cast<uint16_t*>(b.BV.p);
  a.FL = reinterpret_cast<uint16_t*>(b.FL.p);
  a.word = b.word.p;
  a.best = b.best.p;
  a.ctl = b.ctl.p;
  a.slots = b.slots.p;
  a.queue = c.queue.p;
  a.reads = c.reads.p;
  a.res_score = c.res_score.p;
  a.res_vertex = c.res_vertex.p;
  a.res_t0 = c.res_t0.p;
  a.res_t1 = c.res_t1.p;
  a.done_ring = c.done_ring.p;
  a.qmask = c.qmask;
  a.special = L.special;
  a.match_n = match_n(c);
  a.bar = b.bar.p;
  a.fl = top.h.first_level;
  for (uint32_t l = 0; l <= a.fl; ++l) a.lvl_off[l] = L.lvl_off[l];
  for (uint32_t l = 0; l < a.fl; ++l)
    if (L.lvl_up_edges[l]) a.up_mask |= 1ull << l;
  const size_t smem = std::max(dev::persist_row_smem<R>(), dev::top_smem_bytes(top.h.K, top.ptrs.chunk_cap));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(dev::PersistShape<R>::threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, dev::k_persist<R>, a));
}

// Runs every queued read to completion through R slots, in blocks of
// `per_graph` row-steps (even, so the two row buffers alternate identically
// in every block). mode: kLaunchStream = every kernel launched from the
// host; kLaunchGraphs = each block captured once as a CUDA graph and
// replayed; kLaunchPersistent = each block one launch of the persistent
// kernel (the CUDA-graph chain where that kernel does not apply).
template <int R, typename ST>
void run_queue(chsga_ctx& c, uint32_t n, uint64_t total_rows, uint32_t mode, uint32_t per_graph) {
  SlotBufs& b = get_bufs<R, ST>(c, true);
  if (c.row_kernel == RowKernel::Tiled) row_tiles<R, ST>(c);  // allocates: never inside a capture
  reset_slots<R>(c, b, n);
  const bool profile = (c.flags & CHSGA_FLAG_PROFILE) != 0;
  if (profile) mode = kLaunchStream;
  uint32_t pgrid = 0;
  if (mode == kLaunchPersistent) {
    pgrid = persist_grid<R, ST>(c);
    if (!pgrid) mode = kLaunchGraphs;
  }
  bool use_graphs = mode == kLaunchGraphs;
  std::unique_ptr<StepEvents> sev;
  if (profile) sev = std::make_unique<StepEvents>();
  c.prof = chsga_profile{};
  c.prof.launch_mode = mode;
  per_graph = std::max<uint32_t>(2, per_graph + (per_graph & 1));
  c.h_ctl.alloc(1);
  cudaEvent_t ev[2];
  CK(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  ST* rows[2] = {reinterpret_cast<ST*>(b.rows[0].p), reinterpret_cast<ST*>(b.rows[1].p)};
  auto enqueue_block = [&](cudaStream_t s) {
    for (uint32_t i = 0; i < per_graph; ++i)
      row_step<R, true, ST>(c, b, rows[i & 1], rows[(i + 1) & 1], s);
  };
  if (use_graphs) {
    cudaStream_t cap;
    CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    enqueue_block(cap);
    CK(cudaStreamEndCapture(cap, &graph));
    CK(cudaGraphInstantiate(&exec, graph, 0));
    CK(cudaStreamDestroy(cap));
  }
  // device time from the first admission: the graph above is built on the
  // host first, so its capture and instantiation stay out of total_ms
  cudaEvent_t t_start, t_stop;
  CK(cudaEventCreate(&t_start));
  CK(cudaEventCreate(&t_stop));
  CK(cudaEventRecord(t_start, c.st));
  launch_advance<R>(c, b, 0, c.st);  // admit the first reads
  auto launch_block = [&]() {
    if (mode == kLaunchPersistent) {
      if constexpr (std::is_same_v<ST, uint16_t>) launch_persist<R>(c, b, pgrid, per_graph, c.st);
    } else if (use_graphs) {
      CK(cudaGraphLaunch(exec, c.st));
    } else if (profile) {
      for (uint32_t i = 0; i < per_graph; ++i) {
        row_step<R, true, ST>(c, b, rows[i & 1], rows[(i + 1) & 1], c.st, sev.get());
        sev->add(c.prof);
      }
    } else {
      enqueue_block(c.st);
    }
  };
  // R == 1 runs exactly one row per step, so the step count is known; the
  // batched engine polls its done counter, one block behind the device.
  uint64_t launched = 0;
  if (R == 1) {
    const uint64_t blocks = (total_rows + per_graph - 1) / per_graph;
    for (uint64_t i = 0; i < blocks; ++i) launch_block();
    launched = blocks;
    CK(cudaStreamSynchronize(c.st));
  } else {
    const uint64_t max_blocks = total_rows / per_graph + 4;
    while (true) {
      launch_block();
      CK(cudaMemcpyAsync(c.h_ctl.p, b.ctl.p, sizeof(dev::StepCtl), cudaMemcpyDeviceToHost, c.st));
      CK(cudaEventRecord(ev[launched & 1], c.st));
      ++launched;
      if (launched >= 2) {
        CK(cudaEventSynchronize(ev[(launched - 2) & 1]));
        // the pinned copy may already hold a newer value; both are progress
        if (c.h_ctl.p->done >= n) break;
      }
      require(launched <= max_blocks + 2, CHSGA_ERR_INTERNAL, "batched engine made no progress");
    }
    CK(cudaStreamSynchronize(c.st));
    require(c.h_ctl.p->done == n, CHSGA_ERR_INTERNAL, "batched engine lost reads");
  }
  CK(cudaEventRecord(t_stop, c.st));
  CK(cudaEventSynchronize(t_stop));
  float dev_ms = 0;
  CK(cudaEventElapsedTime(&dev_ms, t_start, t_stop));
  cudaEventDestroy(t_start);
  cudaEventDestroy(t_stop);
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  dev::StepCtl fin{};
  CK(cudaMemcpy(&fin, b.ctl.p, sizeof(fin), cudaMemcpyDeviceToHost));
  require_step_ok(fin.error);
  c.prof.total_ms = dev_ms;
  c.prof.rows = total_rows;
  c.prof.steps = fin.steps;
  // every kernel launched, the early-exit ones of steps after the last read included
  c.prof.launches = mode == kLaunchPersistent ? 1 + launched
                                              : 1 + (uint64_t)kernels_per_step(c) * launched * per_graph;
  c.prof.row_launches = profile ? fin.steps : launched * per_graph;
}

void upload_graph(chsga_ctx& c, const chsga_graph_host& g) {
  HostLayout L = build_layout(g);
  // the previous graph (if any) stays alive while another context shares it
  auto lg = std::make_shared<LoadedGraph>();
  GraphDev& d = lg->gd;
  cudaStream_t s = c.st;
  d.lab2.upload(L.lab2, s);
  d.lab_sp.upload(L.lab_sp, s);
  d.lab4.upload(L.lab4, s);
  d.sv_off.upload(L.sv_off, s);
  d.sv_dev.upload(L.sv_dev, s);
  d.vin_off.upload(L.vin_off, s);
  d.vin_src.upload(L.vin_src, s);
  d.vin_srcv.upload(L.vin_srcv, s);
  d.dv_first.upload(L.dv_first, s);
  d.dv_len.upload(L.dv_len, s);
  d.up_off.upload(L.up_off, s);
  d.dn_off.upload(L.dn_off, s);
  d.istr_off.upload(L.istr_off, s);
  d.istr_src.upload(L.istr_src, s);
  d.dv_s.upload(L.dv_s, s);
  std::vector<int2> up(L.up_in.size()), dn(L.dn_in.size());
  for (size_t i = 0; i < up.size(); ++i) up[i] = make_int2(L.up_in[i].src, L.up_in[i].w);
  for (size_t i = 0; i < dn.size(); ++i) dn[i] = make_int2(L.dn_in[i].src, L.dn_in[i].w);
  d.up_in.upload(up, s);
  d.dn_in.upload(dn, s);
  auto to4 = [](const std::vector<uint32_t>& v) {
    std::vector<uint4> o(v.size() / 4);
    std::memcpy(o.data(), v.data(), o.size() * sizeof(uint4));
    return o;
  };
  d.dn_head.upload(to4(L.dn_head), s);
  d.up_head.upload(to4(L.up_head), s);
  d.fin.upload(to4(L.fin), s);
  {
    // runs of 32 consecutive string vertices, longest (in chars) first; ties by index
    const uint32_t nruns = (L.S + 31) / 32;
    std::vector<uint32_t> order(nruns);
    std::vector<uint32_t> len(nruns);
    for (uint32_t r = 0; r < nruns; ++r) {
      order[r] = r;
      len[r] = L.sv_off[std::min<uint64_t>((uint64_t)32 * r + 32, L.S)] - L.sv_off[(uint64_t)32 * r];
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return len[a] > len[b]; });
    d.delta_order.upload(order, s);
    CK(cudaStreamSynchronize(s));  // the host vectors die with this scope
  }
  auto top = make_top(L, d, kTopDefaultVertices, s);
  {
    HostT1 t1 = build_t1(L);
    if (t1.ok) {
      d.t1_desc.upload(to4(t1.desc), s);
      d.t1_vrec.upload(to4(t1.vrec), s);
      d.t1_heads.upload(t1.heads, s);
      lg->t1 = dev::T1Ptrs{d.t1_desc.p, d.t1_heads.p, d.t1_vrec.p, t1.ntiles()};
    }
    CK(cudaStreamSynchronize(s));  // the host vectors die with this scope
  }
  lg->gp = dev::GraphPtrs{L.N,          L.S,          L.special,    d.lab2.p,     d.lab_sp.p,
                          d.lab4.p,     d.sv_off.p,   d.sv_dev.p,   d.vin_off.p,  d.vin_src.p,
                          d.vin_srcv.p, d.dv_first.p, d.dv_len.p,   d.dv_s.p,     d.up_off.p,
                          d.up_in.p,    d.dn_off.p,   d.dn_in.p,    d.istr_off.p, d.istr_src.p,
                          d.dn_head.p,  d.up_head.p,  d.fin.p,
                          (uint32_t)L.vin_srcv.size(), (uint32_t)L.up_in.size(), (uint32_t)L.dn_in.size()};
  lg->nul_label = false;
  for (uint32_t i = 0; i < g.num_chars; ++i) {
    lg->nul_label |= g.labels[i] == '\0';
    lg->n_label |= g.labels[i] == 'N';
  }
  lg->pitch = ((size_t)L.N + 15) / 16 * 16;
  lg->L = std::move(L);
  lg->top = std::move(top);
  c.g = std::move(lg);
  c.bufs.clear();
  c.row_tiles.clear();
  c.tops.clear();
  c.top_sel = nullptr;
  c.loaded = true;
}

template <int R>
void scores_with(chsga_ctx& c, const char* const* reads, const uint32_t* lens, uint32_t n,
                 int32_t* out, uint32_t mode, uint32_t per_graph, uint32_t row_bits) {
  // length-0 reads never reach the device: the reference scores row 0
  // against read[0] == '\0', i.e. 1 unless a label byte is 0
  std::vector<const char*> rp;
  std::vector<uint32_t> rl, idx;
  uint64_t rows = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (lens[i] == 0) {
      out[i] = empty_score(c);
      continue;
    }
    rp.push_back(reads[i]);
    rl.push_back(lens[i]);
    idx.push_back(i);
    rows += lens[i];
  }
  c.last_ids = idx;
  if (rp.empty()) return;
  upload_reads(c, rp.data(), rl.data(), (uint32_t)rp.size(), R > 1);
  // every value of row i is at most i + 1 (row 0 is 0/1, a row adds at most
  // the deletion cost 1, the closure only lowers), so reads shorter than
  // kRow16Max rows are stored exactly in 16 bits
  const uint32_t max_len = *std::max_element(rl.begin(), rl.end());
  const bool narrow = row_bits == 16 || (row_bits == 0 && max_len <= kRow16Max);
  require(!(row_bits == 16 && max_len > kRow16Max), CHSGA_ERR_INVALID_ARG,
          "16-bit rows need reads of at most 65000 bases");
  if (narrow) {
    run_queue<R, uint16_t>(c, (uint32_t)rp.size(), rows, mode, per_graph);
  } else {
    run_queue<R, int>(c, (uint32_t)rp.size(), rows, mode, per_graph);
  }
  c.prof.row_bits = narrow ? 16 : 32;
  std::vector<int32_t> res(rp.size());
  CK(cudaMemcpy(res.data(), c.res_score.p, res.size() * 4, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < idx.size(); ++i) out[idx[i]] = res[i];
}

// ---- traceback --------------------------------------------------------------

struct TbState {
  std::vector<dev::WalkOp> path;  // reverse order
};

// Forward rows [a+1, b] of the single read from row a (on the device at
// matrix row 0), writing row i to matrix + (i - a) * pitch; rows are final
// (FIXUP), in ST storage.
template <typename ST>
void forward_rows(chsga_ctx& c, SlotBufs& b, uint32_t len, int64_t a, int64_t b_row,
                  ST* matrix /* rows a..b at stride c.g->pitch, row a already present */) {
  const size_t N = c.g->pitch;
  // slot 0 at row a+1 of read 0
  dev::SlotState s{0, len, (uint32_t)(a + 1), 0, 0};
  CK(cudaMemcpyAsync(b.slots.p, &s, sizeof(s), cudaMemcpyHostToDevice, c.st));
  dev::StepCtl ctl{};
  ctl.q_count = 0;
  CK(cudaMemcpyAsync(b.ctl.p, &ctl, sizeof(ctl), cudaMemcpyHostToDevice, c.st));
  unsigned long long inf = ~0ull;
  CK(cudaMemcpyAsync(b.best.p, &inf, 8, cudaMemcpyHostToDevice, c.st));
  CK(cudaStreamSynchronize(c.st));
  launch_advance<1>(c, b, 1, c.st);
  // the row-step reads the previous row's per-vertex first/last scores; row a
  // comes from a checkpoint, so derive them from it
  dev::k_fl_from_row<ST><<<nblocks(c.g->L.S), 256, 0, c.st>>>(c.g->gp, matrix, reinterpret_cast<ST*>(b.FL.p));
  check_launch();
  for (int64_t i = a + 1; i <= b_row; ++i)
    row_step<1, false, ST>(c, b, matrix + (size_t)(i - 1 - a) * N, matrix + (size_t)(i - a) * N, c.st);
  check_device_error(c, b);
}

template <typename MT>
void walk(chsga_ctx& c, const MT* M, int64_t lo, int64_t hi, uint32_t start, uint32_t len,
          std::vector<dev::WalkOp>& path, uint32_t* landing) {
  const uint32_t max_ops = (uint32_t)(2 * (hi - lo) + 2 * (uint64_t)len + 16);
  DevArr<dev::WalkOp> ops;
  ops.alloc(max_ops);
  DevArr<dev::WalkOut> out;
  out.alloc(1);
  dev::k_walk<MT><<<1, 1, 0, c.st>>>(c.g->gp, M, c.g->pitch, lo, hi, start, c.reads.p, ops.p, max_ops, out.p,
                                     match_n(c));
  check_launch();
  dev::WalkOut h{};
  CK(cudaMemcpyAsync(&h, out.p, sizeof(h), cudaMemcpyDeviceToHost, c.st));
  CK(cudaStreamSynchronize(c.st));
  if (h.status == 7)
    fail(CHSGA_ERR_NO_PATH, "score-matrix traceback: no valid predecessor at row " +
                                std::to_string(h.fail_row));
  require(h.status == 0, CHSGA_ERR_INTERNAL, "traceback walk exceeded its op budget");
  size_t old = path.size();
  path.resize(old + h.nops);
  if (h.nops)
    CK(cudaMemcpy(path.data() + old, ops.p, h.nops * sizeof(dev::WalkOp), cudaMemcpyDeviceToHost));
  *landing = h.vertex;
}

// ops of a walked path (collected end first) into a caller-owned result
void fill_result(chsga_tb_result* res, std::vector<dev::WalkOp>& path, int32_t score) {
  std::reverse(path.begin(), path.end());
  res->num_ops = path.size();
  res->ops = (chsga_op*)std::malloc(std::max<size_t>(1, path.size()) * sizeof(chsga_op));
  require(res->ops != nullptr, CHSGA_ERR_OOM, "host out of memory");
  for (size_t i = 0; i < path.size(); ++i) {
    res->ops[i].row = path[i].row;
    res->ops[i].vertex = path[i].vertex;
    res->ops[i].op = (uint8_t)path[i].op;
    std::memset(res->ops[i].pad, 0, 3);
  }
  res->score = score;
}

// Rows per sub-segment when a segment of `span` + 1 rows does not fit the
// device: the longest k2 for which the ceil(span / k2) sub-checkpoint rows
// plus one sub-segment of k2 + 1 rows fit in `fit` rows; 0 if none does.
uint64_t sub_segment_rows(uint64_t span, uint64_t fit) {
  for (uint64_t k2 = std::min<uint64_t>(span, fit); k2 >= 1; --k2)
    if ((span + k2 - 1) / k2 + k2 + 1 <= fit) return k2;
  return 0;
}

// Pinned host rows of the checkpointed traceback, per row storage.
template <typename ST>
PinnedArr<ST>& ckpt_host(chsga_ctx& c);
template <>
PinnedArr<int32_t>& ckpt_host<int32_t>(chsga_ctx& c) {
  return c.h_ckpt;
}
template <>
PinnedArr<uint16_t>& ckpt_host<uint16_t>(chsga_ctx& c) {
  return c.h_ckpt16;
}

// Checkpoint files hold raw int32 rows (the reference's format,
// src/traceback.hpp:215-227) whatever the rows are stored in.
void write_ckpt(const std::string& dir, int64_t row, const int32_t* d, uint64_t n) {
  write_ckpt_row(dir, row, d, n);
}
void write_ckpt(const std::string& dir, int64_t row, const uint16_t* d, uint64_t n) {
  std::vector<int32_t> w(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) w[i] = d[i];
  write_ckpt_row(dir, row, w.data(), n);
}

// One read's traceback with rows stored as ST: int32, or uint16 for reads
// of at most kRow16Max bases (every value of row i is at most i + 1, so the
// rows are the same numbers in half the bytes).
template <typename ST>
void traceback_rows(chsga_ctx& c, const char* read, uint32_t len, const chsga_tb_opts* o,
                    chsga_tb_result* res) {
  require(len > 0, CHSGA_ERR_INVALID_ARG, "traceback of an empty read");
  const size_t N = c.g->pitch;   // row stride of every matrix below
  const size_t NC = c.g->L.N;    // chars per row
  const int64_t k = (o && o->k > 0) ? o->k : 500;
  const uint64_t cap = (o && o->cap_bytes) ? o->cap_bytes : c.cap;
  const std::string dir = (o && o->dir) ? o->dir : "";
  const bool keep = o && o->keep_files;
  const char* rp[1] = {read};
  upload_reads(c, rp, &len, 1);
  SlotBufs& b = get_bufs<1, ST>(c, false);
  // the full-matrix / checkpointed decision counts int32 rows, as the
  // reference does (src/traceback.hpp:614-645), whatever ST is
  const uint64_t store = (uint64_t)len * NC * 4;
  const uint64_t row_bytes = (uint64_t)NC * sizeof(ST);  // one stored row
  std::vector<dev::WalkOp> path;
  uint32_t best_v = 0;
  int32_t best_s = 0;
  auto harvest = [&]() {
    check_device_error(c, b);
    CK(cudaMemcpy(&best_s, c.res_score.p, 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&best_v, c.res_vertex.p, 4, cudaMemcpyDeviceToHost));
  };
  res->checkpointed = 0;
  res->num_checkpoints = 0;
  if (store <= cap) {
    // one spare row: row 0 reads no previous row, but its input pointer
    // must not alias the row it writes
    DevArr<ST> M;
    M.alloc((size_t)(len + 1) * N);
    reset_slots<1>(c, b, 1);
    launch_advance<1>(c, b, 0, c.st);
    for (uint32_t i = 0; i < len; ++i)
      row_step<1, false, ST>(c, b, M.p + (size_t)(i ? i - 1 : len) * N, M.p + (size_t)i * N, c.st);
    harvest();
    uint32_t v = best_v;
    if (len > 1) walk(c, M.p, 0, len - 1, best_v, len, path, &v);
    path.push_back(dev::WalkOp{0, v, CHSGA_OP_MATCHSUB});
  } else {
    // forward with checkpoints every k rows (src/traceback.hpp:855-892)
    res->checkpointed = 1;
    const uint64_t nck = (len - 1) / (uint64_t)k + 1;
    res->num_checkpoints = nck;
    PinnedArr<ST>& hck = ckpt_host<ST>(c);
    hck.alloc(nck * NC);
    DevArr<ST> ring;
    ring.alloc(3 * N);
    cudaEvent_t done_ev[3];
    for (auto& e : done_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    bool busy[3] = {false, false, false};
    reset_slots<1>(c, b, 1);
    launch_advance<1>(c, b, 0, c.st);
    // three row buffers: the previous row, the row being computed, and a
    // checkpoint row whose copy to pinned host memory may still be running
    int prev = 1;
    for (uint32_t i = 0; i < len; ++i) {
      int cur = -1;
      for (int j = 0; j < 3 && cur < 0; ++j)
        if (j != prev && !busy[j]) cur = j;
      if (cur < 0) {
        cur = (prev + 1) % 3;
        CK(cudaEventSynchronize(done_ev[cur]));
        busy[cur] = false;
      }
      row_step<1, false, ST>(c, b, ring.p + (size_t)prev * N, ring.p + (size_t)cur * N, c.st);
      if (i % k == 0) {
        cudaEvent_t ready;
        CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        CK(cudaEventRecord(ready, c.st));
        CK(cudaStreamWaitEvent(c.side, ready, 0));
        CK(cudaMemcpyAsync(hck.p + (size_t)(i / k) * NC, ring.p + (size_t)cur * N, row_bytes,
                           cudaMemcpyDeviceToHost, c.side));
        CK(cudaEventRecord(done_ev[cur], c.side));
        busy[cur] = true;
        cudaEventDestroy(ready);
      }
      prev = cur;
    }
    harvest();
    CK(cudaStreamSynchronize(c.side));
    for (auto& e : done_ev) cudaEventDestroy(e);
    ring.release();
    if (!dir.empty())
      for (uint64_t j = 0; j < nck; ++j)
        write_ckpt(dir, (int64_t)(j * k), hck.p + (size_t)j * NC, NC);
    // backward, one segment at a time (src/traceback.hpp:945-1011)
    int64_t cur_row = len - 1;
    uint32_t cur_v = best_v;
    // like the reference, the cap only decides between the two paths
    // (traceback.hpp:614-645); segment recompute is sized by device memory
    const uint64_t budget = std::max<uint64_t>(c.cap, cap);
    // segment buffers live across segments (equal segments reuse them; a
    // buffer whose size changes is released before anything is allocated,
    // so the device holds one segment's plan at a time)
    DevArr<ST> seg, sub;
    auto plan = [&](size_t seg_elems, size_t sub_elems) {
      if (seg.n != seg_elems) seg.release();
      if (sub.n != sub_elems) sub.release();
      if (seg_elems) seg.alloc(seg_elems);
      if (sub_elems) sub.alloc(sub_elems);
    };
    while (cur_row > 0) {
      int64_t seg_start = (cur_row % k == 0) ? (cur_row - k) : (cur_row / k * k);
      if (seg_start < 0) seg_start = 0;
      const int64_t seg_end = cur_row;
      const ST* ck = hck.p + (size_t)(seg_start / k) * NC;
      const uint64_t rows = (uint64_t)(seg_end - seg_start + 1);
      uint32_t landing = cur_v;
      const uint64_t pitch_bytes = (uint64_t)N * sizeof(ST);
      if (rows * pitch_bytes <= budget || rows <= 2) {
        plan(rows * N, 0);
        CK(cudaMemcpyAsync(seg.p, ck, row_bytes, cudaMemcpyHostToDevice, c.st));
        forward_rows(c, b, len, seg_start, seg_end, seg.p);
        walk(c, seg.p, seg_start, seg_end, cur_v, len, path, &landing);
      } else {
        // two levels: sub-segments of k2 rows, as long as the device budget
        // allows; a first pass keeps the row at the start of each and ends
        // with the last sub-segment on the device, which is walked at once;
        // the earlier ones are recomputed from their sub-checkpoints
        const uint64_t span = (uint64_t)(seg_end - seg_start);
        const uint64_t k2 = sub_segment_rows(span, budget / pitch_bytes);
        require(k2 >= 1, CHSGA_ERR_OOM,
                "traceback segment does not fit the byte cap even with two-level checkpoints");
        const uint64_t nsub = (span + k2 - 1) / k2;
        plan((k2 + 1) * N, nsub * N);
        CK(cudaMemcpyAsync(sub.p, ck, row_bytes, cudaMemcpyHostToDevice, c.st));
        CK(cudaMemcpyAsync(seg.p, ck, row_bytes, cudaMemcpyHostToDevice, c.st));
        int64_t r0 = seg_start;
        for (uint64_t j = 1; j < nsub; ++j) {
          const int64_t r1 = seg_start + (int64_t)(j * k2);
          forward_rows(c, b, len, r0, r1, seg.p);
          CK(cudaMemcpyAsync(sub.p + j * N, seg.p + (size_t)(r1 - r0) * N, row_bytes,
                             cudaMemcpyDeviceToDevice, c.st));
          CK(cudaMemcpyAsync(seg.p, seg.p + (size_t)(r1 - r0) * N, row_bytes,
                             cudaMemcpyDeviceToDevice, c.st));
          r0 = r1;
        }
        // r0 < seg_end: the last sub-segment holds 1..k2 rows after r0
        forward_rows(c, b, len, r0, seg_end, seg.p);
        uint32_t v = cur_v;
        {
          uint32_t l2 = v;
          walk(c, seg.p, r0, seg_end, v, len, path, &l2);
          v = l2;
        }
        int64_t row = r0;
        while (row > seg_start) {
          const int64_t s0 = row - (int64_t)k2;
          CK(cudaMemcpyAsync(seg.p, sub.p + (size_t)((s0 - seg_start) / (int64_t)k2) * N, row_bytes,
                             cudaMemcpyDeviceToDevice, c.st));
          forward_rows(c, b, len, s0, row, seg.p);
          uint32_t l2 = v;
          walk(c, seg.p, s0, row, v, len, path, &l2);
          v = l2;
          row = s0;
        }
        landing = v;
      }
      if (!dir.empty() && !keep && seg_start > 0)
        std::filesystem::remove(ckpt_row_path(dir, seg_start));
      cur_row = seg_start;
      cur_v = landing;
    }
    path.push_back(dev::WalkOp{0, cur_v, CHSGA_OP_MATCHSUB});
    if (!dir.empty() && !keep) std::filesystem::remove(ckpt_row_path(dir, 0));
  }
  fill_result(res, path, best_s);
}

void traceback(chsga_ctx& c, const char* read, uint32_t len, const chsga_tb_opts* o,
               chsga_tb_result* res) {
  if (len <= kRow16Max)
    traceback_rows<uint16_t>(c, read, len, o, res);
  else
    traceback_rows<int32_t>(c, read, len, o, res);
}

// Publishes queue entries [0, q_count) to k_advance (one thread, stream-ordered).
__global__ void k_publish(dev::StepCtl* ctl, uint32_t q_count) { ctl->q_count = q_count; }

// ---- batched full-matrix traceback --------------------------------------------
//
// Reads whose full matrix fits the cap run together as the slots of the
// batched engine in FIXUP mode (every row final); after each row-step
// k_store_rows copies each active slot's row into that read's own 16-bit
// matrix (stream-ordered allocations, published to the device queue only
// once the matrix exists and fits the device budget). A finished read is
// walked on the side stream, one engine block behind, while the next block
// runs; its matrix is then freed. Same matrix values and the same walk as
// the one-read path, so the same ops.
template <int R>
void traceback_batched(chsga_ctx& parent, const char* const* reads, const uint32_t* lens,
                       const std::vector<uint32_t>& idx, chsga_tb_result* out) {
  std::unique_ptr<chsga_ctx, void (*)(chsga_ctx*)> hold(fork_context(parent), chsga_close);
  chsga_ctx& c = *hold;
  const uint32_t nf = (uint32_t)idx.size();
  std::vector<const char*> rp(nf);
  std::vector<uint32_t> rl(nf);
  std::vector<uint64_t> roff(nf);
  uint64_t off = 0, max_ops = 16;
  for (uint32_t i = 0; i < nf; ++i) {
    rp[i] = reads[idx[i]];
    rl[i] = lens[idx[i]];
    roff[i] = off;
    off += rl[i];
    max_ops = std::max<uint64_t>(max_ops, 4ull * rl[i] + 16);
  }
  upload_reads(c, rp.data(), rl.data(), nf);  // queue entry i = read i, published below
  c.done_ring.alloc(nf);
  SlotBufs& b = get_bufs<R, uint16_t>(c, true);
  reset_slots<R>(c, b, 0);
  launch_advance<R>(c, b, 0, c.st);
  DevArr<uint16_t*> mats;
  mats.alloc(nf);
  CK(cudaMemsetAsync(mats.p, 0, nf * sizeof(uint16_t*), c.st));
  const size_t pitch = c.g->pitch;
  const RowSink sink{mats.p, pitch};
  constexpr uint32_t per = 8;
  uint16_t* rows[2] = {reinterpret_cast<uint16_t*>(b.rows[0].p), reinterpret_cast<uint16_t*>(b.rows[1].p)};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  {
    cudaStream_t cap;
    CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    for (uint32_t i = 0; i < per; ++i)
      row_step<R, false, uint16_t>(c, b, rows[i & 1], rows[(i + 1) & 1], cap, nullptr, &sink);
    CK(cudaStreamEndCapture(cap, &graph));
    CK(cudaGraphInstantiate(&exec, graph, 0));
    CK(cudaStreamDestroy(cap));
  }
  struct GraphHold {
    cudaGraph_t g;
    cudaGraphExec_t e;
    ~GraphHold() {
      if (e) cudaGraphExecDestroy(e);
      if (g) cudaGraphDestroy(g);
    }
  } gh{graph, exec};
  PinnedArr<dev::StepCtl> hctl;
  hctl.alloc(2);
  PinnedArr<dev::CompletionRec> hring;
  hring.alloc(2 * (size_t)nf);
  cudaEvent_t ev[2];
  for (auto& e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  struct EvHold {
    cudaEvent_t* e;
    ~EvHold() {
      cudaEventDestroy(e[0]);
      cudaEventDestroy(e[1]);
    }
  } eh{ev};
  // walk outputs of one harvest (at most R reads finish per row-step)
  const uint32_t wcap = R * per + R;
  DevArr<dev::WalkOp> ops_buf;
  ops_buf.alloc(max_ops * wcap);
  DevArr<dev::WalkOut> wout;
  wout.alloc(wcap);
  std::vector<dev::WalkOut> hout(wcap);
  std::vector<dev::WalkOp> hops(max_ops);
  // matrices held at once: what is free once the engine's buffers exist;
  // the stream-ordered pool keeps freed matrices for the next reads instead
  // of unmapping them at every synchronisation
  const uint64_t budget = (uint64_t)(device_free_bytes(c) * 0.8);
  {
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, c.device));
    uint64_t keep = budget;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  std::vector<uint16_t*> hm(nf, nullptr);
  uint64_t used = 0;
  uint32_t next = 0, hdone = 0;
  uint64_t launched = 0;
  // the walks of every read finished by a harvested block, launched back to
  // back on the side stream (the engine stream runs the next block), then
  // one synchronisation for all of them
  auto harvest = [&](int k) {
    CK(cudaEventSynchronize(ev[k]));
    const dev::StepCtl& st = hctl.p[k];
    require_step_ok(st.error);
    for (uint32_t i0 = hdone; i0 < st.done; i0 += wcap) {
      const uint32_t i1 = std::min<uint32_t>(st.done, i0 + wcap);
      for (uint32_t i = i0; i < i1; ++i) {
        const dev::CompletionRec& r = hring.p[(size_t)k * nf + i];
        const uint32_t id = (uint32_t)r.id, len = rl[id], j = i - i0;
        if (len > 1)
          dev::k_walk<uint16_t><<<1, 1, 0, c.side>>>(c.g->gp, hm[id], pitch, 0, (long long)len - 1,
                                                      r.vertex, c.reads.p + roff[id],
                                                      ops_buf.p + (size_t)j * max_ops, (uint32_t)max_ops,
                                                      wout.p + j, match_n(c));
      }
      check_launch();
      CK(cudaMemcpyAsync(hout.data(), wout.p, (i1 - i0) * sizeof(dev::WalkOut), cudaMemcpyDeviceToHost,
                         c.side));
      CK(cudaStreamSynchronize(c.side));
      for (uint32_t i = i0; i < i1; ++i) {
        const dev::CompletionRec& r = hring.p[(size_t)k * nf + i];
        const uint32_t id = (uint32_t)r.id, len = rl[id], j = i - i0;
        std::vector<dev::WalkOp> path;
        uint32_t v = r.vertex;
        if (len > 1) {
          const dev::WalkOut& h = hout[j];
          if (h.status == 7)
            fail(CHSGA_ERR_NO_PATH, "score-matrix traceback: no valid predecessor at row " +
                                        std::to_string(h.fail_row));
          require(h.status == 0, CHSGA_ERR_INTERNAL, "traceback walk exceeded its op budget");
          if (h.nops)
            CK(cudaMemcpy(hops.data(), ops_buf.p + (size_t)j * max_ops, h.nops * sizeof(dev::WalkOp),
                          cudaMemcpyDeviceToHost));
          path.assign(hops.begin(), hops.begin() + h.nops);
          v = h.vertex;
        }
        path.push_back(dev::WalkOp{0, v, CHSGA_OP_MATCHSUB});
        fill_result(&out[idx[id]], path, r.score);
        CK(cudaFreeAsync(hm[id], c.side));
        hm[id] = nullptr;
        used -= (uint64_t)len * pitch * 2;
      }
    }
    hdone = st.done;
  };
  try {
    while (hdone < nf) {
      const uint32_t pub0 = next;
      while (next < nf) {
        const uint64_t mb = (uint64_t)rl[next] * pitch * 2;
        // always admit when nothing else holds a matrix, so the loop progresses
        if (used + mb > budget && used > 0) break;
        void* p = nullptr;
        CK(cudaMallocAsync(&p, mb, c.st));
        hm[next] = static_cast<uint16_t*>(p);
        dev::k_set_ptr<<<1, 1, 0, c.st>>>(mats.p, next, hm[next]);
        used += mb;
        ++next;
      }
      if (next > pub0) k_publish<<<1, 1, 0, c.st>>>(b.ctl.p, next);
      const int k = (int)(launched & 1);
      CK(cudaGraphLaunch(exec, c.st));
      CK(cudaMemcpyAsync(hctl.p + k, b.ctl.p, sizeof(dev::StepCtl), cudaMemcpyDeviceToHost, c.st));
      CK(cudaMemcpyAsync(hring.p + (size_t)k * nf, c.done_ring.p, nf * sizeof(dev::CompletionRec),
                         cudaMemcpyDeviceToHost, c.st));
      CK(cudaEventRecord(ev[k], c.st));
      ++launched;
      if (launched >= 2) harvest((int)((launched - 2) & 1));
      require(launched < 4ull * (off + 16) + 64, CHSGA_ERR_INTERNAL, "batched traceback made no progress");
    }
    CK(cudaStreamSynchronize(c.st));
    CK(cudaStreamSynchronize(c.side));
  } catch (...) {
    cudaStreamSynchronize(c.st);
    cudaStreamSynchronize(c.side);
    for (auto* p : hm)
      if (p) cudaFreeAsync(p, c.st);
    cudaStreamSynchronize(c.st);
    throw;
  }
}

// ---- score-only alignment without device allocation -------------------------
//
// For callers that may not allocate GPU memory once they are running (a
// service whose free HBM belongs to its own pool after start-up, a loop that
// cannot afford the device-wide synchronisation of cudaMalloc): every
// per-call buffer of the one-read-per-step score path comes from this fixed
// array. The driver reserves it on each GPU where it loads this file's device
// code, until the process exits. On the host, `noalloc_scratch` only names
// the symbol; its device address on the current GPU comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char noalloc_scratch[CHSGA_NOALLOC_SCRATCH_BYTES];

constexpr int kNoallocMaxDevices = 64;

struct NoallocDevice {
  std::mutex mu;                  // held for a whole call: calls on a device never overlap
  unsigned char* base = nullptr;  // device address of noalloc_scratch on this device
};
NoallocDevice noalloc_devices[kNoallocMaxDevices];

// Byte offsets of the per-call buffers in the array (each 256-byte aligned).
struct NoallocLayout {
  uint64_t rows[2], bv, fl, slots, word, best, ctl, reads, lens, queue, slot_of, res_score,
      res_vertex, res_t0, res_t1, out, end;
};

NoallocLayout noalloc_layout(uint64_t N, uint64_t S, uint64_t read_bytes, uint64_t n) {
  NoallocLayout l{};
  uint64_t at = 0;
  auto take = [&](uint64_t bytes) {
    const uint64_t o = at;
    at += (std::max<uint64_t>(bytes, 1) + 255) / 256 * 256;
    return o;
  };
  // the same sizes as the context's own buffers for one slot of 16-bit rows
  l.rows[0] = take((N + 32) * sizeof(uint16_t));
  l.rows[1] = take((N + 32) * sizeof(uint16_t));
  l.bv = take(2 * S * sizeof(uint16_t));
  l.fl = take(2 * (S + 16) * sizeof(uint16_t));
  l.slots = take(sizeof(dev::SlotState));
  l.word = take(sizeof(uint32_t));
  l.best = take(sizeof(unsigned long long));
  l.ctl = take(sizeof(dev::StepCtl));
  l.reads = take(read_bytes);
  l.lens = take(n * sizeof(uint32_t));
  l.queue = take(n * sizeof(dev::ReadDesc));
  l.slot_of = take(n * sizeof(int32_t));
  l.res_score = take(n * sizeof(int32_t));
  l.res_vertex = take(n * sizeof(uint32_t));
  l.res_t0 = take(n * sizeof(unsigned long long));
  l.res_t1 = take(n * sizeof(unsigned long long));
  l.out = take(n * sizeof(int32_t));
  l.end = at;
  return l;
}

struct NoallocBufs {
  uint16_t* rows[2];
  uint16_t* BV;
  uint16_t* FL;
  dev::SlotState* slots;
  uint32_t* word;
  unsigned long long* best;
  dev::StepCtl* ctl;
  unsigned char* reads;
  uint32_t* lens;
  dev::ReadDesc* queue;
  int32_t* slot_of;
  int32_t* res_score;
  uint32_t* res_vertex;
  unsigned long long *res_t0, *res_t1;
  int32_t* out;
};

// One block. Builds the read queue from the lengths: the non-empty reads in
// caller order, ids 0..m-1, offsets = prefix sums of all lengths (where the
// host copied the bytes); slot_of[i] = queue id of caller read i, -1 when it
// is empty. Puts the slot idle and the control block at zero with m queued
// reads: the array holds the previous call's values.
__global__ void __launch_bounds__(1024) k_noalloc_prepare(const uint32_t* __restrict__ lens, uint32_t n,
                                                          dev::ReadDesc* __restrict__ queue,
                                                          int32_t* __restrict__ slot_of,
                                                          dev::SlotState* __restrict__ slots,
                                                          dev::StepCtl* __restrict__ ctl,
                                                          unsigned long long* __restrict__ best) {
  __shared__ unsigned long long s_off[1024];
  __shared__ uint32_t s_cnt[1024];
  const uint64_t per = ((uint64_t)n + 1023) / 1024;
  const uint64_t a = threadIdx.x * per;
  const uint64_t lo = a < n ? a : n, hi = lo + per < n ? lo + per : n;
  unsigned long long off = 0;
  uint32_t cnt = 0;
  for (uint64_t i = lo; i < hi; ++i) {
    off += lens[i];
    cnt += lens[i] != 0;
  }
  s_off[threadIdx.x] = off;
  s_cnt[threadIdx.x] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long o = 0;
    uint32_t k = 0;
    for (int t = 0; t < 1024; ++t) {
      const unsigned long long a = s_off[t];
      const uint32_t b = s_cnt[t];
      s_off[t] = o;
      s_cnt[t] = k;
      o += a;
      k += b;
    }
    dev::StepCtl z{};
    z.q_count = k;
    *ctl = z;
    slots[0] = dev::SlotState{0, 0, 0, -1, 0};
    best[0] = ~0ull;
  }
  __syncthreads();
  off = s_off[threadIdx.x];
  cnt = s_cnt[threadIdx.x];
  for (uint64_t i = lo; i < hi; ++i) {
    const uint32_t len = lens[i];
    if (len) {
      queue[cnt] = dev::ReadDesc{off, len, (int32_t)cnt};
      slot_of[i] = (int32_t)cnt;
      ++cnt;
    } else {
      slot_of[i] = -1;
    }
    off += len;
  }
}

__global__ void k_noalloc_finish(const int32_t* __restrict__ slot_of,
                                 const int32_t* __restrict__ res_score, uint32_t n,
                                 int32_t empty_score, int32_t* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const int32_t q = slot_of[i];
    out[i] = q < 0 ? empty_score : res_score[q];
  }
}

// The row-step of chsga_align_scores (one slot, 16-bit rows, deferred
// closure) on the buffers of the fixed array.
void noalloc_row_step(chsga_ctx& c, const NoallocBufs& b, const uint16_t* D, uint16_t* T) {
  const cudaStream_t s = c.st;
  const HostLayout& L = c.g->L;
  const TopDev& top = *c.g->top;
  constexpr int G = Lanes<1>::G;
  dev::k_row_direct<1, true, uint16_t><<<nblocks((uint64_t)L.S * G), 256, 0, s>>>(
      c.g->gp, D, T, b.BV, b.FL, b.word, b.best, b.ctl);
  const uint32_t fl = top.h.first_level;
  for (uint32_t l = 0; l < fl; ++l) {
    if (L.lvl_up_edges[l] == 0) continue;
    const uint32_t lo = L.lvl_off[l], hi = L.lvl_off[l + 1];
    dev::k_pull<1, uint16_t><<<nblocks((uint64_t)(hi - lo) * G), 256, 0, s>>>(
        b.BV, lo, hi, c.g->gd.up_off.p, c.g->gd.up_in.p, 0, b.ctl);
  }
  if (top.h.K) {
    if (!top.h.upg.empty())
      dev::k_pull<1, uint16_t><<<nblocks((uint64_t)top.h.K * G), 256, 0, s>>>(
          b.BV, top.h.K0, L.S, top.upg_off.p, top.upg.p, top.h.K0, b.ctl);
    dev::k_top<1, uint16_t><<<1, kTopThreads, dev::top_smem_bytes(top.h.K, top.ptrs.chunk_cap), s>>>(b.BV, top.ptrs,
                                                                               b.word, b.ctl);
  }
  if (fl == 0) {
    dev::k_down<1, false, uint16_t><<<nblocks((uint64_t)L.S * G), 256, 0, s>>>(
        c.g->gp, b.BV, T, b.FL, 0, 0, L.S, b.word, b.best, b.ctl);
  } else {
    for (int l = (int)fl - 1; l >= 0; --l) {
      const uint32_t lo = L.lvl_off[l], mid = L.lvl_off[l + 1];
      const uint32_t hi = (l == (int)fl - 1) ? L.S : mid;
      dev::k_down<1, false, uint16_t><<<nblocks((uint64_t)(hi - lo) * G), 256, 0, s>>>(
          c.g->gp, b.BV, T, b.FL, lo, mid, hi, b.word, b.best, b.ctl);
    }
  }
  dev::k_advance<1><<<1, 128, 0, s>>>(b.slots, b.queue, b.reads, b.best, b.res_score, b.res_vertex,
                                      b.res_t0, b.res_t1, b.word, b.ctl, L.special, 0, 0xFFFFFFFFu,
                                      nullptr, match_n(c));
  check_launch();
}

void scores_noalloc_enqueue(chsga_ctx& c, const NoallocBufs& b, const char* const* reads,
                            const uint32_t* lens, uint32_t n, uint64_t total, uint32_t m,
                            int32_t* out);

void scores_noalloc(chsga_ctx& c, const char* const* reads, const uint32_t* lens, uint32_t n,
                    int32_t* out) {
  require(c.device >= 0 && c.device < kNoallocMaxDevices, CHSGA_ERR_UNSUPPORTED,
          "chsga_align_scores_noalloc supports device ordinals below 64");
  NoallocDevice& d = noalloc_devices[c.device];
  std::lock_guard<std::mutex> lock(d.mu);
  if (!d.base) {  // set-up, once per device; the context made this device current
    unsigned char* ptr = nullptr;
    CK(cudaGetSymbolAddress((void**)&ptr, noalloc_scratch));
    CK(cudaFuncSetAttribute(dev::k_top<1, uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)dev::top_smem_bytes(kTopMaxVertices)));
    d.base = ptr;
  }
  uint64_t total = 0;
  uint32_t m = 0, max_len = 0;
  for (uint32_t i = 0; i < n; ++i) {
    require(reads[i] != nullptr || lens[i] == 0, CHSGA_ERR_INVALID_ARG, "null read");
    total += lens[i];
    m += lens[i] != 0;
    max_len = std::max(max_len, lens[i]);
  }
  require(max_len <= kRow16Max, CHSGA_ERR_UNSUPPORTED,
          "chsga_align_scores_noalloc keeps 16-bit rows: reads of at most 65000 bases");
  const NoallocLayout l = noalloc_layout(c.g->L.N, c.g->L.S, total, n);
  require(l.end <= CHSGA_NOALLOC_SCRATCH_BYTES, CHSGA_ERR_OOM,
          "chsga_align_scores_noalloc needs " + std::to_string(l.end) +
              " bytes of its fixed device array for this graph and these reads; the array holds " +
              std::to_string((uint64_t)CHSGA_NOALLOC_SCRATCH_BYTES) + " (CHSGA_NOALLOC_SCRATCH_BYTES)");
  if (n == 0) return;
  unsigned char* base = d.base;
  NoallocBufs b{};
  b.rows[0] = reinterpret_cast<uint16_t*>(base + l.rows[0]);
  b.rows[1] = reinterpret_cast<uint16_t*>(base + l.rows[1]);
  b.BV = reinterpret_cast<uint16_t*>(base + l.bv);
  b.FL = reinterpret_cast<uint16_t*>(base + l.fl);
  b.slots = reinterpret_cast<dev::SlotState*>(base + l.slots);
  b.word = reinterpret_cast<uint32_t*>(base + l.word);
  b.best = reinterpret_cast<unsigned long long*>(base + l.best);
  b.ctl = reinterpret_cast<dev::StepCtl*>(base + l.ctl);
  b.reads = base + l.reads;
  b.lens = reinterpret_cast<uint32_t*>(base + l.lens);
  b.queue = reinterpret_cast<dev::ReadDesc*>(base + l.queue);
  b.slot_of = reinterpret_cast<int32_t*>(base + l.slot_of);
  b.res_score = reinterpret_cast<int32_t*>(base + l.res_score);
  b.res_vertex = reinterpret_cast<uint32_t*>(base + l.res_vertex);
  b.res_t0 = reinterpret_cast<unsigned long long*>(base + l.res_t0);
  b.res_t1 = reinterpret_cast<unsigned long long*>(base + l.res_t1);
  b.out = reinterpret_cast<int32_t*>(base + l.out);
  const cudaStream_t s = c.st;
  // the lock must not be released while work on the shared array is still
  // queued: any failure after the first enqueue waits for the stream first
  try {
    scores_noalloc_enqueue(c, b, reads, lens, n, total, m, out);
  } catch (...) {
    cudaStreamSynchronize(s);
    throw;
  }
}

void scores_noalloc_enqueue(chsga_ctx& c, const NoallocBufs& b, const char* const* reads,
                            const uint32_t* lens, uint32_t n, uint64_t total, uint32_t m,
                            int32_t* out) {
  const cudaStream_t s = c.st;
  // copies from pageable caller memory: each returns once its source is read
  CK(cudaMemcpyAsync(b.lens, lens, (size_t)n * 4, cudaMemcpyHostToDevice, s));
  uint64_t off = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (lens[i]) CK(cudaMemcpyAsync(b.reads + off, reads[i], lens[i], cudaMemcpyHostToDevice, s));
    off += lens[i];
  }
  k_noalloc_prepare<<<1, 1024, 0, s>>>(b.lens, n, b.queue, b.slot_of, b.slots, b.ctl, b.best);
  check_launch();
  if (m) {
    // admit the first read, then one row per step: `total` steps finish every read
    dev::k_advance<1><<<1, 128, 0, s>>>(b.slots, b.queue, b.reads, b.best, b.res_score,
                                        b.res_vertex, b.res_t0, b.res_t1, b.word, b.ctl,
                                        c.g->L.special, 0, 0xFFFFFFFFu, nullptr, match_n(c));
    check_launch();
    for (uint64_t k = 0; k < total; ++k) noalloc_row_step(c, b, b.rows[k & 1], b.rows[(k + 1) & 1]);
  }
  k_noalloc_finish<<<nblocks(n), 256, 0, s>>>(b.slot_of, b.res_score, n, empty_score(c), b.out);
  check_launch();
  dev::StepCtl fin{};
  CK(cudaMemcpyAsync(&fin, b.ctl, sizeof(fin), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(out, b.out, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  require(fin.error == 0, CHSGA_ERR_TIMEOUT,
          "a bounded device-side wait expired (code " + std::to_string(fin.error) + ")");
  require(fin.done == m, CHSGA_ERR_INTERNAL, "allocation-free path lost reads");
}

// Applies a call's row-kernel and level-grouping choices to the context
// and puts the previous ones back when the call ends.
struct CallKnobs {
  chsga_ctx& c;
  RowKernel rk;
  const TopDev* ts;
  CallKnobs(chsga_ctx& cx, uint32_t row_kernel, uint32_t top_vertices)
      : c(cx), rk(cx.row_kernel), ts(cx.top_sel) {
    require(row_kernel <= CHSGA_ROW_DELTA, CHSGA_ERR_INVALID_ARG, "row_kernel must be CHSGA_ROW_*");
    if (row_kernel == CHSGA_ROW_DIRECT) c.row_kernel = RowKernel::Direct;
    if (row_kernel == CHSGA_ROW_TILED) c.row_kernel = RowKernel::Tiled;
    if (row_kernel == CHSGA_ROW_DPX) c.row_kernel = RowKernel::Dpx;
    if (row_kernel == CHSGA_ROW_STREAM) c.row_kernel = RowKernel::Stream;
    if (row_kernel == CHSGA_ROW_DELTA) c.row_kernel = RowKernel::Delta;
    c.top_sel = top_for(c, top_vertices);
  }
  ~CallKnobs() {
    c.row_kernel = rk;
    c.top_sel = ts;
  }
};

void scores_batched(chsga_ctx& c, const char* const* reads, const uint32_t* lens, uint32_t n,
                    const chsga_batch_opts* o, int32_t* out) {
  const uint32_t slots = o && o->slots ? o->slots : 64;
  const uint32_t graphs = o ? o->use_graphs : kLaunchGraphs;
  require(graphs <= kLaunchPersistent, CHSGA_ERR_INVALID_ARG, "use_graphs must be CHSGA_LAUNCH_*");
  const uint32_t per = o && o->steps_per_graph ? o->steps_per_graph : 8;
  const uint32_t rb = o ? o->row_bits : 0;
  require(rb == 0 || rb == 16 || rb == 32, CHSGA_ERR_INVALID_ARG, "row_bits must be 0, 16 or 32");
  CallKnobs knobs(c, o ? o->row_kernel : 0, o ? o->top_vertices : 0);
  switch (slots) {
    case 1: scores_with<1>(c, reads, lens, n, out, graphs, per, rb); break;
    case 2: scores_with<2>(c, reads, lens, n, out, graphs, per, rb); break;
    case 4: scores_with<4>(c, reads, lens, n, out, graphs, per, rb); break;
    case 8: scores_with<8>(c, reads, lens, n, out, graphs, per, rb); break;
    case 16: scores_with<16>(c, reads, lens, n, out, graphs, per, rb); break;
    case 32: scores_with<32>(c, reads, lens, n, out, graphs, per, rb); break;
    case 64: scores_with<64>(c, reads, lens, n, out, graphs, per, rb); break;
    case 128: scores_with<128>(c, reads, lens, n, out, graphs, per, rb); break;
    default: fail(CHSGA_ERR_INVALID_ARG, "slots must be 1, 2, 4, 8, 16, 32, 64 or 128");
  }
}

// Coordinate search over the batched engine's knobs on a read sample:
// slots, then steps per graph, then the row kernel, then the level
// grouping, each stage keeping the fastest by device time. With a cost
// model, the slot stage only runs the candidates of highest predicted
// throughput. Every run must return the first run's scores.
chsga_batch_opts autotune(chsga_ctx& c, const char* const* reads, const uint32_t* lens, uint32_t n,
                          const chsga_tune_opts* o, std::vector<chsga_tune_trial>& trials) {
  const uint32_t repeats = o && o->repeats ? o->repeats : 2;
  uint64_t sum_len = 0;
  for (uint32_t i = 0; i < n; ++i) sum_len += lens[i];
  const double cells = (double)sum_len * c.g->L.N;
  std::vector<int32_t> ref(n), got(n);
  bool have_ref = false;
  auto run = [&](const chsga_batch_opts& b, double predicted) {
    double best_ms = 1e300;
    for (uint32_t r = 0; r < repeats; ++r) {
      scores_batched(c, reads, lens, n, &b, got.data());
      best_ms = std::min(best_ms, (double)c.prof.total_ms);
      if (!have_ref) {
        ref = got;
        have_ref = true;
      }
      require(got == ref, CHSGA_ERR_INTERNAL, "autotune candidates disagree on the scores");
    }
    const double g = cells / (best_ms * 1e-3) / 1e9;
    trials.push_back(chsga_tune_trial{b.slots, b.steps_per_graph, b.row_kernel, b.top_vertices, predicted, g});
    return g;
  };
  chsga_batch_opts cur{};
  cur.slots = 64;
  cur.steps_per_graph = 8;
  cur.use_graphs = 1;
  // slots
  std::vector<std::pair<double, uint32_t>> cand;  // (predicted gcups, slots)
  for (uint32_t R : {16u, 32u, 64u, 128u}) {
    double pred = 0;
    if (o && o->cost_model) {
      // per-read time at R slots; R reads run at once
      std::vector<float> x((size_t)n * CHSGA_CM_FEATURES), y((size_t)n * CHSGA_CM_OUTPUTS);
      for (uint32_t i = 0; i < n; ++i)
        request_features(c, lens[i], CHSGA_REQ_SCORE, R, 0, 0, &x[(size_t)i * CHSGA_CM_FEATURES]);
      const chsga_status st = chsga_cm_predict(o->cost_model, x.data(), n, y.data());
      require(st == CHSGA_OK, st, "cost model prediction failed");
      double t_ms = 0;
      for (uint32_t i = 0; i < n; ++i) t_ms += y[(size_t)i * CHSGA_CM_OUTPUTS];
      pred = cells / (t_ms / R * 1e-3) / 1e9;
    }
    cand.push_back({pred, R});
  }
  if (o && o->cost_model) {
    std::stable_sort(cand.begin(), cand.end(), [](auto& a, auto& b) { return a.first > b.first; });
    const uint32_t top = o->measure_top ? o->measure_top : 4;
    for (size_t i = top; i < cand.size(); ++i)
      trials.push_back(chsga_tune_trial{cand[i].second, 8, 0, 0, cand[i].first, 0.0});
    cand.resize(std::min<size_t>(cand.size(), top));
  }
  double best_g = -1;
  chsga_batch_opts best = cur;
  for (auto& [pred, R] : cand) {
    chsga_batch_opts b = cur;
    b.slots = R;
    const double g = run(b, pred);
    if (g > best_g) best_g = g, best = b;
  }
  // steps per graph
  cur = best;
  for (uint32_t per : {4u, 16u}) {
    chsga_batch_opts b = cur;
    b.steps_per_graph = per;
    const double g = run(b, 0);
    if (g > best_g) best_g = g, best = b;
  }
  // row kernel
  cur = best;
  for (uint32_t rk : {(uint32_t)CHSGA_ROW_STREAM, (uint32_t)CHSGA_ROW_DPX, (uint32_t)CHSGA_ROW_DIRECT,
                      (uint32_t)CHSGA_ROW_TILED}) {
    if (rk == CHSGA_ROW_TILED && cur.slots < 32) continue;
    if (rk == CHSGA_ROW_DPX && cur.slots < 64) continue;        // AUTO already is DPX there
    if (rk == CHSGA_ROW_STREAM && cur.slots != 128) continue;   // AUTO is STREAM at 64, DELTA at 128
    chsga_batch_opts b = cur;
    b.row_kernel = rk;
    const double g = run(b, 0);
    if (g > best_g) best_g = g, best = b;
  }
  // level grouping
  cur = best;
  for (uint32_t K : {kTopMaxVertices, 3000u}) {
    chsga_batch_opts b = cur;
    b.top_vertices = K;
    const double g = run(b, 0);
    if (g > best_g) best_g = g, best = b;
  }
  return best;
}

template <typename F>
chsga_status guarded_ctx(chsga_ctx* c, F&& f) {
  try {
    if (c) set_device(*c);
    f();
    check_indices();
    return CHSGA_OK;
  } catch (const ChsgaError& e) {
    if (c) c->err = e.what();
    g_last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    if (c) c->err = "host out of memory";
    return CHSGA_ERR_OOM;
  } catch (const std::exception& e) {
    if (c) c->err = e.what();
    g_last_error = e.what();
    return CHSGA_ERR_INTERNAL;
  }
}

// ---- continuous score lane (serving) -----------------------------------------


__global__ void k_clock(unsigned long long* out) { *out = dev::global_ns(); }

int64_t host_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

template <int R, typename ST>
class ScoreLaneImpl final : public ScoreLane {
 public:
  ScoreLaneImpl(chsga_ctx& parent, uint32_t per_graph, uint32_t cap, uint64_t arena)
      : c_(fork_context(parent)), cap_(cap), arena_(arena) {
    chsga_ctx& c = *c_;
    per_ = std::max<uint32_t>(2, per_graph + (per_graph & 1));
    c.qmask = cap - 1;
    c.reads.alloc(arena + 64);
    c.queue.alloc(cap);
    c.res_score.alloc(cap);
    c.res_vertex.alloc(cap);
    c.res_t0.alloc(cap);
    c.res_t1.alloc(cap);
    c.done_ring.alloc(cap);
    b_ = &get_bufs<R, ST>(c, true);
    if (c.row_kernel == RowKernel::Tiled) row_tiles<R, ST>(c);  // allocates: before the capture
    reset_slots<R>(c, *b_, 0);
    launch_advance<R>(c, *b_, 0, c.st);  // every slot idle
    harena_.alloc(arena + 64);
    hq_.alloc(cap);
    hctl_.alloc(2);
    hring_.alloc(2 * (size_t)cap);
    for (auto& e : ev_) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaStream_t cap_st;
    CK(cudaStreamCreateWithFlags(&cap_st, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(cap_st, cudaStreamCaptureModeThreadLocal));
    ST* rows[2] = {reinterpret_cast<ST*>(b_->rows[0].p), reinterpret_cast<ST*>(b_->rows[1].p)};
    for (uint32_t i = 0; i < per_; ++i) row_step<R, true, ST>(c, *b_, rows[i & 1], rows[(i + 1) & 1], cap_st);
    CK(cudaStreamEndCapture(cap_st, &graph_));
    CK(cudaGraphInstantiate(&exec_, graph_, 0));
    CK(cudaStreamDestroy(cap_st));
    calibrate_clock();
  }

  ~ScoreLaneImpl() override {
    cudaStreamSynchronize(c_->st);
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    for (auto& e : ev_) cudaEventDestroy(e);
    chsga_close(c_);
  }

  uint32_t capacity() const override { return cap_; }
  uint64_t arena_bytes() const override { return arena_; }
  unsigned char* staging() override { return harena_.p; }
  uint64_t blocks() const override { return launched_; }
  uint32_t kernels_per_block() const override { return kernels_per_step(*c_) * per_; }

  void inject_wait_timeout() override {
    dev::k_wait_selftest<<<1, 32, 0, c_->st>>>(b_->ctl.p, 4096);
    check_launch();
  }

  void publish(uint64_t lo, uint64_t hi, const LaneRead* reads, uint32_t n) override {
    chsga_ctx& c = *c_;
    require(hi <= arena_ && lo <= hi, CHSGA_ERR_INTERNAL, "arena range");
    if (hi > lo)
      CK(cudaMemcpyAsync(c.reads.p + lo, harena_.p + lo, hi - lo, cudaMemcpyHostToDevice, c.st));
    const uint32_t mask = cap_ - 1;
    for (uint32_t i = 0; i < n; ++i) {
      require(reads[i].id < cap_ && reads[i].off + reads[i].len <= arena_, CHSGA_ERR_INTERNAL,
              "lane read out of range");
      hq_.p[(qpub_ + i) & mask] = dev::ReadDesc{reads[i].off, reads[i].len, (int32_t)reads[i].id};
    }
    const uint32_t first = qpub_ & mask;
    const uint32_t n1 = std::min<uint32_t>(n, cap_ - first);
    if (n1)
      CK(cudaMemcpyAsync(c.queue.p + first, hq_.p + first, n1 * sizeof(dev::ReadDesc),
                         cudaMemcpyHostToDevice, c.st));
    if (n > n1)
      CK(cudaMemcpyAsync(c.queue.p, hq_.p, (n - n1) * sizeof(dev::ReadDesc), cudaMemcpyHostToDevice,
                         c.st));
    qpub_ += n;
    k_publish<<<1, 1, 0, c.st>>>(b_->ctl.p, qpub_);
    check_launch();
  }

  void step(std::vector<LaneDone>& out) override {
    chsga_ctx& c = *c_;
    const int k = (int)(launched_ & 1);
    CK(cudaGraphLaunch(exec_, c.st));
    CK(cudaMemcpyAsync(hctl_.p + k, b_->ctl.p, sizeof(dev::StepCtl), cudaMemcpyDeviceToHost, c.st));
    CK(cudaMemcpyAsync(hring_.p + (size_t)k * cap_, c.done_ring.p, (size_t)cap_ * sizeof(dev::CompletionRec),
                       cudaMemcpyDeviceToHost, c.st));
    CK(cudaEventRecord(ev_[k], c.st));
    ++launched_;
    if (launched_ >= 2) harvest((int)((launched_ - 2) & 1), out);
  }

  void drain(std::vector<LaneDone>& out) override {
    if (launched_ == 0) return;
    CK(cudaStreamSynchronize(c_->st));
    harvest((int)((launched_ - 1) & 1), out);
  }

 private:
  void harvest(int k, std::vector<LaneDone>& out) {
    CK(cudaEventSynchronize(ev_[k]));
    const dev::StepCtl& s = hctl_.p[k];
    require_step_ok(s.error);
    const uint32_t mask = cap_ - 1;
    for (uint32_t i = hdone_; i != s.done; ++i) {
      const dev::CompletionRec& r = hring_.p[(size_t)k * cap_ + (i & mask)];
      out.push_back(LaneDone{(uint32_t)r.id, r.score, r.vertex, (int64_t)r.t0 - clock_off_,
                             (int64_t)r.t1 - clock_off_});
    }
    hdone_ = s.done;
  }

  // device global timer minus host steady clock, from the tightest of a few
  // round trips
  void calibrate_clock() {
    DevArr<unsigned long long> t;
    t.alloc(1);
    int64_t best_rt = INT64_MAX;
    for (int i = 0; i < 8; ++i) {
      CK(cudaStreamSynchronize(c_->st));
      const int64_t a = host_ns();
      k_clock<<<1, 1, 0, c_->st>>>(t.p);
      unsigned long long d = 0;
      CK(cudaMemcpyAsync(&d, t.p, 8, cudaMemcpyDeviceToHost, c_->st));
      CK(cudaStreamSynchronize(c_->st));
      const int64_t b = host_ns();
      if (b - a < best_rt) {
        best_rt = b - a;
        clock_off_ = (int64_t)d - (a + b) / 2;
      }
    }
  }

  chsga_ctx* c_;
  SlotBufs* b_ = nullptr;
  uint32_t cap_;
  uint64_t arena_;
  uint32_t per_ = 8;
  uint32_t qpub_ = 0, hdone_ = 0;
  uint64_t launched_ = 0;
  int64_t clock_off_ = 0;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  PinnedArr<unsigned char> harena_;
  PinnedArr<dev::ReadDesc> hq_;
  PinnedArr<dev::StepCtl> hctl_;
  PinnedArr<dev::CompletionRec> hring_;
};

template <typename ST>
std::unique_ptr<ScoreLane> lane_for(chsga_ctx& p, uint32_t slots, uint32_t per, uint32_t cap,
                                    uint64_t arena) {
  switch (slots) {
    case 2: return std::make_unique<ScoreLaneImpl<2, ST>>(p, per, cap, arena);
    case 4: return std::make_unique<ScoreLaneImpl<4, ST>>(p, per, cap, arena);
    case 8: return std::make_unique<ScoreLaneImpl<8, ST>>(p, per, cap, arena);
    case 16: return std::make_unique<ScoreLaneImpl<16, ST>>(p, per, cap, arena);
    case 32: return std::make_unique<ScoreLaneImpl<32, ST>>(p, per, cap, arena);
    case 64: return std::make_unique<ScoreLaneImpl<64, ST>>(p, per, cap, arena);
    case 128: return std::make_unique<ScoreLaneImpl<128, ST>>(p, per, cap, arena);
    default: fail(CHSGA_ERR_INVALID_ARG, "slots must be 2, 4, 8, 16, 32, 64 or 128");
  }
}

}  // namespace

chsga_ctx* fork_context(chsga_ctx& p) {
  require(p.loaded && p.g, CHSGA_ERR_INVALID_ARG, "no graph loaded");
  auto c = std::make_unique<chsga_ctx>();
  c->device = p.device;
  c->flags = p.flags & ~(uint32_t)CHSGA_FLAG_PROFILE;
  c->cap = p.cap;
  c->num_sms = p.num_sms;
  c->row_kernel = p.row_kernel;
  c->plain_mode = p.plain_mode;
  c->pdl = p.pdl;
  c->pull_coop = p.pull_coop;
  c->pull_lean = p.pull_lean;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
  c->g = p.g;
  c->loaded = true;
  return c.release();
}

uint64_t traceback_device_bytes(const chsga_ctx& c, uint32_t len, const chsga_tb_opts* o) {
  // rows as traceback_rows stores them; the path choice counts int32 rows
  const uint64_t pb = (uint64_t)c.g->pitch * (len <= kRow16Max ? 2 : 4), row_bytes = (uint64_t)c.g->L.N * 4;
  const int64_t k = (o && o->k > 0) ? o->k : 500;
  const uint64_t cap = (o && o->cap_bytes) ? o->cap_bytes : c.cap;
  const uint64_t read = (len + 255) / 256 * 256;
  if ((uint64_t)len * row_bytes <= cap) return ((uint64_t)len + 1) * pb + read;
  // checkpointed: three forward rows, then the largest recompute segment
  const uint64_t budget = std::max<uint64_t>(c.cap, cap);
  const uint64_t seg = std::min<uint64_t>((uint64_t)k, len ? len - 1 : 0) + 1;
  uint64_t peak = seg * pb;
  if (!(seg * pb <= budget || seg <= 2)) {
    const uint64_t span = seg - 1;
    const uint64_t k2 = std::max<uint64_t>(1, sub_segment_rows(span, budget / pb));
    peak = ((span + k2 - 1) / k2 + k2 + 1) * pb;
  }
  return std::max<uint64_t>(3 * pb, peak) + read;
}

uint64_t graph_chars(const chsga_ctx& c) { return c.g->L.N; }
uint64_t graph_string_vertices(const chsga_ctx& c) { return c.g->L.S; }
int32_t empty_read_score(const chsga_ctx& c) { return empty_score(c); }

void bind_device(const chsga_ctx& c) { CK(cudaSetDevice(c.device)); }

int64_t meter_reset() {
  t_peak_bytes = t_live_bytes;
  return t_live_bytes;
}

uint64_t meter_peak_since(int64_t base) { return (uint64_t)std::max<int64_t>(0, t_peak_bytes - base); }

void request_features(const chsga_ctx& c, uint32_t len, uint32_t mode, uint32_t slots, int64_t k,
                      uint64_t cap_bytes, float* x) {
  const HostLayout& L = c.g->L;
  const uint64_t cap = cap_bytes ? cap_bytes : c.cap;
  const bool tb = mode == CHSGA_REQ_TRACEBACK;
  const bool ck = tb && (uint64_t)len * L.N * 4 > cap;
  x[0] = (float)std::log2((double)len + 1);
  x[1] = (float)std::log2((double)std::max<uint32_t>(L.N, 1));
  x[2] = (float)std::log2((double)std::max<uint32_t>(L.S, 1));
  x[3] = (float)std::log2((double)(L.up_in.size() + L.dn_in.size()) + 1);
  x[4] = (float)std::log2((double)L.levels + 1);
  x[5] = (float)std::log2((double)std::max<uint32_t>(slots, 1));
  x[6] = tb ? 1.f : 0.f;
  x[7] = ck ? (float)std::log2((double)std::max<int64_t>(k > 0 ? k : 500, 1)) : 0.f;
}

uint64_t device_free_bytes(const chsga_ctx& c) {
  CK(cudaSetDevice(c.device));
  size_t f = 0, t = 0;
  CK(cudaMemGetInfo(&f, &t));
  return f;
}

std::unique_ptr<ScoreLane> make_score_lane(chsga_ctx& parent, uint32_t slots, uint32_t per_graph,
                                           uint32_t capacity, uint64_t arena_bytes,
                                           uint32_t row_bits) {
  require(capacity >= 2 && (capacity & (capacity - 1)) == 0, CHSGA_ERR_INVALID_ARG,
          "queue capacity must be a power of two");
  require(row_bits == 16 || row_bits == 32, CHSGA_ERR_INVALID_ARG, "row_bits must be 16 or 32");
  if (row_bits == 16) return lane_for<uint16_t>(parent, slots, per_graph, capacity, arena_bytes);
  return lane_for<int>(parent, slots, per_graph, capacity, arena_bytes);
}

}  // namespace chsga

using namespace chsga;

extern "C" {

chsga_status chsga_open(const chsga_opts* opts, chsga_ctx** out) {
  return guarded_ctx(nullptr, [&] {
    require(out != nullptr, CHSGA_ERR_INVALID_ARG, "null output");
    auto c = std::make_unique<chsga_ctx>();
    c->device = opts ? opts->device : 0;
    c->flags = opts ? opts->flags : 0;
    int count = 0;
    CK(cudaGetDeviceCount(&count));
    require(c->device >= 0 && c->device < count, CHSGA_ERR_INVALID_ARG, "no such CUDA device");
    CK(cudaSetDevice(c->device));
    cudaDeviceProp prop{};
    CK(cudaGetDeviceProperties(&prop, c->device));
    require(prop.major >= 10, CHSGA_ERR_UNSUPPORTED,
            std::string("libchsga is built for sm_100a; device is ") + prop.name);
    c->num_sms = prop.multiProcessorCount;
    if (const char* rk = std::getenv("CHSGA_ROW_KERNEL")) {
      if (std::string(rk) == "direct") c->row_kernel = RowKernel::Direct;
      if (std::string(rk) == "tiled") c->row_kernel = RowKernel::Tiled;
      if (std::string(rk) == "dpx") c->row_kernel = RowKernel::Dpx;
      if (std::string(rk) == "stream") c->row_kernel = RowKernel::Stream;
      if (std::string(rk) == "delta") c->row_kernel = RowKernel::Delta;
    }
    // CHSGA_PLAIN_LAUNCH=stream|graphs|persistent: how chsga_align_scores
    // runs its row-steps (default graphs)
    if (const char* pl = std::getenv("CHSGA_PLAIN_LAUNCH")) {
      if (std::string(pl) == "stream") c->plain_mode = CHSGA_LAUNCH_STREAM;
      if (std::string(pl) == "graphs") c->plain_mode = CHSGA_LAUNCH_GRAPHS;
      if (std::string(pl) == "persistent") c->plain_mode = CHSGA_LAUNCH_PERSISTENT;
    }
    if (const char* pd = std::getenv("CHSGA_PDL")) c->pdl = std::string(pd) != "0";
    if (const char* pc = std::getenv("CHSGA_PULL_COOP")) c->pull_coop = std::string(pc) == "1";
    if (const char* pn = std::getenv("CHSGA_PULL_LEAN")) c->pull_lean = std::string(pn) != "0";
    CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    c->cap = (opts && opts->hbm_cap_bytes) ? opts->hbm_cap_bytes : (uint64_t)(free_b * 0.85);
    *out = c.release();
  });
}

void chsga_close(chsga_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->st);
  c->bufs.clear();
  c->g.reset();
  if (c->st) cudaStreamDestroy(c->st);
  if (c->side) cudaStreamDestroy(c->side);
  delete c;
}

const char* chsga_last_error(chsga_ctx* c) { return c ? c->err.c_str() : g_last_error.c_str(); }

chsga_status chsga_load_graph(chsga_ctx* c, const chsga_graph_host* g) {
  return guarded_ctx(c, [&] {
    require(c && g, CHSGA_ERR_INVALID_ARG, "null argument");
    upload_graph(*c, *g);
  });
}

chsga_status chsga_load_host_graph(chsga_ctx* c, const chsga_host_graph* g) {
  return guarded_ctx(c, [&] {
    require(c && g, CHSGA_ERR_INVALID_ARG, "null argument");
    validate_host_graph(*g);
    chsga_graph_host v{};
    require(chsga_graph_view(g, &v) == CHSGA_OK, CHSGA_ERR_INTERNAL, "graph view");
    upload_graph(*c, v);
  });
}

chsga_status chsga_align_scores(chsga_ctx* c, const char* const* reads, const uint32_t* lens,
                                uint32_t n, int32_t* scores_out) {
  return guarded_ctx(c, [&] {
    require(c && (n == 0 || (reads && lens && scores_out)), CHSGA_ERR_INVALID_ARG, "null argument");
    require(c->loaded, CHSGA_ERR_INVALID_ARG, "no graph loaded");
    scores_with<1>(*c, reads, lens, n, scores_out, c->plain_mode, 16,
                   (uint32_t)std::strtoul(std::getenv("CHSGA_ROW_BITS") ? std::getenv("CHSGA_ROW_BITS") : "0",
                                          nullptr, 10));
  });
}

chsga_status chsga_align_scores_batched(chsga_ctx* c, const char* const* reads,
                                        const uint32_t* lens, uint32_t n,
                                        const chsga_batch_opts* o, int32_t* scores_out) {
  return guarded_ctx(c, [&] {
    require(c && (n == 0 || (reads && lens && scores_out)), CHSGA_ERR_INVALID_ARG, "null argument");
    require(c->loaded, CHSGA_ERR_INVALID_ARG, "no graph loaded");
    scores_batched(*c, reads, lens, n, o, scores_out);
  });
}

chsga_status chsga_autotune(chsga_ctx* c, const char* const* reads, const uint32_t* lens,
                            uint32_t n, const chsga_tune_opts* opts, chsga_batch_opts* best,
                            chsga_tune_trial* trials, uint32_t max_trials, uint32_t* n_trials) {
  return guarded_ctx(c, [&] {
    require(c && reads && lens && n > 0 && best, CHSGA_ERR_INVALID_ARG, "bad argument");
    require(c->loaded, CHSGA_ERR_INVALID_ARG, "no graph loaded");
    std::vector<chsga_tune_trial> t;
    *best = autotune(*c, reads, lens, n, opts, t);
    const uint32_t m = std::min<uint32_t>(max_trials, (uint32_t)t.size());
    if (trials)
      for (uint32_t i = 0; i < m; ++i) trials[i] = t[i];
    if (n_trials) *n_trials = (uint32_t)t.size();
  });
}

chsga_status chsga_align_scores_noalloc(chsga_ctx* c, const char* const* reads,
                                        const uint32_t* lens, uint32_t n, int32_t* scores_out) {
  return guarded_ctx(c, [&] {
    require(c && (n == 0 || (reads && lens && scores_out)), CHSGA_ERR_INVALID_ARG, "null argument");
    require(c->loaded, CHSGA_ERR_INVALID_ARG, "no graph loaded");
    scores_noalloc(*c, reads, lens, n, scores_out);
  });
}

chsga_status chsga_align_rows(chsga_ctx* c, const char* read, uint32_t len, int32_t* rows_out) {
  return guarded_ctx(c, [&] {
    require(c && read && rows_out && len > 0, CHSGA_ERR_INVALID_ARG, "bad argument");
    require(c->loaded, CHSGA_ERR_INVALID_ARG, "no graph loaded");
    const size_t N = c->g->pitch, NC = c->g->L.N;
    const char* rp[1] = {read};
    upload_reads(*c, rp, &len, 1);
    SlotBufs& b = get_bufs<1, int>(*c, false);
    DevArr<int> M;
    M.alloc((size_t)(len + 1) * N);
    reset_slots<1>(*c, b, 1);
    launch_advance<1>(*c, b, 0, c->st);
    for (uint32_t i = 0; i < len; ++i)
      row_step<1, false, int>(*c, b, M.p + (size_t)(i ? i - 1 : len) * N, M.p + (size_t)i * N, c->st);
    check_device_error(*c, b);
    CK(cudaMemcpy2D(rows_out, NC * 4, M.p, N * 4, NC * 4, len, cudaMemcpyDeviceToHost));
  });
}

chsga_status chsga_align_traceback(chsga_ctx* c, const char* read, uint32_t len,
                                   const chsga_tb_opts* opts, chsga_tb_result* out) {
  return guarded_ctx(c, [&] {
    require(c && read && out, CHSGA_ERR_INVALID_ARG, "null argument");
    require(c->loaded, CHSGA_ERR_INVALID_ARG, "no graph loaded");
    std::memset(out, 0, sizeof(*out));
    traceback(*c, read, len, opts, out);
  });
}

chsga_status chsga_align_traceback_batched(chsga_ctx* c, const char* const* reads,
                                           const uint32_t* lens, uint32_t n,
                                           const chsga_tb_opts* opts, uint32_t slots,
                                           chsga_tb_result* out) {
  return guarded_ctx(c, [&] {
    require(c && (n == 0 || (reads && lens && out)), CHSGA_ERR_INVALID_ARG, "null argument");
    require(c->loaded, CHSGA_ERR_INVALID_ARG, "no graph loaded");
    if (!slots) slots = 64;
    require(slots == 4 || slots == 8 || slots == 16 || slots == 32 || slots == 64, CHSGA_ERR_INVALID_ARG,
            "slots must be 4, 8, 16, 32 or 64");
    for (uint32_t i = 0; i < n; ++i) {
      require(reads[i] && lens[i] > 0, CHSGA_ERR_INVALID_ARG, "traceback of an empty read");
      std::memset(&out[i], 0, sizeof(out[i]));
    }
    // the one-read path's choice between the full matrix and checkpoints
    const uint64_t cap = (opts && opts->cap_bytes) ? opts->cap_bytes : c->cap;
    const uint64_t row_bytes = (uint64_t)c->g->L.N * 4;
    std::vector<uint32_t> full, rest;
    for (uint32_t i = 0; i < n; ++i) {
      // (a full-matrix traceback never writes checkpoint files, so a
      // checkpoint directory does not keep a read off the batched path)
      if (lens[i] <= kRow16Max && (uint64_t)lens[i] * row_bytes <= cap)
        full.push_back(i);
      else
        rest.push_back(i);
    }
    std::stable_sort(full.begin(), full.end(), [&](uint32_t a, uint32_t b) { return lens[a] > lens[b]; });
    try {
      // groups of reads (longest first) whose 16-bit matrices fit together
      // `slots` at a time; a group whose matrices are large runs with fewer
      // slots (idle slots would still cost a full row-step each)
      const uint64_t mem = (uint64_t)(device_free_bytes(*c) * 0.6);
      const uint64_t pitch_b = (uint64_t)c->g->pitch * 2;
      size_t g0 = 0;
      while (g0 < full.size()) {
        const uint64_t mb = (uint64_t)lens[full[g0]] * pitch_b;  // the group's largest matrix
        uint32_t fit = (uint32_t)std::min<uint64_t>(slots, std::max<uint64_t>(1, mem / std::max<uint64_t>(mb, 1)));
        uint32_t R = 64;
        while (R > fit && R > 4) R >>= 1;
        // the group: reads while a matrix at most half as large cannot run with more slots
        size_t g1 = g0 + 1;
        while (g1 < full.size() && (uint64_t)lens[full[g1]] * pitch_b * 2 > mb) ++g1;
        std::vector<uint32_t> grp(full.begin() + g0, full.begin() + g1);
        if (grp.size() == 1) {
          rest.push_back(grp[0]);
        } else {
          switch (std::min(R, slots)) {
            case 4: traceback_batched<4>(*c, reads, lens, grp, out); break;
            case 8: traceback_batched<8>(*c, reads, lens, grp, out); break;
            case 16: traceback_batched<16>(*c, reads, lens, grp, out); break;
            case 32: traceback_batched<32>(*c, reads, lens, grp, out); break;
            default: traceback_batched<64>(*c, reads, lens, grp, out); break;
          }
        }
        g0 = g1;
      }
      for (uint32_t i : rest) traceback(*c, reads[i], lens[i], opts, &out[i]);
    } catch (...) {
      for (uint32_t i = 0; i < n; ++i) chsga_tb_result_free(&out[i]);
      throw;
    }
  });
}

void chsga_tb_result_free(chsga_tb_result* r) {
  if (!r) return;
  std::free(r->ops);
  r->ops = nullptr;
  r->num_ops = 0;
}

uint64_t chsga_ops_to_cigar(const chsga_op* ops, uint64_t n, char* buf, uint64_t cap) {
  std::string cig;
  auto ch = [](uint8_t op) { return op == CHSGA_OP_DELETE ? 'D' : op == CHSGA_OP_MATCHSUB ? 'M' : 'I'; };
  if (n > 0) {
    char prev = ch(ops[0].op);
    uint64_t run = 1;
    for (uint64_t i = 1; i < n; ++i) {
      char x = ch(ops[i].op);
      if (x == prev) {
        ++run;
      } else {
        cig += std::to_string(run);
        cig += prev;
        prev = x;
        run = 1;
      }
    }
    cig += std::to_string(run);
    cig += prev;
  }
  if (buf && cap) {
    size_t m = std::min<size_t>(cap - 1, cig.size());
    std::memcpy(buf, cig.data(), m);
    buf[m] = '\0';
  }
  return cig.size();
}

chsga_status chsga_get_read_times(chsga_ctx* c, uint64_t* admit_ns, uint64_t* done_ns,
                                  uint32_t n) {
  return guarded_ctx(c, [&] {
    require(c && admit_ns && done_ns, CHSGA_ERR_INVALID_ARG, "null argument");
    require(n == c->last_ids.size() || n == 0, CHSGA_ERR_INVALID_ARG,
            "n must equal the number of non-empty reads of the last score call");
    std::vector<unsigned long long> a(n), d(n);
    if (n) {
      CK(cudaMemcpy(a.data(), c->res_t0.p, n * 8, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(d.data(), c->res_t1.p, n * 8, cudaMemcpyDeviceToHost));
    }
    for (uint32_t i = 0; i < n; ++i) {
      admit_ns[i] = a[i];
      done_ns[i] = d[i];
    }
  });
}

chsga_status chsga_cm_features(chsga_ctx* c, uint32_t read_len, uint32_t mode, uint32_t slots,
                               int64_t k, uint64_t cap_bytes, float* x_out) {
  return guarded_ctx(c, [&] {
    require(c && x_out, CHSGA_ERR_INVALID_ARG, "null argument");
    require(c->loaded, CHSGA_ERR_INVALID_ARG, "no graph loaded");
    request_features(*c, read_len, mode, slots, k, cap_bytes, x_out);
  });
}

chsga_status chsga_selftest_wait(chsga_ctx* c, uint32_t polls) {
  return guarded_ctx(c, [&] {
    require(c != nullptr, CHSGA_ERR_INVALID_ARG, "null argument");
    SlotBufs b;
    b.ctl.alloc(1);
    CK(cudaMemsetAsync(b.ctl.p, 0, sizeof(dev::StepCtl), c->st));
    dev::k_wait_selftest<<<1, 32, 0, c->st>>>(b.ctl.p, polls);
    check_launch();
    check_device_error(*c, b);
  });
}

chsga_status chsga_selftest_grid_wait(chsga_ctx* c, uint32_t limit_us) {
  return guarded_ctx(c, [&] {
    require(c != nullptr, CHSGA_ERR_INVALID_ARG, "null argument");
    require(limit_us > 0 && limit_us <= 1000000, CHSGA_ERR_INVALID_ARG, "limit_us must be 1 .. 1000000");
    SlotBufs b;
    b.ctl.alloc(1);
    b.bar.alloc(1);
    CK(cudaMemsetAsync(b.ctl.p, 0, sizeof(dev::StepCtl), c->st));
    CK(cudaMemsetAsync(b.bar.p, 0, sizeof(dev::GridBar), c->st));
    dev::k_grid_selftest<<<2, 32, 0, c->st>>>(b.bar.p, b.ctl.p, (unsigned long long)limit_us * 1000ull);
    check_launch();
    dev::GridBar gb{};
    CK(cudaMemcpyAsync(&gb, b.bar.p, sizeof(gb), cudaMemcpyDeviceToHost, c->st));
    check_device_error(*c, b);  // throws CHSGA_ERR_TIMEOUT when the wait gave up
    require(false, CHSGA_ERR_INTERNAL,
            "the grid barrier wait did not give up (abort word " + std::to_string(gb.abort) + ")");
  });
}

chsga_status chsga_get_profile(chsga_ctx* c, chsga_profile* out) {
  return guarded_ctx(c, [&] {
    require(c && out, CHSGA_ERR_INVALID_ARG, "null argument");
    *out = c->prof;
  });
}

}  // extern "C"
