// Witness searches of the hierarchy builder on the device (see pch_gpu.hpp).
//
// One thread runs one bounded Dijkstra. Only relaxations within the bound
// are kept: the search never pops an entry above it, and every query
// threshold is at most the bound, so a vertex left out answers each query
// like one whose tentative distance exceeds the bound. The kept distances
// (below 2^32: a larger bound sends the task to the host) live in a
// per-thread open-addressing table (kHash slots, at most kHashMaxFill used,
// entries of earlier tasks told apart by a generation stamp) and the queue
// in a per-thread binary heap of distance << 32 | vertex keys, which order
// by distance, then vertex id, as the CPU's std::priority_queue of pairs
// does; both pop the same sequence and stop at the same pop. A search that
// would outgrow either structure is reported as kPchOverflow and redone by
// the caller on the CPU.
#include <cuda_runtime.h>

#include <string>

#include "common.hpp"
#include "pch_gpu.hpp"

namespace chsga {

#define CKP(x)                                                                               \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess)                                                                   \
      fail(e_ == cudaErrorMemoryAllocation ? CHSGA_ERR_OOM : CHSGA_ERR_CUDA,                 \
           std::string("hierarchy builder: ") + #x + ": " + cudaGetErrorString(e_));        \
  } while (0)

namespace {

constexpr uint32_t kHashBits = 7, kHash = 1u << kHashBits, kHashMaxFill = 96, kHeap = 128;
constexpr uint32_t kNoDist = 0xFFFFFFFFu;
constexpr int kSearchThreads = 128;

__global__ void __launch_bounds__(kSearchThreads)
    k_witness(const uint32_t* __restrict__ off, const uint64_t* __restrict__ arcs,
              const uint32_t* __restrict__ thru, const uint32_t* __restrict__ tu,
              const uint32_t* __restrict__ ts, const uint32_t* __restrict__ tw, uint64_t ntasks,
              uint32_t pop_limit, uint64_t* __restrict__ masks) {
  uint32_t hkey[kHash], hdist[kHash];
  uint16_t hgen[kHash];
  uint64_t heap[kHeap];
  for (uint32_t i = 0; i < kHash; ++i) hgen[i] = 0;
  uint16_t gen = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += stride) {
    if (++gen == 0) {
      for (uint32_t i = 0; i < kHash; ++i) hgen[i] = 0;
      gen = 1;
    }
    const uint32_t u = tu[t];
    const uint32_t u0 = off[u], u1 = off[u + 1];
    uint64_t max_out = 0;
    for (uint32_t j = u0; j < u1; ++j) max_out = max(max_out, arcs[j] >> 32);
    const bool score = ts != nullptr;
    const uint32_t s = score ? ts[t] : u;
    const uint64_t w_in = score ? (uint64_t)tw[t] : 0;
    const uint64_t bound64 = score ? w_in + thru[u] + max_out : max_out;
    if (u1 - u0 > kPchMaskDegree || bound64 >= kNoDist) {
      masks[t] = kPchOverflow;
      continue;
    }
    const uint32_t bound = (uint32_t)bound64;
    uint32_t fill = 0, qn = 0;
    bool ovf = false;
    // slot holding v, or the empty slot where v would go (the table is never
    // more than three quarters full, so the probe ends)
    auto slot = [&](uint32_t v) {
      uint32_t h = (v * 0x9E3779B1u) >> (32 - kHashBits);
      while (hgen[h] == gen && hkey[h] != v) h = (h + 1) & (kHash - 1);
      return h;
    };
    auto dist = [&](uint32_t v) {
      const uint32_t h = slot(v);
      return hgen[h] == gen ? hdist[h] : kNoDist;
    };
    // d < dist(v) and d within the bound: record it and queue (d, v)
    auto relax = [&](uint32_t v, uint64_t d) {
      if (d > bound) return;
      const uint32_t h = slot(v);
      const bool present = hgen[h] == gen;
      if (present && hdist[h] <= d) return;
      if (qn == kHeap || (!present && fill == kHashMaxFill)) {
        ovf = true;
        return;
      }
      if (!present) {
        ++fill;
        hgen[h] = gen;
        hkey[h] = v;
      }
      hdist[h] = (uint32_t)d;
      const uint64_t key = d << 32 | v;
      uint32_t i = qn++;
      while (i > 0) {
        const uint32_t p = (i - 1) >> 1;
        if (heap[p] <= key) break;
        heap[i] = heap[p];
        i = p;
      }
      heap[i] = key;
    };
    auto pop = [&]() {
      const uint64_t last = heap[--qn];
      if (qn == 0) return;
      uint32_t i = 0;
      while (true) {
        uint32_t c = 2 * i + 1;
        if (c >= qn) break;
        if (c + 1 < qn && heap[c + 1] < heap[c]) ++c;
        if (heap[c] >= last) break;
        heap[i] = heap[c];
        i = c;
      }
      heap[i] = last;
    };
    for (uint32_t j = off[s]; j < off[s + 1] && !ovf; ++j) relax((uint32_t)arcs[j], arcs[j] >> 32);
    uint32_t pops = 0;
    // every queued entry is within the bound, so the bound check of the
    // host search never ends this loop early
    while (!ovf && qn > 0 && pops < pop_limit) {
      const uint32_t d = (uint32_t)(heap[0] >> 32);
      const uint32_t x = (uint32_t)heap[0];
      pop();
      if (dist(x) < d) continue;  // stale entry
      ++pops;
      const uint64_t base = (uint64_t)d + thru[x];
      for (uint32_t j = off[x]; j < off[x + 1] && !ovf; ++j) {
        const uint32_t v = (uint32_t)arcs[j];
        if (v != s) relax(v, base + (arcs[j] >> 32));
      }
    }
    if (ovf) {
      masks[t] = kPchOverflow;
      continue;
    }
    uint64_t m = 0;
    for (uint32_t j = u0; j < u1; ++j) {
      const uint32_t b = (uint32_t)arcs[j];
      const uint64_t wb = arcs[j] >> 32;
      const bool bit = score ? (b != s && dist(b) >= w_in + wb + thru[u]) : dist(b) >= wb;
      if (bit) m |= 1ull << (j - u0);
    }
    if (score && dist(u) >= w_in) m |= 1ull << 62;
    masks[t] = m;
  }
}

template <typename T>
struct Buf {
  T* p = nullptr;
  size_t cap = 0;
  void fit(size_t n) {
    if (n <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    CKP(cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T)));
    cap = std::max<size_t>(n, 1);
  }
  void put(const std::vector<T>& v, cudaStream_t s) {
    fit(v.size());
    if (!v.empty()) CKP(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

struct PchGpuImpl {
  int device = 0;
  uint32_t pop_limit = 500;
  uint32_t n = 0;
  int blocks = 0;
  cudaStream_t st = nullptr;
  Buf<uint32_t> thru, off, tu, ts, tw;
  Buf<uint64_t> arcs, masks;
};

PchGpu::PchGpu(int device, uint32_t pop_limit) : p_(std::make_unique<PchGpuImpl>()) {
  int count = 0;
  CKP(cudaGetDeviceCount(&count));
  require(device >= 0 && device < count, CHSGA_ERR_INVALID_ARG,
          "hierarchy builder: no CUDA device " + std::to_string(device));
  p_->device = device;
  p_->pop_limit = pop_limit;
  CKP(cudaSetDevice(device));
  int sms = 0;
  CKP(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  p_->blocks = sms * 4;
  CKP(cudaStreamCreateWithFlags(&p_->st, cudaStreamNonBlocking));
}

PchGpu::~PchGpu() {
  if (p_ && p_->st) {
    cudaSetDevice(p_->device);
    cudaStreamSynchronize(p_->st);
    cudaStreamDestroy(p_->st);
  }
}

void PchGpu::set_overlay(const std::vector<uint32_t>& off, const std::vector<uint64_t>& arcs,
                         const std::vector<uint32_t>& through) {
  require(!off.empty() && off.size() == through.size() + 1 && off.back() == arcs.size(),
          CHSGA_ERR_INTERNAL, "hierarchy builder: overlay size");
  const uint32_t n = (uint32_t)through.size();
  int64_t bad = 0;
#pragma omp parallel for reduction(+ : bad)
  for (int64_t i = 0; i < (int64_t)arcs.size(); ++i) bad += (uint32_t)arcs[i] >= n;
  require(bad == 0, CHSGA_ERR_INTERNAL, "hierarchy builder: arc target");
  p_->n = n;
  CKP(cudaSetDevice(p_->device));
  p_->off.put(off, p_->st);
  p_->arcs.put(arcs, p_->st);
  p_->thru.put(through, p_->st);
}

void PchGpu::run(const std::vector<uint32_t>& tu, const std::vector<uint32_t>& ts,
                 const std::vector<uint32_t>& tw, std::vector<uint64_t>& masks) {
  const bool score = !ts.empty();
  require(!score || (ts.size() == tu.size() && tw.size() == tu.size()), CHSGA_ERR_INTERNAL,
          "hierarchy builder: task arrays");
  masks.resize(tu.size());
  if (tu.empty()) return;
  for (uint32_t u : tu) require(u < p_->n, CHSGA_ERR_INTERNAL, "hierarchy builder: task vertex");
  for (uint32_t s : ts) require(s < p_->n, CHSGA_ERR_INTERNAL, "hierarchy builder: search source");
  CKP(cudaSetDevice(p_->device));
  p_->tu.put(tu, p_->st);
  if (score) {
    p_->ts.put(ts, p_->st);
    p_->tw.put(tw, p_->st);
  }
  p_->masks.fit(tu.size());
  const uint64_t nt = tu.size();
  const int blocks = (int)std::min<uint64_t>((uint64_t)p_->blocks, (nt + kSearchThreads - 1) / kSearchThreads);
  k_witness<<<blocks, kSearchThreads, 0, p_->st>>>(p_->off.p, p_->arcs.p, p_->thru.p, p_->tu.p,
                                                   score ? p_->ts.p : nullptr, score ? p_->tw.p : nullptr,
                                                   nt, p_->pop_limit, p_->masks.p);
  CKP(cudaGetLastError());
  CKP(cudaMemcpyAsync(masks.data(), p_->masks.p, nt * sizeof(uint64_t), cudaMemcpyDeviceToHost, p_->st));
  CKP(cudaStreamSynchronize(p_->st));
}

}  // namespace chsga
