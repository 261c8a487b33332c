// The persistent row-step kernel: one cooperative launch advances every
// slot through a block of row-steps (src/align.hpp:430-463 per slot), each
// row-step the same phases as the launch chain of engine.cu::row_step --
// the row update, the upward levels below the top region, the edges from
// below into the top region, the top region (block r sweeps slot r), the
// downward levels, the slot advance -- separated by grid barriers instead of
// kernel boundaries. Score-only (deferred closure), 16-bit rows.
//
// Every block runs every phase with a grid-stride loop over that phase's
// work items (tiles, vertices, runs of vertices, hierarchy positions), using
// the same per-item code as the separate kernels. Data written by other
// blocks earlier in the launch is read with plain or L2 loads, never the
// read-only path (COH = true).
//
// Grid barrier: a block's thread 0 adds one arrival to a global counter;
// the last arrival resets the counter and bumps a generation word, the
// others spin on the generation with acquire loads. Every spin is bounded
// by the device's global timer: a block that gives up sets StepCtl::error
// and an abort word that every other spin also watches, and returns; the
// host turns the error into CHSGA_ERR_TIMEOUT. A launch needs all of its
// blocks resident at once, which the cooperative launch guarantees.
#pragma once

#include "kernels.cuh"

namespace chsga {
namespace dev {

// The arrival counter, the generation word and the abort word sit on
// separate 128-byte lines, so the blocks spinning on the generation do not
// slow the arrivals down.
struct GridBar {
  unsigned int count;  // arrivals at the current barrier
  unsigned int pad0[31];
  unsigned int gen;    // barriers completed (only grows)
  unsigned int pad1[31];
  unsigned int abort;  // nonzero: some block gave up waiting
  unsigned int pad2[31];
};

constexpr uint32_t ERR_GRID_WAIT = 4;
constexpr unsigned long long kGridWaitNs = 4000000000ull;  // 4 s on the global timer

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int atom_add_acq_rel(unsigned int* p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void red_add_release(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Every block of the grid meets here. False when this block's wait gave up
// or another block's did (the caller returns at once). The block barrier
// orders every thread's writes before thread 0's release-acquire arrival;
// the acquire load that sees the new generation orders the reads after it.
__device__ __forceinline__ bool grid_sync(GridBar* gb, unsigned int& gen, StepCtl* ctl,
                                          unsigned long long limit_ns = kGridWaitNs) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int g0 = gen;
    if (atom_add_acq_rel(&gb->count, 1u) == gridDim.x - 1) {
      gb->count = 0;  // nobody arrives again before the generation moves
      red_add_release(&gb->gen, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned int polls = 0;
      while (ld_acquire_u32(&gb->gen) == g0) {
        if ((++polls & 63u) == 0 &&
            (ld_cg_u32(&gb->abort) != 0 || global_ns() - t0 > limit_ns)) {
          ok = 0;
          break;
        }
      }
    }
    // a block that gave up after arriving lets the barrier complete; the
    // others still leave here rather than at the next one
    if (ok && ld_cg_u32(&gb->abort) != 0) ok = 0;
    if (!ok) {
      atomicExch(&gb->abort, 1u);
      atomicOr(&ctl->error, ERR_GRID_WAIT);
    }
    gen = g0 + 1;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// The grid barrier's timeout path on a barrier that can never complete:
// launched with two blocks, block 1 leaves at once and block 0 waits for it
// until limit_ns runs out, then flags the control block as a persistent
// launch whose wait expired would.
__global__ void k_grid_selftest(GridBar* gb, StepCtl* ctl, unsigned long long limit_ns) {
  if (blockIdx.x != 0) return;
  unsigned int gen = 0;
  if (threadIdx.x == 0) gen = ld_cg_u32(&gb->gen);
  grid_sync(gb, gen, ctl, limit_ns);
}

constexpr int kPersistMaxLevels = 64;

struct PersistArgs {
  GraphPtrs g;
  T1Ptrs t1;
  TopPtrs top;
  const uint32_t* upg_off;  // edges from below into the top region
  const int2* upg;
  uint32_t has_upg;
  uint32_t steps;  // row-steps of this launch (even: the two rows alternate)
  uint16_t* rows[2];
  uint16_t* BV;
  uint16_t* FL;
  uint32_t* word;
  unsigned long long* best;
  StepCtl* ctl;
  SlotState* slots;
  const ReadDesc* queue;
  const unsigned char* reads;
  int32_t* res_score;
  uint32_t* res_vertex;
  unsigned long long* res_t0;
  unsigned long long* res_t1;
  CompletionRec* done_ring;
  uint32_t qmask;
  int special;
  int match_n;
  GridBar* bar;
  uint32_t fl;  // levels below the top region
  uint32_t lvl_off[kPersistMaxLevels + 1];
  unsigned long long up_mask;  // bit l: level l has upward pull lists
};

// Threads per block (one block per SM): 1024 (64 registers a thread) up to 4
// slots; 768 (80 registers) for 8 to 32 slots and 640 (96 registers) for 64
// and 128, whose row phases (k_row_dpx's and k_row_stream's bodies) need
// more registers beside the other phases.
template <int R>
struct PersistShape {
  static constexpr int threads = R >= 64 ? 640 : R >= 8 ? 768 : 1024;
  static constexpr int warps = threads / 32;
};

// Dynamic shared memory of a launch: the largest of the row phase's needs
// and the top region's.
template <int R>
__host__ __device__ constexpr size_t persist_row_smem() {
  return R == 1    ? (size_t)PersistShape<R>::warps * kT1VertMax * 12
         : R >= 64 ? (size_t)PersistShape<R>::warps * kStreamRing * R * 2
                   : 0;
}

template <int R>
__global__ void __launch_bounds__(PersistShape<R>::threads, 1) k_persist(PersistArgs a) {
  constexpr int TH = PersistShape<R>::threads, NW = PersistShape<R>::warps;
  extern __shared__ __align__(16) unsigned char psm[];
  __shared__ unsigned long long sm_best[R];
  unsigned int gen = 0;
  if (threadIdx.x == 0) gen = ld_cg_u32(&a.bar->gen);
  const uint32_t warp = threadIdx.x >> 5;
  const uint32_t gwarp = blockIdx.x * NW + warp, nwarps = gridDim.x * NW;
  const uint64_t gtid = (uint64_t)blockIdx.x * TH + threadIdx.x, nthreads = (uint64_t)gridDim.x * TH;
  const GraphPtrs& g = a.g;
  const uint32_t S = g.S;
  for (uint32_t step = 0; step < a.steps; ++step) {
    const uint16_t* D = a.rows[step & 1];
    uint16_t* T = a.rows[(step + 1) & 1];
    // the control block and slot words as the last advance left them
    const bool active = ld_cg_u32(&a.ctl->any_active) != 0;
    const bool ending_any = ld_cg_u32(&a.ctl->any_ending) != 0;
    if (active) {
      if (ending_any) {
        for (int r = threadIdx.x; r < R; r += TH) sm_best[r] = ~0ull;
        __syncthreads();
      }
      // ---- row phase
      if constexpr (R == 1) {
        int* s_G = reinterpret_cast<int*>(psm) + warp * kT1VertMax;
        int* s_X = reinterpret_cast<int*>(psm) + (NW + warp) * kT1VertMax;
        uint32_t* s_d = reinterpret_cast<uint32_t*>(psm) + (2 * NW + warp) * kT1VertMax;
        const uint32_t w = ld_cg_u32(a.word);
        unsigned long long mn = ~0ull;
        for (uint32_t tile = gwarp; tile < a.t1.ntiles; tile += nwarps)
          row_t1_tile<true, true>(g, a.t1, t1_head(g, a.t1, tile), D, T, a.BV, a.FL, w, s_G, s_X, s_d, mn);
        if (ending_any) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
          if ((threadIdx.x & 31) == 0 && mn != ~0ull) atomicMin(sm_best, mn);
        }
      } else if constexpr (R >= 64) {
        uint16_t* ring = reinterpret_cast<uint16_t*>(psm) + (size_t)warp * kStreamRing * R;
        for (uint32_t run = gwarp; run * 32 < S; run += nwarps)
          stream_run<R, true, true>(g, run, run_head(g, run), D, T, a.BV, a.FL, a.word, ring, sm_best,
                                    ending_any);
      } else {
        constexpr int G = Pairs<R>::G;
        for (uint64_t it = gtid; it < (uint64_t)S * G; it += nthreads)
          dpx_vertex<R, true, true>(g, (uint32_t)(it / G), (int)(it % G), D, T, a.BV, a.FL, a.word,
                                    sm_best, ending_any);
      }
      // the block's rows and boundary scores were written through the
      // generic proxy; the top phase refills this shared memory by bulk copies
      fence_async_shared();
      if (!grid_sync(a.bar, gen, a.ctl)) return;
      // ---- upward levels below the top region
      for (uint32_t l = 0; l < a.fl; ++l) {
        if (!((a.up_mask >> l) & 1ull)) continue;
        const uint32_t lo = a.lvl_off[l], hi = a.lvl_off[l + 1];
        if constexpr (R >= 8) {
          constexpr int G = R / 8;
          for (uint64_t it = gtid; it < (uint64_t)(hi - lo) * G; it += nthreads) {
            const uint32_t d = lo + (uint32_t)(it / G);
            pull_lv16_item<R, true>(a.BV, d, (int)(it % G), pull_head(d, g.up_head, g.up_in, g.n_up),
                                    g.up_in);
          }
        } else {
          constexpr int G = Lanes<R>::G;
          for (uint64_t it = gtid; it < (uint64_t)(hi - lo) * G; it += nthreads) {
            const uint32_t d = lo + (uint32_t)(it / G);
            pull_lv_item<R, uint16_t, true>(a.BV, d, (int)(it % G), pull_head(d, g.up_head, g.up_in, g.n_up),
                                            g.up_in);
          }
        }
        if (!grid_sync(a.bar, gen, a.ctl)) return;
      }
      // ---- top region: edges from below, then block r sweeps slot r
      if (a.top.K) {
        if (a.has_upg) {
          constexpr int G = Lanes<R>::G;
          for (uint64_t it = gtid; it < (uint64_t)a.top.K * G; it += nthreads)
            pull_item<R, uint16_t, true>(a.BV, a.top.K0 + (uint32_t)(it / G), (int)(it % G), a.upg_off,
                                         a.upg, a.top.K0);
          if (!grid_sync(a.bar, gen, a.ctl)) return;
        }
        bool ok = true;
        if (blockIdx.x < R && (ld_cg_u32(a.word + blockIdx.x) & SW_CLOSURE))
          ok = top_body<R, uint16_t>(a.BV, a.top, a.ctl, (int)blockIdx.x, psm);
        if (!ok && threadIdx.x == 0) atomicExch(&a.bar->abort, 1u);
        if (!grid_sync(a.bar, gen, a.ctl) || !ok) return;
      }
      // ---- downward levels (the highest one also finalises the top region)
      auto down = [&](uint32_t lo, uint32_t mid, uint32_t hi) {
        if constexpr (R >= 8) {
          constexpr int G = R / 8;
          for (uint64_t it = gtid; it < (uint64_t)(hi - lo) * G; it += nthreads) {
            const uint32_t d = lo + (uint32_t)(it / G);
            down16_item<R, true>(g, a.BV, a.FL, d, (int)(it % G), down_head(g, d, mid), a.word, sm_best,
                                 ending_any);
          }
        } else {
          constexpr int G = Lanes<R>::G;
          for (uint64_t it = gtid; it < (uint64_t)(hi - lo) * G; it += nthreads) {
            const uint32_t d = lo + (uint32_t)(it / G);
            down_item<R, false, uint16_t, true>(g, a.BV, T, a.FL, d, (int)(it % G), down_head(g, d, mid), a.word,
                                                sm_best, ending_any);
          }
        }
      };
      if (a.fl == 0) {
        down(0, 0, S);
      } else {
        for (int l = (int)a.fl - 1; l >= 0; --l) {
          const uint32_t lo = a.lvl_off[l], mid = a.lvl_off[l + 1];
          down(lo, mid, l == (int)a.fl - 1 ? S : mid);
          if (l > 0 && !grid_sync(a.bar, gen, a.ctl)) return;
        }
      }
      if (ending_any) flush_min<R>(sm_best, a.best);
      if (!grid_sync(a.bar, gen, a.ctl)) return;
    }
    // ---- advance: block 0 moves every slot to its next row
    if (blockIdx.x == 0)
      advance_body<R>(a.slots, a.queue, a.reads, a.best, a.res_score, a.res_vertex, a.res_t0, a.res_t1,
                      a.word, a.ctl, a.special, 0, a.qmask, a.done_ring, a.match_n);
    if (!grid_sync(a.bar, gen, a.ctl)) return;
  }
}

}  // namespace dev
}  // namespace chsga
