// sm_100a kernels of the ConSGA DP. One template parameter R = number of
// read slots advanced together; every score array is slot-interleaved
// (score of char c for slot r at c*R + r), so R = 1 is the plain
// one-read-per-launch path and R > 1 the batched path, with the graph and
// hierarchy loads of a row-step shared by all slots.
//
// Thread mapping: a group of G = min(R, 32) lanes owns one vertex; each lane
// owns V = R / G consecutive slots and moves them with one 4/8/16-byte access.
//
// A row-step of one read (src/align.hpp:430-463) is:
//   k_row         fused_deletion_substitution (align.hpp:245-277) and the
//                 within-vertex forward scan (align.hpp:362-373), one pass;
//                 writes the first/last scores of every vertex into BV
//   k_pull        one upward hierarchy level (align.hpp:296-314), pull form
//   k_top         every level of the top region, up and down, in shared memory
//   k_down        one downward level (align.hpp:317-343) plus the final
//                 within-vertex propagation (align.hpp:381-396) of the vertices
//                 it finalises, which only needs the vertex's own first score
//   k_advance     moves every slot to its next row, harvests finished reads
//                 and refills slots from the device read queue
// Row 0 of a read is only the initial match/substitution row
// (align.hpp:205-210, 421); it gets no hierarchy closure.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace chsga {
namespace dev {

struct GraphPtrs {
  uint32_t N, S;
  int special;
  const uint32_t* lab2;
  const uint32_t* lab_sp;
  const uint32_t* sv_off;
  const uint32_t* sv_dev;
  const uint32_t* vin_off;
  const uint32_t* vin_src;
  const uint32_t* vin_srcv;
  const uint32_t* dv_first;
  const uint32_t* dv_len;
  const uint32_t* up_off;
  const int2* up_in;
  const uint32_t* dn_off;
  const int2* dn_in;
  const uint32_t* istr_off;
  const uint32_t* istr_src;
};

// Per-slot word for the current row-step, written by k_advance.
constexpr uint32_t SW_CODE = 0xFFu;         // read base code: 0..3 A,C,G,T, 4 special, 5 none
constexpr uint32_t SW_INIT = 1u << 8;       // row 0: match/substitution only
constexpr uint32_t SW_CLOSURE = 1u << 9;    // row >= 1: hierarchy closure applies
constexpr uint32_t SW_ENDING = 1u << 10;    // last row of the read: reduce its minimum
constexpr uint32_t SW_ACTIVE = 1u << 11;

struct SlotState {
  unsigned long long off;  // first base of the read in the device read buffer
  uint32_t len;
  uint32_t row;            // row computed by the current row-step
  int32_t id;              // read index, -1 = idle
  uint32_t pad;
};

struct ReadDesc {
  unsigned long long off;
  uint32_t len;
  int32_t id;
};

struct StepCtl {        // device-resident control block
  uint32_t any_active;  // some slot has a row to compute
  uint32_t any_ending;  // some slot is on its last row
  uint32_t q_head;      // next queue entry to admit
  uint32_t q_count;     // queue entries published by the host
  uint32_t done;        // reads finished
  uint32_t steps;       // row-steps with work
  uint32_t pad[2];
};

template <int R>
struct Lanes {
  static constexpr int G = R < 32 ? R : 32;
  static constexpr int V = R < 32 ? 1 : R / 32;
};

template <int V>
struct IV {
  int v[V];
};

template <int V>
__device__ __forceinline__ IV<V> ld_nc(const int* p) {
  IV<V> o;
  if constexpr (V == 1) {
    o.v[0] = __ldg(p);
  } else if constexpr (V == 2) {
    int2 t = __ldg(reinterpret_cast<const int2*>(p));
    o.v[0] = t.x;
    o.v[1] = t.y;
  } else {
    int4 t = __ldg(reinterpret_cast<const int4*>(p));
    o.v[0] = t.x;
    o.v[1] = t.y;
    o.v[2] = t.z;
    o.v[3] = t.w;
  }
  return o;
}

template <int V>
__device__ __forceinline__ IV<V> ld(const int* p) {
  IV<V> o;
  if constexpr (V == 1) {
    o.v[0] = *p;
  } else if constexpr (V == 2) {
    int2 t = *reinterpret_cast<const int2*>(p);
    o.v[0] = t.x;
    o.v[1] = t.y;
  } else {
    int4 t = *reinterpret_cast<const int4*>(p);
    o.v[0] = t.x;
    o.v[1] = t.y;
    o.v[2] = t.z;
    o.v[3] = t.w;
  }
  return o;
}

template <int V>
__device__ __forceinline__ void st(int* p, const IV<V>& x) {
  if constexpr (V == 1) {
    *p = x.v[0];
  } else if constexpr (V == 2) {
    *reinterpret_cast<int2*>(p) = make_int2(x.v[0], x.v[1]);
  } else {
    *reinterpret_cast<int4*>(p) = make_int4(x.v[0], x.v[1], x.v[2], x.v[3]);
  }
}

// Label key of char c: 0..3 for A,C,G,T, 4 for the special byte.
__device__ __forceinline__ uint32_t label_key(const GraphPtrs& g, uint32_t c) {
  const uint32_t code = (__ldg(g.lab2 + (c >> 4)) >> ((c & 15u) * 2u)) & 3u;
  const uint32_t sp = (__ldg(g.lab_sp + (c >> 5)) >> (c & 31u)) & 1u;
  return sp ? 4u : code;
}

// Read base -> code comparable with label_key (match_sub, csr_align.hpp:41-50:
// a base matches a label only if the bytes are equal).
__device__ __forceinline__ uint32_t base_code(int b, int special) {
  switch (b) {
    case 'A': return 0u;
    case 'C': return 1u;
    case 'G': return 2u;
    case 'T': return 3u;
    default: return b == special ? 4u : 5u;
  }
}

__device__ __forceinline__ unsigned long long pack_min(int score, uint32_t c) {
  return ((unsigned long long)(uint32_t)score << 32) | c;
}

// Block-wide minimum per slot, one global atomic per slot per block.
template <int R>
__device__ __forceinline__ void flush_min(unsigned long long* sm_best, unsigned long long* best) {
  __syncthreads();
  for (int r = threadIdx.x; r < R; r += blockDim.x)
    if (sm_best[r] != ~0ull) atomicMin(best + r, sm_best[r]);
}

// ---------------------------------------------------------------------------
// k_row: one pass over the string vertices in char order. For vertex s and
// each slot: the first char takes min(D[f]+1, min over in-edges D[u]+delta),
// every later char c takes min(D[c]+1, D[c-1]+delta, T[c-1]+1): the chain
// in-edge c-1 -> c plus the within-vertex forward scan. Row 0 takes delta.
// ---------------------------------------------------------------------------
template <int R>
__global__ void __launch_bounds__(256) k_row(GraphPtrs g, const int* __restrict__ D,
                                             int* __restrict__ T, int* __restrict__ BV,
                                             const uint32_t* __restrict__ slot_word,
                                             unsigned long long* __restrict__ best,
                                             const StepCtl* __restrict__ ctl) {
  constexpr int G = Lanes<R>::G, V = Lanes<R>::V;
  __shared__ unsigned long long sm_best[R];
  const bool ending_any = ctl->any_ending != 0;
  if (!ctl->any_active) return;
  if (ending_any) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) sm_best[r] = ~0ull;
    __syncthreads();
  }
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t s = (uint32_t)(gt / G);
  const int lane = (int)(gt % G);
  if (s < g.S) {
    uint32_t code[V];
    bool init[V], ending[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const uint32_t w = __ldg(slot_word + lane * V + v);
      code[v] = w & SW_CODE;
      init[v] = (w & SW_INIT) != 0;
      ending[v] = (w & SW_ENDING) != 0;
    }
    const uint32_t f = __ldg(g.sv_off + s), e = __ldg(g.sv_off + s + 1);
    const uint32_t d = __ldg(g.sv_dev + s);
    const size_t so = (size_t)lane * V;
    int bmin[V];
    uint32_t barg[V];
    // first char
    IV<V> dprev = ld_nc<V>(D + (size_t)f * R + so);
    IV<V> t;
    {
      const uint32_t key = label_key(g, f);
      int delta[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        delta[v] = key == code[v] ? 0 : 1;
        t.v[v] = dprev.v[v] + 1;
      }
      const uint32_t k0 = __ldg(g.vin_off + s), k1 = __ldg(g.vin_off + s + 1);
      for (uint32_t k = k0; k < k1; ++k) {
        const uint32_t u = __ldg(g.vin_src + k);
        const IV<V> du = ld_nc<V>(D + (size_t)u * R + so);
#pragma unroll
        for (int v = 0; v < V; ++v) t.v[v] = min(t.v[v], du.v[v] + delta[v]);
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        if (init[v]) t.v[v] = delta[v];
        bmin[v] = t.v[v];
        barg[v] = f;
      }
    }
    st<V>(T + (size_t)f * R + so, t);
    st<V>(BV + (size_t)(2 * d) * R + so, t);
    for (uint32_t c = f + 1; c < e; ++c) {
      const uint32_t key = label_key(g, c);
      const IV<V> dc = ld_nc<V>(D + (size_t)c * R + so);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int delta = key == code[v] ? 0 : 1;
        int x = min(dc.v[v] + 1, dprev.v[v] + delta);
        x = min(x, t.v[v] + 1);
        if (init[v]) x = delta;
        t.v[v] = x;
        if (x < bmin[v]) {
          bmin[v] = x;
          barg[v] = c;
        }
      }
      dprev = dc;
      st<V>(T + (size_t)c * R + so, t);
    }
    if (e - f > 1) st<V>(BV + (size_t)(2 * d + 1) * R + so, t);
    if (ending_any) {
#pragma unroll
      for (int v = 0; v < V; ++v)
        if (ending[v]) atomicMin(sm_best + lane * V + v, pack_min(bmin[v], barg[v]));
    }
  }
  if (ending_any) flush_min<R>(sm_best, best);
}

// ---------------------------------------------------------------------------
// k_pull: hierarchy positions [lo, hi): BV[2d] = min(BV[2d], BV[src] + w)
// over the list off[d-base]..off[d-base+1]. Every source lies on another
// level, finished before this launch, so the gathers use the read-only path.
// ---------------------------------------------------------------------------
template <int R>
__global__ void __launch_bounds__(256) k_pull(int* __restrict__ BV, uint32_t lo, uint32_t hi,
                                              const uint32_t* __restrict__ off,
                                              const int2* __restrict__ edges, uint32_t base,
                                              const StepCtl* __restrict__ ctl) {
  constexpr int G = Lanes<R>::G, V = Lanes<R>::V;
  if (!ctl->any_active) return;
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t d = lo + (uint32_t)(gt / G);
  const int lane = (int)(gt % G);
  if (d >= hi) return;
  const size_t so = (size_t)lane * V;
  const uint32_t k0 = __ldg(off + (d - base)), k1 = __ldg(off + (d - base) + 1);
  if (k0 == k1) return;
  int* p = BV + (size_t)(2 * d) * R + so;
  IV<V> f = ld<V>(p);
  bool changed = false;
  for (uint32_t k = k0; k < k1; ++k) {
    const int2 ew = __ldg(edges + k);
    const IV<V> x = ld_nc<V>(BV + (size_t)ew.x * R + so);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int c = x.v[v] + ew.y;
      if (c < f.v[v]) {
        f.v[v] = c;
        changed = true;
      }
    }
  }
  if (changed) st<V>(p, f);
}

// ---------------------------------------------------------------------------
// k_down: positions [lo, hi). Those below `mid` first pull their downward
// in-edges (sources on higher levels, final); every position then finalises
// its vertex's chars: if the first score fell below the row value, write it
// and propagate first + (p - first) forward while it improves
// (align.hpp:381-396). Slots without closure (row 0, idle) are untouched.
// ---------------------------------------------------------------------------
template <int R>
__global__ void __launch_bounds__(256) k_down(GraphPtrs g, int* __restrict__ BV, int* __restrict__ T,
                                              uint32_t lo, uint32_t mid, uint32_t hi,
                                              const uint32_t* __restrict__ slot_word,
                                              unsigned long long* __restrict__ best,
                                              const StepCtl* __restrict__ ctl) {
  constexpr int G = Lanes<R>::G, V = Lanes<R>::V;
  __shared__ unsigned long long sm_best[R];
  const bool ending_any = ctl->any_ending != 0;
  if (!ctl->any_active) return;
  if (ending_any) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) sm_best[r] = ~0ull;
    __syncthreads();
  }
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t d = lo + (uint32_t)(gt / G);
  const int lane = (int)(gt % G);
  if (d < hi) {
    const size_t so = (size_t)lane * V;
    int* p = BV + (size_t)(2 * d) * R + so;
    IV<V> f = ld<V>(p);
    if (d < mid) {
      const uint32_t k0 = __ldg(g.dn_off + d), k1 = __ldg(g.dn_off + d + 1);
      bool changed = false;
      for (uint32_t k = k0; k < k1; ++k) {
        const int2 ew = __ldg(g.dn_in + k);
        const IV<V> x = ld_nc<V>(BV + (size_t)ew.x * R + so);
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const int c = x.v[v] + ew.y;
          if (c < f.v[v]) {
            f.v[v] = c;
            changed = true;
          }
        }
      }
      if (changed) st<V>(p, f);
    }
    const uint32_t first = __ldg(g.dv_first + d), len = __ldg(g.dv_len + d);
    const IV<V> t0 = ld<V>(T + (size_t)first * R + so);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if (f.v[v] >= t0.v[v]) continue;
      const uint32_t w = __ldg(slot_word + so + v);
      if (!(w & SW_CLOSURE)) continue;
      const bool ending = (w & SW_ENDING) != 0;
      const int fv = f.v[v];
      T[(size_t)first * R + so + v] = fv;
      if (ending) atomicMin(sm_best + so + v, pack_min(fv, first));
      for (uint32_t q = 1; q < len; ++q) {
        int* tp = T + (size_t)(first + q) * R + so + v;
        const int cand = fv + (int)q;
        if (cand < *tp) {
          *tp = cand;
          if (ending) atomicMin(sm_best + so + v, pack_min(cand, first + q));
        } else {
          break;
        }
      }
    }
  }
  if (ending_any) flush_min<R>(sm_best, best);
}

// ---------------------------------------------------------------------------
// k_top: hierarchy positions [K0, S), one CTA per slot. Stages first/last
// scores in shared memory, then runs the upward levels low -> high and the
// downward levels high -> low with a block barrier between levels. Edges
// from below the region were applied by k_pull before this launch.
// ---------------------------------------------------------------------------
struct TopPtrs {
  uint32_t K0, K, nlev;
  const uint32_t* lvl_off;  // nlev+1, local
  const uint32_t* upl_off;
  const int2* upl;
  const uint32_t* dn_off;
  const int2* dn;
  const uint32_t* dv_len;   // global, by hierarchy position
};

template <int R>
__global__ void __launch_bounds__(1024) k_top(int* __restrict__ BV, TopPtrs t,
                                              const uint32_t* __restrict__ slot_word,
                                              const StepCtl* __restrict__ ctl) {
  extern __shared__ int sm[];  // 2*K ints: [2j] first, [2j+1] last
  if (!ctl->any_active) return;
  const int r = blockIdx.x;
  if (!(slot_word[r] & SW_CLOSURE)) return;
  for (uint32_t j = threadIdx.x; j < t.K; j += blockDim.x) {
    const size_t d = t.K0 + j;
    sm[2 * j] = BV[(2 * d) * R + r];
    if (__ldg(t.dv_len + d) > 1) sm[2 * j + 1] = BV[(2 * d + 1) * R + r];
  }
  __syncthreads();
  for (uint32_t l = 0; l < t.nlev; ++l) {
    const uint32_t lo = t.lvl_off[l], hi = t.lvl_off[l + 1];
    for (uint32_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
      int f = sm[2 * j];
      for (uint32_t k = t.upl_off[j]; k < t.upl_off[j + 1]; ++k) {
        const int2 ew = t.upl[k];
        f = min(f, sm[ew.x] + ew.y);
      }
      sm[2 * j] = f;
    }
    __syncthreads();
  }
  for (uint32_t l = t.nlev; l-- > 0;) {
    const uint32_t lo = t.lvl_off[l], hi = t.lvl_off[l + 1];
    for (uint32_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
      int f = sm[2 * j];
      for (uint32_t k = t.dn_off[j]; k < t.dn_off[j + 1]; ++k) {
        const int2 ew = t.dn[k];
        f = min(f, sm[ew.x] + ew.y);
      }
      sm[2 * j] = f;
    }
    __syncthreads();
  }
  for (uint32_t j = threadIdx.x; j < t.K; j += blockDim.x) BV[(2 * (size_t)(t.K0 + j)) * R + r] = sm[2 * j];
}

// ---------------------------------------------------------------------------
// k_advance: one block. Slots that computed their last row hand in their
// minimum (score and smallest char index reaching it); idle slots admit the
// next queued reads in order; every slot gets its word for the next step.
// prime != 0 only recomputes the words (used after the host sets slots).
// ---------------------------------------------------------------------------
template <int R>
__global__ void __launch_bounds__(128) k_advance(SlotState* __restrict__ slots,
                                                 const ReadDesc* __restrict__ queue,
                                                 const unsigned char* __restrict__ reads,
                                                 unsigned long long* __restrict__ best,
                                                 int32_t* __restrict__ res_score,
                                                 uint32_t* __restrict__ res_vertex,
                                                 uint32_t* __restrict__ slot_word,
                                                 StepCtl* __restrict__ ctl, int special,
                                                 int prime) {
  __shared__ uint32_t s_need[128];
  __shared__ uint32_t s_base, s_take, s_active, s_ending;
  const int r = threadIdx.x;
  SlotState st{};
  bool need = false;
  if (r == 0) {
    s_active = 0;
    s_ending = 0;
  }
  if (r < R) {
    st = slots[r];
    if (!prime && st.id >= 0) {
      if (st.row + 1 >= st.len) {
        const unsigned long long b = best[r];
        res_score[st.id] = (int32_t)(b >> 32);
        res_vertex[st.id] = (uint32_t)(b & 0xffffffffu);
        atomicAdd(&ctl->done, 1u);
        st.id = -1;
      } else {
        st.row += 1;
      }
    }
    need = !prime && st.id < 0;
  }
  s_need[r] = need ? 1u : 0u;
  __syncthreads();
  if (r == 0) {
    uint32_t total = 0;
    for (int i = 0; i < R && i < 128; ++i) {
      const uint32_t n = s_need[i];
      s_need[i] = total;
      total += n;
    }
    const uint32_t avail = ctl->q_count - ctl->q_head;
    s_take = total < avail ? total : avail;
    s_base = ctl->q_head;
    ctl->q_head += s_take;
  }
  __syncthreads();
  if (r < R) {
    if (need && s_need[r] < s_take) {
      const ReadDesc q = queue[s_base + s_need[r]];
      st.off = q.off;
      st.len = q.len;
      st.row = 0;
      st.id = q.id;
      best[r] = ~0ull;
    }
    uint32_t w = 0;
    if (st.id >= 0) {
      w = base_code(reads[st.off + st.row], special) | SW_ACTIVE;
      w |= st.row == 0 ? SW_INIT : SW_CLOSURE;
      if (st.row + 1 == st.len) w |= SW_ENDING;
      atomicOr(&s_active, 1u);
      if (w & SW_ENDING) atomicOr(&s_ending, 1u);
    }
    slots[r] = st;
    slot_word[r] = w;
  }
  __syncthreads();
  if (r == 0) {
    ctl->any_active = s_active;
    ctl->any_ending = s_ending;
    if (s_active) ctl->steps += 1;
  }
}

// ---------------------------------------------------------------------------
// k_walk: single-thread traceback by score equality over rows
// [row_lo, row_hi] of a score matrix (row i at M + (i - row_lo) * N),
// walk_traceback_from_scores (src/traceback.hpp:483-586). Tie order:
// INSERT from the previous char of the same vertex, INSERT from the last
// char of the first string in-neighbour (in-CSR order) that fits, DELETE,
// MATCHSUB from the first char in-neighbour (in-CSR order) that fits.
// Stops on reaching row_lo; ops are written in reverse order.
// ---------------------------------------------------------------------------
struct WalkOut {
  uint32_t vertex;   // vertex reached at row_lo
  uint32_t nops;
  int32_t status;    // 0 ok, 7 no predecessor, 8 op budget exhausted
  int32_t fail_row;
};

struct WalkOp {
  long long row;
  uint32_t vertex;
  uint32_t op;
};

__global__ void k_walk(GraphPtrs g, const int* __restrict__ M, long long row_lo, long long row_hi,
                       uint32_t start, const unsigned char* __restrict__ read, WalkOp* __restrict__ ops,
                       uint32_t max_ops, WalkOut* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const size_t N = g.N;
  uint32_t cur = start;
  long long row = row_hi;
  // string vertex of `cur`: binary search over sv_off
  uint32_t lo = 0, hi = g.S;
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) / 2;
    if (g.sv_off[m] <= cur) lo = m; else hi = m;
  }
  uint32_t sv = lo;
  uint32_t n = 0;
  out->status = 0;
  while (row > row_lo) {
    if (n >= max_ops) {
      out->status = 8;
      out->fail_row = (int)row;
      break;
    }
    const int* Rw = M + (size_t)(row - row_lo) * N;
    const int* Pw = M + (size_t)(row - 1 - row_lo) * N;
    const int s = Rw[cur];
    const uint32_t first = g.sv_off[sv];
    uint32_t op = 255, src = cur, src_sv = sv;
    if (cur > first && Rw[cur - 1] + 1 == s) {
      op = 2;
      src = cur - 1;
    }
    if (op == 255 && cur == first) {
      for (uint32_t k = g.istr_off[sv]; k < g.istr_off[sv + 1]; ++k) {
        const uint32_t u = g.istr_src[k];
        const uint32_t ul = g.sv_off[u + 1] - 1;
        if (Rw[ul] + 1 == s) {
          op = 2;
          src = ul;
          src_sv = u;
          break;
        }
      }
    }
    if (op == 255 && Pw[cur] + 1 == s) op = 0;
    if (op == 255) {
      const uint32_t key = label_key(g, cur);
      const int delta = key == base_code(read[row], g.special) ? 0 : 1;
      if (cur > first) {
        if (Pw[cur - 1] + delta == s) {
          op = 1;
          src = cur - 1;
        }
      } else {
        for (uint32_t k = g.vin_off[sv]; k < g.vin_off[sv + 1]; ++k) {
          const uint32_t u = g.vin_src[k];
          if (Pw[u] + delta == s) {
            op = 1;
            src = u;
            src_sv = g.vin_srcv[k];
            break;
          }
        }
      }
    }
    if (op == 255) {
      out->status = 7;
      out->fail_row = (int)row;
      break;
    }
    ops[n++] = WalkOp{row, cur, op};
    cur = src;
    sv = src_sv;
    if (op != 2) --row;
  }
  out->vertex = cur;
  out->nops = n;
}

}  // namespace dev
}  // namespace chsga
