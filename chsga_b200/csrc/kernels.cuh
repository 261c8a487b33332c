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
//   k_down        one downward level (align.hpp:317-343). The final
//                 within-vertex propagation (align.hpp:381-396) only ever
//                 lowers char c of vertex s to F[s] + (c - first(s)), F[s] the
//                 swept first score, so it is either written into the row here
//                 (FIXUP: rows that are kept, i.e. traceback) or applied when
//                 the next row-step reads the row (score-only: k_row<DEFER>)
//   k_advance     moves every slot to its next row, harvests finished reads
//                 and refills slots from the device read queue
// Row 0 of a read is only the initial match/substitution row
// (align.hpp:205-210, 421); it gets no hierarchy closure.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "device_graph.hpp"  // tile limits shared with the host-side tile builder

namespace chsga {
namespace dev {

struct GraphPtrs {
  uint32_t N, S;
  int special;
  const uint32_t* lab2;
  const uint32_t* lab_sp;
  const uint32_t* lab4;  // 4-bit label key per char, 8 per word
  const uint32_t* sv_off;
  const uint32_t* sv_dev;
  const uint32_t* vin_off;
  const uint32_t* vin_src;
  const uint32_t* vin_srcv;  // string vertex of each first-char in-edge source (the
                             // source is that vertex's last char)
  const uint32_t* dv_first;
  const uint32_t* dv_len;
  const uint32_t* dv_s;  // original id of hierarchy vertex d
  const uint32_t* up_off;
  const int2* up_in;
  const uint32_t* dn_off;
  const int2* dn_in;
  const uint32_t* istr_off;
  const uint32_t* istr_src;
  // per hierarchy position: {list begin, list end, first source, first
  // weight} of the down pull list; two uint4 {begin, end, src0, w0},
  // {src1, w1, 0, 0} of the up pull list; and {first char, length, string
  // vertex, 0} -- 16-byte loads instead of a chain of word loads
  const uint4* dn_head;
  const uint4* up_head;
  const uint4* fin;
  uint32_t n_vin, n_up, n_dn;  // entries of vin_srcv, up_in, dn_in (index checks)
};

// ---------------------------------------------------------------------------
// Index checks of the CHSGA_CHECKED build (make CHECKED=1): every index a
// kernel reads from a graph array before using it as an address is checked
// against the size of what it indexes. An index out of range records the
// check site and the index (the first failure wins) and is replaced by 0, so
// the access stays inside the array; the host turns the record into
// CHSGA_ERR_INTERNAL after the call. No trap, no fault. Without
// CHSGA_CHECKED the checks compile to the index itself.
// ---------------------------------------------------------------------------
#ifdef CHSGA_CHECKED
static __device__ unsigned int g_chk_fail;
static __device__ unsigned long long g_chk_first;  // site << 40 | index
__device__ __forceinline__ void chk_fail(uint64_t i, uint32_t site) {
  if (atomicCAS(&g_chk_fail, 0u, 1u) == 0u)
    atomicExch(&g_chk_first, ((unsigned long long)site << 40) | (i & 0xFFFFFFFFFFull));
}
__device__ __forceinline__ uint32_t chk_index(uint64_t i, uint64_t n, uint32_t site) {
  if (i < n) return (uint32_t)i;
  chk_fail(i, site);
  return 0;
}
// an index below n, else 0
#define CHSGA_CHK(i, n, site) (::chsga::dev::chk_index((uint64_t)(i), (uint64_t)(n), (site)))
// lo <= hi <= n, else the empty range 0..0
#define CHSGA_CHK_RANGE(lo, hi, n, site)                                                  \
  do {                                                                                    \
    if (!((uint64_t)(lo) <= (uint64_t)(hi) && (uint64_t)(hi) <= (uint64_t)(n))) {         \
      ::chsga::dev::chk_fail((uint64_t)(hi), (site));                                     \
      (lo) = 0;                                                                           \
      (hi) = 0;                                                                           \
    }                                                                                     \
  } while (0)
// the chars f .. e-1 of one vertex: f < e <= n, else the one char 0
#define CHSGA_CHK_CHARS(f, e, n, site)                                                    \
  do {                                                                                    \
    if (!((uint64_t)(f) < (uint64_t)(e) && (uint64_t)(e) <= (uint64_t)(n))) {            \
      ::chsga::dev::chk_fail((uint64_t)(e), (site));                                      \
      (f) = 0;                                                                            \
      (e) = 1;                                                                            \
    }                                                                                     \
  } while (0)
#else
#define CHSGA_CHK(i, n, site) (i)
#define CHSGA_CHK_RANGE(lo, hi, n, site) \
  do {                                   \
  } while (0)
#define CHSGA_CHK_CHARS(f, e, n, site) \
  do {                                 \
  } while (0)
#endif

// Per-slot word for the current row-step, written by k_advance.
constexpr uint32_t SW_CODE = 0xFFu;         // read base code: 0..3 A,C,G,T, 4 special, 5 none
constexpr uint32_t SW_INIT = 1u << 8;       // row 0: match/substitution only
constexpr uint32_t SW_CLOSURE = 1u << 9;    // row >= 1: hierarchy closure applies
constexpr uint32_t SW_ENDING = 1u << 10;    // last row of the read: reduce its minimum
constexpr uint32_t SW_ACTIVE = 1u << 11;
constexpr uint32_t SW_FIX = 1u << 12;      // row >= 2: previous row had a closure to apply
constexpr uint32_t SW_MASK_SHIFT = 16;     // bits 16..20: mismatch mask over label keys
constexpr uint32_t SW_MASK = 0x1Fu;

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

// One finished read, appended by k_advance to a completion ring (serving).
struct CompletionRec {
  int32_t id;
  int32_t score;
  uint32_t vertex;
  uint32_t pad;
  unsigned long long t0, t1;  // admission / completion, device global timer ns
};

struct StepCtl {        // device-resident control block
  uint32_t any_active;  // some slot has a row to compute
  uint32_t any_ending;  // some slot is on its last row
  uint32_t q_head;      // next queue entry to admit
  uint32_t q_count;     // queue entries published by the host
  uint32_t done;        // reads finished
  uint32_t steps;       // row-steps with work
  uint32_t error;       // nonzero: a bounded device-side wait gave up
  uint32_t run_next;    // k_row_delta: runs handed out after each warp's first (k_advance resets it)
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

// 16-bit row storage: the same accessors over uint16_t (values widened to
// int in registers). Every DP value of row i is at most i + 1, so rows of
// reads shorter than 65535 fit exactly.
template <int V>
__device__ __forceinline__ IV<V> ld_nc(const uint16_t* p) {
  IV<V> o;
  if constexpr (V == 1) {
    o.v[0] = __ldg(reinterpret_cast<const unsigned short*>(p));
  } else if constexpr (V == 2) {
    const uint32_t t = __ldg(reinterpret_cast<const unsigned int*>(p));
    o.v[0] = (int)(t & 0xFFFFu);
    o.v[1] = (int)(t >> 16);
  } else {
    const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
    o.v[0] = (int)(t.x & 0xFFFFu);
    o.v[1] = (int)(t.x >> 16);
    o.v[2] = (int)(t.y & 0xFFFFu);
    o.v[3] = (int)(t.y >> 16);
  }
  return o;
}

template <int V>
__device__ __forceinline__ IV<V> ld(const uint16_t* p) {
  IV<V> o;
  if constexpr (V == 1) {
    o.v[0] = *p;
  } else if constexpr (V == 2) {
    const uint32_t t = *reinterpret_cast<const uint32_t*>(p);
    o.v[0] = (int)(t & 0xFFFFu);
    o.v[1] = (int)(t >> 16);
  } else {
    const uint2 t = *reinterpret_cast<const uint2*>(p);
    o.v[0] = (int)(t.x & 0xFFFFu);
    o.v[1] = (int)(t.x >> 16);
    o.v[2] = (int)(t.y & 0xFFFFu);
    o.v[3] = (int)(t.y >> 16);
  }
  return o;
}

template <int V>
__device__ __forceinline__ void st(uint16_t* p, const IV<V>& x) {
  if constexpr (V == 1) {
    *p = (uint16_t)x.v[0];
  } else if constexpr (V == 2) {
    *reinterpret_cast<uint32_t*>(p) = (uint32_t)x.v[0] | ((uint32_t)x.v[1] << 16);
  } else {
    *reinterpret_cast<uint2*>(p) = make_uint2((uint32_t)x.v[0] | ((uint32_t)x.v[1] << 16),
                                              (uint32_t)x.v[2] | ((uint32_t)x.v[3] << 16));
  }
}

// Source loads of the sweep and row kernels: the read-only path (__ldg) when
// the data was written by an earlier launch, plain loads inside the
// persistent row-step kernel (COH), where other blocks of the same launch
// wrote it before the last grid barrier.
template <int V, bool COH, typename ST>
__device__ __forceinline__ IV<V> ld_src(const ST* p) {
  if constexpr (COH) return ld<V>(p);
  else return ld_nc<V>(p);
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

// Bit k set: a label of key k (0..3 A,C,G,T, 4 the special byte) scores a
// substitution against read byte b, i.e. match_sub (csr_align.hpp:41-50):
// mismatchN (ALPHABET_SIZE 5) matches equal bytes only; matchN
// (ALPHABET_SIZE 4, match_n != 0) also matches an 'N' on either side.
__device__ __forceinline__ uint32_t mismatch_mask(int b, int special, int match_n) {
  if (match_n && b == 'N') return 0u;
  uint32_t m = SW_MASK & ~(1u << base_code(b, special));
  if (match_n && special == 'N') m &= ~(1u << 4);
  return m;
}

// Programmatic dependent launch: a row-step kernel launched while the kernel
// before it on the stream drains waits here until that kernel has finished
// and its writes are visible (a no-op for a kernel launched the usual way).
// Once every block of this kernel has passed the wait, the next kernel of the
// chain may launch into the SMs this one frees and load its graph constants
// before its own wait. Every block of a chain kernel calls this before it
// reads anything a kernel writes, and before it exits, so a kernel completes
// only after the one before it.
__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
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
// Bulk asynchronous copies (TMA engine, non-tensor form) into shared memory,
// completing on an mbarrier. Source and destination 16-byte aligned, size a
// multiple of 16. Every wait is bounded: on expiry the kernel records an
// error code in StepCtl::error and stops.
// ---------------------------------------------------------------------------
constexpr uint32_t kWaitLimit = 1u << 22;  // try_wait polls (each may suspend briefly)
constexpr uint32_t ERR_TOP_WAIT = 1;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_inval(unsigned long long* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of transaction, then the copy.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          unsigned long long* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Waits for phase `parity` of the barrier; false if the poll budget ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity,
                                          uint32_t limit = kWaitLimit) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// k_row: one pass over the string vertices in char order. For vertex s and
// each slot: the first char takes min(D[f]+1, min over in-edges D[u]+delta),
// every later char c takes min(D[c]+1, D[c-1]+delta, T[c-1]+1): the chain
// in-edge c-1 -> c plus the within-vertex forward scan. Row 0 takes delta.
//
// The previous row's final first and last scores of every string vertex are
// kept in char order, FL[(2s + j) * R + r] (j = 0 first, 1 last; written by
// k_down). A first char's in-edge sources are last chars of other vertices,
// so their final values are read from FL. With DEFER, D holds the previous
// row before its within-vertex propagation, and every chain value is read as
// min(D[c], FL_first(s) + c - first(s)).
// ---------------------------------------------------------------------------
template <int R, bool DEFER, typename ST>
__global__ void __launch_bounds__(256, 3) k_row_direct(GraphPtrs g, const ST* __restrict__ D,
                                                       ST* __restrict__ T, ST* __restrict__ BV,
                                                       const ST* __restrict__ FL,
                                                       const uint32_t* __restrict__ slot_word,
                                                       unsigned long long* __restrict__ best,
                                                       const StepCtl* __restrict__ ctl) {
  pdl_wait();
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
    bool init[V], ending[V], fix[V];
    bool any_fix = false;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const uint32_t w = __ldg(slot_word + lane * V + v);
      code[v] = (w >> SW_MASK_SHIFT) & SW_MASK;  // mismatch mask
      init[v] = (w & SW_INIT) != 0;
      ending[v] = (w & SW_ENDING) != 0;
      fix[v] = DEFER && (w & SW_FIX) != 0;
      any_fix |= fix[v];
    }
    uint32_t f = __ldg(g.sv_off + s), e = __ldg(g.sv_off + s + 1);
    CHSGA_CHK_CHARS(f, e, g.N, 1);
    const uint32_t d = CHSGA_CHK(__ldg(g.sv_dev + s), g.S, 3);
    const size_t so = (size_t)lane * V;
    constexpr int kBig = 0x3fffffff;
    IV<V> F;
#pragma unroll
    for (int v = 0; v < V; ++v) F.v[v] = kBig;
    if (DEFER && any_fix) {
      const IV<V> x = ld_nc<V>(FL + (size_t)(2 * s) * R + so);
#pragma unroll
      for (int v = 0; v < V; ++v)
        if (fix[v]) F.v[v] = x.v[v];
    }
    int bmin[V];
    uint32_t barg[V];
    IV<V> dprev = ld_nc<V>(D + (size_t)f * R + so);
    IV<V> t;
    {
      const uint32_t key = label_key(g, f);
      int delta[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        if (DEFER) dprev.v[v] = min(dprev.v[v], F.v[v]);
        delta[v] = (int)((code[v] >> key) & 1u);
        t.v[v] = dprev.v[v] + 1;
      }
      uint32_t k0 = __ldg(g.vin_off + s), k1 = __ldg(g.vin_off + s + 1);
      CHSGA_CHK_RANGE(k0, k1, g.n_vin, 4);
      for (uint32_t k = k0; k < k1; ++k) {
        const uint32_t su = CHSGA_CHK(__ldg(g.vin_srcv + k), g.S, 5);
        const IV<V> du = ld_nc<V>(FL + (size_t)(2 * su + 1) * R + so);
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
    for (uint32_t c0 = f + 1; c0 < e; c0 += 4) {
      const uint32_t n = min(4u, e - c0);
      IV<V> dq[4];
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k)
        if (k < n) dq[k] = ld_nc<V>(D + (size_t)(c0 + k) * R + so);
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k) {
        if (k < n) {
          const uint32_t c = c0 + k;
          const uint32_t key = label_key(g, c);
#pragma unroll
          for (int v = 0; v < V; ++v) {
            if (DEFER) dq[k].v[v] = min(dq[k].v[v], F.v[v] + (int)(c - f));
            const int delta = (int)((code[v] >> key) & 1u);
            int x = min(dq[k].v[v] + 1, dprev.v[v] + delta);
            x = min(x, t.v[v] + 1);
            if (init[v]) x = delta;
            t.v[v] = x;
            if (x < bmin[v]) {
              bmin[v] = x;
              barg[v] = c;
            }
          }
          dprev = dq[k];
          st<V>(T + (size_t)c * R + so, t);
        }
      }
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
// k_row_dpx: k_row_direct for 16-bit rows on the DPX units. Two slots share
// one 32-bit register (one 16-bit score each) and every min/add of the
// recurrence runs on both at once: the chain char c becomes
//   x = min(dprev + delta, min(T[c-1] + 1, D[c] + 1))   (two __viaddmin_u16x2)
// No half ever wraps: every score is at most 65000 (rows are 16-bit only for
// reads of at most 65000 bases), +1 and +delta stay below 65536, and the
// deferred term F + (c - first) stays below 65536 because the engine runs
// this kernel only when every string vertex has at most 512 chars.
// Lanes: G = min(32, R/2) per vertex, P = R / (2G) register pairs each.
// ---------------------------------------------------------------------------
template <int R>
struct Pairs {
  static constexpr int G = (R / 2) < 32 ? (R / 2) : 32;
  static constexpr int P = R / (2 * G);
};

template <int P>
struct U2 {
  uint32_t h[P];
};

template <int P>
__device__ __forceinline__ U2<P> ldp_nc(const uint16_t* p) {
  U2<P> o;
  if constexpr (P == 1) {
    o.h[0] = __ldg(reinterpret_cast<const unsigned int*>(p));
  } else {
    const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
    o.h[0] = t.x;
    o.h[1] = t.y;
  }
  return o;
}

template <int P, bool COH>
__device__ __forceinline__ U2<P> ldp_src(const uint16_t* p) {
  if constexpr (COH) {
    U2<P> o;
    if constexpr (P == 1) {
      o.h[0] = *reinterpret_cast<const uint32_t*>(p);
    } else {
      const uint2 t = *reinterpret_cast<const uint2*>(p);
      o.h[0] = t.x;
      o.h[1] = t.y;
    }
    return o;
  } else {
    return ldp_nc<P>(p);
  }
}

template <int P>
__device__ __forceinline__ void stp(uint16_t* p, const U2<P>& x) {
  if constexpr (P == 1) {
    *reinterpret_cast<uint32_t*>(p) = x.h[0];
  } else {
    *reinterpret_cast<uint2*>(p) = make_uint2(x.h[0], x.h[1]);
  }
}

// (a & m) | (b & ~m) in one LOP3
__device__ __forceinline__ uint32_t sel(uint32_t a, uint32_t b, uint32_t m) {
  uint32_t r;
  asm("lop3.b32 %0, %1, %2, %3, 0xE4;" : "=r"(r) : "r"(a), "r"(b), "r"(m));
  return r;
}

// Label keys of consecutive chars: a 64-bit window over the 4-bit key array.
struct KeyWindow {
  const uint32_t* w;
  uint64_t win;
  uint32_t nx;  // the word after the window, loaded a word (8 chars) before it is needed
  uint32_t sh;
  KeyWindow() = default;
  __device__ __forceinline__ KeyWindow(const uint32_t* lab4, uint32_t c) {
    w = lab4 + (c >> 3);
    win = (uint64_t)__ldg(w) | ((uint64_t)__ldg(w + 1) << 32);
    nx = __ldg(w + 2);
    sh = (c & 7u) * 4u;
  }
  __device__ __forceinline__ uint32_t next() {
    const uint32_t k = (uint32_t)(win >> sh) & 0xFu;
    sh += 4;
    if (sh == 32) {
      ++w;
      win = (win >> 32) | ((uint64_t)nx << 32);
      nx = __ldg(w + 2);
      sh = 0;
    }
    return k;
  }
  // the keys of the next four chars, 4 bits each; the window must be at a
  // char c with c % 4 == 0
  __device__ __forceinline__ uint32_t next4() {
    const uint32_t k = (uint32_t)(win >> sh) & 0xFFFFu;
    sh += 16;
    if (sh == 32) {
      ++w;
      win = (win >> 32) | ((uint64_t)nx << 32);
      nx = __ldg(w + 2);
      sh = 0;
    }
    return k;
  }
};

// The chain chars of one vertex (c = f+1 .. f+len-1); TRACK also keeps the
// per-slot minimum and its smallest char for slots on their last row.
template <int R, bool DEFER, bool TRACK, int P, bool COH = false>
__device__ __forceinline__ void dpx_chain(const uint16_t* __restrict__ dp, uint16_t* __restrict__ tp,
                                          uint32_t len, uint32_t f, KeyWindow& kw, U2<P>& t,
                                          U2<P>& dprev, const U2<P>& F, bool any_fix,
                                          const uint32_t (&dtab)[P], const uint32_t (&imask)[P],
                                          const uint32_t (&fmask)[P], int (&bmin)[2 * P],
                                          uint32_t (&barg)[2 * P]) {
  constexpr uint32_t ONES = 0x00010001u;
  constexpr int DEPTH = 8;
  uint32_t off2 = 0;
  for (uint32_t q0 = 1; q0 < len; q0 += DEPTH) {
    const uint32_t n = min((uint32_t)DEPTH, len - q0);
    U2<P> dq[DEPTH];
#pragma unroll
    for (int k = 0; k < DEPTH; ++k)
      if (k < (int)n) dq[k] = ldp_src<P, COH>(dp + (size_t)k * R);
#pragma unroll
    for (int k = 0; k < DEPTH; ++k) {
      if (k < (int)n) {
        const uint32_t key = kw.next();
        off2 += ONES;
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const uint32_t delta = (dtab[p] >> key) & ONES;
          if (DEFER && any_fix)
            dq[k].h[p] = sel(__viaddmin_u16x2(F.h[p], off2, dq[k].h[p]), dq[k].h[p], fmask[p]);
          uint32_t x = __viaddmin_u16x2(t.h[p], ONES, dq[k].h[p] + ONES);
          x = __viaddmin_u16x2(dprev.h[p], delta, x);
          t.h[p] = sel(delta, x, imask[p]);
        }
        dprev = dq[k];
        stp<P>(tp + (size_t)k * R, t);
        if (TRACK) {
          const uint32_t c = f + q0 + k;
#pragma unroll
          for (int p = 0; p < P; ++p) {
            const int lo = (int)(t.h[p] & 0xFFFFu), hi = (int)(t.h[p] >> 16);
            if (lo < bmin[2 * p]) {
              bmin[2 * p] = lo;
              barg[2 * p] = c;
            }
            if (hi < bmin[2 * p + 1]) {
              bmin[2 * p + 1] = hi;
              barg[2 * p + 1] = c;
            }
          }
        }
      }
    }
    dp += (size_t)DEPTH * R;
    tp += (size_t)DEPTH * R;
  }
}

// The update of string vertex s for the lane's 2P slots (k_row_dpx's body).
template <int R, bool DEFER, bool COH>
__device__ __forceinline__ void dpx_vertex(const GraphPtrs& g, uint32_t s, int lane, const uint16_t* D,
                                           uint16_t* T, uint16_t* BV, const uint16_t* FL,
                                           const uint32_t* slot_word, unsigned long long* sm_best,
                                           bool ending_any) {
  constexpr int P = Pairs<R>::P;
  constexpr uint32_t ONES = 0x00010001u;
    const size_t so = (size_t)lane * 2 * P;  // first slot of this lane
    // per register pair: delta table over label keys (bit k of each half =
    // mismatch of key k), row-0 mask, deferred-propagation mask
    uint32_t dtab[P], imask[P], fmask[P];
    bool any_fix = false, any_end = false;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      dtab[p] = imask[p] = fmask[p] = 0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint32_t w = COH ? slot_word[so + 2 * p + h] : __ldg(slot_word + so + 2 * p + h);
        dtab[p] |= ((w >> SW_MASK_SHIFT) & SW_MASK) << (16 * h);
        if (w & SW_INIT) imask[p] |= 0xFFFFu << (16 * h);
        if (DEFER && (w & SW_FIX)) fmask[p] |= 0xFFFFu << (16 * h);
        any_end |= (w & SW_ENDING) != 0;
      }
      any_fix |= fmask[p] != 0;
    }
    uint32_t f = __ldg(g.sv_off + s), e = __ldg(g.sv_off + s + 1);
    CHSGA_CHK_CHARS(f, e, g.N, 1);
    const uint32_t d = CHSGA_CHK(__ldg(g.sv_dev + s), g.S, 3);
    uint32_t k0 = __ldg(g.vin_off + s), k1 = __ldg(g.vin_off + s + 1);
    CHSGA_CHK_RANGE(k0, k1, g.n_vin, 4);
    KeyWindow kw(g.lab4, f);
    U2<P> F;
#pragma unroll
    for (int p = 0; p < P; ++p) F.h[p] = 0;
    if (DEFER && any_fix) F = ldp_src<P, COH>(FL + (size_t)(2 * s) * R + so);
    const uint16_t* dp = D + (size_t)f * R + so;
    uint16_t* tp = T + (size_t)f * R + so;
    U2<P> dprev = ldp_src<P, COH>(dp);
    U2<P> t;
    {
      const uint32_t key = kw.next();
      uint32_t delta[P];
#pragma unroll
      for (int p = 0; p < P; ++p) {
        delta[p] = (dtab[p] >> key) & ONES;
        if (DEFER && any_fix) dprev.h[p] = sel(__vminu2(dprev.h[p], F.h[p]), dprev.h[p], fmask[p]);
        t.h[p] = dprev.h[p] + ONES;
      }
      for (uint32_t k = k0; k < k1; ++k) {
        const uint32_t su = CHSGA_CHK(__ldg(g.vin_srcv + k), g.S, 5);
        const U2<P> du = ldp_src<P, COH>(FL + (size_t)(2 * su + 1) * R + so);
#pragma unroll
        for (int p = 0; p < P; ++p) t.h[p] = __viaddmin_u16x2(du.h[p], delta[p], t.h[p]);
      }
#pragma unroll
      for (int p = 0; p < P; ++p) t.h[p] = sel(delta[p], t.h[p], imask[p]);
    }
    stp<P>(tp, t);
    stp<P>(BV + (size_t)(2 * d) * R + so, t);
    int bmin[2 * P];
    uint32_t barg[2 * P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      bmin[2 * p] = (int)(t.h[p] & 0xFFFFu);
      bmin[2 * p + 1] = (int)(t.h[p] >> 16);
      barg[2 * p] = barg[2 * p + 1] = f;
    }
    const uint32_t len = e - f;
    if (ending_any && any_end) {
      dpx_chain<R, DEFER, true, P, COH>(dp + R, tp + R, len, f, kw, t, dprev, F, any_fix, dtab, imask,
                                   fmask, bmin, barg);
    } else {
      dpx_chain<R, DEFER, false, P, COH>(dp + R, tp + R, len, f, kw, t, dprev, F, any_fix, dtab, imask,
                                    fmask, bmin, barg);
    }
    if (len > 1) stp<P>(BV + (size_t)(2 * d + 1) * R + so, t);
    if (ending_any && any_end) {
#pragma unroll
      for (int q = 0; q < 2 * P; ++q) {
        const uint32_t w = COH ? slot_word[so + q] : __ldg(slot_word + so + q);
        if (w & SW_ENDING) atomicMin(sm_best + so + q, pack_min(bmin[q], barg[q]));
      }
    }
  }

template <int R, bool DEFER>
__global__ void __launch_bounds__(256, 4) k_row_dpx(GraphPtrs g, const uint16_t* __restrict__ D,
                                                    uint16_t* __restrict__ T,
                                                    uint16_t* __restrict__ BV,
                                                    const uint16_t* __restrict__ FL,
                                                    const uint32_t* __restrict__ slot_word,
                                                    unsigned long long* __restrict__ best,
                                                    const StepCtl* __restrict__ ctl) {
  pdl_wait();
  constexpr int G = Pairs<R>::G;
  __shared__ unsigned long long sm_best[R];
  const bool ending_any = ctl->any_ending != 0;
  if (!ctl->any_active) return;
  if (ending_any) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) sm_best[r] = ~0ull;
    __syncthreads();
  }
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t s = (uint32_t)(gt / G);
  if (s < g.S) dpx_vertex<R, DEFER, false>(g, s, (int)(gt % G), D, T, BV, FL, slot_word, sm_best, ending_any);
  if (ending_any) flush_min<R>(sm_best, best);
}

// ---------------------------------------------------------------------------
// k_row_stream (R >= 64): k_row_dpx with one warp walking a run of 32
// consecutive string vertices, whose chars are consecutive too. The warp's
// previous-row scores stream through a ring of kStreamRing rows in shared
// memory: every lane copies its own 2P scores of a row with cp.async
// (kStreamRing rows in flight per lane, one commit group per row) and reads
// back only what it copied, so no lane waits for another. The next vertex's
// final first score F and the final last scores of its first two in-edge
// sources are loaded into registers while the current vertex computes; the
// run's vertex words and first 64 in-edge sources come in coalesced loads,
// one vertex per lane, broadcast by shuffles. Every branch depends only on
// warp-uniform values. Slots on their last row keep one running minimum
// per warp; chars are visited in increasing order, so a strict comparison
// keeps the smallest char among equal scores.
// ---------------------------------------------------------------------------
// Measured on B200 (6.4 M-char graph, 128 slots): 16 rows in flight per lane
// with 4-warp blocks, 6 per SM, beat deeper rings (32 or 48 rows take the
// shared memory the L1 needs for the in-edge and label loads) and 8-warp
// blocks.
#ifndef CHSGA_STREAM_RING
#define CHSGA_STREAM_RING 16  // rows in flight per warp (build-time tuning)
#endif
#ifndef CHSGA_STREAM_WARPS
#define CHSGA_STREAM_WARPS 4  // warps per block (build-time tuning)
#endif
#ifndef CHSGA_STREAM_BLOCKS
#define CHSGA_STREAM_BLOCKS 6  // blocks per SM the register budget is sized for
#endif
constexpr int kStreamRing = CHSGA_STREAM_RING;
constexpr int kStreamWarps = CHSGA_STREAM_WARPS;

__host__ __device__ constexpr size_t stream_smem_bytes(int R) {
  return (size_t)kStreamWarps * kStreamRing * R * 2;
}

template <int P>
__device__ __forceinline__ void cp_async_row(uint16_t* dst, const uint16_t* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst)), "l"(src),
               "n"(4 * P)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int P>
struct StreamVertex {
  uint32_t f, len, d, k0, k1;
  U2<P> F;
  U2<P> u[2];  // final last scores of the first two in-edge sources
};

template <int P>
__device__ __forceinline__ U2<P> lds_u2(const uint16_t* p) {
  U2<P> o;
  if constexpr (P == 1) {
    o.h[0] = *reinterpret_cast<const uint32_t*>(p);
  } else {
    const uint2 t = *reinterpret_cast<const uint2*>(p);
    o.h[0] = t.x;
    o.h[1] = t.y;
  }
  return o;
}

// The graph constants of lane j of a k_row_stream run: vertex s0 + j's char
// range, hierarchy position and first-char in-edge range (zeros past the
// graph). Loaded before the kernel's pdl_wait.
struct RunHead {
  uint32_t mf, me, md, mk0, mk1;
};

__device__ __forceinline__ RunHead run_head(const GraphPtrs& g, uint32_t run_index) {
  RunHead r{0, 0, 0, 0, 0};
  const uint32_t s0 = run_index * 32, lane = threadIdx.x & 31;
  if (lane < min(32u, g.S - s0)) {
    const uint32_t s = s0 + lane;
    r.mf = __ldg(g.sv_off + s);
    r.me = __ldg(g.sv_off + s + 1);
    r.md = CHSGA_CHK(__ldg(g.sv_dev + s), g.S, 3);
    r.mk0 = __ldg(g.vin_off + s);
    r.mk1 = __ldg(g.vin_off + s + 1);
    CHSGA_CHK_CHARS(r.mf, r.me, g.N, 1);
    CHSGA_CHK_RANGE(r.mk0, r.mk1, g.n_vin, 4);
  }
  return r;
}

// One warp's run of 32 string vertices starting at s0 = 32 * run_index (k_row_stream's
// body); warp_ring = the warp's kStreamRing x R ring in shared memory.
template <int R, bool DEFER, bool COH>
__device__ __forceinline__ void stream_run(const GraphPtrs& g, uint32_t run_index, const RunHead& rh,
                                           const uint16_t* D, uint16_t* T, uint16_t* BV, const uint16_t* FL,
                                           const uint32_t* slot_word, uint16_t* warp_ring,
                                           unsigned long long* sm_best, bool ending_any) {
  constexpr int P = Pairs<R>::P;
  constexpr int W = kStreamRing;
  constexpr uint32_t ONES = 0x00010001u;
  constexpr unsigned FULL = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const uint32_t s0 = run_index * 32;
    const size_t so = (size_t)lane * 2 * P;
    // this lane's ring: row slot k at ring + k * R (the warp's 32 lanes side by side)
    uint16_t* ring = warp_ring + so;
    uint32_t dtab[P], imask[P], fmask[P];
    bool any_fix = false, any_end = false;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      dtab[p] = imask[p] = fmask[p] = 0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint32_t w = COH ? slot_word[so + 2 * p + h] : __ldg(slot_word + so + 2 * p + h);
        dtab[p] |= ((w >> SW_MASK_SHIFT) & SW_MASK) << (16 * h);
        if (w & SW_INIT) imask[p] |= 0xFFFFu << (16 * h);
        if (DEFER && (w & SW_FIX)) fmask[p] |= 0xFFFFu << (16 * h);
        any_end |= (w & SW_ENDING) != 0;
      }
      any_fix |= fmask[p] != 0;
    }
    any_fix = __any_sync(FULL, any_fix);
    const bool track = ending_any && __any_sync(FULL, any_end);
    // the run's vertex words, vertex s0 + lane on each lane
    const uint32_t nv = min(32u, g.S - s0);
    const uint32_t mf = rh.mf, me = rh.me, md = rh.md, mk0 = rh.mk0, mk1 = rh.mk1;
    const uint32_t cb = __shfl_sync(FULL, mf, 0), ce = __shfl_sync(FULL, me, nv - 1);
    // previous-row scores of the run's chars cb .. ce-1: row c goes to slot
    // (c - cb) % W; one commit group per row, empty past the run
    const uint16_t* dsrc = D + so;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      if (cb + k < ce) cp_async_row<P>(ring + (size_t)k * R, dsrc + (size_t)(cb + k) * R);
      cp_async_commit();
    }
    const uint32_t kb = __shfl_sync(FULL, mk0, 0), ke = __shfl_sync(FULL, mk1, nv - 1);
    const uint32_t src_a = kb + lane < ke ? CHSGA_CHK(__ldg(g.vin_srcv + kb + lane), g.S, 5) : 0u;
    const uint32_t src_b = kb + 32 + lane < ke ? CHSGA_CHK(__ldg(g.vin_srcv + kb + 32 + lane), g.S, 5) : 0u;
    // source vertex of in-edge k (k warp-uniform)
    auto src_at = [&](uint32_t k) -> uint32_t {
      const uint32_t i = k - kb;
      const uint32_t a = __shfl_sync(FULL, src_a, i & 31), b = __shfl_sync(FULL, src_b, i & 31);
      return i < 32 ? a : i < 64 ? b : CHSGA_CHK(__ldg(g.vin_srcv + k), g.S, 5);
    };
    auto prefetch = [&](uint32_t i, StreamVertex<P>& v) {
      v.f = __shfl_sync(FULL, mf, i);
      v.len = __shfl_sync(FULL, me, i) - v.f;
      v.d = __shfl_sync(FULL, md, i);
      v.k0 = __shfl_sync(FULL, mk0, i);
      v.k1 = __shfl_sync(FULL, mk1, i);
#pragma unroll
      for (int p = 0; p < P; ++p) v.F.h[p] = v.u[0].h[p] = v.u[1].h[p] = 0;
      if (DEFER && any_fix) v.F = ldp_src<P, COH>(FL + (size_t)(2 * (s0 + i)) * R + so);
#pragma unroll
      for (int j = 0; j < 2; ++j)
        if (v.k0 + j < v.k1) v.u[j] = ldp_src<P, COH>(FL + (size_t)(2 * src_at(v.k0 + j) + 1) * R + so);
    };
    // The char stream cb .. ce-1: `slot` is the ring row of the current char
    // (its copy is the oldest of W pending groups), `gnext` the global row
    // W chars ahead that refills the slot once the current value is used,
    // `left` how many chars remain to be fetched, `tp` the current char's
    // row of T.
    uint16_t* slot = ring;
    uint16_t* const ring_end = ring + (size_t)W * R;
    const uint16_t* gnext = dsrc + (size_t)(cb + W) * R;
    int32_t left = (int32_t)(ce - cb) - W;
    uint16_t* tp = T + (size_t)cb * R + so;
    auto take = [&]() -> U2<P> {
      cp_async_wait<W - 1>();
      return lds_u2<P>(slot);
    };
    auto refill = [&]() {
      if (left > 0) cp_async_row<P>(slot, gnext);
      cp_async_commit();
      gnext += R;
      --left;
      slot += R;
      if (slot == ring_end) slot = ring;
      tp += R;
    };
    int bmin[2 * P];
    uint32_t barg[2 * P];
#pragma unroll
    for (int q = 0; q < 2 * P; ++q) {
      bmin[q] = 0x7fffffff;
      barg[q] = 0;
    }
    auto track_char = [&](const U2<P>& t, uint32_t c) {
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const int lo = (int)(t.h[p] & 0xFFFFu), hi = (int)(t.h[p] >> 16);
        if (lo < bmin[2 * p]) {
          bmin[2 * p] = lo;
          barg[2 * p] = c;
        }
        if (hi < bmin[2 * p + 1]) {
          bmin[2 * p + 1] = hi;
          barg[2 * p + 1] = c;
        }
      }
    };
    KeyWindow kw(g.lab4, cb);
    StreamVertex<P> cur, nxt;
    prefetch(0, cur);
    // the vertex loop, once with and once without the last-row minimum
    auto run = [&](auto track_tag) {
      constexpr bool TRACK = decltype(track_tag)::value;
      for (uint32_t i = 0; i < nv; ++i) {
        if (i + 1 < nv) prefetch(i + 1, nxt);
        const uint32_t f = cur.f, len = cur.len;
        const U2<P> F = cur.F;
        U2<P> t, dprev = take();
        // first char: min(D[f] + 1, min over in-edges of last(u) + delta)
        {
          const uint32_t key = kw.next();
          uint32_t delta[P];
#pragma unroll
          for (int p = 0; p < P; ++p) {
            delta[p] = (dtab[p] >> key) & ONES;
            if (DEFER && any_fix) dprev.h[p] = sel(__vminu2(dprev.h[p], F.h[p]), dprev.h[p], fmask[p]);
            t.h[p] = dprev.h[p] + ONES;
          }
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (cur.k0 + j < cur.k1)
#pragma unroll
              for (int p = 0; p < P; ++p) t.h[p] = __viaddmin_u16x2(cur.u[j].h[p], delta[p], t.h[p]);
          for (uint32_t k = cur.k0 + 2; k < cur.k1; ++k) {
            const U2<P> du = ldp_src<P, COH>(FL + (size_t)(2 * src_at(k) + 1) * R + so);
#pragma unroll
            for (int p = 0; p < P; ++p) t.h[p] = __viaddmin_u16x2(du.h[p], delta[p], t.h[p]);
          }
#pragma unroll
          for (int p = 0; p < P; ++p) t.h[p] = sel(delta[p], t.h[p], imask[p]);
        }
        stp<P>(tp, t);
        stp<P>(BV + (size_t)(2 * cur.d) * R + so, t);
        if (TRACK) track_char(t, f);
        refill();
        // chain chars: off2 = q in both halves
        uint32_t off2 = 0;
        for (uint32_t q = 1; q < len; ++q) {
          U2<P> dq = take();
          const uint32_t key = kw.next();
          off2 += ONES;
#pragma unroll
          for (int p = 0; p < P; ++p) {
            const uint32_t delta = (dtab[p] >> key) & ONES;
            if (DEFER && any_fix)
              dq.h[p] = sel(__viaddmin_u16x2(F.h[p], off2, dq.h[p]), dq.h[p], fmask[p]);
            uint32_t x = __viaddmin_u16x2(t.h[p], ONES, dq.h[p] + ONES);
            x = __viaddmin_u16x2(dprev.h[p], delta, x);
            t.h[p] = sel(delta, x, imask[p]);
          }
          dprev = dq;
          stp<P>(tp, t);
          if (TRACK) track_char(t, f + q);
          refill();
        }
        if (len > 1) stp<P>(BV + (size_t)(2 * cur.d + 1) * R + so, t);
        cur = nxt;
      }
    };
    if (track)
      run(std::true_type{});
    else
      run(std::false_type{});
    cp_async_wait<0>();
    if (track) {
#pragma unroll
      for (int q = 0; q < 2 * P; ++q) {
        const uint32_t w = COH ? slot_word[so + q] : __ldg(slot_word + so + q);
        if ((w & SW_ENDING) && bmin[q] != 0x7fffffff)
          atomicMin(sm_best + so + q, pack_min(bmin[q], barg[q]));
      }
    }
  }

template <int R, bool DEFER>
__global__ void __launch_bounds__(kStreamWarps * 32, CHSGA_STREAM_BLOCKS) k_row_stream(
    GraphPtrs g, const uint16_t* __restrict__ D, uint16_t* __restrict__ T, uint16_t* __restrict__ BV,
    const uint16_t* __restrict__ FL, const uint32_t* __restrict__ slot_word,
    unsigned long long* __restrict__ best, const StepCtl* __restrict__ ctl) {
  static_assert(Pairs<R>::G == 32, "one full warp per vertex");
  extern __shared__ __align__(16) uint16_t ring_smem[];
  __shared__ unsigned long long sm_best[R];
  const uint32_t run = (uint32_t)((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5);
  RunHead rh{0, 0, 0, 0, 0};
  if (run * 32 < g.S) rh = run_head(g, run);
  pdl_wait();
  const bool ending_any = ctl->any_ending != 0;
  if (!ctl->any_active) return;
  if (ending_any) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) sm_best[r] = ~0ull;
    __syncthreads();
  }
  if (run * 32 < g.S)
    stream_run<R, DEFER, false>(g, run, rh, D, T, BV, FL, slot_word,
                                ring_smem + (size_t)(threadIdx.x >> 5) * kStreamRing * R, sm_best,
                                ending_any);
  if (ending_any) flush_min<R>(sm_best, best);
}

// ---------------------------------------------------------------------------
// Delta rows (128 slots, score-only). Within a string vertex two consecutive
// chars' scores differ by at most 1 in every row: row 0 holds 0/1; a row's
// raw update keeps the bound when the previous final row has it (a chain
// char takes min(D[c] + 1, D[c-1] + delta, T[c-1] + 1) and D is 1-Lipschitz
// along the chain), and the closure only lowers a vertex's chars to
// min(T[c], F + (c - first)), a line of slope 1. So a row is stored as the
// raw first score of every vertex (16 bits per slot, "H") and, for every
// char, T[c] - T[c-1] + 1 in {0, 1, 2} (2 bits per slot, "Z"): 0.26 bytes
// per cell instead of 2. Z: chars in groups of 4; group q, lane L (slots
// 4L .. 4L+3) is the 32-bit word q * 32 + L, byte c & 3 for char c, slot
// 4L + j at bits 2j .. 2j+1 (a first char's byte is unused). H[s * 128 + r]
// follows Z at a 256-byte boundary. A delta outside {0, 1, 2} for an active
// slot would mean the bound failed: the kernel sets ERR_ROW_DELTA and the
// call fails instead of returning a wrong score.
// ---------------------------------------------------------------------------
constexpr uint32_t ERR_ROW_DELTA = 8;
#ifndef CHSGA_DELTA_RING
#define CHSGA_DELTA_RING 16  // Z words in flight per lane (4 chars each; build-time tuning)
#endif
constexpr int kDeltaRing = CHSGA_DELTA_RING;

__host__ __device__ constexpr size_t delta_z_bytes(size_t N) { return ((N + 3) / 4 + 1) * 32 * 4; }
__host__ __device__ constexpr size_t delta_h_offset(size_t N) { return (delta_z_bytes(N) + 255) / 256 * 256; }
__host__ __device__ constexpr size_t delta_row_bytes(size_t N, size_t S) {
  return delta_h_offset(N) + S * 128 * 2 + 256;
}
__host__ __device__ constexpr size_t delta_smem_bytes() { return (size_t)kStreamWarps * kDeltaRing * 32 * 4; }

__device__ __forceinline__ void cp_async_word(uint32_t* dst, const uint32_t* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

// the four 2-bit deltas in the low byte of b as two u16x2 words (slots 0,1
// and 2,3): b | b << 14 puts bits 2-3 at 16-17 and bits 6-7 at 20-21
__device__ __forceinline__ void delta_expand(uint32_t b, uint32_t& e0, uint32_t& e1) {
  b &= 0xFFu;  // the other bytes of the word would reach bits 16-21
  const uint32_t t = b | (b << 14);
  e0 = t & 0x00030003u;
  e1 = (t >> 4) & 0x00030003u;
}

template <bool COH>
__device__ __forceinline__ void delta_run(const GraphPtrs& g, uint32_t run_index, const RunHead& rh,
                                          const uint32_t* DZ,
                                          const uint16_t* DH, uint32_t* TZ, uint16_t* TH, uint16_t* BV,
                                          const uint16_t* FL, const uint32_t* slot_word, uint32_t* warp_ring,
                                          const uint2* lut, const uint2* dtl, unsigned long long* sm_best,
                                          bool ending_any, StepCtl* ctl) {
  constexpr int R = 128, P = 2, W = kDeltaRing;
  // a first score that no closure candidate F + (c - first) can beat: above
  // every score (at most 65001) and, plus a vertex offset (at most 511), still
  // below 2^16
  constexpr uint32_t NO_CLOSURE = 0xFDFFFDFFu;
  constexpr uint32_t ONES = 0x00010001u;
  constexpr unsigned FULL = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const uint32_t s0 = run_index * 32;
  const size_t so = (size_t)lane * 4;
  uint32_t* ring = warp_ring + lane;  // word k of this lane at ring[k * 32]
  // (the mismatch increments of every key come from the block's table dtl)
  uint32_t imask[P], fmask[P], amask[P];
  bool any_fix = false, any_end = false;
#pragma unroll
  for (int p = 0; p < P; ++p) {
    imask[p] = fmask[p] = amask[p] = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t w = COH ? slot_word[so + 2 * p + h] : __ldg(slot_word + so + 2 * p + h);
      if (w & SW_INIT) imask[p] |= 0xFFFFu << (16 * h);
      if (w & SW_FIX) fmask[p] |= 0xFFFFu << (16 * h);
      if (w & SW_ACTIVE) amask[p] |= 0xFFFFu << (16 * h);
      any_end |= (w & SW_ENDING) != 0;
    }
    any_fix |= fmask[p] != 0;
    // an idle slot computes a row-0 row of a read that matches everywhere
    // (its mismatch mask is empty): all 0, so every slot's scores stay in
    // 0..65535 and the pair arithmetic below never carries between halves.
    // The rows a slot on row 0 reads are the ones its previous read (or the
    // row-0 path) left, also in range; only the first step of a call reads
    // rows no step of the call wrote, and there every slot is on row 0 or
    // idle, so both halves of every pair are replaced by their row-0 values
    imask[p] |= ~amask[p];
  }
  any_fix = __any_sync(FULL, any_fix);
  const bool any_init = __any_sync(FULL, (imask[0] | imask[1]) != 0);
  const bool track = ending_any && __any_sync(FULL, any_end);
  const uint32_t nv = min(32u, g.S - s0);
  const uint32_t mf = rh.mf, me = rh.me, md = rh.md, mk0 = rh.mk0, mk1 = rh.mk1;
  const uint32_t cb = __shfl_sync(FULL, mf, 0), ce = __shfl_sync(FULL, me, nv - 1);
  // previous-row Z words of the run's char groups q0 .. q1, W in flight
  const uint32_t q0 = cb >> 2, q1 = (ce - 1) >> 2;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    if (q0 + k <= q1) cp_async_word(ring + k * 32, DZ + (size_t)(q0 + k) * 32 + lane);
    cp_async_commit();
  }
  uint32_t rslot = 0;                 // ring word of the current group
  uint32_t qnext = q0 + W;            // next group to fetch
  auto take_word = [&]() -> uint32_t {
    cp_async_wait<W - 1>();
    const uint32_t w = ring[rslot * 32];
    if (qnext <= q1) cp_async_word(ring + rslot * 32, DZ + (size_t)qnext * 32 + lane);
    cp_async_commit();
    ++qnext;
    rslot = (rslot + 1) % W;
    return w;
  };
  const uint32_t kb = __shfl_sync(FULL, mk0, 0), ke = __shfl_sync(FULL, mk1, nv - 1);
  const uint32_t src_a = kb + lane < ke ? CHSGA_CHK(__ldg(g.vin_srcv + kb + lane), g.S, 5) : 0u;
  const uint32_t src_b = kb + 32 + lane < ke ? CHSGA_CHK(__ldg(g.vin_srcv + kb + 32 + lane), g.S, 5) : 0u;
  auto src_at = [&](uint32_t k) -> uint32_t {
    const uint32_t i = k - kb;
    const uint32_t a = __shfl_sync(FULL, src_a, i & 31), b = __shfl_sync(FULL, src_b, i & 31);
    return i < 32 ? a : i < 64 ? b : CHSGA_CHK(__ldg(g.vin_srcv + k), g.S, 5);
  };
  struct DV {
    uint32_t f, len, d, k0, k1;
    U2<P> F, H, u[2];
  };
  auto prefetch = [&](uint32_t i, DV& v) {
    v.f = __shfl_sync(FULL, mf, i);
    v.len = __shfl_sync(FULL, me, i) - v.f;
    v.d = __shfl_sync(FULL, md, i);
    v.k0 = __shfl_sync(FULL, mk0, i);
    v.k1 = __shfl_sync(FULL, mk1, i);
#pragma unroll
    for (int p = 0; p < P; ++p) v.F.h[p] = v.u[0].h[p] = v.u[1].h[p] = 0;
    v.H = ldp_src<P, COH>(DH + (size_t)(s0 + i) * R + so);
    // the vertex's final first score of the previous row: BV[2d], which this
    // warp alone overwrites, later, with the new row's raw first score
    if (any_fix) v.F = ldp_src<P, true>(BV + (size_t)(2 * v.d) * R + so);
#pragma unroll
    for (int j = 0; j < 2; ++j)
      if (v.k0 + j < v.k1) v.u[j] = ldp_src<P, COH>(FL + (size_t)(2 * src_at(v.k0 + j) + 1) * R + so);
  };
  int bmin[2 * P];
  uint32_t barg[2 * P];
#pragma unroll
  for (int q = 0; q < 2 * P; ++q) {
    bmin[q] = 0x7fffffff;
    barg[q] = 0;
  }
  auto track_char = [&](const U2<P>& t, uint32_t c) {
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const int lo = (int)(t.h[p] & 0xFFFFu), hi = (int)(t.h[p] >> 16);
      if (lo < bmin[2 * p]) {
        bmin[2 * p] = lo;
        barg[2 * p] = c;
      }
      if (hi < bmin[2 * p + 1]) {
        bmin[2 * p + 1] = hi;
        barg[2 * p + 1] = c;
      }
    }
  };
  // output: the bytes of the current group shift in from the top of zout;
  // a whole group is one word store, the run's first and last groups (shared
  // with the neighbouring runs) are stored byte by byte
  // the group's input word is fetched where its output word is stored, so a
  // char takes one branch
  uint32_t zin = 0, zout = 0, bad = 0;
  auto put = [&](uint32_t c, uint32_t byte) {
    zout = __funnelshift_r(zout, byte, 8);
    if ((c & 3u) == 3u) {
      uint32_t* dst = TZ + (size_t)(c >> 2) * 32 + lane;
      if (c >= cb + 3) {
        *dst = zout;
      } else {
        unsigned char* db = reinterpret_cast<unsigned char*>(dst);
        for (uint32_t b = cb & 3u; b < 4; ++b) db[b] = (unsigned char)(zout >> (8 * b));
      }
      if (c + 1 < ce) zin = take_word();
    }
  };
  KeyWindow kw(g.lab4, cb);
  DV cur, nxt;
  prefetch(0, cur);
  zin = take_word();  // the run's first group
  auto run = [&](auto track_tag, auto fix_tag, auto init_tag) {
    constexpr bool TRACK = decltype(track_tag)::value;
    constexpr bool FIX = decltype(fix_tag)::value;    // some slot of the warp applies a deferred closure
    constexpr bool INIT = decltype(init_tag)::value;  // some slot of the warp is on row 0 (or idle)
    for (uint32_t i = 0; i < nv; ++i) {
      if (i + 1 < nv) prefetch(i + 1, nxt);
      const uint32_t f = cur.f, len = cur.len;
      // slots without the deferred closure take NO_CLOSURE, so it never wins
      U2<P> F;
#pragma unroll
      for (int p = 0; p < P; ++p) F.h[p] = sel(cur.F.h[p], NO_CLOSURE, fmask[p]);
      U2<P> t, draw = cur.H, dprev = cur.H;
      // first char: its byte of the group is unused
      {
        const uint32_t key = kw.next();
        const uint2 dl = dtl[key * 32];  // the char's mismatch increments, both pairs
        const uint32_t delta[P] = {dl.x, dl.y};
#pragma unroll
        for (int p = 0; p < P; ++p) {
          if (FIX) dprev.h[p] = __vminu2(dprev.h[p], F.h[p]);
          t.h[p] = dprev.h[p] + ONES;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j)
          if (cur.k0 + j < cur.k1)
#pragma unroll
            for (int p = 0; p < P; ++p) t.h[p] = __viaddmin_u16x2(cur.u[j].h[p], delta[p], t.h[p]);
        for (uint32_t k = cur.k0 + 2; k < cur.k1; ++k) {
          const U2<P> du = ldp_src<P, COH>(FL + (size_t)(2 * src_at(k) + 1) * R + so);
#pragma unroll
          for (int p = 0; p < P; ++p) t.h[p] = __viaddmin_u16x2(du.h[p], delta[p], t.h[p]);
        }
#pragma unroll
        for (int p = 0; p < P; ++p)
          if (INIT) t.h[p] = sel(delta[p], t.h[p], imask[p]);
      }
      stp<P>(TH + (size_t)(s0 + i) * R + so, t);
      stp<P>(BV + (size_t)(2 * cur.d) * R + so, t);
      put(f, 0u);
      if (TRACK) track_char(t, f);
      uint32_t off2 = 0;
      // one chain char from its input byte (its four slots' 2-bit fields)
      // and its label key; returns its output byte in bits 0-7 (bits 16-21
      // hold leftovers that the caller drops)
      auto step = [&](uint32_t byte_in, uint32_t key) -> uint32_t {
        // the pair increments of the byte, -1..1 per half: a 32-bit add is
        // exact since no half leaves 0..65535 (scores stay in 0..65001,
        // consecutive chars differ by at most 1)
        const uint2 e = lut[byte_in];
        draw.h[0] += e.x;
        draw.h[1] += e.y;
        U2<P> dq = draw;
        off2 += ONES;
        const U2<P> tp = t;
        const uint2 dl = dtl[key * 32];
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const uint32_t delta = p == 0 ? dl.x : dl.y;
          if (FIX) dq.h[p] = __viaddmin_u16x2(F.h[p], off2, dq.h[p]);
          uint32_t x = __viaddmin_u16x2(t.h[p], ONES, dq.h[p] + ONES);
          x = __viaddmin_u16x2(dprev.h[p], delta, x);
          t.h[p] = INIT ? sel(delta, x, imask[p]) : x;
        }
        dprev = dq;
        // T[c] - T[c-1] + 1 per slot, 2 bits each
        const uint32_t d0 = t.h[0] + ONES - tp.h[0];
        const uint32_t d1 = t.h[1] + ONES - tp.h[1];
        bad |= d0 | d1;
        // 0..2 in every half (idle slots included): low halves at bits 0
        // and 4, high halves at 16 and 20, folded into one byte
        const uint32_t dd = d0 | (d1 << 4);
        return dd | (dd >> 14);
      };
      // one char at a time up to a group boundary: selector = byte c & 3 of
      // zin, then three zero bytes of the second operand (an index below 256)
      auto one = [&](uint32_t c) {
        put(c, step(__byte_perm(zin, 0u, (c & 3u) | 0x4440u), kw.next()) & 0xFFu);
        if (TRACK) track_char(t, c);
      };
      uint32_t c = f + 1;
      const uint32_t cend = f + len;
      for (; c < cend && (c & 3u); ++c) one(c);
      // whole groups inside the vertex: constant byte positions, the four
      // keys from one window read, one word store (a group that starts
      // after cb lies wholly in this run)
      for (; c + 4 <= cend; c += 4) {
        const uint32_t k4 = kw.next4();
        uint32_t word = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const uint32_t o = step(__byte_perm(zin, 0u, 0x4440u | (uint32_t)j), (k4 >> (4 * j)) & 0xFu);
          // byte j of word := byte 0 of o
          word = __byte_perm(word, o, j == 0 ? 0x3214u : j == 1 ? 0x3240u : j == 2 ? 0x3410u : 0x4210u);
          if (TRACK) track_char(t, c + j);
        }
        TZ[(size_t)(c >> 2) * 32 + lane] = word;
        zout = word;
        if (c + 4 < ce) zin = take_word();
      }
      for (; c < cend; ++c) one(c);
      if (len > 1) stp<P>(BV + (size_t)(2 * cur.d + 1) * R + so, t);
      cur = nxt;
    }
  };
  auto with_init = [&](auto track_tag, auto fix_tag) {
    if (any_init)
      run(track_tag, fix_tag, std::true_type{});
    else
      run(track_tag, fix_tag, std::false_type{});
  };
  if (track) {
    if (any_fix)
      with_init(std::true_type{}, std::true_type{});
    else
      with_init(std::true_type{}, std::false_type{});
  } else {
    if (any_fix)
      with_init(std::false_type{}, std::true_type{});
    else
      with_init(std::false_type{}, std::false_type{});
  }
  // the run's last group when it ends inside a group
  if (((ce - 1) & 3u) != 3u) {
    const uint32_t g0 = (ce - 1) & ~3u, k = ce - g0;  // bytes of the group this run holds
    unsigned char* db = reinterpret_cast<unsigned char*>(TZ + (size_t)(g0 >> 2) * 32 + lane);
    const uint32_t first = cb > g0 ? cb - g0 : 0u;
    for (uint32_t b = first; b < k; ++b) db[b] = (unsigned char)(zout >> (8 * (4 - k + b)));
  }
  cp_async_wait<0>();
  if (bad & 0xFFFCFFFCu) atomicOr(&ctl->error, ERR_ROW_DELTA);
  if (track) {
#pragma unroll
    for (int q = 0; q < 2 * P; ++q) {
      const uint32_t w = COH ? slot_word[so + q] : __ldg(slot_word + so + q);
      if ((w & SW_ENDING) && bmin[q] != 0x7fffffff) atomicMin(sm_best + so + q, pack_min(bmin[q], barg[q]));
    }
  }
}

#ifndef CHSGA_DELTA_BLOCKS
#define CHSGA_DELTA_BLOCKS CHSGA_STREAM_BLOCKS  // blocks per SM the register budget is sized for
#endif
// Runs are taken longest first: run_order lists the run indices by
// decreasing char count (built on the host). Warp w of the grid takes entry
// w, then entries from the launch's counter (StepCtl::run_next, reset by
// k_advance) until the list is done, so the last runs to finish are the
// short ones. The grid is at most the resident blocks.
__global__ void __launch_bounds__(kStreamWarps * 32, CHSGA_DELTA_BLOCKS) k_row_delta(
    GraphPtrs g, const uint16_t* __restrict__ D, uint16_t* __restrict__ T, uint16_t* __restrict__ BV,
    const uint16_t* __restrict__ FL, const uint32_t* __restrict__ slot_word,
    unsigned long long* __restrict__ best, StepCtl* __restrict__ ctl, const uint32_t* __restrict__ run_order,
    uint32_t nruns) {
  constexpr unsigned FULL = 0xFFFFFFFFu;
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
  uint32_t k = (uint32_t)((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5);
  uint32_t run = k < nruns ? CHSGA_CHK(__ldg(run_order + k), nruns, 7) : 0u;
  RunHead rh{0, 0, 0, 0, 0};
  if (k < nruns) rh = run_head(g, run);
  pdl_wait();
  extern __shared__ __align__(16) uint32_t dring_smem[];
  __shared__ unsigned long long sm_best[128];
  const bool ending_any = ctl->any_ending != 0;
  if (!ctl->any_active) return;
  if (ending_any) {
    for (int r = threadIdx.x; r < 128; r += blockDim.x) sm_best[r] = ~0ull;
    __syncthreads();
  }
  // byte -> increments of the two slot pairs (the 2-bit fields minus 1)
  __shared__ uint2 s_lut[256];
  for (int v = threadIdx.x; v < 256; v += blockDim.x) {
    uint32_t e0, e1;
    delta_expand((uint32_t)v, e0, e1);
    s_lut[v] = make_uint2(e0 - 0x00010001u, e1 - 0x00010001u);
  }
  // label key -> mismatch increments of lane L's two slot pairs (slots 4L ..
  // 4L + 3, 1 in a half where the slot's read base mismatches the key)
  __shared__ uint2 s_dtab[16 * 32];
  for (int i = threadIdx.x; i < 16 * 32; i += blockDim.x) {
    const uint32_t key = (uint32_t)i >> 5, L = (uint32_t)i & 31u;
    uint32_t v[2];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const uint32_t m0 = (__ldg(slot_word + 4 * L + 2 * p) >> SW_MASK_SHIFT) & SW_MASK;
      const uint32_t m1 = (__ldg(slot_word + 4 * L + 2 * p + 1) >> SW_MASK_SHIFT) & SW_MASK;
      v[p] = ((m0 >> key) & 1u) | (((m1 >> key) & 1u) << 16);
    }
    s_dtab[i] = make_uint2(v[0], v[1]);
  }
  __syncthreads();
  const size_t hoff = delta_h_offset(g.N);
  while (k < nruns) {
    delta_run<false>(g, run, rh, reinterpret_cast<const uint32_t*>(D),
                     reinterpret_cast<const uint16_t*>(reinterpret_cast<const unsigned char*>(D) + hoff),
                     reinterpret_cast<uint32_t*>(T),
                     reinterpret_cast<uint16_t*>(reinterpret_cast<unsigned char*>(T) + hoff), BV, FL, slot_word,
                     dring_smem + (size_t)(threadIdx.x >> 5) * kDeltaRing * 32, s_lut, s_dtab + (threadIdx.x & 31),
                     sm_best, ending_any, ctl);
    uint32_t nk = 0;
    if ((threadIdx.x & 31) == 0) nk = nwarps + atomicAdd(&ctl->run_next, 1u);
    k = __shfl_sync(FULL, nk, 0);
    if (k < nruns) {
      run = CHSGA_CHK(__ldg(run_order + k), nruns, 7);
      rh = run_head(g, run);
    }
  }
  if (ending_any) flush_min<128>(sm_best, best);
}

// ---------------------------------------------------------------------------
// Loads of data that other blocks of the same launch may have written (the
// persistent row-step kernel's rows, boundary scores and slot words): L2
// only (ld.global.cg), never the read-only path, which assumes the data does
// not change while the kernel runs. COH = false keeps __ldg for kernels that
// only read what earlier launches wrote.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 ld_cg_v4(const void* p) {
  uint4 r;
  asm volatile("ld.global.cg.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p));
  return r;
}
__device__ __forceinline__ uint32_t ld_cg_u32(const void* p) {
  uint32_t r;
  asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(r) : "l"(p));
  return r;
}
__device__ __forceinline__ int ld_cg_u16(const void* p) {
  unsigned short r;
  asm volatile("ld.global.cg.u16 %0, [%1];" : "=h"(r) : "l"(p));
  return (int)r;
}
template <bool COH>
__device__ __forceinline__ uint4 ldv4(const void* p) {
  if constexpr (COH) return ld_cg_v4(p);
  else return __ldg(reinterpret_cast<const uint4*>(p));
}
template <bool COH>
__device__ __forceinline__ uint32_t ldu32(const uint32_t* p) {
  if constexpr (COH) return ld_cg_u32(p);
  else return __ldg(p);
}
template <bool COH>
__device__ __forceinline__ int ldu16(const uint16_t* p) {
  if constexpr (COH) return ld_cg_u16(p);
  else return (int)__ldg(reinterpret_cast<const unsigned short*>(p));
}

// ---------------------------------------------------------------------------
// k_row_t1 (R = 1, 16-bit rows): the row update of one read, one warp per
// tile of whole consecutive string vertices (at most 32 aligned chunks of 8
// chars and 64 vertices, built on the host). Lane j owns chunk q0 + j: its 8
// previous-row scores in one 16-byte load, its 8 label keys in one word and
// its head bits (first chars of vertices) in one byte. Lanes v and v + 32
// load vertex v's record (first char, hierarchy position, first in-edge
// sources) and the previous row's final scores it needs; the warp keeps them
// in shared memory.
//
// Within a vertex T[c] = min(X[c], T[c-1] + 1), with X[c] = min(D'[c] + 1,
// D'[c-1] + delta) for a chain char and X[f] = min(D'[f] + 1, min over
// in-edges of FL_last(u) + delta) for the first char, D' being the previous
// row with its deferred propagation applied (as in k_row_direct). A lane
// runs the recurrence over its 8 chars from no carry. The carry into lane j
// is the composition of the earlier lanes' maps x -> min(a, x + b) (a = the
// lane's last value, b = 8, or none when the lane holds a first char), a
// min-plus scan in 5 shuffle steps; chars before the lane's first head then
// take min(T, carry + distance). Row 0 takes delta only.
// ---------------------------------------------------------------------------
struct T1Ptrs {
  const uint4* desc;     // per tile {first char, end char, first vertex, end vertex}
  const uint8_t* heads;  // per 8-char chunk: bit i = char 8q + i starts a vertex
  const uint4* vrec;     // per vertex {first char, position | many << 31, src0, src1}
  uint32_t ntiles;
};
constexpr int kT1Warps = 8;       // warps per block of k_row_t1
constexpr int kT1VertMax = 64;    // vertices per tile (kT1MaxVerts on the host)

// The graph constants of one lane of a k_row_t1 tile: the tile descriptor,
// the lane's chunk of label keys and head bits, and the record of vertex
// `lane` of the tile. Loaded before the kernel's pdl_wait. In the checked
// build a descriptor outside the graph, or larger than a warp's lanes and
// vertex slots, comes back as the empty tile {0, 0, 0, 0} and is skipped
// whole (every lane reads the same descriptor).
struct T1Head {
  uint4 td, r0;
  uint32_t keys, hb;
};

__device__ __forceinline__ T1Head t1_head(const GraphPtrs& g, const T1Ptrs& t, uint32_t tile) {
  const int lane = threadIdx.x & 31;
  T1Head r{};
  r.td = __ldg(t.desc + tile);
#ifdef CHSGA_CHECKED
  const uint4 td = r.td;
  if (!(td.x < td.y && td.y <= g.N && td.z < td.w && td.w <= g.S && td.w - td.z <= (uint32_t)kT1VertMax &&
        ((td.y - 1) >> 3) - (td.x >> 3) < 32u)) {
    if (lane == 0) chk_fail(tile, 6);
    r.td = make_uint4(0, 0, 0, 0);
    return r;
  }
#endif
  const uint32_t q = (r.td.x >> 3) + lane;
  if (q <= ((r.td.y - 1) >> 3)) {
    r.keys = __ldg(g.lab4 + q);
    r.hb = __ldg(t.heads + q);
  }
  if ((uint32_t)lane < r.td.w - r.td.z) r.r0 = __ldg(t.vrec + r.td.z + lane);
  return r;
}

template <bool DEFER, bool COH>
__device__ __forceinline__ void row_t1_tile(const GraphPtrs& g, const T1Ptrs& t, const T1Head& th,
                                            const uint16_t* D, uint16_t* T, uint16_t* BV,
                                            const uint16_t* FL, uint32_t w, int* s_G, int* s_X,
                                            uint32_t* s_d, unsigned long long& mn) {
  constexpr unsigned FULL = 0xFFFFFFFFu;
  constexpr int BIG = 0x3fffffff;
  const int lane = threadIdx.x & 31;
  const uint4 td = th.td;
#ifdef CHSGA_CHECKED
  if (td.y == 0) return;
#endif
  const uint32_t cb = td.x, ce = td.y, sb = td.z, nv = td.w - td.z;
  const uint32_t q = (cb >> 3) + lane;
  const bool lv = q <= ((ce - 1) >> 3);
  const bool init = (w & SW_INIT) != 0;
  const bool fix = DEFER && (w & SW_FIX) != 0;
  const bool ending = (w & SW_ENDING) != 0;
  const uint32_t mask = (w >> SW_MASK_SHIFT) & SW_MASK;
  uint4 dq = make_uint4(0, 0, 0, 0);
  uint32_t keys = 0, hb = 0, inm = 0;
  if (lv) {
    dq = ldv4<COH>(D + 8 * (size_t)q);
    keys = th.keys;
    hb = th.hb;
    const uint32_t c0 = 8 * q;
    const uint32_t lo = cb > c0 ? cb - c0 : 0u;
    const uint32_t hi = ce - c0 < 8u ? ce - c0 : 8u;
    inm = (0xFFu >> (8u - hi)) & (0xFFu << lo) & 0xFFu;
    hb &= inm;
  }
  for (uint32_t v = lane; v < nv; v += 32) {
    const uint32_t sv = sb + v;
    const uint4 r = v == (uint32_t)lane ? th.r0 : __ldg(t.vrec + sv);
    int G = 0, X = BIG;
    if (fix) G = ldu16<COH>(FL + 2 * (size_t)sv) - (int)r.x;
    if (!init) {
      if (r.z != 0xFFFFFFFFu) X = ldu16<COH>(FL + 2 * (size_t)CHSGA_CHK(r.z, g.S, 10) + 1);
      if (r.w != 0xFFFFFFFFu) X = min(X, ldu16<COH>(FL + 2 * (size_t)CHSGA_CHK(r.w, g.S, 10) + 1));
      if (r.y & 0x80000000u) {
        uint32_t k0 = __ldg(g.vin_off + sv) + 2, k1 = __ldg(g.vin_off + sv + 1);
        CHSGA_CHK_RANGE(k0, k1, g.n_vin, 4);
        for (uint32_t k = k0; k < k1; ++k)
          X = min(X, ldu16<COH>(FL + 2 * (size_t)CHSGA_CHK(__ldg(g.vin_srcv + k), g.S, 5) + 1));
      }
    }
    s_G[v] = G;
    s_X[v] = X;
    s_d[v] = CHSGA_CHK(r.y & 0x7FFFFFFFu, g.S, 9);
  }
  __syncwarp();
  // vertex index (within the tile) of the char before this lane's first head
  const int nh = __popc(hb);
  int incl = nh;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int x = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += x;
  }
  const int vbase = incl - nh - 1;
  // previous-row scores, the deferred propagation applied
  int dp[8];
  {
    const uint32_t wv[4] = {dq.x, dq.y, dq.z, dq.w};
    int vi = vbase;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      dp[i] = (int)((wv[i >> 1] >> (16 * (i & 1))) & 0xFFFFu);
      vi += (hb >> i) & 1;
      if (fix && ((inm >> i) & 1)) dp[i] = min(dp[i], s_G[vi] + (int)(8 * q + i));
    }
  }
  const int dm1 = __shfl_up_sync(FULL, dp[7], 1);
  int tl[8];
  int first_head = 8;
  {
    int a = BIG, vi = vbase;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const bool head = (hb >> i) & 1;
      vi += head;
      const int delta = (int)((mask >> ((keys >> (4 * i)) & 0xFu)) & 1u);
      int x;
      if (init) {
        x = delta;
      } else {
        x = dp[i] + 1;
        if (head) {
          x = min(x, s_X[vi] + delta);
        } else {
          x = min(x, (i ? dp[i - 1] : dm1) + delta);
          x = min(x, a + 1);
        }
      }
      if (head && first_head == 8) first_head = i;
      a = x;
      tl[i] = x;
    }
  }
  // carry across lanes: inclusive min-plus scan of (last value, distance)
  int A = tl[7], B = (hb || init) ? BIG : 8;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int Ap = __shfl_up_sync(FULL, A, o), Bp = __shfl_up_sync(FULL, B, o);
    if (lane >= o) {
      A = min(A, Ap + B);
      B = min(BIG, Bp + B);
    }
  }
  const int carry = __shfl_up_sync(FULL, A, 1);
  if (!init && lane > 0) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (i < first_head) tl[i] = min(tl[i], carry + i + 1);
  }
  // final scores: the row, the vertex boundary scores, the last-row minimum
  const uint32_t nb0 = (uint32_t)__shfl_down_sync(FULL, (int)hb, 1) & 1u;
  if (inm) {
    uint32_t ow[4] = {0, 0, 0, 0};
    int vi = vbase;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const bool head = (hb >> i) & 1;
      vi += head;
      ow[i >> 1] |= ((uint32_t)tl[i] & 0xFFFFu) << (16 * (i & 1));
      if ((inm >> i) & 1) {
        const uint32_t c = 8 * q + i;
        if (head) BV[2 * (size_t)s_d[vi]] = (uint16_t)tl[i];
        const bool last = (c + 1 == ce) || (i < 7 ? ((hb >> (i + 1)) & 1u) != 0 : nb0 != 0);
        if (last && !head) BV[2 * (size_t)s_d[vi] + 1] = (uint16_t)tl[i];
        if (ending) mn = min(mn, pack_min(tl[i], c));
        if (inm != 0xFFu) T[8 * (size_t)q + i] = (uint16_t)tl[i];
      }
    }
    if (inm == 0xFFu)
      *reinterpret_cast<uint4*>(T + 8 * (size_t)q) = make_uint4(ow[0], ow[1], ow[2], ow[3]);
  }
  __syncwarp();  // s_G / s_X / s_d are reused by the warp's next tile
}

#ifndef CHSGA_T1_BLOCKS
#define CHSGA_T1_BLOCKS 6  // blocks per SM the register budget is sized for (build-time tuning)
#endif
template <bool DEFER>
__global__ void __launch_bounds__(kT1Warps * 32, CHSGA_T1_BLOCKS) k_row_t1(GraphPtrs g, T1Ptrs t,
                                                          const uint16_t* __restrict__ D,
                                                          uint16_t* __restrict__ T,
                                                          uint16_t* __restrict__ BV,
                                                          const uint16_t* __restrict__ FL,
                                                          const uint32_t* __restrict__ slot_word,
                                                          unsigned long long* __restrict__ best,
                                                          const StepCtl* __restrict__ ctl) {
  __shared__ int s_G[kT1Warps][kT1VertMax], s_X[kT1Warps][kT1VertMax];
  __shared__ uint32_t s_d[kT1Warps][kT1VertMax];
  __shared__ unsigned long long sm_best[1];
  const int wp = threadIdx.x >> 5;
  const uint32_t tile = blockIdx.x * kT1Warps + wp;
  T1Head th{};
  if (tile < t.ntiles) th = t1_head(g, t, tile);
  pdl_wait();
  if (!ctl->any_active) return;
  const bool ending = ctl->any_ending != 0;
  if (ending) {
    if (threadIdx.x == 0) sm_best[0] = ~0ull;
    __syncthreads();
  }
  unsigned long long mn = ~0ull;
  if (tile < t.ntiles)
    row_t1_tile<DEFER, false>(g, t, th, D, T, BV, FL, __ldg(slot_word), s_G[wp], s_X[wp], s_d[wp], mn);
  if (ending) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
    if ((threadIdx.x & 31) == 0 && mn != ~0ull) atomicMin(sm_best, mn);
    flush_min<1>(sm_best, best);
  }
}

// ---------------------------------------------------------------------------
// k_row_tiled (R >= 32, one warp per vertex): the same update with every
// input of a tile of consecutive vertices staged in shared memory by TMA
// bulk copies. A producer warp walks the block's tiles and, per tile, copies
// the previous-row scores of its chars, the FL block of its vertices, the
// tile's descriptor (vertex and in-edge records, built on the host) and the
// FL last scores of in-edge sources outside the tile into one of nslots
// buffers; 16 consumer warps compute tiles from shared memory, so no
// dependent global load sits on their critical path. full/empty mbarriers
// hand buffers back and forth; all waits are bounded.
//
// Tile record: r0 = {s0, s1, c0, c1 | long << 31}, r1 = {descriptor word
// offset, descriptor bytes, external count, external list word offset}.
// Descriptor: per vertex {first char, length, hierarchy position,
// first edge << 16 | edge count}, then per in-edge one word: source vertex
// - s0 if inside the tile, else 0x80000000 | external index. A long tile (one
// vertex longer than the score buffer) reads its chars from global memory.
// ---------------------------------------------------------------------------
constexpr int kRowCons = 16;     // consumer warps per block
constexpr int kRowMaxSlots = (int)kTileSlotsMax;
constexpr int kRowThreads = (kRowCons + 1) * 32;
constexpr uint32_t ERR_ROW_WAIT = 2;

struct RowTiles {
  const int4* rec;          // 2 per tile
  const uint32_t* desc;     // descriptors (16-byte aligned per tile)
  uint32_t ntiles;
  uint32_t nslots;          // buffers per block
  uint32_t d_cap, fl_cap, desc_cap, ext_cap;  // byte size of each slot region
};

__host__ __device__ constexpr uint32_t row_slot_bytes(const RowTiles& t) {
  return t.d_cap + t.fl_cap + t.desc_cap + t.ext_cap;
}
__host__ __device__ constexpr size_t row_smem_bytes(uint32_t slot_bytes, uint32_t nslots, int R) {
  return (size_t)nslots * slot_bytes + (size_t)kRowMaxSlots * 16 + (size_t)R * 8 + 16;
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Bulk copy into shared memory completing on `bar` without an arrival (the
// arrival with the whole tile's byte count is made separately).
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_expect(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

template <int R, bool DEFER, typename ST>
__global__ void __launch_bounds__(kRowThreads, 1) k_row_tiled(GraphPtrs g, RowTiles rt,
                                                             const ST* __restrict__ D,
                                                             ST* __restrict__ T, ST* __restrict__ BV,
                                                             const ST* __restrict__ FL,
                                                             const uint32_t* __restrict__ slot_word,
                                                             unsigned long long* __restrict__ best,
                                                             StepCtl* __restrict__ ctl) {
  pdl_wait();
  static_assert(R >= 32, "one warp per vertex");
  constexpr int V = Lanes<R>::V;
  constexpr uint32_t PC = R * sizeof(ST);  // bytes per char (and per FL entry)
  extern __shared__ __align__(16) unsigned char row_smem[];
  __shared__ int s_fail;
  if (!ctl->any_active) return;
  const bool ending_any = ctl->any_ending != 0;
  const int warp = threadIdx.x >> 5, wl = threadIdx.x & 31;
  const uint32_t SB = row_slot_bytes(rt);
  unsigned long long* full = reinterpret_cast<unsigned long long*>(row_smem + (size_t)rt.nslots * SB);
  unsigned long long* empty = full + kRowMaxSlots;
  unsigned long long* sm_best = empty + kRowMaxSlots;
  if (ending_any)
    for (int r = threadIdx.x; r < R; r += blockDim.x) sm_best[r] = ~0ull;
  if (threadIdx.x == 0) {
    s_fail = 0;
    for (uint32_t k = 0; k < rt.nslots; ++k) {
      mbar_init(&full[k], 1);
      mbar_init(&empty[k], 1);
    }
    fence_async_shared();
  }
  __syncthreads();
  // this block's tiles: t = blockIdx.x + i * gridDim.x; tile i uses buffer
  // i % nslots and consumer warp i % nslots (nslots <= kRowCons)
  const uint32_t nt =
      rt.ntiles > blockIdx.x ? (rt.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  if (warp == kRowCons) {
    uint32_t last_parity = 0, used = 0;  // lane 0's record of every buffer's last fill
    for (uint32_t i = 0; i < nt; ++i) {
      const uint32_t k = i % rt.nslots;
      int stop = 0;
      if (wl == 0) {
        stop = *(volatile int*)&s_fail;
        if (!stop && i >= rt.nslots && !mbar_wait(&empty[k], ((i / rt.nslots) - 1) & 1)) {
          s_fail = 1;
          stop = 1;
        }
      }
      if (__shfl_sync(0xffffffffu, stop, 0)) break;
      const uint32_t t = blockIdx.x + i * gridDim.x;
      const int4 r0 = rt.rec[2 * t], r1 = rt.rec[2 * t + 1];
      unsigned char* slot = row_smem + (size_t)k * SB;
      const uint32_t s0 = (uint32_t)r0.x, s1 = (uint32_t)r0.y, c0 = (uint32_t)r0.z;
      const bool lng = r0.w < 0;
      const uint32_t c1 = (uint32_t)(r0.w & 0x7fffffff);
      const uint32_t dbytes = lng ? 0u : (c1 - c0) * PC;
      const uint32_t flbytes = 2 * (s1 - s0) * PC;
      const uint32_t total = dbytes + flbytes + (uint32_t)r1.y + (uint32_t)r1.z * PC;
      if (wl == 0) {
        fence_async_shared();
        mbar_expect(&full[k], total);
        if (dbytes) bulk_copy(slot, D + (size_t)c0 * R, dbytes, &full[k]);
        bulk_copy(slot + rt.d_cap, FL + (size_t)(2 * s0) * R, flbytes, &full[k]);
        bulk_copy(slot + rt.d_cap + rt.fl_cap, rt.desc + (size_t)r1.x, (uint32_t)r1.y, &full[k]);
        last_parity ^= 1u << k;
        used |= 1u << k;
      }
      __syncwarp();
      if (wl < r1.z) {
        const uint32_t su = rt.desc[(size_t)r1.w + wl];
        bulk_copy(slot + rt.d_cap + rt.fl_cap + rt.desc_cap + wl * PC, FL + (size_t)(2 * su + 1) * R,
                  PC, &full[k]);
      }
    }
    if (wl == 0 && *(volatile int*)&s_fail) {
      // bounded wait for every buffer's last fill before shared memory goes
      for (uint32_t k = 0; k < rt.nslots; ++k)
        if (used & (1u << k)) mbar_wait(&full[k], ((last_parity >> k) & 1) ^ 1);
    }
  } else {
    const int lane = wl;
    const size_t so = (size_t)lane * V;
    uint32_t code[V];
    bool init[V], ending[V], fix[V];
    bool any_fix = false;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const uint32_t w = __ldg(slot_word + so + v);
      code[v] = (w >> SW_MASK_SHIFT) & SW_MASK;  // mismatch mask
      init[v] = (w & SW_INIT) != 0;
      ending[v] = (w & SW_ENDING) != 0;
      fix[v] = DEFER && (w & SW_FIX) != 0;
      any_fix |= fix[v];
    }
    int bmin[V];
    uint32_t barg[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      bmin[v] = 0x7fffffff;
      barg[v] = 0;
    }
    constexpr int kBig = 0x3fffffff;
    // consumer warp w owns buffer w and takes tiles w, w + nslots, ...: each
    // buffer's fills are consumed in order, so a parity wait can never be
    // satisfied by an older fill of the same buffer
    for (uint32_t i = warp; warp < (int)rt.nslots && i < nt; i += rt.nslots) {
      const uint32_t k = i % rt.nslots;
      const bool ok = mbar_wait(&full[k], (i / rt.nslots) & 1);
      if (__any_sync(0xffffffffu, !ok || *(volatile int*)&s_fail)) {
        s_fail = 1;
        break;
      }
      const uint32_t t = blockIdx.x + i * gridDim.x;
      const int4 r0 = rt.rec[2 * t];
      const uint32_t s0 = (uint32_t)r0.x, nv = (uint32_t)r0.y - s0, c0 = (uint32_t)r0.z;
      const bool lng = r0.w < 0;
      const unsigned char* slot = row_smem + (size_t)k * SB;
      const ST* Dt = lng ? D + (size_t)c0 * R : reinterpret_cast<const ST*>(slot);
      const ST* FLt = reinterpret_cast<const ST*>(slot + rt.d_cap);
      const uint32_t* dsc = reinterpret_cast<const uint32_t*>(slot + rt.d_cap + rt.fl_cap);
      const ST* EXt = reinterpret_cast<const ST*>(slot + rt.d_cap + rt.fl_cap + rt.desc_cap);
      const uint32_t* erec = dsc + 4 * nv;
      for (uint32_t j = 0; j < nv; ++j) {
        const uint4 vr = *reinterpret_cast<const uint4*>(dsc + 4 * j);
        const uint32_t f = vr.x, len = vr.y, d = vr.z;
        const uint32_t eb = vr.w >> 16, ec = vr.w & 0xFFFFu;
        IV<V> F;
#pragma unroll
        for (int v = 0; v < V; ++v) F.v[v] = kBig;
        if (DEFER && any_fix) {
          const IV<V> x = ld<V>(FLt + (size_t)(2 * j) * R + so);
#pragma unroll
          for (int v = 0; v < V; ++v)
            if (fix[v]) F.v[v] = x.v[v];
        }
        const ST* Dv = Dt + (size_t)(f - c0) * R + so;
        IV<V> dprev = ld<V>(Dv);
        IV<V> tv;
        {
          const uint32_t key = label_key(g, f);
          int delta[V];
#pragma unroll
          for (int v = 0; v < V; ++v) {
            if (DEFER) dprev.v[v] = min(dprev.v[v], F.v[v]);
            delta[v] = (int)((code[v] >> key) & 1u);
            tv.v[v] = dprev.v[v] + 1;
          }
          for (uint32_t q = 0; q < ec; ++q) {
            const uint32_t loc = erec[eb + q];
            const ST* src = (loc & 0x80000000u)
                                ? EXt + (size_t)(loc & 0x7fffffffu) * R + so
                                : FLt + (size_t)(2 * loc + 1) * R + so;
            const IV<V> du = ld<V>(src);
#pragma unroll
            for (int v = 0; v < V; ++v) tv.v[v] = min(tv.v[v], du.v[v] + delta[v]);
          }
#pragma unroll
          for (int v = 0; v < V; ++v) {
            if (init[v]) tv.v[v] = delta[v];
            if (tv.v[v] < bmin[v]) {
              bmin[v] = tv.v[v];
              barg[v] = f;
            }
          }
        }
        st<V>(T + (size_t)f * R + so, tv);
        st<V>(BV + (size_t)(2 * d) * R + so, tv);
        for (uint32_t q0 = 1; q0 < len; q0 += 4) {
          const uint32_t n = min(4u, len - q0);
          IV<V> dq[4];
#pragma unroll
          for (uint32_t q = 0; q < 4; ++q)
            if (q < n) dq[q] = ld<V>(Dv + (size_t)(q0 + q) * R);
#pragma unroll
          for (uint32_t q = 0; q < 4; ++q) {
            if (q < n) {
              const uint32_t c = f + q0 + q;
              const uint32_t key = label_key(g, c);
#pragma unroll
              for (int v = 0; v < V; ++v) {
                if (DEFER) dq[q].v[v] = min(dq[q].v[v], F.v[v] + (int)(q0 + q));
                const int delta = (int)((code[v] >> key) & 1u);
                int x = min(dq[q].v[v] + 1, dprev.v[v] + delta);
                x = min(x, tv.v[v] + 1);
                if (init[v]) x = delta;
                tv.v[v] = x;
                if (x < bmin[v]) {
                  bmin[v] = x;
                  barg[v] = c;
                }
              }
              dprev = dq[q];
              st<V>(T + (size_t)c * R + so, tv);
            }
          }
        }
        if (len > 1) st<V>(BV + (size_t)(2 * d + 1) * R + so, tv);
      }
      __syncwarp();
      if (wl == 0) mbar_arrive(&empty[k]);
    }
    if (ending_any) {
#pragma unroll
      for (int v = 0; v < V; ++v)
        if (ending[v] && bmin[v] != 0x7fffffff)
          atomicMin(sm_best + so + v, pack_min(bmin[v], barg[v]));
    }
  }
  __syncthreads();
  if (s_fail && threadIdx.x == 0) atomicOr(&ctl->error, ERR_ROW_WAIT);
  if (ending_any)
    for (int r = threadIdx.x; r < R; r += blockDim.x)
      if (sm_best[r] != ~0ull) atomicMin(best + r, sm_best[r]);
}

// ---------------------------------------------------------------------------
// k_pull: hierarchy positions [lo, hi): BV[2d] = min(BV[2d], BV[src] + w)
// over the list off[d-base]..off[d-base+1]. Every source lies on another
// level, finished before this launch, so the gathers use the read-only path.
// ---------------------------------------------------------------------------
template <int R, typename ST, bool COH>
__device__ __forceinline__ void pull_item(ST* BV, uint32_t d, int lane, const uint32_t* __restrict__ off,
                                          const int2* __restrict__ edges, uint32_t base) {
  constexpr int V = Lanes<R>::V;
  const size_t so = (size_t)lane * V;
  const uint32_t k0 = __ldg(off + (d - base)), k1 = __ldg(off + (d - base) + 1);
  if (k0 == k1) return;
  ST* p = BV + (size_t)(2 * d) * R + so;
  IV<V> f = ld<V>(p);
  bool changed = false;
  for (uint32_t k = k0; k < k1; ++k) {
    const int2 ew = __ldg(edges + k);
    const IV<V> x = ld_src<V, COH>(BV + (size_t)CHSGA_CHK(ew.x, 2 * (uint64_t)d, 12) * R + so);
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

template <int R, typename ST>
__global__ void __launch_bounds__(256) k_pull(ST* __restrict__ BV, uint32_t lo, uint32_t hi,
                                              const uint32_t* __restrict__ off,
                                              const int2* __restrict__ edges, uint32_t base,
                                              const StepCtl* __restrict__ ctl) {
  pdl_wait();
  constexpr int G = Lanes<R>::G;
  if (!ctl->any_active) return;
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t d = lo + (uint32_t)(gt / G);
  if (d >= hi) return;
  pull_item<R, ST, false>(BV, d, (int)(gt % G), off, edges, base);
}

// The graph constants of one k_pull_lv / k_pull_lv16 target: its list head
// (edge range, first two sources and weights) and the four edges after those
// two. Nothing here is written during a run, so the kernel loads it before
// its pdl_wait, while the kernel before it drains.
constexpr int kPullHeadEdges = 4;
template <int NE>
struct PullHeadT {
  uint4 h, h2;
  int2 e[NE > 0 ? NE : 1];  // unused when NE = 0
};
using PullHead = PullHeadT<kPullHeadEdges>;

// NE = the edges after the head's two that come with it (0 or kPullHeadEdges)
template <int NE = kPullHeadEdges>
__device__ __forceinline__ PullHeadT<NE> pull_head(uint32_t d, const uint4* __restrict__ head,
                                                   const int2* __restrict__ edges, uint32_t n_edges) {
  PullHeadT<NE> r;
  r.h = __ldg(head + 2 * (size_t)d);
  r.h2 = __ldg(head + 2 * (size_t)d + 1);
  CHSGA_CHK_RANGE(r.h.x, r.h.y, n_edges, 11);
  const uint32_t k = r.h.x + 2;
#pragma unroll
  for (int q = 0; q < NE; ++q) r.e[q] = k + q < r.h.y ? __ldg(edges + k + q) : make_int2(0, 0);
  return r;
}

// ---------------------------------------------------------------------------
// k_pull_lv: one upward level [lo, hi) below the top region, the k_pull
// update with the list head of each position in two 16-byte loads (the
// first two sources are gathered without waiting for an edge load).
// ---------------------------------------------------------------------------
template <int R, typename ST, bool COH>
__device__ __forceinline__ void pull_lv_item(ST* BV, uint32_t d, int lane, const PullHead& hd,
                                             const int2* __restrict__ edges) {
  constexpr int V = Lanes<R>::V;
  uint4 h = hd.h, h2 = hd.h2;
  if (h.x == h.y) return;
  h.z = CHSGA_CHK(h.z, 2 * (uint64_t)d, 12);
  h2.x = CHSGA_CHK(h2.x, 2 * (uint64_t)d, 12);
  const size_t so = (size_t)lane * V;
  ST* p = BV + (size_t)(2 * d) * R + so;
  IV<V> f = ld<V>(p);
  bool changed = false;
  auto relax = [&](const IV<V>& x, int w) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int c = x.v[v] + w;
      if (c < f.v[v]) {
        f.v[v] = c;
        changed = true;
      }
    }
  };
  const IV<V> x0 = ld_src<V, COH>(BV + (size_t)h.z * R + so);
  if (h.y - h.x > 1) {
    const IV<V> x1 = ld_src<V, COH>(BV + (size_t)h2.x * R + so);
    relax(x0, (int)h.w);
    relax(x1, (int)h2.y);
  } else {
    relax(x0, (int)h.w);
  }
  IV<V> xe[kPullHeadEdges];
#pragma unroll
  for (int q = 0; q < kPullHeadEdges; ++q)
    if (h.x + 2 + q < h.y) xe[q] = ld_src<V, COH>(BV + (size_t)CHSGA_CHK(hd.e[q].x, 2 * (uint64_t)d, 12) * R + so);
#pragma unroll
  for (int q = 0; q < kPullHeadEdges; ++q)
    if (h.x + 2 + q < h.y) relax(xe[q], hd.e[q].y);
  for (uint32_t k = h.x + 2 + kPullHeadEdges; k < h.y; ++k) {
    const int2 ew = __ldg(edges + k);
    relax(ld_src<V, COH>(BV + (size_t)CHSGA_CHK(ew.x, 2 * (uint64_t)d, 12) * R + so), ew.y);
  }
  if (changed) st<V>(p, f);
}

template <int R, typename ST>
__global__ void __launch_bounds__(256) k_pull_lv(ST* __restrict__ BV, uint32_t lo, uint32_t hi,
                                                 const uint4* __restrict__ head,
                                                 const int2* __restrict__ edges, uint32_t n_edges,
                                                 const StepCtl* __restrict__ ctl) {
  constexpr int G = Lanes<R>::G;
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t d = lo + (uint32_t)(gt / G);
  PullHead hd{};
  if (d < hi) hd = pull_head(d, head, edges, n_edges);
  pdl_wait();
  if (!ctl->any_active || d >= hi) return;
  pull_lv_item<R, ST, false>(BV, d, (int)(gt % G), hd, edges);
}

// ---------------------------------------------------------------------------
// k_pull_lv16: k_pull_lv for 16-bit rows and R >= 8 slots. A lane holds 8
// slots (16 bytes) as four u16x2 words and relaxes them with a saturating
// add and a min, so a position takes R / 8 lanes and a warp keeps twice the
// bytes in flight of the one-word-per-slot form. Saturation is exact here:
// every stored score is below 65535, so a sum that clamps never wins the
// min, as in the int form. Edges beyond the two in the head are fetched four
// at a time, their sources gathered together.
// ---------------------------------------------------------------------------
// MAXE = 2: every target of the level has at most the head's two edges (the
// host knows each level's largest list), so the form has no edge loop and
// needs about half the registers (26 against 48 at 128 slots): eight blocks
// per SM instead of five. MAXE = 4: at most the head's two and the two
// prefetched after them, every gather at once, no loop (38 registers, six
// blocks per SM). MAXE = 0: any number of edges.
template <int R, bool COH, int MAXE = 0, int NE = kPullHeadEdges>
__device__ __forceinline__ void pull_lv16_item(uint16_t* BV, uint32_t d, int lane, const PullHeadT<NE>& hd,
                                               const int2* __restrict__ edges) {
  static_assert(R >= 8 && R % 8 == 0, "8 slots per lane");
  static_assert(MAXE == 0 || MAXE == 2 || MAXE == 4, "edge bound");
  static_assert(MAXE == 2 || NE >= MAXE - 2, "the prefetched edges");
  constexpr int B = kPullHeadEdges;
  uint4 h = hd.h, h2 = hd.h2;
  if (h.x == h.y) return;
  h.z = CHSGA_CHK(h.z, 2 * (uint64_t)d, 12);
  h2.x = CHSGA_CHK(h2.x, 2 * (uint64_t)d, 12);
  const size_t so = (size_t)lane * 8;
  uint4* p = reinterpret_cast<uint4*>(BV + (size_t)(2 * d) * R + so);
  auto src = [&](uint32_t i) { return ldv4<COH>(BV + (size_t)i * R + so); };
  const uint4 f0 = *p;
  uint4 f = f0;
  auto relax = [&](const uint4& x, uint32_t w) {
    const uint32_t ww = min(w, 0xFFFFu) * 0x10001u;
    f.x = __vminu2(f.x, __vaddus2(x.x, ww));
    f.y = __vminu2(f.y, __vaddus2(x.y, ww));
    f.z = __vminu2(f.z, __vaddus2(x.z, ww));
    f.w = __vminu2(f.w, __vaddus2(x.w, ww));
  };
  const bool two = h.y - h.x > 1;
  const uint4 x0 = src(h.z);
  uint4 x1 = x0;
  if (two) x1 = src(h2.x);
  if constexpr (MAXE == 2) {
    relax(x0, h.w);
    if (two) relax(x1, h2.y);
    if (f.x != f0.x || f.y != f0.y || f.z != f0.z || f.w != f0.w) *p = f;
    return;
  }
  if constexpr (MAXE == 4) {
    // the head's two edges and the two prefetched after them, gathered at once
    const bool three = h.y - h.x > 2, four = h.y - h.x > 3;
    uint4 x2 = x0, x3 = x0;
    if (three) x2 = src(CHSGA_CHK((uint32_t)hd.e[0].x, 2 * (uint64_t)d, 12));
    if (four) x3 = src(CHSGA_CHK((uint32_t)hd.e[1].x, 2 * (uint64_t)d, 12));
    relax(x0, h.w);
    if (two) relax(x1, h2.y);
    if (three) relax(x2, (uint32_t)hd.e[0].y);
    if (four) relax(x3, (uint32_t)hd.e[1].y);
    if (f.x != f0.x || f.y != f0.y || f.z != f0.z || f.w != f0.w) *p = f;
    return;
  }
  uint32_t k = h.x + 2;
  int2 e[B];
#pragma unroll
  for (int q = 0; q < B; ++q) e[q] = hd.e[q];
  relax(x0, h.w);
  if (two) relax(x1, h2.y);
  for (; k < h.y; k += B) {
    uint4 x[B];
#pragma unroll
    for (int q = 0; q < B; ++q)
      if (k + q < h.y) x[q] = src(CHSGA_CHK((uint32_t)e[q].x, 2 * (uint64_t)d, 12));
#pragma unroll
    for (int q = 0; q < B; ++q)
      if (k + q < h.y) relax(x[q], (uint32_t)e[q].y);
    if (k + B < h.y) {
#pragma unroll
      for (int q = 0; q < B; ++q)
        e[q] = k + B + q < h.y ? __ldg(edges + k + B + q) : make_int2(0, 0);
    }
  }
  if (f.x != f0.x || f.y != f0.y || f.z != f0.z || f.w != f0.w) *p = f;
}

template <int R, int MAXE = 0>
__global__ void __launch_bounds__(256) k_pull_lv16(uint16_t* __restrict__ BV, uint32_t lo,
                                                   uint32_t hi, const uint4* __restrict__ head,
                                                   const int2* __restrict__ edges, uint32_t n_edges,
                                                   const StepCtl* __restrict__ ctl) {
  constexpr int G = R / 8;
  constexpr int NE = MAXE == 2 ? 0 : MAXE == 4 ? 2 : kPullHeadEdges;
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t d = lo + (uint32_t)(gt / G);
  PullHeadT<NE> hd{};
  if (d < hi) hd = pull_head<NE>(d, head, edges, n_edges);
  pdl_wait();
  if (!ctl->any_active || d >= hi) return;
  pull_lv16_item<R, false, MAXE, NE>(BV, d, (int)(gt % G), hd, edges);
}

// ---------------------------------------------------------------------------
// k_pull_lv16c: k_pull_lv16 with the target's edge list loaded by its lane
// group at once. A target's G = R / 8 lanes (G >= 8) each load one edge of
// the list after the two in the head, shuffles hand every edge to every lane,
// and each lane then issues the gathers of up to kPullBatch edges before it
// uses any of them. The chain of dependent loads per target is head ->
// edges -> gathers (the first two gathers start from the head), instead of
// one round trip per batch of four edges.
// ---------------------------------------------------------------------------
constexpr int kPullBatch = 8;

template <int R, bool COH>
__device__ __forceinline__ void pull_lv16c_item(uint16_t* BV, uint32_t d, int lane,
                                                const uint4* __restrict__ head,
                                                const int2* __restrict__ edges, uint32_t n_edges) {
  constexpr int G = R / 8;
  static_assert(G >= 8 && G <= 32 && (G & (G - 1)) == 0, "a lane group of 8 to 32 lanes per target");
  uint4 h = __ldg(head + 2 * (size_t)d);
  uint4 h2 = __ldg(head + 2 * (size_t)d + 1);
  if (h.x == h.y) return;
  CHSGA_CHK_RANGE(h.x, h.y, n_edges, 11);
  if (h.x == h.y) return;
  h.z = CHSGA_CHK(h.z, 2 * (uint64_t)d, 12);
  h2.x = CHSGA_CHK(h2.x, 2 * (uint64_t)d, 12);
  // every lane of the group has this target: the group's lanes are G
  // consecutive lanes of the warp
  const int wl = threadIdx.x & 31;
  const unsigned gmask = G == 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (wl & ~(G - 1)));
  const size_t so = (size_t)lane * 8;
  uint4* p = reinterpret_cast<uint4*>(BV + (size_t)(2 * d) * R + so);
  auto src = [&](uint32_t i) { return ldv4<COH>(BV + (size_t)i * R + so); };
  const uint4 f0 = *p;
  uint4 f = f0;
  auto relax = [&](const uint4& x, uint32_t w) {
    const uint32_t ww = min(w, 0xFFFFu) * 0x10001u;
    f.x = __vminu2(f.x, __vaddus2(x.x, ww));
    f.y = __vminu2(f.y, __vaddus2(x.y, ww));
    f.z = __vminu2(f.z, __vaddus2(x.z, ww));
    f.w = __vminu2(f.w, __vaddus2(x.w, ww));
  };
  const bool two = h.y - h.x > 1;
  const uint32_t base0 = h.x + 2;
  // this lane's edge of the first group-sized window after the head's two
  const int2 mine = base0 + (uint32_t)lane < h.y ? __ldg(edges + base0 + lane) : make_int2(0, 0);
  const uint4 x0 = src(h.z);
  uint4 x1 = x0;
  if (two) x1 = src(h2.x);
  relax(x0, h.w);
  if (two) relax(x1, h2.y);
  int2 win = mine;
  for (uint32_t base = base0; base < h.y; base += G) {
    if (base != base0)
      win = base + (uint32_t)lane < h.y ? __ldg(edges + base + lane) : make_int2(0, 0);
    const uint32_t cnt = min((uint32_t)G, h.y - base);
    for (uint32_t q = 0; q < cnt; q += kPullBatch) {
      uint4 x[kPullBatch];
      uint32_t w[kPullBatch];
#pragma unroll
      for (int b = 0; b < kPullBatch; ++b) {
        if (q + b < cnt) {
          const uint32_t sidx = (uint32_t)__shfl_sync(gmask, win.x, (int)(q + b), G);
          w[b] = (uint32_t)__shfl_sync(gmask, win.y, (int)(q + b), G);
          x[b] = src(CHSGA_CHK(sidx, 2 * (uint64_t)d, 12));
        }
      }
#pragma unroll
      for (int b = 0; b < kPullBatch; ++b)
        if (q + b < cnt) relax(x[b], w[b]);
    }
  }
  if (f.x != f0.x || f.y != f0.y || f.z != f0.z || f.w != f0.w) *p = f;
}

template <int R>
__global__ void __launch_bounds__(256) k_pull_lv16c(uint16_t* __restrict__ BV, uint32_t lo,
                                                    uint32_t hi, const uint4* __restrict__ head,
                                                    const int2* __restrict__ edges, uint32_t n_edges,
                                                    const StepCtl* __restrict__ ctl) {
  pdl_wait();
  constexpr int G = R / 8;
  if (!ctl->any_active) return;
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t d = lo + (uint32_t)(gt / G);
  if (d >= hi) return;  // whole lane groups: 256 threads hold whole groups
  pull_lv16c_item<R, false>(BV, d, (int)(gt % G), head, edges, n_edges);
}

// The graph constants of one k_down / k_down16 position: its downward list
// head (edge range, first source and weight; none at or above `mid`), its
// vertex (first char, length, string vertex) and its second in-edge. Loaded
// before the kernel's pdl_wait, like PullHead.
struct DownHead {
  uint4 h, m;
  int2 e1;
};

__device__ __forceinline__ DownHead down_head(const GraphPtrs& g, uint32_t d, uint32_t mid) {
  DownHead r;
  r.h = d < mid ? __ldg(g.dn_head + d) : make_uint4(0, 0, 0, 0);
  r.m = __ldg(g.fin + d);
  CHSGA_CHK_RANGE(r.h.x, r.h.y, g.n_dn, 13);
  r.e1 = r.h.x + 1 < r.h.y ? __ldg(g.dn_in + r.h.x + 1) : make_int2(0, 0);
  return r;
}

// ---------------------------------------------------------------------------
// k_down: positions [lo, hi). Those below `mid` first pull their downward
// in-edges (sources on higher levels, final); every position then finalises
// its vertex's chars: if the first score fell below the row value, write it
// and propagate first + (p - first) forward while it improves
// (align.hpp:381-396). Slots without closure (row 0, idle) are untouched.
// ---------------------------------------------------------------------------
template <int R, bool FIXUP, typename ST, bool COH>
__device__ __forceinline__ void down_item(const GraphPtrs& g, ST* BV, ST* T, ST* FL, uint32_t d, int lane,
                                          const DownHead& hd, const uint32_t* slot_word,
                                          unsigned long long* sm_best, bool ending_any) {
  constexpr int V = Lanes<R>::V;
  {
    const size_t so = (size_t)lane * V;
    ST* p = BV + (size_t)(2 * d) * R + so;
    // the list head and vertex words came with the head; the first score and
    // the raw last score load together (the last entry is never written
    // here; for a one-char vertex it is unused)
    uint4 h = hd.h;
    uint4 m = hd.m;
    h.z = CHSGA_CHK(h.z, 2 * (uint64_t)g.S, 14);
    m.z = CHSGA_CHK(m.z, g.S, 15);
#ifdef CHSGA_CHECKED
    // the vertex's chars first .. first + len - 1 (the fix-up writes them)
    if (!(m.y >= 1 && m.x < g.N && m.y <= g.N - m.x)) {
      chk_fail(m.x, 16);
      m.x = 0;
      m.y = 1;
    }
#endif
    IV<V> f = ld<V>(p);
    IV<V> raw{};
    if (m.y > 1) raw = ld<V>(BV + (size_t)(2 * d + 1) * R + so);
    if (h.y > h.x) {
      bool changed = false;
      auto relax = [&](const IV<V>& x, int w) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const int c = x.v[v] + w;
          if (c < f.v[v]) {
            f.v[v] = c;
            changed = true;
          }
        }
      };
      const IV<V> x0 = ld_src<V, COH>(BV + (size_t)h.z * R + so);
      if (h.y > h.x + 1) {
        const IV<V> x1 = ld_src<V, COH>(BV + (size_t)CHSGA_CHK(hd.e1.x, 2 * (uint64_t)g.S, 14) * R + so);
        relax(x0, (int)h.w);
        relax(x1, hd.e1.y);
      } else {
        relax(x0, (int)h.w);
      }
      for (uint32_t k = h.x + 2; k < h.y; ++k) {
        const int2 ew = __ldg(g.dn_in + k);
        relax(ld_src<V, COH>(BV + (size_t)CHSGA_CHK(ew.x, 2 * (uint64_t)g.S, 14) * R + so), ew.y);
      }
      if (changed) st<V>(p, f);
    }
    const uint32_t first = m.x, len = m.y;
    {
      // final first and last scores of the vertex, in char order, for the
      // next row-step (the last char ends at min(raw last, F + len - 1))
      const uint32_t sv = m.z;
      IV<V> lf = f;
      if (len > 1) {
#pragma unroll
        for (int v = 0; v < V; ++v) lf.v[v] = min(raw.v[v], f.v[v] + (int)(len - 1));
      }
      st<V>(FL + (size_t)(2 * sv) * R + so, f);
      st<V>(FL + (size_t)(2 * sv + 1) * R + so, lf);
    }
    if (!FIXUP) {
      // the row stays raw; a slot on its last row needs min over the final
      // scores = min(min over raw scores [k_row], min over swept first scores)
      if (ending_any) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const uint32_t w = COH ? slot_word[so + v] : __ldg(slot_word + so + v);
          if ((w & SW_CLOSURE) && (w & SW_ENDING))
            atomicMin(sm_best + so + v, pack_min(f.v[v], first));
        }
      }
    } else {
    IV<V> tq = ld<V>(T + (size_t)first * R + so);
    bool act[V], endg[V];
    bool any = false;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const uint32_t w = COH ? slot_word[so + v] : __ldg(slot_word + so + v);
      act[v] = (w & SW_CLOSURE) && f.v[v] < tq.v[v];
      endg[v] = act[v] && (w & SW_ENDING);
      if (act[v]) {
        tq.v[v] = f.v[v];
        if (endg[v]) atomicMin(sm_best + so + v, pack_min(f.v[v], first));
      }
      any |= act[v];
    }
    if (any) {
      st<V>(T + (size_t)first * R + so, tq);
      // first + q while it improves, every slot of the lane in one pass per char
      for (uint32_t q = 1; q < len && any; ++q) {
        ST* tp = T + (size_t)(first + q) * R + so;
        IV<V> x = ld<V>(tp);
        any = false;
#pragma unroll
        for (int v = 0; v < V; ++v) {
          if (!act[v]) continue;
          const int cand = f.v[v] + (int)q;
          if (cand < x.v[v]) {
            x.v[v] = cand;
            if (endg[v]) atomicMin(sm_best + so + v, pack_min(cand, first + q));
            any = true;
          } else {
            act[v] = false;
          }
        }
        st<V>(tp, x);
      }
    }
    }
  }
}

template <int R, bool FIXUP, typename ST>
__global__ void __launch_bounds__(256) k_down(GraphPtrs g, ST* __restrict__ BV, ST* __restrict__ T,
                                              ST* __restrict__ FL, uint32_t lo, uint32_t mid,
                                              uint32_t hi,
                                              const uint32_t* __restrict__ slot_word,
                                              unsigned long long* __restrict__ best,
                                              const StepCtl* __restrict__ ctl) {
  constexpr int G = Lanes<R>::G;
  __shared__ unsigned long long sm_best[R];
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t d = lo + (uint32_t)(gt / G);
  DownHead hd{};
  if (d < hi) hd = down_head(g, d, mid);
  pdl_wait();
  const bool ending_any = ctl->any_ending != 0;
  if (!ctl->any_active) return;
  if (ending_any) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) sm_best[r] = ~0ull;
    __syncthreads();
  }
  if (d < hi)
    down_item<R, FIXUP, ST, false>(g, BV, T, FL, d, (int)(gt % G), hd, slot_word, sm_best, ending_any);
  if (ending_any) flush_min<R>(sm_best, best);
}

// ---------------------------------------------------------------------------
// k_down16: k_down without the row fix-up (score-only steps) for 16-bit rows
// and R >= 8 slots, 8 slots per lane as four u16x2 words: the downward pull
// by saturating add and min (exact, as in k_pull_lv16), then the vertex's
// final first and last scores into FL and the first scores of slots on
// their last row into the per-slot minimum.
// ---------------------------------------------------------------------------
template <int R, bool COH, bool WF = true>
__device__ __forceinline__ void down16_item(const GraphPtrs& g, uint16_t* BV, uint16_t* FL, uint32_t d,
                                            int lane, const DownHead& hd, const uint32_t* slot_word,
                                            unsigned long long* sm_best, bool ending_any) {
  static_assert(R >= 8 && R % 8 == 0, "8 slots per lane");
  const size_t so = (size_t)lane * 8;
  uint4* p = reinterpret_cast<uint4*>(BV + (size_t)(2 * d) * R + so);
  auto src = [&](uint32_t i) { return ldv4<COH>(BV + (size_t)i * R + so); };
  uint4 h = hd.h;
  uint4 m = hd.m;
  h.z = CHSGA_CHK(h.z, 2 * (uint64_t)g.S, 14);
  m.z = CHSGA_CHK(m.z, g.S, 15);
  const uint4 f0 = *p;
  // the raw last score only matters for a vertex of two or more chars
  const uint4 raw = m.y > 1 ? *reinterpret_cast<const uint4*>(BV + (size_t)(2 * d + 1) * R + so)
                            : make_uint4(0, 0, 0, 0);
  uint4 f = f0;
  auto relax = [&](const uint4& x, uint32_t w) {
    const uint32_t ww = min(w, 0xFFFFu) * 0x10001u;
    f.x = __vminu2(f.x, __vaddus2(x.x, ww));
    f.y = __vminu2(f.y, __vaddus2(x.y, ww));
    f.z = __vminu2(f.z, __vaddus2(x.z, ww));
    f.w = __vminu2(f.w, __vaddus2(x.w, ww));
  };
  if (h.y > h.x) {
    const uint4 x0 = src(h.z);
    if (h.y > h.x + 1) {
      const uint4 x1 = src(CHSGA_CHK((uint32_t)hd.e1.x, 2 * (uint64_t)g.S, 14));
      relax(x0, h.w);
      relax(x1, (uint32_t)hd.e1.y);
    } else {
      relax(x0, h.w);
    }
    for (uint32_t k = h.x + 2; k < h.y; ++k) {
      const int2 ew = __ldg(g.dn_in + k);
      relax(src(CHSGA_CHK((uint32_t)ew.x, 2 * (uint64_t)g.S, 14)), (uint32_t)ew.y);
    }
    if (f.x != f0.x || f.y != f0.y || f.z != f0.z || f.w != f0.w) *p = f;
  }
  const uint32_t first = m.x, len = m.y, sv = m.z;
  uint4 lf = f;
  if (len > 1) {
    const uint32_t ww = min(len - 1, 0xFFFFu) * 0x10001u;
    lf.x = __vminu2(raw.x, __vaddus2(f.x, ww));
    lf.y = __vminu2(raw.y, __vaddus2(f.y, ww));
    lf.z = __vminu2(raw.z, __vaddus2(f.z, ww));
    lf.w = __vminu2(raw.w, __vaddus2(f.w, ww));
  }
  // WF = false (the delta rows read a vertex's final first score from BV[2d],
  // where it also is): only the last score goes to FL
  if (WF) *reinterpret_cast<uint4*>(FL + (size_t)(2 * sv) * R + so) = f;
  *reinterpret_cast<uint4*>(FL + (size_t)(2 * sv + 1) * R + so) = lf;
  if (ending_any) {
    const uint32_t fw[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const uint32_t w = COH ? slot_word[so + v] : __ldg(slot_word + so + v);
      if ((w & SW_CLOSURE) && (w & SW_ENDING))
        atomicMin(sm_best + so + v, pack_min((int)((fw[v >> 1] >> (16 * (v & 1))) & 0xFFFFu), first));
    }
  }
}

template <int R, bool WF = true>
__global__ void __launch_bounds__(256) k_down16(GraphPtrs g, uint16_t* __restrict__ BV,
                                                uint16_t* __restrict__ FL, uint32_t lo,
                                                uint32_t mid, uint32_t hi,
                                                const uint32_t* __restrict__ slot_word,
                                                unsigned long long* __restrict__ best,
                                                const StepCtl* __restrict__ ctl) {
  constexpr int G = R / 8;
  __shared__ unsigned long long sm_best[R];
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t d = lo + (uint32_t)(gt / G);
  DownHead hd{};
  if (d < hi) hd = down_head(g, d, mid);
  pdl_wait();
  const bool ending_any = ctl->any_ending != 0;
  if (!ctl->any_active) return;
  if (ending_any) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) sm_best[r] = ~0ull;
    __syncthreads();
  }
  if (d < hi) down16_item<R, false, WF>(g, BV, FL, d, (int)(gt % G), hd, slot_word, sm_best, ending_any);
  if (ending_any) flush_min<R>(sm_best, best);
}

// ---------------------------------------------------------------------------
// k_top: hierarchy positions [K0, S), one CTA per slot. The first/last
// scores of the region are staged in shared memory; the region's upward
// levels (low -> high) and downward levels (high -> low) then run as a
// sequence of edge chunks, each chunk a contiguous array of
// {target << 16 | source, weight} that thread 0 brings into one of
// kTopBufs shared buffers with a bulk copy, kTopBufs - 1 chunks ahead of
// the one the block relaxes (atomic min into the target's first score).
// Every thread reads the next chunk's edge count while the current one
// runs, so no global load sits between two chunks. A block chunk never
// spans two levels and ends with a block barrier, so every level sees its
// sources final; a warp chunk (negative count) holds a run of small levels,
// each padded to whole 32-edge rounds that warp 0 runs in order, separated
// by warp barriers. Edges from below the region were applied by k_pull
// before launch.
// ---------------------------------------------------------------------------
constexpr uint32_t kTopChunk = 1024;     // edges per chunk (8 KiB): the smallest chunk size
constexpr uint32_t kTopChunkMax = 4096;  // largest chunk size, for regions that leave room
constexpr uint32_t kTopBufs = 4;         // chunk buffers (copies in flight + the one in use)

struct TopPtrs {
  uint32_t K0, K, nchunks;
  const int2* chunk;   // nchunks x {first edge, edge count (even; < 0: warp chunk)}
  const int2* edges;   // chunk edges in schedule order, 16-byte aligned chunks
  const uint32_t* dv_len;  // global, by hierarchy position
  uint32_t chunk_cap;  // edges per chunk buffer
};

__host__ __device__ constexpr size_t top_smem_bytes(uint32_t K, uint32_t chunk_cap = kTopChunk) {
  return ((size_t)(2 * K + 2) * 4 + 15) / 16 * 16 + kTopBufs * (size_t)chunk_cap * 8 + kTopBufs * 8;
}

// Chunk size of a region of K vertices: the largest power of two up to
// kTopChunkMax whose buffers keep the block within `smem_cap` bytes, so
// fewer block barriers split the big levels (chunks of one level need none
// between them but for the buffer ring).
inline uint32_t top_chunk_for(uint32_t K, size_t smem_cap) {
  uint32_t c = kTopChunkMax;
  while (c > kTopChunk && top_smem_bytes(K, c) > smem_cap) c /= 2;
  return c;
}

// Edge count of a chunk of the top-region schedule (negative: warp chunk);
// the checked build clamps it to the chunk buffer.
__device__ __forceinline__ int top_chunk_count(int y, uint32_t cap) {
#ifdef CHSGA_CHECKED
  if ((uint32_t)abs(y) > cap) {
    chk_fail((uint32_t)abs(y), 19);
    return y < 0 ? -(int)cap : (int)cap;
  }
#endif
  return y;
}

// The region's sweeps for slot r by the whole block (top_smem: the block's
// dynamic shared memory, top_smem_bytes of the region). Returns false when a
// bounded wait expired (StepCtl::error is set).
template <int R, typename ST>
__device__ __forceinline__ bool top_body(ST* BV, const TopPtrs& t, StepCtl* ctl, int r,
                                         unsigned char* top_smem) {
  int* sm = reinterpret_cast<int*>(top_smem);  // [2j] first, [2j+1] last, [2K] scratch
  int2* ebuf = reinterpret_cast<int2*>(top_smem + ((size_t)(2 * t.K + 2) * 4 + 15) / 16 * 16);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(ebuf + kTopBufs * t.chunk_cap);
  // the buffers may hold what this block last wrote there through the
  // generic proxy (another phase of the persistent kernel): order those
  // writes before the bulk copies
  fence_async_shared();
  if (threadIdx.x == 0) {
    for (uint32_t b = 0; b < kTopBufs; ++b) mbar_init(&bar[b], 1);
    fence_async_shared();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t c = 0; c < kTopBufs && c < t.nchunks; ++c) {
      const int2 ch = t.chunk[c];
      bulk_load(ebuf + c * t.chunk_cap, t.edges + ch.x, (uint32_t)abs(top_chunk_count(ch.y, t.chunk_cap)) * 8,
                &bar[c]);
    }
  }
  int n_next = t.nchunks ? __ldg(&t.chunk[0].y) : 0;
  // stage the region's scores (independent loads, unrolled)
  const size_t K0 = t.K0;
  for (uint32_t j0 = threadIdx.x; j0 < t.K; j0 += 4 * blockDim.x) {
    int fv[4], lv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t j = j0 + u * blockDim.x;
      if (j < t.K) {
        const size_t d = K0 + j;
        if constexpr (R == 1 && sizeof(ST) == 4) {
          const int2 x = *reinterpret_cast<const int2*>(BV + 2 * d);
          fv[u] = x.x;
          lv[u] = x.y;
        } else {
          fv[u] = BV[(2 * d) * R + r];
          lv[u] = BV[(2 * d + 1) * R + r];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t j = j0 + u * blockDim.x;
      if (j < t.K) {
        sm[2 * j] = fv[u];
        sm[2 * j + 1] = lv[u];
      }
    }
  }
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    sm[2 * t.K] = 0;
    s_fail = 0;
  }
  __syncthreads();
  uint32_t c = 0;
  for (; c < t.nchunks; ++c) {
    const uint32_t b = c % kTopBufs;
    const int n = top_chunk_count(n_next, t.chunk_cap);
    if (c + 1 < t.nchunks) n_next = __ldg(&t.chunk[c + 1].y);
    // a thread whose wait expires flags it, skips the chunk and still
    // reaches the barrier below, so the whole block leaves the loop together
    const bool ok = mbar_wait(&bar[b], (c / kTopBufs) & 1);
    if (!ok) s_fail = 1;
    const int2* e = ebuf + b * t.chunk_cap;
    if (ok && n >= 0) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int2 x = e[i];
        atomicMin(&sm[2 * CHSGA_CHK(x.x >> 16, t.K + 1, 17)], sm[CHSGA_CHK(x.x & 0xFFFF, 2 * t.K + 2, 18)] + x.y);
      }
    } else if (ok && threadIdx.x < 32) {
      // warp chunk: a run of small levels in rounds of 32 edges, each level
      // whole rounds, the rounds ordered by the warp barrier. The buffer is
      // complete and unchanging while the chunk runs, so a round's edge is
      // loaded before the barrier that ends the round before it
      const int m = -n;  // a multiple of 32: every lane runs every round
      int2 x = (int)threadIdx.x < m ? e[threadIdx.x] : make_int2(0, 0);
      for (int i = threadIdx.x; i < m; i += 32) {
        const int2 xn = i + 32 < m ? e[i + 32] : x;
        atomicMin(&sm[2 * CHSGA_CHK(x.x >> 16, t.K + 1, 17)], sm[CHSGA_CHK(x.x & 0xFFFF, 2 * t.K + 2, 18)] + x.y);
        __syncwarp();
        x = xn;
      }
    }
    __syncthreads();
    if (s_fail) break;
    if (threadIdx.x == 0 && c + kTopBufs < t.nchunks) {
      fence_async_shared();
      const int2 ch = t.chunk[c + kTopBufs];
      bulk_load(ebuf + b * t.chunk_cap, t.edges + ch.x, (uint32_t)abs(top_chunk_count(ch.y, t.chunk_cap)) * 8,
                &bar[b]);
    }
  }
  if (s_fail) {
    // record the failure and give the copies still in flight a bounded wait
    // before the shared memory is released
    if (threadIdx.x == 0) {
      atomicOr(&ctl->error, ERR_TOP_WAIT);
      for (uint32_t k = c; k < c + kTopBufs && k < t.nchunks; ++k)
        mbar_wait(&bar[k % kTopBufs], (k / kTopBufs) & 1);
    }
    __syncthreads();
    return false;
  }
  for (uint32_t j = threadIdx.x; j < t.K; j += blockDim.x) BV[(2 * (K0 + j)) * R + r] = (ST)sm[2 * j];
  // every copy was waited for: the barriers' memory may serve other uses
  if (threadIdx.x == 0)
    for (uint32_t b = 0; b < kTopBufs; ++b) mbar_inval(&bar[b]);
  __syncthreads();
  return true;
}

template <int R, typename ST>
__global__ void __launch_bounds__(1024) k_top(ST* __restrict__ BV, TopPtrs t,
                                              const uint32_t* __restrict__ slot_word,
                                              StepCtl* __restrict__ ctl) {
  pdl_wait();
  extern __shared__ __align__(16) unsigned char top_smem[];
  if (!ctl->any_active) return;
  const int r = blockIdx.x;
  if (!(slot_word[r] & SW_CLOSURE)) return;
  top_body<R, ST>(BV, t, ctl, r, top_smem);
}

// ---------------------------------------------------------------------------
// k_store_rows: after a FIXUP row-step (rows final), copies the row every
// active slot just computed from the slot-interleaved row T into that read's
// own matrix: row slots[r].row of mats[slots[r].id], `pitch` elements per
// row. A block moves a tile of 64 chars x R slots through shared memory, so
// the read of T and each slot's 64-char write are both coalesced. Runs
// before k_advance moves the slots on.
// ---------------------------------------------------------------------------
template <int R>
__global__ void __launch_bounds__(256) k_store_rows(const uint16_t* __restrict__ T,
                                                    const SlotState* __restrict__ slots,
                                                    uint16_t* const* __restrict__ mats,
                                                    size_t pitch, uint32_t N,
                                                    const StepCtl* __restrict__ ctl) {
  pdl_wait();
  constexpr int C = 64;
  __shared__ uint16_t tile[C][R + 2];
  __shared__ uint16_t* dst[R];
  if (!ctl->any_active) return;
  const uint32_t c0 = blockIdx.x * C;
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    const SlotState st = slots[r];
    dst[r] = st.id >= 0 ? mats[st.id] + (size_t)st.row * pitch : nullptr;
  }
  for (int k = threadIdx.x; k < C * R; k += blockDim.x) {
    const int i = k / R, r = k % R;
    const uint32_t c = c0 + i;
    tile[i][r] = c < N ? T[(size_t)c * R + r] : (uint16_t)0;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < C * R; k += blockDim.x) {
    const int r = k / C, i = k % C;
    const uint32_t c = c0 + i;
    if (dst[r] && c < N) dst[r][c] = tile[i][r];
  }
}

__global__ void k_set_ptr(uint16_t** mats, uint32_t i, uint16_t* p) { mats[i] = p; }

// ---------------------------------------------------------------------------
// k_wait_selftest: the bounded mbarrier wait of k_top on a barrier that
// nothing completes. It gives up after `polls` polls and reports through the
// control block as k_top does, so the host's timeout path can be checked
// without any real wait failing.
// ---------------------------------------------------------------------------
__global__ void k_wait_selftest(StepCtl* __restrict__ ctl, uint32_t polls) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_async_shared();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0, polls)) atomicOr(&ctl->error, ERR_TOP_WAIT);
}

// ---------------------------------------------------------------------------
// k_fl_from_row: FL of a final row that was not produced by the preceding
// row-step (a checkpoint row a segment restarts from): first and last score
// of every string vertex, read from the row (R = 1, int32 or 16-bit rows).
// ---------------------------------------------------------------------------
template <typename ST>
__global__ void k_fl_from_row(GraphPtrs g, const ST* __restrict__ row, ST* __restrict__ FL) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.S) return;
  FL[2 * s] = row[g.sv_off[s]];
  FL[2 * s + 1] = row[g.sv_off[s + 1] - 1];
}

// ---------------------------------------------------------------------------
// k_advance: one block. Slots that computed their last row hand in their
// minimum (score and smallest char index reaching it); idle slots admit the
// next queued reads in order; every slot gets its word for the next step.
// Admission and completion times (device global timer, ns) are recorded per
// read. prime != 0 only recomputes the words (used after the host sets slots).
// Serving: the queue is a ring (entry i at queue[i & qmask]) that the host
// refills while the engine runs, ids index the result arrays, and every
// finished read is also appended to done_ring (entry ctl->done & qmask).
// ---------------------------------------------------------------------------
// The body runs on the first 128 threads of a block (R <= 128); the other
// threads only take part in the block barriers.
template <int R>
__device__ __forceinline__ void advance_body(SlotState* slots, const ReadDesc* queue,
                                             const unsigned char* reads, unsigned long long* best,
                                             int32_t* res_score, uint32_t* res_vertex,
                                             unsigned long long* res_t0, unsigned long long* res_t1,
                                             uint32_t* slot_word, StepCtl* ctl, int special, int prime,
                                             uint32_t qmask, CompletionRec* done_ring, int match_n) {
  static_assert(R <= 128, "one thread per slot");
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
        const unsigned long long t1 = global_ns();
        res_score[st.id] = (int32_t)(b >> 32);
        res_vertex[st.id] = (uint32_t)(b & 0xffffffffu);
        res_t1[st.id] = t1;
        const uint32_t k = atomicAdd(&ctl->done, 1u);
        if (done_ring)
          done_ring[k & qmask] = CompletionRec{st.id, (int32_t)(b >> 32), (uint32_t)(b & 0xffffffffu), 0u,
                                               res_t0[st.id], t1};
        st.id = -1;
      } else {
        st.row += 1;
      }
    }
    need = !prime && st.id < 0;
  }
  if (r < 128) s_need[r] = need ? 1u : 0u;
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
      const ReadDesc q = queue[(s_base + s_need[r]) & qmask];
      st.off = q.off;
      st.len = q.len;
      st.row = 0;
      st.id = q.id;
      best[r] = ~0ull;
      res_t0[q.id] = global_ns();
    }
    uint32_t w = 0;
    if (st.id >= 0) {
      const int byte = reads[st.off + st.row];
      w = base_code(byte, special) | (mismatch_mask(byte, special, match_n) << SW_MASK_SHIFT) |
          SW_ACTIVE;
      w |= st.row == 0 ? SW_INIT : SW_CLOSURE;
      if (st.row >= 2) w |= SW_FIX;
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
    ctl->run_next = 0;
    if (s_active) ctl->steps += 1;
  }
}

template <int R>
__global__ void __launch_bounds__(128) k_advance(SlotState* __restrict__ slots,
                                                 const ReadDesc* __restrict__ queue,
                                                 const unsigned char* __restrict__ reads,
                                                 unsigned long long* __restrict__ best,
                                                 int32_t* __restrict__ res_score,
                                                 uint32_t* __restrict__ res_vertex,
                                                 unsigned long long* __restrict__ res_t0,
                                                 unsigned long long* __restrict__ res_t1,
                                                 uint32_t* __restrict__ slot_word,
                                                 StepCtl* __restrict__ ctl, int special,
                                                 int prime, uint32_t qmask = 0xFFFFFFFFu,
                                                 CompletionRec* __restrict__ done_ring = nullptr,
                                                 int match_n = 0) {
  pdl_wait();
  advance_body<R>(slots, queue, reads, best, res_score, res_vertex, res_t0, res_t1, slot_word, ctl,
                  special, prime, qmask, done_ring, match_n);
}

// ---------------------------------------------------------------------------
// k_walk: single-thread traceback by score equality over rows
// [row_lo, row_hi] of a score matrix (row i at M + (i - row_lo) * pitch),
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

template <typename MT>
__global__ void k_walk(GraphPtrs g, const MT* __restrict__ M, size_t pitch, long long row_lo,
                       long long row_hi, uint32_t start, const unsigned char* __restrict__ read,
                       WalkOp* __restrict__ ops, uint32_t max_ops, WalkOut* __restrict__ out,
                       int match_n) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const size_t N = pitch;
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
    const MT* Rw = M + (size_t)(row - row_lo) * N;
    const MT* Pw = M + (size_t)(row - 1 - row_lo) * N;
    const int s = (int)Rw[cur];
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
      const int delta = (int)((mismatch_mask(read[row], g.special, match_n) >> key) & 1u);
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
