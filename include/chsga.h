/*
 * chsga.h - C-ABI of libchsga, a B200 (sm_100a) implementation of CHSGA's
 * per-read sequence-to-graph alignment DP (ConSGA score-only and traceback).
 *
 * The reference is header-only C++ (src/align.hpp, src/traceback.hpp) driven
 * by src/ConSGA.cpp and src/ConSGA_traceback.cpp. Each entry point below names
 * the reference interface it replaces. Plain pointers and sizes only; no
 * exception crosses this boundary: every call returns a chsga_status and the
 * message of the last failure is kept per context (chsga_last_error) or per
 * thread for calls without a context (chsga_last_error_global).
 *
 * Scoring is the reference's fixed mismatchN scheme: match 0, substitution 1,
 * deletion 1, insertion 1 (src/ConSGA.cpp:216, src/ConSGA_traceback.cpp:128),
 * int32 arithmetic. Naming follows the reference: DELETE consumes a read base
 * and stays on the graph vertex, INSERT moves along graph edges in one row.
 */
#ifndef CHSGA_H
#define CHSGA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t chsga_status;
enum {
  CHSGA_OK = 0,
  CHSGA_ERR_INVALID_ARG = 1, /* bad pointer, size or option */
  CHSGA_ERR_IO = 2,          /* file missing, unreadable or short */
  CHSGA_ERR_FORMAT = 3,      /* file or array contents malformed */
  CHSGA_ERR_CUDA = 4,        /* CUDA runtime error */
  CHSGA_ERR_OOM = 5,         /* device memory or byte cap exceeded */
  CHSGA_ERR_UNSUPPORTED = 6, /* input outside what the GPU path handles */
  CHSGA_ERR_NO_PATH = 7,     /* traceback found no predecessor (src/traceback.hpp:571-575) */
  CHSGA_ERR_TIMEOUT = 8,     /* a bounded device-side wait gave up */
  CHSGA_ERR_INTERNAL = 9,
  CHSGA_ERR_BUSY = 10        /* server queue full: retry after chsga_server_poll */
};

/* Backpointer / path operation codes, src/traceback.hpp:168-170. */
enum { CHSGA_OP_DELETE = 0, CHSGA_OP_MATCHSUB = 1, CHSGA_OP_INSERT = 2 };

/* ------------------------------------------------------------------------- */
/* Host-side input description. These mirror what the reference drivers hold */
/* after loading their files (src/ConSGA.cpp:154-206).                       */
/* ------------------------------------------------------------------------- */

/* Out-CSR of a graph as read by read_graph() from an AdjacencyGraph file. */
typedef struct {
  uint64_t n;             /* vertices */
  uint64_t m;             /* edges */
  const uint64_t* offset; /* n+1 */
  const uint32_t* target; /* m */
  const uint32_t* weight; /* m integer weights; NULL means every weight is 1 */
} chsga_csr;

/* The contraction hierarchy, rank-ordered as build_pch's setOrderedLayer()
 * leaves it (src/CHoverrides/build_pch.hpp:1132-1220) and as align.hpp:279-345
 * indexes it through PchQuery::GC. */
typedef struct {
  uint64_t n;                   /* string vertices */
  uint64_t m;                   /* upward edges (GC.E) */
  uint64_t rm;                  /* downward in-edges (GC.in_E) */
  uint64_t num_layers;
  uint64_t num_cc;
  const uint32_t* rank;         /* n: rank of original string vertex i */
  const uint32_t* level;        /* n: level, indexed by rank */
  const uint32_t* layer_offset; /* num_layers+1: first rank of each (cc, level) layer */
  const uint32_t* cc_offset;    /* num_cc+1: first layer of each connected component */
  const uint64_t* up_offset;    /* n+1, by rank */
  const uint32_t* up_v;         /* m: head rank of u -> v, v in a higher layer */
  const uint32_t* up_w;         /* m */
  const uint64_t* down_offset;  /* n+1, by rank */
  const uint32_t* down_v;       /* rm: tail rank of v -> u, v in a higher layer */
  const uint32_t* down_w;       /* rm */
} chsga_pch;

typedef struct {
  uint64_t num_chars;             /* N = number of labels */
  const char* labels;             /* N bytes: -l file with newlines removed */
  chsga_csr char_graph;           /* -I: out-CSR over the N chars */
  chsga_csr string_graph;         /* -i: out-CSR over the S string vertices */
  const uint64_t* label_offsets;  /* -o: S+1 char offsets of each string vertex */
  chsga_pch pch;                  /* -c: hierarchy over the string graph */
} chsga_graph_host;

/* ------------------------------------------------------------------------- */
/* Host graph objects: file loading, synthetic generation, hierarchy build.  */
/* ------------------------------------------------------------------------- */

typedef struct chsga_host_graph chsga_host_graph;

/* Loads the five input files of ConSGA (-I -i -c -l -o), src/ConSGA.cpp:154-197. */
chsga_status chsga_graph_read_files(const char* char_adj, const char* string_adj,
                                    const char* pch_file, const char* labels_file,
                                    const char* label_offsets_file, chsga_host_graph** out);
/* Borrowed view of the arrays (valid until chsga_graph_free). */
chsga_status chsga_graph_view(const chsga_host_graph* g, chsga_graph_host* view);
void chsga_graph_free(chsga_host_graph* g);

/* Writes prefix + {".char.adj", ".string.adj", ".char.labels",
 * ".string.label_offsets", ".string.out"} in the reference's layouts
 * (src/csr_to_adj.cpp:46-114); ".string.out" is the hierarchy file. */
chsga_status chsga_graph_write_files(const chsga_host_graph* g, const char* prefix);

/* Graph ingest, the reference's handlegraph_to_csr -> csr_to_adj pipeline
 * (src/handlegraph_to_csr.cpp:44-247, src/csr_to_adj.cpp). libbdsg's
 * PackedGraph is not available, so the bidirected graph is read from GFA v1
 * (numeric segment ids, blunt links): node i becomes string vertex 2i
 * (forward) and 2i + 1 (reverse complement), the out-edges of an oriented
 * handle are the handles its right side links to (sorted), sequences are
 * upper-cased with other bytes as N, and the char graph is the expansion.
 * chsga_gfa_to_csr_text writes handlegraph_to_csr's two CSR text files;
 * chsga_csr_text_to_adj is csr_to_adj (AdjacencyGraph, labels, label
 * offsets, byte-identical); chsga_graph_from_gfa / _from_csr_text build a
 * host graph without a hierarchy (call chsga_build_pch). */
chsga_status chsga_gfa_to_csr_text(const char* gfa_path, const char* string_csr_out,
                                   const char* char_csr_out);
chsga_status chsga_csr_text_to_adj(const char* csr_path, const char* adj_out, const char* labels_out,
                                   const char* label_offsets_out);
chsga_status chsga_graph_from_gfa(const char* gfa_path, chsga_host_graph** out);
chsga_status chsga_graph_from_csr_text(const char* string_csr, const char* char_csr,
                                       chsga_host_graph** out);

/* Seeded variant-bubble DAG (backbone + SNP / indel / alternative-allele
 * bubbles, string vertices split to [vlen_min, vlen_max] chars). The char
 * graph is the expansion of src/handlegraph_to_csr.cpp:165-247; ids are in
 * topological order. No hierarchy is attached: call chsga_build_pch. */
typedef struct {
  uint64_t backbone_len;
  uint64_t seed;
  double bubble_gap_mean;  /* mean backbone distance between bubbles (geometric) */
  double p_snp, p_indel, p_alt; /* bubble-type mixture, sums to 1 */
  uint32_t indel_min, indel_max; /* indel allele length */
  uint32_t alt_min, alt_max;     /* alternative-allele length (both branches) */
  uint32_t vlen_min, vlen_max;   /* string vertex label length */
} chsga_gen_graph_cfg;
chsga_status chsga_gen_graph(const chsga_gen_graph_cfg* cfg, chsga_host_graph** out);

/* Contraction hierarchy over the string graph, restating build_pch
 * (src/CHoverrides/build_pch.cpp:6-131, build_pch.hpp:912-1341): witness
 * search bounded by max_pop_count, shortcut weights w1+w2+len(mid)-1 when
 * use_label_lengths (build_pch -v), levels max(level[nbr], level[u]+1),
 * rank by (cc, level, id). Replaces any hierarchy already attached. */
typedef struct {
  uint32_t max_pop_count;   /* -p, default 500 */
  double sample_bound;      /* -s, default 1 */
  uint64_t weight_bound;    /* -k, 0 = unbounded */
  int use_label_lengths;    /* -v given */
  uint64_t seed;            /* contraction priority permutation */
  int threads;              /* 0 = all */
  int print_detail;         /* -d */
  int use_gpu;              /* nonzero: each round's witness searches run on CUDA device
                             * `device` (same hierarchy: a search that outgrows the device's
                             * per-thread tables is redone on the host) */
  int device;
} chsga_pch_opts;
chsga_status chsga_build_pch(chsga_host_graph* g, const chsga_pch_opts* opts);

/* Reads: the concatenated bases plus offsets. */
typedef struct chsga_reads chsga_reads;
/* FASTA/FASTQ (gzip or plain), bases upper-cased, at most max_reads records
 * (0 = all). The reference caps at 5 (src/load_reads.hpp:5-40). */
chsga_status chsga_reads_load(const char* path, uint64_t max_reads, chsga_reads** out);
chsga_status chsga_reads_from_arrays(const char* data, const uint64_t* offsets, uint64_t n,
                                     chsga_reads** out);
uint64_t chsga_reads_count(const chsga_reads* r);
const char* chsga_reads_data(const chsga_reads* r);
const uint64_t* chsga_reads_offsets(const chsga_reads* r); /* count+1 */
chsga_status chsga_reads_write_fasta(const chsga_reads* r, const char* path);
void chsga_reads_free(chsga_reads* r);

/* Seeded reads from random source-to-sink paths at uniform offsets, with
 * substitutions, 1..indel_len_max indels and N bases. Lengths are fixed
 * (len_min == len_max) or log-uniform in [len_min, len_max]. */
typedef struct {
  uint64_t count;
  uint64_t seed;
  uint32_t len_min, len_max;
  double sub_rate, indel_rate, n_rate;
  uint32_t indel_len_max;
} chsga_gen_reads_cfg;
chsga_status chsga_gen_reads(const chsga_host_graph* g, const chsga_gen_reads_cfg* cfg,
                             chsga_reads** out);

/* Graph statistics (for logs, the cost model and the benchmark). */
typedef struct {
  uint64_t num_chars, num_char_edges, num_strings, num_string_edges;
  uint64_t pch_up_edges, pch_down_edges, pch_levels, pch_layers, pch_ccs;
  uint64_t max_label_len, single_char_strings;
} chsga_graph_stats;
chsga_status chsga_graph_get_stats(const chsga_host_graph* g, chsga_graph_stats* out);

/* Pre-flight check of a graph for the device layout, on the host only:
 * builds the layout the kernels use (labels, string vertices, hierarchy
 * order, pull lists, top region) and, for slots >= 32, the shared-memory
 * tiles of the row kernel, and checks every bound and alignment the kernels
 * rely on. No reference counterpart. */
typedef struct {
  uint64_t num_levels, top_first_level, top_vertices;
  uint64_t tiled;            /* 1 if the tile-staged row kernel applies */
  uint64_t tiles, long_tiles, slot_bytes, slots_per_block, smem_bytes;
  /* below the top region: positions with a non-empty upward / downward pull
   * list and the edges of those lists (the grid-wide sweep kernels' work) */
  uint64_t sweep_up_targets, sweep_up_edges, sweep_down_targets, sweep_down_edges;
} chsga_layout_stats;
chsga_status chsga_check_layout(const chsga_host_graph* g, uint32_t slots, uint32_t row_bits,
                                uint32_t top_vertices /* 0 = 8000, as chsga_batch_opts */,
                                chsga_layout_stats* out);

const char* chsga_last_error_global(void);

/* ------------------------------------------------------------------------- */
/* Device context and alignment                                              */
/* ------------------------------------------------------------------------- */

typedef struct chsga_ctx chsga_ctx;

typedef struct {
  int device;              /* CUDA device ordinal */
  uint64_t hbm_cap_bytes;  /* byte cap for the full score matrix; 0 = 85% of free HBM */
  uint32_t flags;          /* CHSGA_FLAG_* */
} chsga_opts;
enum {
  CHSGA_FLAG_PROFILE = 1u, /* per-phase CUDA-event timing into chsga_profile */
  /* matchN scoring, the reference's ALPHABET_SIZE=4 builds (ConSGA_matchN_dag,
   * ConSGA_traceback_matchN_dag): an 'N' in the read or in a label matches
   * every base (csr_align.hpp:45-46). Default: mismatchN, ALPHABET_SIZE=5,
   * where only equal bytes match. */
  CHSGA_FLAG_MATCH_N = 2u
};

/* Context with its own streams. One context per host thread. */
chsga_status chsga_open(const chsga_opts* opts, chsga_ctx** out);
void chsga_close(chsga_ctx* ctx);
const char* chsga_last_error(chsga_ctx* ctx);

/* Copies the graph and hierarchy to the device (the context owns the copies).
 * Replaces the inputs of InCSR/build_in_csr (src/align.hpp:214-242), the
 * rank->original map (src/ConSGA.cpp:203-206) and VertexLabelMapper. */
chsga_status chsga_load_graph(chsga_ctx* ctx, const chsga_graph_host* g);
chsga_status chsga_load_host_graph(chsga_ctx* ctx, const chsga_host_graph* g);

/* Score-only, one read per launch sequence: align_combo<int> (src/align.hpp:470-531).
 * scores_out[i] = min over the last row of read i. A read of length 0 gets
 * what the reference computes for it, row 0 against the byte '\0': 0 if a
 * label matches that byte (a '\0' label, or an 'N' under matchN), else 1. */
chsga_status chsga_align_scores(chsga_ctx* ctx, const char* const* reads, const uint32_t* lens,
                                uint32_t n, int32_t* scores_out);

/* Every final DP row of one read (after the graph-skip closure), row-major
 * len x N int32: what align_read_combo leaves in edits_src after each row
 * (src/align.hpp:430-463). For parity checks on small graphs. */
chsga_status chsga_align_rows(chsga_ctx* ctx, const char* read, uint32_t len, int32_t* rows_out);

/* Batched score-only: all reads through one slot-interleaved engine that
 * advances up to `slots` reads together, row by row; finished slots are
 * refilled on the device. No reference counterpart (the reference aligns
 * reads serially, src/align.hpp:488); results equal chsga_align_scores. */
typedef struct {
  uint32_t slots;         /* reads advanced together: 1,2,4,8,16,32,64,128; 0 = 64 */
  uint32_t steps_per_graph; /* row-steps per CUDA graph or persistent launch; 0 = default */
  uint32_t use_graphs;    /* launch mode, CHSGA_LAUNCH_*: 0 = every kernel launched from the host,
                             1 = CUDA-graph capture of the row-step sequence, 2 = the persistent
                             kernel (where it applies, else 1) */
  uint32_t row_bits;      /* storage of the score rows: 0 = 16 when every read is at most
                             65000 bases (each value of row i is at most i + 1, so this is
                             exact; arithmetic stays int32), else 32; or force 16 / 32 */
  uint32_t row_kernel;    /* CHSGA_ROW_*: which row kernel runs; 0 = AUTO */
  uint32_t top_vertices;  /* level grouping: hierarchy vertices (highest levels first) swept
                             by the one-CTA-per-slot top kernel, the levels below one grid
                             launch each; 0 = 8000; at most 23000 (the most shared memory
                             holds) */
} chsga_batch_opts;
/* Row kernels. With 16-bit rows, slots >= 2 and no string vertex label over
 * 512 chars, AUTO runs DELTA for score-only steps at 128 slots, STREAM for
 * other steps at 64 slots and up, DPX below, else DIRECT; one slot runs the
 * tile kernel (one warp per tile of whole vertices, one lane per 8 chars).
 * DELTA (128 slots, score-only) = STREAM over rows stored
 * as the raw first score of every vertex (16 bits per slot) and, per char,
 * the difference to the char before in 2 bits per slot (consecutive chars of
 * a vertex differ by at most 1 in every row): about 0.4 bytes per cell (0.25
 * for the differences, the rest for the first scores, 11.6 chars per vertex
 * on the config-2 graph) instead of 2, bound by instruction issue rather than
 * memory.
 * DIRECT = one thread group per string vertex, 16- or 32-bit rows;
 * TILED = shared-memory tiles of consecutive string vertices staged by TMA
 * bulk copies (slots >= 32); DPX = two 16-bit scores per register on the
 * DPX min/add units, one thread group per string vertex; STREAM = DPX with
 * one warp per run of 32 consecutive string vertices, loading the next
 * vertex's inputs while the current one computes (slots >= 64). */
/* Launch modes of the row-step sequence (chsga_batch_opts::use_graphs).
 * PERSISTENT runs a block of steps_per_graph row-steps as one cooperative
 * launch of the persistent row-step kernel: the row update, every hierarchy
 * level and the slot advance as phases of one kernel, separated by bounded
 * grid barriers. It applies to 16-bit rows with the AUTO row kernel and
 * string vertices of at most 512 chars (one slot: at most ~240); otherwise
 * GRAPHS runs. */
enum {
  CHSGA_LAUNCH_STREAM = 0,
  CHSGA_LAUNCH_GRAPHS = 1,
  CHSGA_LAUNCH_PERSISTENT = 2
};
enum {
  CHSGA_ROW_AUTO = 0,
  CHSGA_ROW_DIRECT = 1,
  CHSGA_ROW_TILED = 2,
  CHSGA_ROW_DPX = 3,
  CHSGA_ROW_STREAM = 4,
  CHSGA_ROW_DELTA = 5
};
chsga_status chsga_align_scores_batched(chsga_ctx* ctx, const char* const* reads,
                                        const uint32_t* lens, uint32_t n,
                                        const chsga_batch_opts* opts, int32_t* scores_out);

/* Score-only alignment that allocates no device memory. It has no
 * counterpart in the reference.
 *
 * Some callers may not allocate GPU memory once they are running: a
 * service that hands the free HBM to its own pool at start-up, or a loop
 * that cannot afford the device-wide synchronisation cudaMalloc may imply.
 * They load the graph at start-up (chsga_load_graph allocates the graph's
 * arrays then) and align with this call. It returns the same scores as
 * chsga_align_scores for the same reads. Every per-call buffer comes from
 * one fixed array of CHSGA_NOALLOC_SCRATCH_BYTES inside the library: read
 * bytes, read queue, two 16-bit score rows, per-vertex boundary scores,
 * slot state and results. The call makes no cudaMalloc, no cudaFree and no
 * other allocating call.
 *
 * - The CUDA driver reserves the array on each GPU where it loads the
 *   library's device code, and the GPU keeps it until the process exits.
 * - The first call on a device looks up the array's device address, so
 *   make that first call before any stream capture starts. The library
 *   keeps that address for the life of the process: resetting the device
 *   (cudaDeviceReset, or tearing down its primary context) after the first
 *   call is not supported.
 * - The call fails with CHSGA_ERR_OOM, and runs nothing, when the graph and
 *   the reads need more than the array holds. The need is about
 *   4 N + 8 S + (read bytes) + 52 n bytes, where N = chars and S = string
 *   vertices, each part rounded up to 256 bytes.
 * - It fails with CHSGA_ERR_UNSUPPORTED for a read longer than 65000 bases,
 *   because its rows are 16-bit.
 * - All calls on one device share the array, which keeps the last call's
 *   contents. The call clears the slot, queue and control state before it
 *   starts. Calls whose GPU work overlapped would race on the array. The
 *   library holds a per-device lock for the whole call, and the call
 *   returns only after its GPU work is done, so calls made through it do
 *   not overlap.
 * - chsga_get_profile and chsga_get_read_times do not report on this call. */
#define CHSGA_NOALLOC_SCRATCH_BYTES (32u << 20)
chsga_status chsga_align_scores_noalloc(chsga_ctx* ctx, const char* const* reads,
                                        const uint32_t* lens, uint32_t n, int32_t* scores_out);

/* Traceback of one read: align_read_with_traceback<int> (src/traceback.hpp:588-1031).
 * If len x N x 4 bytes fit under the byte cap the full score matrix stays in
 * HBM and the path is walked by score equality (src/traceback.hpp:483-586);
 * otherwise rows 0, k, 2k, ... are copied to pinned host memory and segments
 * are recomputed on the device before the walk. */
typedef struct {
  int64_t k;              /* checkpoint interval, default 500 (-k) */
  const char* dir;        /* if non-NULL, checkpoint rows are also written as
                             dir/row_<i>.bin (src/traceback.hpp:215-227) */
  int keep_files;         /* 0: erase row files after use, like cleanup=true */
  uint64_t cap_bytes;     /* 0: context cap; forces the checkpointed path when small */
} chsga_tb_opts;

typedef struct {
  int64_t row;      /* read position; INSERT keeps the row */
  uint32_t vertex;  /* char index */
  uint8_t op;       /* CHSGA_OP_* */
  uint8_t pad[3];
} chsga_op;         /* AlignOp, src/traceback.hpp:185-189 */

typedef struct {
  chsga_op* ops;      /* forward order, owned by the library */
  uint64_t num_ops;
  int32_t score;      /* min over the last row */
  uint32_t checkpointed; /* 1 if the checkpointed path ran */
  uint64_t num_checkpoints;
} chsga_tb_result;
chsga_status chsga_align_traceback(chsga_ctx* ctx, const char* read, uint32_t len,
                                   const chsga_tb_opts* opts, chsga_tb_result* out);
void chsga_tb_result_free(chsga_tb_result* r);

/* Tracebacks of many reads; each result equals chsga_align_traceback on that
 * read. Reads whose full matrix fits the cap (and are at most 65000 bases,
 * with no checkpoint directory requested) run together as slots of the
 * batched engine with every row final: after each row-step the rows are
 * copied into one 16-bit matrix per read, and a read is walked as soon as it
 * finishes. Reads are taken longest first in groups of similar length, each
 * group with as many slots (4 to `slots`, a power of two; 0 = 64) as its
 * matrices fit in device memory together. The others take the one-read
 * path. Batching has no reference counterpart (the reference
 * traces reads one after another, src/ConSGA_traceback.cpp:160-180). */
chsga_status chsga_align_traceback_batched(chsga_ctx* ctx, const char* const* reads,
                                           const uint32_t* lens, uint32_t n,
                                           const chsga_tb_opts* opts, uint32_t slots,
                                           chsga_tb_result* out);

/* ops_to_cigar (src/traceback.hpp:1081-1110): run-length string with D
 * (DELETE), M (MATCHSUB), I (INSERT). Writes at most cap bytes including the
 * terminator; returns the full length needed (excluding the terminator). */
uint64_t chsga_ops_to_cigar(const chsga_op* ops, uint64_t n, char* buf, uint64_t cap);

/* Device timing of the last score call. total_ms: CUDA-event time of the
 * whole device sequence (every row-step, reads already resident; the batched
 * engine's CUDA graph is built on the host before the first event). With
 * CHSGA_FLAG_PROFILE (CUDA graphs off, one sync per row-step) the five kernel
 * groups of every row-step are timed with CUDA events: row_ms (k_row),
 * sweep_up_ms (upward level kernels), top_ms (top region), sweep_down_ms
 * (downward levels with the final propagation), other_ms (slot advance). */
typedef struct {
  double row_ms, sweep_up_ms, top_ms, sweep_down_ms, other_ms, total_ms;
  uint64_t row_bits;      /* 16 or 32: storage width of the score rows */
  uint64_t rows;          /* read rows computed */
  uint64_t steps;         /* row-steps that had work */
  uint64_t launches;      /* kernels launched by those steps */
  uint64_t row_launches;  /* k_row launches (row phases of the persistent kernel) */
  uint64_t launch_mode;   /* how the row-steps ran: CHSGA_LAUNCH_* */
} chsga_profile;
chsga_status chsga_get_profile(chsga_ctx* ctx, chsga_profile* out);

/* Per-read admission and completion times of the last score call (device
 * global timer, ns), in the order of the non-empty reads passed in. No
 * reference counterpart: used for per-read latency percentiles. */
chsga_status chsga_get_read_times(chsga_ctx* ctx, uint64_t* admit_ns, uint64_t* done_ns, uint32_t n);

/* Self-test of the device-side failure path, no reference counterpart: one
 * kernel runs the hierarchy sweep's bounded mbarrier wait on a barrier that
 * nothing completes, gives up after `polls` polls and flags the control
 * block; the call then returns CHSGA_ERR_TIMEOUT exactly as an alignment
 * whose wait expired would, and the context stays usable. */
chsga_status chsga_selftest_wait(chsga_ctx* ctx, uint32_t polls);

/* Self-test of the persistent kernel's grid barrier, no reference
 * counterpart: two blocks meet at a barrier that one of them never reaches;
 * the other gives up after limit_us microseconds of the device's global
 * timer, sets the abort word every other waiting block watches and flags
 * the control block. Returns CHSGA_ERR_TIMEOUT as a persistent launch whose
 * barrier expired would; the context stays usable. */
chsga_status chsga_selftest_grid_wait(chsga_ctx* ctx, uint32_t limit_us);

/* ------------------------------------------------------------------------- */
/* Autotuner (no reference counterpart)                                      */
/* ------------------------------------------------------------------------- */

/* Chooses chsga_batch_opts for a read mix: reads per launch (slots),
 * row-steps per CUDA graph, the row kernel and the level grouping
 * (top_vertices). Candidates run chsga_align_scores_batched on the given
 * sample and the fastest (device time) wins; every candidate must return
 * the same scores (else CHSGA_ERR_INTERNAL). With a trained cost model only
 * the `measure_top` candidates of highest predicted throughput are run. */
typedef struct {
  uint32_t slots, steps_per_graph, row_kernel, top_vertices;
  double predicted_gcups;  /* cost model's estimate; 0 without one */
  double measured_gcups;   /* 0 when not run */
} chsga_tune_trial;

typedef struct {
  struct chsga_cost_model* cost_model;  /* optional ranking of the candidates */
  uint32_t measure_top;                 /* with a cost model: candidates run; 0 = 4 */
  uint32_t repeats;                     /* timed runs per candidate, fastest kept; 0 = 2 */
} chsga_tune_opts;

chsga_status chsga_autotune(chsga_ctx* ctx, const char* const* reads, const uint32_t* lens,
                            uint32_t n, const chsga_tune_opts* opts, chsga_batch_opts* best,
                            chsga_tune_trial* trials, uint32_t max_trials, uint32_t* n_trials);

/* ------------------------------------------------------------------------- */
/* Serving loop (no reference counterpart: the reference aligns a fixed read */
/* set serially, src/align.hpp:488)                                          */
/* ------------------------------------------------------------------------- */

/* A server takes reads as they arrive and keeps the context's graph and
 * hierarchy resident. Score requests run through a continuously refilled
 * batched engine: `slots` reads advance together, a finished slot takes the
 * next queued read on the device, and reads submitted while others run are
 * published between CUDA-graph blocks of row-steps. Traceback requests run
 * on `tb_workers` worker contexts that share the graph; each is admitted
 * when its projected device footprint (full matrix, or the checkpointed
 * path's rows) fits what the running ones leave of `hbm_budget_bytes`.
 * Results are the same as chsga_align_scores / chsga_align_traceback on
 * the same read, whatever else is in flight. The server is internally
 * synchronised: any thread may submit and poll. The context must outlive
 * the server and must not be reloaded while it runs. */
typedef struct chsga_server chsga_server;

typedef struct {
  uint32_t slots;            /* score reads advanced together: 2..128 (power of 2); 0 = 128 */
  uint32_t steps_per_graph;  /* row-steps per CUDA-graph launch; 0 = 8 */
  uint32_t queue_capacity;   /* score reads queued or running on the device (power of 2); 0 = 4096 */
  uint32_t tb_workers;       /* traceback requests running at once; 0 = 2 */
  uint64_t arena_bytes;      /* device bytes for the bases of queued score reads; 0 = 64 MiB */
  uint64_t hbm_budget_bytes; /* device bytes running traceback requests may hold; 0 = 50% of free */
  int64_t tb_k;              /* checkpoint interval of traceback requests; 0 = 500 */
  uint64_t tb_cap_bytes;     /* full-matrix byte cap of a traceback request; 0 = the context's */
  uint32_t row_bits;         /* score rows: 16 (reads <= 65000 bases) or 32; 0 = 16 */
  uint32_t max_pending;      /* requests waiting for admission before submit says BUSY; 0 = 2^20 */
  struct chsga_cost_model* cost_model; /* predicts traceback time and footprint (may be NULL) */
  uint32_t footprint;        /* projection used for admission, CHSGA_FP_*; 0 = PLAN */
  uint32_t order;            /* admission order of waiting score reads, CHSGA_ORDER_*; 0 = FIFO */
} chsga_server_opts;

/* FIFO: arrival order (latency-fair). LONGEST: the longest waiting read
 * first (throughput: long reads start early and the engine does not end a
 * stream with a few long reads running alone in mostly idle slots). */
enum { CHSGA_ORDER_FIFO = 0, CHSGA_ORDER_LONGEST = 1 };

/* How a traceback request's device footprint is projected for admission:
 * PLAN     the allocation plan of the traceback (full matrix, or the
 *          checkpointed path's row ring and largest recompute segment);
 * MODEL    the cost model's prediction (cost_model must be set);
 * ANALYTIC the |V| x |read| fallback, 4 N len bytes (a full matrix). */
enum { CHSGA_FP_PLAN = 0, CHSGA_FP_MODEL = 1, CHSGA_FP_ANALYTIC = 2 };

enum { CHSGA_REQ_SCORE = 0, CHSGA_REQ_TRACEBACK = 1 };

typedef struct {
  uint64_t ticket;       /* from chsga_server_submit */
  int32_t status;        /* chsga_status of this request */
  int32_t score;
  uint32_t vertex;       /* score requests: smallest char index reaching the score */
  uint32_t mode;         /* CHSGA_REQ_* */
  uint32_t read_len;
  uint32_t pad;
  int64_t submit_ns;     /* host steady-clock ns: submitted, */
  int64_t start_ns;      /* admitted to the device, */
  int64_t done_ns;       /* finished */
  uint64_t projected_bytes; /* traceback: footprint admission counted */
  uint64_t peak_bytes;      /* traceback: device bytes the request allocated at its peak */
  float predicted_ms;       /* traceback with a cost model: predicted time, else 0 */
  uint32_t pad2;
  chsga_tb_result tb;    /* traceback requests; free with chsga_tb_result_free */
} chsga_server_result;

typedef struct {
  uint64_t submitted, completed, failed, pending, running;
  uint64_t cells;            /* sum over completed requests of read length x N */
  double wall_s;             /* first submit to last completion */
  double gcups;              /* cells / wall_s / 1e9 */
  double p50_ms, p99_ms;     /* latency submit -> done, all completed requests */
  double score_p50_ms, score_p99_ms, tb_p50_ms, tb_p99_ms;
  uint64_t peak_tb_bytes;    /* largest projected footprint held by running tracebacks */
  uint64_t blocks;           /* CUDA-graph blocks launched by the score lane */
  uint64_t gpu_launches;     /* kernels launched by the score lane */
} chsga_server_stats;

chsga_status chsga_server_open(chsga_ctx* ctx, const chsga_server_opts* opts, chsga_server** out);
/* Queues one request (the read is copied). CHSGA_ERR_BUSY when max_pending
 * requests already wait; CHSGA_ERR_OOM when a traceback could never fit the
 * budget; CHSGA_ERR_UNSUPPORTED for a score read over 65000 bases with
 * 16-bit rows. */
/* Self-test of the serving loop's failure path, no reference counterpart:
 * at its next block of row-steps the score lane also runs a bounded
 * device-side wait that cannot succeed (as chsga_selftest_wait does)
 * against its control block. The lane then fails as it would after any
 * expired device wait: every waiting and running score request completes
 * with CHSGA_ERR_TIMEOUT, later score submissions are refused with it, and
 * the context stays usable (a new server on it aligns as before). Nothing
 * happens until score work is on the lane. */
chsga_status chsga_server_selftest_fail(chsga_server* srv);

chsga_status chsga_server_submit(chsga_server* s, const char* read, uint32_t len, uint32_t mode,
                                 uint64_t* ticket);
/* Moves up to `max` finished results to `out`; waits up to wait_ms (-1 =
 * until one is ready, 0 = not at all) when none is ready. */
chsga_status chsga_server_poll(chsga_server* s, chsga_server_result* out, uint32_t max,
                               uint32_t* n_out, int32_t wait_ms);
chsga_status chsga_server_stats_get(chsga_server* s, chsga_server_stats* out);
/* Waits until every submitted request has finished (results stay pollable). */
chsga_status chsga_server_drain(chsga_server* s);
/* Drains, stops the engine and workers, frees unpolled results. */
void chsga_server_close(chsga_server* s);
const char* chsga_server_last_error(chsga_server* s);

/* ------------------------------------------------------------------------- */
/* Learned cost model (no reference counterpart)                             */
/* ------------------------------------------------------------------------- */

/* FP32 MLP, 8 features -> 64 -> 64 -> 2 outputs (ReLU), trained and run by
 * the library's own CUDA kernels. Outputs: per-read device time in ms and
 * peak device bytes, learned in log space. It feeds the serving loop's
 * admission control (chsga_server_opts.cost_model) and the autotuner; the
 * fallback without it is the analytic |V| x |read| model; it never changes
 * a score. Parameters: W1[8][64] b1[64] W2[64][64] b2[64] W3[64][2] b3[2];
 * normalisation: x mean[8], x std[8], log-target mean[2], log-target std[2]. */
#define CHSGA_CM_FEATURES 8
#define CHSGA_CM_HIDDEN 64
#define CHSGA_CM_OUTPUTS 2
#define CHSGA_CM_NUM_PARAMS 4866
#define CHSGA_CM_NUM_NORM 20
typedef struct chsga_cost_model chsga_cost_model;

typedef struct {
  uint32_t epochs;     /* 0 = 200 */
  uint32_t batch;      /* mini-batch size, 0 = 256 */
  float lr;            /* Adam step, 0 = 3e-3 */
  uint32_t keep_norm;  /* 1: keep the current normalisation instead of fitting it */
  uint64_t seed;       /* shuffling */
} chsga_cm_train_opts;

chsga_status chsga_cm_create(int device, uint64_t seed, chsga_cost_model** out);
void chsga_cm_free(chsga_cost_model* m);
const char* chsga_cm_last_error(chsga_cost_model* m);
uint32_t chsga_cm_num_params(void);
chsga_status chsga_cm_get_params(chsga_cost_model* m, float* params, float* norm);
chsga_status chsga_cm_set_params(chsga_cost_model* m, const float* params, const float* norm);
/* x: n x 8 features; y: n x 2 targets (time ms, bytes; both > 0). Loss
 * 1/(2n) sum (o - t)^2 over standardised log targets t, and its gradient
 * with respect to the parameters (for gradient checks). */
chsga_status chsga_cm_loss_grad(chsga_cost_model* m, const float* x, const float* y, uint32_t n,
                                float* loss, float* grad);
/* Adam on mini-batches; fits the normalisation first unless keep_norm. */
chsga_status chsga_cm_train(chsga_cost_model* m, const float* x, const float* y, uint32_t n,
                            const chsga_cm_train_opts* opts, float* final_loss);
/* y_out: n x 2 predictions (time ms, bytes). */
chsga_status chsga_cm_predict(chsga_cost_model* m, const float* x, uint32_t n, float* y_out);
chsga_status chsga_cm_save(chsga_cost_model* m, const char* path);
chsga_status chsga_cm_load(chsga_cost_model* m, const char* path);
/* Features of one request on the context's graph: log2(len + 1), log2 N,
 * log2 S, log2(hierarchy edges + 1), log2(hierarchy levels + 1),
 * log2(slots), traceback (0/1), log2(k) when the traceback is checkpointed
 * under cap_bytes (0 = the context's cap) else 0. */
chsga_status chsga_cm_features(chsga_ctx* ctx, uint32_t read_len, uint32_t mode, uint32_t slots,
                               int64_t k, uint64_t cap_bytes, float* x_out);

#ifdef __cplusplus
}
#endif
#endif /* CHSGA_H */
