"""Python binding of libchsga (include/chsga.h) via ctypes.

libchsga is a B200 (sm_100a) implementation of CHSGA's ConSGA alignment DP:
score-only alignment (``align_combo``, src/align.hpp:470-531 of the
reference) and traceback (``align_read_with_traceback``,
src/traceback.hpp:588-1031). This module only marshals arguments; every
computation runs in the shared library, and importing fails loudly when the
library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# CHSGA_LIBRARY: another build of the library (the checked build,
# chsga_b200/lib_checked/libchsga.so)
LIB_PATH = os.environ.get("CHSGA_LIBRARY") or os.path.join(_HERE, "lib", "libchsga.so")
BIN_DIR = os.path.join(_HERE, "bin")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C {_HERE}` "
        "(or __graft_entry__.build())")

_lib = C.CDLL(LIB_PATH)

OK, ERR_INVALID_ARG, ERR_IO, ERR_FORMAT, ERR_CUDA, ERR_OOM, ERR_UNSUPPORTED, \
    ERR_NO_PATH, ERR_TIMEOUT, ERR_INTERNAL, ERR_BUSY = range(11)
OP_DELETE, OP_MATCHSUB, OP_INSERT = 0, 1, 2
REQ_SCORE, REQ_TRACEBACK = 0, 1
FP_PLAN, FP_MODEL, FP_ANALYTIC = 0, 1, 2
ORDER_FIFO, ORDER_LONGEST = 0, 1
ROW_AUTO, ROW_DIRECT, ROW_TILED, ROW_DPX, ROW_STREAM, ROW_DELTA = 0, 1, 2, 3, 4, 5
LAUNCH_STREAM, LAUNCH_GRAPHS, LAUNCH_PERSISTENT = 0, 1, 2
FLAG_PROFILE = 1
FLAG_MATCH_N = 2
NOALLOC_SCRATCH_BYTES = 32 << 20  # CHSGA_NOALLOC_SCRATCH_BYTES

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)


class ChsgaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"chsga status {status}: {msg}")
        self.status = status


class CsrT(C.Structure):
    _fields_ = [("n", C.c_uint64), ("m", C.c_uint64), ("offset", u64p), ("target", u32p),
                ("weight", u32p)]


class PchT(C.Structure):
    _fields_ = [("n", C.c_uint64), ("m", C.c_uint64), ("rm", C.c_uint64),
                ("num_layers", C.c_uint64), ("num_cc", C.c_uint64),
                ("rank", u32p), ("level", u32p), ("layer_offset", u32p), ("cc_offset", u32p),
                ("up_offset", u64p), ("up_v", u32p), ("up_w", u32p),
                ("down_offset", u64p), ("down_v", u32p), ("down_w", u32p)]


class GraphHostT(C.Structure):
    _fields_ = [("num_chars", C.c_uint64), ("labels", C.c_char_p), ("char_graph", CsrT),
                ("string_graph", CsrT), ("label_offsets", u64p), ("pch", PchT)]


class GenGraphCfg(C.Structure):
    _fields_ = [("backbone_len", C.c_uint64), ("seed", C.c_uint64), ("bubble_gap_mean", C.c_double),
                ("p_snp", C.c_double), ("p_indel", C.c_double), ("p_alt", C.c_double),
                ("indel_min", C.c_uint32), ("indel_max", C.c_uint32),
                ("alt_min", C.c_uint32), ("alt_max", C.c_uint32),
                ("vlen_min", C.c_uint32), ("vlen_max", C.c_uint32)]


class PchOpts(C.Structure):
    _fields_ = [("max_pop_count", C.c_uint32), ("sample_bound", C.c_double),
                ("weight_bound", C.c_uint64), ("use_label_lengths", C.c_int),
                ("seed", C.c_uint64), ("threads", C.c_int), ("print_detail", C.c_int),
                ("use_gpu", C.c_int), ("device", C.c_int)]


class GenReadsCfg(C.Structure):
    _fields_ = [("count", C.c_uint64), ("seed", C.c_uint64), ("len_min", C.c_uint32),
                ("len_max", C.c_uint32), ("sub_rate", C.c_double), ("indel_rate", C.c_double),
                ("n_rate", C.c_double), ("indel_len_max", C.c_uint32)]


class GraphStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in (
        "num_chars", "num_char_edges", "num_strings", "num_string_edges", "pch_up_edges",
        "pch_down_edges", "pch_levels", "pch_layers", "pch_ccs", "max_label_len",
        "single_char_strings")]


class LayoutStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in (
        "num_levels", "top_first_level", "top_vertices", "tiled", "tiles", "long_tiles",
        "slot_bytes", "slots_per_block", "smem_bytes", "sweep_up_targets", "sweep_up_edges",
        "sweep_down_targets", "sweep_down_edges")]


class OptsT(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_cap_bytes", C.c_uint64), ("flags", C.c_uint32)]


class BatchOpts(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("steps_per_graph", C.c_uint32), ("use_graphs", C.c_uint32),
                ("row_bits", C.c_uint32), ("row_kernel", C.c_uint32), ("top_vertices", C.c_uint32)]


class TuneTrial(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("steps_per_graph", C.c_uint32), ("row_kernel", C.c_uint32),
                ("top_vertices", C.c_uint32), ("predicted_gcups", C.c_double),
                ("measured_gcups", C.c_double)]


class TuneOpts(C.Structure):
    _fields_ = [("cost_model", C.c_void_p), ("measure_top", C.c_uint32), ("repeats", C.c_uint32)]


class TbOpts(C.Structure):
    _fields_ = [("k", C.c_int64), ("dir", C.c_char_p), ("keep_files", C.c_int),
                ("cap_bytes", C.c_uint64)]


class OpT(C.Structure):
    _fields_ = [("row", C.c_int64), ("vertex", C.c_uint32), ("op", C.c_uint8),
                ("pad", C.c_uint8 * 3)]


class TbResult(C.Structure):
    _fields_ = [("ops", C.POINTER(OpT)), ("num_ops", C.c_uint64), ("score", C.c_int32),
                ("checkpointed", C.c_uint32), ("num_checkpoints", C.c_uint64)]


class ProfileT(C.Structure):
    _fields_ = [("row_ms", C.c_double), ("sweep_up_ms", C.c_double), ("top_ms", C.c_double),
                ("sweep_down_ms", C.c_double), ("other_ms", C.c_double), ("total_ms", C.c_double),
                ("row_bits", C.c_uint64), ("rows", C.c_uint64), ("steps", C.c_uint64),
                ("launches", C.c_uint64),
                ("row_launches", C.c_uint64), ("launch_mode", C.c_uint64)]


class ServerOpts(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("steps_per_graph", C.c_uint32),
                ("queue_capacity", C.c_uint32), ("tb_workers", C.c_uint32),
                ("arena_bytes", C.c_uint64), ("hbm_budget_bytes", C.c_uint64), ("tb_k", C.c_int64),
                ("tb_cap_bytes", C.c_uint64), ("row_bits", C.c_uint32), ("max_pending", C.c_uint32),
                ("cost_model", C.c_void_p), ("footprint", C.c_uint32), ("order", C.c_uint32)]


class ServerResult(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int32), ("score", C.c_int32),
                ("vertex", C.c_uint32), ("mode", C.c_uint32), ("read_len", C.c_uint32),
                ("pad", C.c_uint32), ("submit_ns", C.c_int64), ("start_ns", C.c_int64),
                ("done_ns", C.c_int64), ("projected_bytes", C.c_uint64), ("peak_bytes", C.c_uint64),
                ("predicted_ms", C.c_float), ("pad2", C.c_uint32), ("tb", TbResult)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("pending", C.c_uint64), ("running", C.c_uint64), ("cells", C.c_uint64),
                ("wall_s", C.c_double), ("gcups", C.c_double), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("score_p50_ms", C.c_double), ("score_p99_ms", C.c_double),
                ("tb_p50_ms", C.c_double), ("tb_p99_ms", C.c_double), ("peak_tb_bytes", C.c_uint64),
                ("blocks", C.c_uint64), ("gpu_launches", C.c_uint64)]


class CmTrainOpts(C.Structure):
    _fields_ = [("epochs", C.c_uint32), ("batch", C.c_uint32), ("lr", C.c_float),
                ("keep_norm", C.c_uint32), ("seed", C.c_uint64)]


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


vp = C.c_void_p
_sig("chsga_last_error_global", C.c_char_p)
_sig("chsga_graph_read_files", C.c_int32, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
     C.c_char_p, C.POINTER(vp))
_sig("chsga_graph_view", C.c_int32, vp, C.POINTER(GraphHostT))
_sig("chsga_gfa_to_csr_text", C.c_int32, C.c_char_p, C.c_char_p, C.c_char_p)
_sig("chsga_csr_text_to_adj", C.c_int32, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p)
_sig("chsga_graph_from_gfa", C.c_int32, C.c_char_p, C.POINTER(vp))
_sig("chsga_graph_from_csr_text", C.c_int32, C.c_char_p, C.c_char_p, C.POINTER(vp))
_sig("chsga_graph_free", None, vp)
_sig("chsga_graph_write_files", C.c_int32, vp, C.c_char_p)
_sig("chsga_gen_graph", C.c_int32, C.POINTER(GenGraphCfg), C.POINTER(vp))
_sig("chsga_build_pch", C.c_int32, vp, C.POINTER(PchOpts))
_sig("chsga_graph_get_stats", C.c_int32, vp, C.POINTER(GraphStats))
_sig("chsga_check_layout", C.c_int32, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(LayoutStats))
_sig("chsga_reads_load", C.c_int32, C.c_char_p, C.c_uint64, C.POINTER(vp))
_sig("chsga_reads_from_arrays", C.c_int32, C.c_char_p, u64p, C.c_uint64, C.POINTER(vp))
_sig("chsga_reads_count", C.c_uint64, vp)
_sig("chsga_reads_data", C.c_void_p, vp)
_sig("chsga_reads_offsets", C.c_void_p, vp)
_sig("chsga_reads_write_fasta", C.c_int32, vp, C.c_char_p)
_sig("chsga_reads_free", None, vp)
_sig("chsga_gen_reads", C.c_int32, vp, C.POINTER(GenReadsCfg), C.POINTER(vp))
_sig("chsga_open", C.c_int32, C.POINTER(OptsT), C.POINTER(vp))
_sig("chsga_close", None, vp)
_sig("chsga_last_error", C.c_char_p, vp)
_sig("chsga_load_graph", C.c_int32, vp, C.POINTER(GraphHostT))
_sig("chsga_load_host_graph", C.c_int32, vp, vp)
_sig("chsga_align_scores", C.c_int32, vp, C.POINTER(C.c_char_p), u32p, C.c_uint32, i32p)
_sig("chsga_align_scores_batched", C.c_int32, vp, C.POINTER(C.c_char_p), u32p, C.c_uint32,
     C.POINTER(BatchOpts), i32p)
_sig("chsga_align_scores_noalloc", C.c_int32, vp, C.POINTER(C.c_char_p), u32p, C.c_uint32, i32p)
_sig("chsga_autotune", C.c_int32, vp, C.POINTER(C.c_char_p), u32p, C.c_uint32, C.POINTER(TuneOpts),
     C.POINTER(BatchOpts), C.POINTER(TuneTrial), C.c_uint32, C.POINTER(C.c_uint32))
_sig("chsga_align_rows", C.c_int32, vp, C.c_char_p, C.c_uint32, i32p)
_sig("chsga_align_traceback", C.c_int32, vp, C.c_char_p, C.c_uint32, C.POINTER(TbOpts),
     C.POINTER(TbResult))
_sig("chsga_tb_result_free", None, C.POINTER(TbResult))
_sig("chsga_align_traceback_batched", C.c_int32, vp, C.POINTER(C.c_char_p), u32p, C.c_uint32,
     C.POINTER(TbOpts), C.c_uint32, C.POINTER(TbResult))
_sig("chsga_ops_to_cigar", C.c_uint64, C.POINTER(OpT), C.c_uint64, C.c_char_p, C.c_uint64)
_sig("chsga_get_profile", C.c_int32, vp, C.POINTER(ProfileT))
_sig("chsga_get_read_times", C.c_int32, vp, u64p, u64p, C.c_uint32)
_sig("chsga_selftest_wait", C.c_int32, vp, C.c_uint32)
_sig("chsga_selftest_grid_wait", C.c_int32, vp, C.c_uint32)
f32p = C.POINTER(C.c_float)
_sig("chsga_cm_create", C.c_int32, C.c_int, C.c_uint64, C.POINTER(vp))
_sig("chsga_cm_free", None, vp)
_sig("chsga_cm_last_error", C.c_char_p, vp)
_sig("chsga_cm_num_params", C.c_uint32)
_sig("chsga_cm_get_params", C.c_int32, vp, f32p, f32p)
_sig("chsga_cm_set_params", C.c_int32, vp, f32p, f32p)
_sig("chsga_cm_loss_grad", C.c_int32, vp, f32p, f32p, C.c_uint32, f32p, f32p)
_sig("chsga_cm_train", C.c_int32, vp, f32p, f32p, C.c_uint32, C.POINTER(CmTrainOpts), f32p)
_sig("chsga_cm_predict", C.c_int32, vp, f32p, C.c_uint32, f32p)
_sig("chsga_cm_save", C.c_int32, vp, C.c_char_p)
_sig("chsga_cm_load", C.c_int32, vp, C.c_char_p)
_sig("chsga_cm_features", C.c_int32, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int64, C.c_uint64,
     f32p)
_sig("chsga_server_open", C.c_int32, vp, C.POINTER(ServerOpts), C.POINTER(vp))
_sig("chsga_server_selftest_fail", C.c_int32, vp)
_sig("chsga_server_submit", C.c_int32, vp, C.c_char_p, C.c_uint32, C.c_uint32,
     C.POINTER(C.c_uint64))
_sig("chsga_server_poll", C.c_int32, vp, C.POINTER(ServerResult), C.c_uint32,
     C.POINTER(C.c_uint32), C.c_int32)
_sig("chsga_server_stats_get", C.c_int32, vp, C.POINTER(ServerStats))
_sig("chsga_server_drain", C.c_int32, vp)
_sig("chsga_server_close", None, vp)
_sig("chsga_server_last_error", C.c_char_p, vp)


def _check(status: int, ctx=None):
    if status != OK:
        msg = (_lib.chsga_last_error(ctx) if ctx else _lib.chsga_last_error_global()) or b""
        raise ChsgaError(status, msg.decode(errors="replace"))


def exported_symbols() -> List[str]:
    """Names declared in include/chsga.h (for the load/export check)."""
    import re
    hdr = os.path.join(_HERE, "..", "include", "chsga.h")
    with open(hdr) as f:
        txt = f.read()
    return sorted(set(re.findall(r"\b(chsga_[a-z0-9_]+)\s*\(", txt)))


# Configurations of the benchmark workloads (graph generator settings).
GRAPH_CONFIGS = {
    # 100 kbp backbone, SNP every ~100 bp and a 1-10 bp indel every ~1 kbp
    "cfg1": dict(backbone_len=100_000, seed=1, bubble_gap_mean=1.0 / (1 / 100 + 1 / 1000),
                 p_snp=(1 / 100) / (1 / 100 + 1 / 1000), p_indel=(1 / 1000) / (1 / 100 + 1 / 1000),
                 p_alt=0.0, indel_min=1, indel_max=10, alt_min=50, alt_max=300,
                 vlen_min=1, vlen_max=32),
    # 5 Mbp backbone, a bubble every ~50 bp: 70% SNP, 20% 1-20 bp indel, 10% 50-300 bp allele
    "cfg2": dict(backbone_len=5_000_000, seed=2, bubble_gap_mean=50.0, p_snp=0.7, p_indel=0.2,
                 p_alt=0.1, indel_min=1, indel_max=20, alt_min=50, alt_max=300,
                 vlen_min=1, vlen_max=32),
    # 100 Mbp backbone, a bubble every ~30 bp, same mix as cfg2
    "cfg4": dict(backbone_len=100_000_000, seed=4, bubble_gap_mean=30.0, p_snp=0.7, p_indel=0.2,
                 p_alt=0.1, indel_min=1, indel_max=20, alt_min=50, alt_max=300,
                 vlen_min=1, vlen_max=32),
}


class Reads:
    """Concatenated read bases plus offsets (owned by the library)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load(cls, path: str, max_reads: int = 5) -> "Reads":
        h = vp()
        _check(_lib.chsga_reads_load(path.encode(), max_reads, C.byref(h)))
        return cls(h)

    @classmethod
    def from_list(cls, seqs: Sequence[bytes]) -> "Reads":
        data = b"".join(seqs)
        offs = np.zeros(len(seqs) + 1, dtype=np.uint64)
        offs[1:] = np.cumsum([len(s) for s in seqs])
        h = vp()
        _check(_lib.chsga_reads_from_arrays(data, offs.ctypes.data_as(u64p), len(seqs), C.byref(h)))
        return cls(h)

    def __len__(self):
        return int(_lib.chsga_reads_count(self._h))

    def to_list(self) -> List[bytes]:
        n = len(self)
        offs = np.ctypeslib.as_array(C.cast(_lib.chsga_reads_offsets(self._h), u64p), (n + 1,))
        total = int(offs[-1])
        data = C.string_at(_lib.chsga_reads_data(self._h), total) if total else b""
        return [data[int(offs[i]):int(offs[i + 1])] for i in range(n)]

    def write_fasta(self, path: str):
        _check(_lib.chsga_reads_write_fasta(self._h, path.encode()))

    def __del__(self):
        if getattr(self, "_h", None):
            _lib.chsga_reads_free(self._h)
            self._h = None


class HostGraph:
    """Alignment inputs held on the host: labels, char graph, string graph,
    label offsets and the contraction hierarchy."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def read_files(cls, char_adj, string_adj, pch, labels, offsets) -> "HostGraph":
        h = vp()
        _check(_lib.chsga_graph_read_files(char_adj.encode(), string_adj.encode(), pch.encode(),
                                           labels.encode(), offsets.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def read_prefix(cls, prefix: str) -> "HostGraph":
        return cls.read_files(*files_for(prefix))

    @classmethod
    def from_gfa(cls, path: str) -> "HostGraph":
        """Both orientations of a GFA v1 graph (handlegraph_to_csr); no hierarchy."""
        h = vp()
        _check(_lib.chsga_graph_from_gfa(path.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_csr_text(cls, string_csr: str, char_csr: str) -> "HostGraph":
        """handlegraph_to_csr's two CSR text files; no hierarchy."""
        h = vp()
        _check(_lib.chsga_graph_from_csr_text(string_csr.encode(), char_csr.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def generate(cls, **cfg) -> "HostGraph":
        c = GenGraphCfg(**cfg)
        h = vp()
        _check(_lib.chsga_gen_graph(C.byref(c), C.byref(h)))
        return cls(h)

    def build_pch(self, max_pop_count=500, sample_bound=1.0, weight_bound=0, use_label_lengths=True,
                  seed=0x5EED, threads=0, print_detail=False, gpu_device=None):
        """Contraction hierarchy; gpu_device runs the witness searches of each
        round on that CUDA device (the same hierarchy as the host builder)."""
        o = PchOpts(max_pop_count, sample_bound, weight_bound, int(use_label_lengths), seed, threads,
                    int(print_detail), int(gpu_device is not None), gpu_device or 0)
        _check(_lib.chsga_build_pch(self._h, C.byref(o)))
        return self

    def write_files(self, prefix: str):
        _check(_lib.chsga_graph_write_files(self._h, prefix.encode()))
        return files_for(prefix)

    def stats(self) -> dict:
        s = GraphStats()
        _check(_lib.chsga_graph_get_stats(self._h, C.byref(s)))
        return {k: int(getattr(s, k)) for k, _ in GraphStats._fields_}

    def check_layout(self, slots: int, row_bits: int, top_vertices: int = 0) -> dict:
        """Host-side pre-flight of the device layout (chsga_check_layout)."""
        st = LayoutStats()
        _check(_lib.chsga_check_layout(self._h, slots, row_bits, top_vertices, C.byref(st)))
        return {k: int(getattr(st, k)) for k, _ in LayoutStats._fields_}

    def view(self) -> GraphHostT:
        v = GraphHostT()
        _check(_lib.chsga_graph_view(self._h, C.byref(v)))
        return v

    def gen_reads(self, count, seed, len_min, len_max=None, sub_rate=0.0, indel_rate=0.0,
                  n_rate=0.0, indel_len_max=3) -> Reads:
        c = GenReadsCfg(count, seed, len_min, len_max or len_min, sub_rate, indel_rate, n_rate,
                        indel_len_max)
        h = vp()
        _check(_lib.chsga_gen_reads(self._h, C.byref(c), C.byref(h)))
        return Reads(h)

    def __del__(self):
        if getattr(self, "_h", None):
            _lib.chsga_graph_free(self._h)
            self._h = None


def files_for(prefix: str) -> Tuple[str, str, str, str, str]:
    """(-I, -i, -c, -l, -o) file names written by HostGraph.write_files."""
    return (prefix + ".char.adj", prefix + ".string.adj", prefix + ".string.out",
            prefix + ".char.labels", prefix + ".string.label_offsets")


def _read_ptrs(reads: Sequence[bytes]):
    arr = (C.c_char_p * len(reads))(*reads)
    lens = np.array([len(r) for r in reads], dtype=np.uint32)
    return arr, lens


class Context:
    """A device context with a loaded graph (chsga_open + chsga_load_graph)."""

    def __init__(self, device: int = 0, hbm_cap_bytes: int = 0, flags: int = 0):
        o = OptsT(device, hbm_cap_bytes, flags)
        h = vp()
        _check(_lib.chsga_open(C.byref(o), C.byref(h)))
        self._h = h

    def _ck(self, st):
        _check(st, self._h)

    def load(self, g: HostGraph) -> "Context":
        self._ck(_lib.chsga_load_host_graph(self._h, g._h))
        return self

    def load_view(self, v: GraphHostT) -> "Context":
        self._ck(_lib.chsga_load_graph(self._h, C.byref(v)))
        return self

    def align_scores(self, reads: Sequence[bytes]) -> np.ndarray:
        """Plain path: one read per launch sequence (align_combo)."""
        arr, lens = _read_ptrs(reads)
        out = np.zeros(len(reads), dtype=np.int32)
        self._ck(_lib.chsga_align_scores(self._h, arr, lens.ctypes.data_as(u32p), len(reads),
                                         out.ctypes.data_as(i32p)))
        return out

    def align_scores_batched(self, reads: Sequence[bytes], slots: int = 64, steps_per_graph: int = 8,
                             use_graphs: int = LAUNCH_GRAPHS, row_bits: int = 0, row_kernel: int = 0,
                             top_vertices: int = 0) -> np.ndarray:
        """chsga_align_scores_batched. use_graphs is the launch mode
        (LAUNCH_STREAM, LAUNCH_GRAPHS or LAUNCH_PERSISTENT; True/False work as 1/0)."""
        arr, lens = _read_ptrs(reads)
        out = np.zeros(len(reads), dtype=np.int32)
        o = BatchOpts(slots, steps_per_graph, int(use_graphs), row_bits, row_kernel, top_vertices)
        self._ck(_lib.chsga_align_scores_batched(self._h, arr, lens.ctypes.data_as(u32p), len(reads),
                                                 C.byref(o), out.ctypes.data_as(i32p)))
        return out

    def align_scores_noalloc(self, reads: Sequence[bytes]) -> np.ndarray:
        """Same scores as align_scores, with no device allocation per call: the
        working memory is a fixed array of NOALLOC_SCRATCH_BYTES in the library."""
        arr, lens = _read_ptrs(reads)
        out = np.zeros(len(reads), dtype=np.int32)
        self._ck(_lib.chsga_align_scores_noalloc(self._h, arr, lens.ctypes.data_as(u32p), len(reads),
                                                 out.ctypes.data_as(i32p)))
        return out

    def autotune(self, reads: Sequence[bytes], cost_model: Optional["CostModel"] = None,
                 measure_top: int = 0, repeats: int = 0):
        """(best batch options as a dict, list of trial dicts)."""
        arr, lens = _read_ptrs(reads)
        o = TuneOpts(cost_model._h if cost_model is not None else None, measure_top, repeats)
        best = BatchOpts()
        trials = (TuneTrial * 64)()
        nt = C.c_uint32()
        self._ck(_lib.chsga_autotune(self._h, arr, lens.ctypes.data_as(u32p), len(reads), C.byref(o),
                                     C.byref(best), trials, 64, C.byref(nt)))
        tr = [{k: getattr(trials[i], k) for k, _ in TuneTrial._fields_} for i in range(min(nt.value, 64))]
        return {k: getattr(best, k) for k, _ in BatchOpts._fields_}, tr

    def align_rows(self, read: bytes, num_chars: int) -> np.ndarray:
        out = np.zeros((len(read), num_chars), dtype=np.int32)
        self._ck(_lib.chsga_align_rows(self._h, read, len(read), out.ctypes.data_as(i32p)))
        return out

    def align_traceback(self, read: bytes, k: int = 500, ckpt_dir: Optional[str] = None,
                        keep_files: bool = False, cap_bytes: int = 0):
        """Returns (ops ndarray[row, vertex, op], score, checkpointed)."""
        o = TbOpts(k, ckpt_dir.encode() if ckpt_dir else None, int(keep_files), cap_bytes)
        r = TbResult()
        self._ck(_lib.chsga_align_traceback(self._h, read, len(read), C.byref(o), C.byref(r)))
        try:
            n = int(r.num_ops)
            ops = np.zeros((n, 3), dtype=np.int64)
            for i in range(n):
                x = r.ops[i]
                ops[i] = (x.row, x.vertex, x.op)
            return ops, int(r.score), bool(r.checkpointed)
        finally:
            _lib.chsga_tb_result_free(C.byref(r))

    def align_traceback_batched(self, reads: Sequence[bytes], slots: int = 32, k: int = 500,
                                cap_bytes: int = 0):
        """[(ops ndarray, score, checkpointed)] per read, as align_traceback."""
        arr, lens = _read_ptrs(reads)
        o = TbOpts(k, None, 0, cap_bytes)
        res = (TbResult * max(1, len(reads)))()
        self._ck(_lib.chsga_align_traceback_batched(self._h, arr, lens.ctypes.data_as(u32p), len(reads),
                                                    C.byref(o), slots, res))
        out = []
        for i in range(len(reads)):
            r = res[i]
            n = int(r.num_ops)
            ops = np.zeros((n, 3), dtype=np.int64)
            for j in range(n):
                x = r.ops[j]
                ops[j] = (x.row, x.vertex, x.op)
            out.append((ops, int(r.score), bool(r.checkpointed)))
            _lib.chsga_tb_result_free(C.byref(r))
        return out

    def read_times(self, n: int):
        """(admit_ns, done_ns) per non-empty read of the last score call."""
        a = np.zeros(n, dtype=np.uint64)
        d = np.zeros(n, dtype=np.uint64)
        self._ck(_lib.chsga_get_read_times(self._h, a.ctypes.data_as(u64p), d.ctypes.data_as(u64p), n))
        return a, d

    def selftest_grid_wait(self, limit_us: int = 2000) -> None:
        """Runs the persistent kernel's grid barrier with one block that never
        arrives (chsga_selftest_grid_wait): raises ChsgaError(ERR_TIMEOUT)."""
        self._ck(_lib.chsga_selftest_grid_wait(self._h, limit_us))

    def selftest_wait(self, polls: int = 4096) -> None:
        """Runs a bounded device wait that cannot succeed (chsga_selftest_wait):
        raises ChsgaError with ERR_TIMEOUT."""
        self._ck(_lib.chsga_selftest_wait(self._h, polls))

    def profile(self) -> dict:
        p = ProfileT()
        self._ck(_lib.chsga_get_profile(self._h, C.byref(p)))
        return {k: getattr(p, k) for k, _ in ProfileT._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _lib.chsga_close(self._h)
            self._h = None

    def __del__(self):
        self.close()


def ops_to_cigar(ops: np.ndarray) -> str:
    """ops_to_cigar (src/traceback.hpp:1081-1110)."""
    if len(ops) == 0:
        return ""
    letters = {OP_DELETE: "D", OP_MATCHSUB: "M", OP_INSERT: "I"}
    out, prev, run = [], letters[int(ops[0][2])], 1
    for r in ops[1:]:
        c = letters[int(r[2])]
        if c == prev:
            run += 1
        else:
            out.append(f"{run}{prev}")
            prev, run = c, 1
    out.append(f"{run}{prev}")
    return "".join(out)


class Server:
    """Serving loop over a loaded Context (chsga_server_*): score requests go
    through the continuously refilled batched engine, traceback requests to
    workers admitted by projected device footprint."""

    def __init__(self, ctx: "Context", cost_model: Optional["CostModel"] = None, **opts):
        o = ServerOpts(**opts)
        if cost_model is not None:
            o.cost_model = cost_model._h
        self._cm = cost_model
        h = vp()
        _check(_lib.chsga_server_open(ctx._h, C.byref(o), C.byref(h)))
        self._h = h
        self._ctx = ctx

    def _ck(self, st):
        if st != OK:
            msg = _lib.chsga_server_last_error(self._h) or b""
            raise ChsgaError(st, msg.decode(errors="replace"))

    def selftest_fail(self) -> None:
        """chsga_server_selftest_fail: the score lane runs a bounded device
        wait that cannot succeed at its next block and fails as after any
        expired wait."""
        self._ck(_lib.chsga_server_selftest_fail(self._h))

    def submit(self, read: bytes, mode: int = REQ_SCORE) -> int:
        t = C.c_uint64()
        self._ck(_lib.chsga_server_submit(self._h, read, len(read), mode, C.byref(t)))
        return t.value

    def try_submit(self, read: bytes, mode: int = REQ_SCORE) -> Optional[int]:
        """submit(), or None when the server answers BUSY."""
        t = C.c_uint64()
        st = _lib.chsga_server_submit(self._h, read, len(read), mode, C.byref(t))
        if st == ERR_BUSY:
            return None
        self._ck(st)
        return t.value

    def poll(self, max_results: int = 256, wait_ms: int = 0) -> List[dict]:
        buf = (ServerResult * max_results)()
        n = C.c_uint32()
        self._ck(_lib.chsga_server_poll(self._h, buf, max_results, C.byref(n), wait_ms))
        out = []
        for i in range(n.value):
            r = buf[i]
            d = {k: getattr(r, k) for k, _ in ServerResult._fields_ if k not in ("tb", "pad", "pad2")}
            if r.mode == REQ_TRACEBACK:
                m = int(r.tb.num_ops)
                ops = np.zeros((m, 3), dtype=np.int64)
                for j in range(m):
                    x = r.tb.ops[j]
                    ops[j] = (x.row, x.vertex, x.op)
                d["ops"] = ops
                d["checkpointed"] = bool(r.tb.checkpointed)
                _lib.chsga_tb_result_free(C.byref(r.tb))
            out.append(d)
        return out

    def drain(self):
        self._ck(_lib.chsga_server_drain(self._h))

    def collect(self) -> Dict[int, dict]:
        """Drains and returns every pending result by ticket."""
        self.drain()
        res = {}
        while True:
            got = self.poll(1024, 0)
            if not got:
                return res
            for d in got:
                res[d["ticket"]] = d

    def stats(self) -> dict:
        t = ServerStats()
        self._ck(_lib.chsga_server_stats_get(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _lib.chsga_server_close(self._h)
            self._h = None

    def __del__(self):
        self.close()


CM_FEATURES, CM_OUTPUTS, CM_NUM_NORM = 8, 2, 20


def _f32(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


class CostModel:
    """The FP32 MLP cost model (chsga_cm_*): trained and run on the GPU by the
    library's own kernels. Targets: (time ms, peak device bytes) per read."""

    def __init__(self, device: int = 0, seed: int = 0):
        h = vp()
        _check(_lib.chsga_cm_create(device, seed, C.byref(h)))
        self._h = h

    def _ck(self, st):
        if st != OK:
            msg = _lib.chsga_cm_last_error(self._h) or b""
            raise ChsgaError(st, msg.decode(errors="replace"))

    @staticmethod
    def num_params() -> int:
        return int(_lib.chsga_cm_num_params())

    def params(self):
        p = np.zeros(self.num_params(), np.float32)
        nm = np.zeros(CM_NUM_NORM, np.float32)
        self._ck(_lib.chsga_cm_get_params(self._h, p.ctypes.data_as(f32p), nm.ctypes.data_as(f32p)))
        return p, nm

    def set_params(self, params=None, norm=None):
        pp = None if params is None else _f32(params)
        nn = None if norm is None else _f32(norm)
        self._ck(_lib.chsga_cm_set_params(self._h, pp.ctypes.data_as(f32p) if pp is not None else None,
                                          nn.ctypes.data_as(f32p) if nn is not None else None))

    def loss_grad(self, x, y):
        x, y = _f32(x, (-1, CM_FEATURES)), _f32(y, (-1, CM_OUTPUTS))
        loss = C.c_float()
        g = np.zeros(self.num_params(), np.float32)
        self._ck(_lib.chsga_cm_loss_grad(self._h, x.ctypes.data_as(f32p), y.ctypes.data_as(f32p), len(x),
                                         C.byref(loss), g.ctypes.data_as(f32p)))
        return float(loss.value), g

    def train(self, x, y, epochs=200, batch=256, lr=3e-3, seed=0, keep_norm=False) -> float:
        x, y = _f32(x, (-1, CM_FEATURES)), _f32(y, (-1, CM_OUTPUTS))
        o = CmTrainOpts(epochs, batch, lr, int(keep_norm), seed)
        loss = C.c_float()
        self._ck(_lib.chsga_cm_train(self._h, x.ctypes.data_as(f32p), y.ctypes.data_as(f32p), len(x),
                                     C.byref(o), C.byref(loss)))
        return float(loss.value)

    def predict(self, x) -> np.ndarray:
        x = _f32(x, (-1, CM_FEATURES))
        out = np.zeros((len(x), CM_OUTPUTS), np.float32)
        self._ck(_lib.chsga_cm_predict(self._h, x.ctypes.data_as(f32p), len(x), out.ctypes.data_as(f32p)))
        return out

    def save(self, path: str):
        self._ck(_lib.chsga_cm_save(self._h, path.encode()))

    def load(self, path: str):
        self._ck(_lib.chsga_cm_load(self._h, path.encode()))

    def close(self):
        if getattr(self, "_h", None):
            _lib.chsga_cm_free(self._h)
            self._h = None

    def __del__(self):
        self.close()


def cm_features(ctx: "Context", read_len: int, mode: int = REQ_SCORE, slots: int = 1, k: int = 500,
                cap_bytes: int = 0) -> np.ndarray:
    x = np.zeros(CM_FEATURES, np.float32)
    _check(_lib.chsga_cm_features(ctx._h, read_len, mode, slots, k, cap_bytes, x.ctypes.data_as(f32p)),
           ctx._h)
    return x


def gfa_to_csr_text(gfa: str, string_csr: str, char_csr: str) -> None:
    _check(_lib.chsga_gfa_to_csr_text(gfa.encode(), string_csr.encode(), char_csr.encode()))


def csr_text_to_adj(csr: str, adj: str, labels: str, label_offsets: str) -> None:
    _check(_lib.chsga_csr_text_to_adj(csr.encode(), adj.encode(), labels.encode(), label_offsets.encode()))
