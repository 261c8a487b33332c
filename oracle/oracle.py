"""ORACLE — test infrastructure, not product code.

ctypes wrappers around
  * oracle/bin/libconsga_oracle.so: the CPU restatement of the reference's
    ConSGA DP (consga_oracle.cpp), and
  * oracle/_ref/libref_{fast,ckpt}.so: the reference's own src/align.hpp and
    src/traceback.hpp compiled against oracle/ref_shim (built here only when
    the reference tree is present; the built files travel with the repo).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "bin", "libconsga_oracle.so")
ORACLE_MATCHN_SO = os.path.join(HERE, "bin", "libconsga_oracle_matchN.so")
REF_FAST_SO = os.path.join(HERE, "_ref", "libref_fast.so")
REF_CKPT_SO = os.path.join(HERE, "_ref", "libref_ckpt.so")
REF_FAST_MATCHN_SO = os.path.join(HERE, "_ref", "libref_fast_matchN.so")
REF_CKPT_MATCHN_SO = os.path.join(HERE, "_ref", "libref_ckpt_matchN.so")
REF_CONSGA = os.path.join(HERE, "_ref", "ConSGA_mismatchN_dag")
REF_CONSGA_TB = os.path.join(HERE, "_ref", "ConSGA_traceback_mismatchN_dag")
REF_CONSGA_MATCHN = os.path.join(HERE, "_ref", "ConSGA_matchN_dag")
REF_CONSGA_TB_MATCHN = os.path.join(HERE, "_ref", "ConSGA_traceback_matchN_dag")
REF_CSR_TO_ADJ = os.path.join(HERE, "_ref", "csr_to_adj")
# the reference source tree (read only); CHSGA_REFERENCE overrides where it lies
REFERENCE_TREE = os.environ.get("CHSGA_REFERENCE", "/root/reference")

u64p = C.POINTER(C.c_uint64)
i32p = C.POINTER(C.c_int32)


def build(with_ref: Optional[bool] = None) -> None:
    """Compiles the restatement and, when the reference tree is present, the
    reference harness (oracle/Makefile)."""
    targets = ["oracle"]
    if with_ref is None:
        with_ref = os.path.isdir(os.path.join(REFERENCE_TREE, "src"))
    if with_ref:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, "-j8", f"REF={REFERENCE_TREE}"] + targets, check=True)


def ref_available(match_n: bool = False) -> bool:
    if match_n:
        return os.path.exists(REF_FAST_MATCHN_SO) and os.path.exists(REF_CKPT_MATCHN_SO)
    return os.path.exists(REF_FAST_SO) and os.path.exists(REF_CKPT_SO)


class _Op(C.Structure):
    _fields_ = [("row", C.c_int64), ("vertex", C.c_uint32), ("op", C.c_uint8),
                ("pad", C.c_uint8 * 3)]


def _pack(reads: Sequence[bytes]):
    data = b"".join(reads)
    offs = np.zeros(len(reads) + 1, dtype=np.uint64)
    offs[1:] = np.cumsum([len(r) for r in reads])
    return data, offs


class Oracle:
    """The restatement (consga_oracle.cpp) over the five ConSGA input files."""

    def __init__(self, files, threads: int = 0, match_n: bool = False):
        self.lib = C.CDLL(ORACLE_MATCHN_SO if match_n else ORACLE_SO)
        L = self.lib
        L.oracle_load.argtypes = [C.c_char_p] * 5 + [C.POINTER(C.c_void_p)]
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_num_chars.restype = C.c_uint64
        L.oracle_num_chars.argtypes = [C.c_void_p]
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_set_threads.argtypes = [C.c_int]
        for f in ("oracle_align_scores", "oracle_exact_scores"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_char_p, u64p, C.c_uint64, i32p]
        L.oracle_align_rows.argtypes = [C.c_void_p, C.c_char_p, C.c_uint64, i32p]
        L.oracle_traceback.argtypes = [C.c_void_p, C.c_char_p, C.c_uint64, C.c_int64, C.c_uint64,
                                       C.c_char_p, C.c_int, C.c_void_p, C.c_uint64, u64p, i32p,
                                       C.POINTER(C.c_int)]
        if threads:
            L.oracle_set_threads(threads)
        h = C.c_void_p()
        rc = L.oracle_load(*[f.encode() for f in files], C.byref(h))
        if rc:
            raise RuntimeError(L.oracle_last_error().decode())
        self.h = h
        self.num_chars = int(L.oracle_num_chars(h))

    def _err(self, rc):
        if rc:
            raise RuntimeError(f"oracle rc={rc}: {self.lib.oracle_last_error().decode()}")

    def scores(self, reads: Sequence[bytes]) -> np.ndarray:
        data, offs = _pack(reads)
        out = np.zeros(len(reads), dtype=np.int32)
        self._err(self.lib.oracle_align_scores(self.h, data, offs.ctypes.data_as(u64p), len(reads),
                                               out.ctypes.data_as(i32p)))
        return out

    def exact_scores(self, reads: Sequence[bytes]) -> np.ndarray:
        data, offs = _pack(reads)
        out = np.zeros(len(reads), dtype=np.int32)
        self._err(self.lib.oracle_exact_scores(self.h, data, offs.ctypes.data_as(u64p), len(reads),
                                               out.ctypes.data_as(i32p)))
        return out

    def rows(self, read: bytes) -> np.ndarray:
        out = np.zeros((len(read), self.num_chars), dtype=np.int32)
        self._err(self.lib.oracle_align_rows(self.h, read, len(read), out.ctypes.data_as(i32p)))
        return out

    def traceback(self, read: bytes, k: int = 500, fast_cap_bytes: int = 400 << 30,
                  ckpt_dir: str = "/tmp/consga_oracle_ckpt", cleanup: bool = True):
        cap = 4 * len(read) + 64
        ops = (_Op * cap)()
        n = C.c_uint64()
        score = C.c_int32()
        ck = C.c_int()
        self._err(self.lib.oracle_traceback(self.h, read, len(read), k, fast_cap_bytes,
                                            ckpt_dir.encode(), int(cleanup), ops, cap, C.byref(n),
                                            C.byref(score), C.byref(ck)))
        arr = np.array([(ops[i].row, ops[i].vertex, ops[i].op) for i in range(min(cap, n.value))],
                       dtype=np.int64).reshape(-1, 3)
        return arr, int(score.value), bool(ck.value)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_free(self.h)
            self.h = None


class RefHarness:
    """The reference's own align.hpp / traceback.hpp (oracle/_ref)."""

    def __init__(self, files, checkpointed: bool = False, threads: int = 0, match_n: bool = False):
        if match_n:
            self.lib = C.CDLL(REF_CKPT_MATCHN_SO if checkpointed else REF_FAST_MATCHN_SO)
        else:
            self.lib = C.CDLL(REF_CKPT_SO if checkpointed else REF_FAST_SO)
        L = self.lib
        L.ref_load.argtypes = [C.c_char_p] * 5 + [C.POINTER(C.c_void_p)]
        L.ref_last_error.restype = C.c_char_p
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_set_threads.argtypes = [C.c_int]
        for f in ("ref_align_scores", "ref_exact_scores"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_char_p, u64p, C.c_uint64, i32p]
        L.ref_align_rows.argtypes = [C.c_void_p, C.c_char_p, C.c_uint64, i32p]
        L.ref_rows_at.argtypes = [C.c_void_p, C.c_char_p, C.c_uint64, u64p, C.c_uint64, i32p]
        L.ref_traceback.argtypes = [C.c_void_p, C.c_char_p, C.c_uint64, C.c_int64, C.c_char_p,
                                    C.c_int, C.c_void_p, C.c_uint64, u64p]
        if threads:
            L.ref_set_threads(threads)
        h = C.c_void_p()
        if L.ref_load(*[f.encode() for f in files], C.byref(h)):
            raise RuntimeError(L.ref_last_error().decode())
        self.h = h
        self.files = files

    def scores(self, reads: Sequence[bytes]) -> np.ndarray:
        data, offs = _pack(reads)
        out = np.zeros(len(reads), dtype=np.int32)
        self.lib.ref_align_scores(self.h, data, offs.ctypes.data_as(u64p), len(reads),
                                  out.ctypes.data_as(i32p))
        return out

    def exact_scores(self, reads: Sequence[bytes]) -> np.ndarray:
        data, offs = _pack(reads)
        out = np.zeros(len(reads), dtype=np.int32)
        self.lib.ref_exact_scores(self.h, data, offs.ctypes.data_as(u64p), len(reads),
                                  out.ctypes.data_as(i32p))
        return out

    def rows(self, read: bytes, num_chars: int) -> np.ndarray:
        out = np.zeros((len(read), num_chars), dtype=np.int32)
        self.lib.ref_align_rows(self.h, read, len(read), out.ctypes.data_as(i32p))
        return out

    def rows_at(self, read: bytes, num_chars: int, want) -> np.ndarray:
        """Rows `want` (ascending) of the read, two rows held at a time."""
        w = np.ascontiguousarray(sorted(want), dtype=np.uint64)
        out = np.zeros((len(w), num_chars), dtype=np.int32)
        if self.lib.ref_rows_at(self.h, read, len(read), w.ctypes.data_as(u64p), len(w),
                                out.ctypes.data_as(i32p)):
            raise RuntimeError("row index beyond the read")
        return out

    def traceback(self, read: bytes, k: int = 500, ckpt_dir: str = "/tmp/ref_ckpt",
                  cleanup: bool = True) -> np.ndarray:
        cap = 4 * len(read) + 64
        ops = (_Op * cap)()
        n = C.c_uint64()
        rc = self.lib.ref_traceback(self.h, read, len(read), k, ckpt_dir.encode(), int(cleanup), ops,
                                    cap, C.byref(n))
        if rc:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return np.array([(ops[i].row, ops[i].vertex, ops[i].op) for i in range(min(cap, n.value))],
                        dtype=np.int64).reshape(-1, 3)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_free(self.h)
            self.h = None


def rescore(ops: np.ndarray, read: bytes, labels: bytes, match_n: bool = False) -> tuple:
    """The verification of src/ConSGA_traceback.cpp:190-209: path score under
    the fixed costs and the last read row the path consumes; match_n scores
    substitutions as the ALPHABET_SIZE=4 build (csr_align.hpp:45-46)."""
    score, read_pos = 0, -1
    N = ord("N")
    for row, v, op in ops:
        if op == 0:
            score += 1
            read_pos = int(row)
        elif op == 1:
            a, b = labels[int(v)], read[int(row)]
            score += 0 if (a == b or (match_n and (a == N or b == N))) else 1
            read_pos = int(row)
        else:
            score += 1
    return score, read_pos

def char_edges(files) -> set:
    """(u, v) pairs of the char graph read from the .char.adj file (files[0])."""
    toks = open(files[0]).read().split()
    n, m = int(toks[1]), int(toks[2])
    off = np.append(np.array(toks[3:3 + n], dtype=np.int64), m)
    tgt = np.array(toks[3 + n:3 + n + m], dtype=np.int64)
    return {(u, int(v)) for u in range(n) for v in tgt[off[u]:off[u + 1]]}


def check_path(ops: np.ndarray, edges: set) -> list:
    """Structure of a traceback path (ops in path order, rows ascending), as
    the reference's walks build it (traceback.hpp:483-586, 945-1011): it
    starts on row 0; a MATCHSUB step moves one row down along a char edge,
    a DELETE step one row down on the same char, an INSERT step along a char
    edge within the row. Returns the offending (previous, step) pairs."""
    ops = [tuple(int(x) for x in op) for op in ops]
    bad = [] if ops and ops[0][0] == 0 else [(None, ops[0] if ops else None)]
    for (pr, pv, _), (r, v, o) in zip(ops[:-1], ops[1:]):
        if o == 1:
            ok = r == pr + 1 and (pv, v) in edges
        elif o == 0:
            ok = r == pr + 1 and v == pv
        else:
            ok = r == pr and (pv, v) in edges
        if not ok:
            bad.append(((pr, pv), (r, v, o)))
    return bad
