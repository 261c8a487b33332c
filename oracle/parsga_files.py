"""Input files of the reference's ParSGA driver (src/ParSGA.cpp) for a graph
of single-char vertices, and a runner for that driver (oracle/_ref/ParSGA,
compiled unchanged). Test infrastructure: ParSGA is the second comparison
method for the score-only DP, never part of the product.

The reference's own writer of these files is src/csr_to_char_graphs.cpp,
whose file output is commented out in the shipped source (lines 351-392)
and which needs the GAP benchmark suite (pvector.h, graph.h, cc.cc,
builder.h), absent from the reference tree. This module restates what it
computes (lines 82-340) and writes it in the layout ParSGA's reader expects
(src/ParSGAoverrides/read_csr.hpp:3-97):

  <prefix>.csr               n, m, n labels (one char each), n+1 offsets, m targets
  <prefix>-<B>.csr           per base B: the match-cut graph, n, m_B, n+1 offsets,
                             m_B targets -- every edge u -> v whose head label
                             differs from B (csr_to_char_graphs.cpp:159-186,
                             ALPHABET_SIZE 5)
  <prefix>-<B>.components    the vertices sorted stably by the label of their
                             connected component in the cut graph, then those
                             labels (lines 82-103: Afforest + stable integer sort)
  <prefix>-<B>-<T>.components  T+1 component-aligned thread offsets for T
                             threads (get_thread_component_offset, lines 54-77)

Component labels: connected components of the cut graph with its edges taken
as undirected, each labelled by its smallest vertex (GAP's Afforest labels
with some vertex of the component; ParSGA only needs every component's
vertices together and in index order, which the stable sort keeps).
"""
import os
import re
import subprocess
from typing import List, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PARSGA_BIN = os.path.join(HERE, "_ref", "ParSGA")
PARSGA_TB_BIN = os.path.join(HERE, "_ref", "ParSGA_traceback")
BASES = "TCGAN"  # src/config.hpp:8-9, ALPHABET_SIZE 5


def available() -> bool:
    return os.path.exists(PARSGA_BIN)


def traceback_available() -> bool:
    return os.path.exists(PARSGA_TB_BIN)


def _components(n: int, src: np.ndarray, dst: np.ndarray) -> np.ndarray:
    """Smallest vertex of each vertex's weakly connected component."""
    parent = np.arange(n, dtype=np.int64)

    def find(x):
        root = x
        while parent[root] != root:
            root = parent[root]
        while parent[x] != root:
            parent[x], x = root, parent[x]
        return root

    for u, v in zip(src.tolist(), dst.tolist()):
        a, b = find(u), find(v)
        if a != b:
            if a < b:
                parent[b] = a
            else:
                parent[a] = b
    return np.array([find(i) for i in range(n)], dtype=np.int64)


def thread_offset(t: int, T: int, n: int) -> int:
    """get_thread_offset (csr_to_char_graphs.cpp:25-31)."""
    extra, floor = n % T, n // T
    return t * (floor + 1) if t <= extra else extra * (floor + 1) + (t - extra) * floor


def thread_component_offsets(T: int, n: int, labels_sorted: np.ndarray) -> List[int]:
    """get_thread_component_offset for t = 0..T-1, then n (lines 54-77,
    97-101): from the even split point, the nearest component boundary at or
    below it, else above it, else -1 when the search reaches the previous
    thread's split point. The reference reads labels_sorted[init + i] without
    a bound; here a position past the end is no boundary."""
    out = []
    for t in range(T):
        init = thread_offset(t, T, n)
        if t == 0:
            out.append(init)
            continue
        prev = thread_offset(t - 1, T, n)
        found = -1
        i = 0
        while i < init:
            if init - i <= prev:
                break
            if init - i == 0 or labels_sorted[init - i] != labels_sorted[init - i - 1]:
                found = init - i
                break
            if init + i < n and labels_sorted[init + i] != labels_sorted[init + i - 1]:
                found = init + i
                break
            i += 1
        out.append(found)
    out.append(n)
    return out


def _ints(a) -> str:
    return " ".join(str(int(x)) for x in a)


def write_inputs(prefix: str, labels: bytes, offsets: np.ndarray, targets: np.ndarray,
                 threads: Sequence[int]) -> None:
    """Writes ParSGA's input files for the char graph (out-CSR offsets,
    targets) with one label byte per vertex."""
    n, m = len(labels), len(targets)
    lab = np.frombuffer(labels, dtype=np.uint8)
    offsets = np.asarray(offsets, dtype=np.int64)
    targets = np.asarray(targets, dtype=np.int64)
    with open(prefix + ".csr", "w") as f:
        f.write(f"{n}\n{m}\n{' '.join(chr(c) for c in lab)}\n{_ints(offsets)}\n{_ints(targets)}\n")
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(offsets))
    for b in BASES:
        keep = lab[targets] != ord(b)
        cut_adj = targets[keep]
        cut_off = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(src[keep], minlength=n), out=cut_off[1:])
        with open(f"{prefix}-{b}.csr", "w") as f:
            f.write(f"{n}\n{len(cut_adj)}\n{_ints(cut_off)}\n{_ints(cut_adj)}\n")
        comp = _components(n, src[keep], cut_adj)
        order = np.argsort(comp, kind="stable")
        with open(f"{prefix}-{b}.components", "w") as f:
            f.write(f"{_ints(order)}\n{_ints(comp[order])}\n")
        for T in threads:
            tco = thread_component_offsets(T, n, comp[order])
            with open(f"{prefix}-{b}-{T}.components", "w") as f:
                f.write(_ints(tco) + "\n")


def run(prefix: str, reads: Sequence[bytes], threads: int, workdir: str) -> np.ndarray:
    """Scores of the reads from the reference's ParSGA driver with `threads`
    OpenMP threads (parallel_align_CSR, src/ParSGAoverrides/csr_align.hpp:
    527-618; uint8 scores). The driver loads at most 5 reads per run
    (src/load_reads.hpp:5), so the reads go five at a time."""
    out = []
    for k in range(0, len(reads), 5):
        fa = os.path.join(workdir, f"parsga_reads_{k}.fa")
        with open(fa, "wb") as f:
            for i, r in enumerate(reads[k:k + 5]):
                f.write(b">r%d\n%s\n" % (i, r))
        res = subprocess.run([PARSGA_BIN, prefix, os.path.join(workdir, "parsga_out"), fa, str(threads)],
                             capture_output=True, text=True, check=True,
                             env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        m = re.search(r"^score: (.*)$", res.stdout, re.M)
        if not m:
            raise RuntimeError("ParSGA printed no score line:\n" + res.stdout[-2000:] + res.stderr[-2000:])
        out.extend(int(x) for x in m.group(1).split())
    return np.array(out, dtype=np.int32)


_TB_READ = re.compile(r'^read\[(\d+)\] = "([^"]*)"\n'
                      r'\s+CIGAR\s+: (\S*)\n'
                      r'\s+path_score\s+: (-?\d+)\s+parallel_ref : (-?\d+)\s+score_ok : (\w+)\n'
                      r'\s+last_row\s+: (-?\d+)\s+expected : (-?\d+)\s+row_ok : (\w+)', re.M)


def run_traceback(prefix: str, reads: Sequence[bytes], threads: int, workdir: str, k: int = 500) -> List[dict]:
    """Tracebacks from the reference's ParSGA traceback driver
    (par_csr_align_reads_with_traceback, src/csr_traceback.hpp:825-1072,
    checkpoints every k rows under workdir) with `threads` OpenMP threads,
    five reads per run (src/load_reads.hpp:5). Per read: the CIGAR, the
    path's score, the forward pass's score (parallel_align_CSR) and the
    driver's own checks that the two agree and that the path ends on the
    read's last row (src/ParSGA_traceback.cpp:172-209). The driver exits 1
    when a check fails; its lines are returned either way."""
    out = []
    for k0 in range(0, len(reads), 5):
        fa = os.path.join(workdir, f"parsga_tb_reads_{k0}.fa")
        with open(fa, "wb") as f:
            for i, r in enumerate(reads[k0:k0 + 5]):
                f.write(b">r%d\n%s\n" % (i, r))
        res = subprocess.run([PARSGA_TB_BIN, "-k", str(k), "-d", os.path.join(workdir, "parsga_tb_ckpt"),
                              prefix, os.path.join(workdir, "parsga_tb_out"), fa, str(threads)],
                             capture_output=True, text=True,
                             env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        if res.returncode not in (0, 1):
            raise RuntimeError(f"ParSGA_traceback exited {res.returncode}:\n" + res.stdout[-2000:]
                               + res.stderr[-2000:])
        got = [{"read": m.group(2).encode(), "cigar": m.group(3), "path_score": int(m.group(4)),
                "forward_score": int(m.group(5)), "score_ok": m.group(6) == "YES",
                "last_row": int(m.group(7)), "row_ok": m.group(9) == "YES"}
               for m in _TB_READ.finditer(res.stdout)]
        if len(got) != len(reads[k0:k0 + 5]):
            raise RuntimeError("ParSGA_traceback printed no traceback for some reads:\n" + res.stdout[-2000:])
        out.extend(got)
    return out


def cigar_read_length(cigar: str) -> int:
    """Read chars a CIGAR of the ParSGA traceback consumes: M and D ops take
    one read row each, I ops none (src/ParSGA_traceback.cpp:178-191)."""
    return sum(int(n) for n, op in re.findall(r"(\d+)([MDI])", cigar) if op in "MD")
