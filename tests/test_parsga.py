"""ParSGA as a second comparison method (src/ParSGA.cpp, parallel_align_CSR
in src/ParSGAoverrides/csr_align.hpp:527-618, and src/ParSGA_traceback.cpp,
par_csr_align_reads_with_traceback in src/csr_traceback.hpp:825-1072), on
graphs of single-char vertices, where ConSGA's sweep quirk cannot arise and
every method computes the exact DP.

The reference's ParSGA driver is compiled unchanged in oracle/_ref; its
per-base match-cut graphs, component orders and thread offsets are written
by oracle/parsga_files.py (a restatement of src/csr_to_char_graphs.cpp:
82-340, whose file output is commented out in the shipped source). Its
scores, at 1, 2 and 4 threads, must equal the reference's serial exact DP
(serial_align_CSR, csr_align.hpp:270-383) and the ConSGA oracle."""
import os

import numpy as np
import pytest

import oracle as orc
import parsga_files as pf
from conftest import gen_graph

pytestmark = pytest.mark.skipif(not (pf.available() and orc.ref_available()),
                                reason="the reference's ParSGA driver is not built (oracle/_ref)")


def _char_csr(files):
    toks = open(files[0]).read().split()
    n, m = int(toks[1]), int(toks[2])
    off = np.append(np.array(toks[3:3 + n], dtype=np.int64), m)
    tgt = np.array(toks[3 + n:3 + n + m], dtype=np.int64)
    return off, tgt


def test_thread_offsets_follow_component_boundaries():
    # components [0,0,0,3,3,5,5,5,5,9]: the even split points 0/4/7 of three
    # threads move to the nearest component boundary (or -1: none found)
    lab = np.array([0, 0, 0, 3, 3, 5, 5, 5, 5, 9])
    assert pf.thread_offset(0, 3, 10) == 0 and pf.thread_offset(1, 3, 10) == 4
    assert pf.thread_offset(2, 3, 10) == 7
    tco = pf.thread_component_offsets(3, 10, lab)
    assert tco[0] == 0 and tco[-1] == 10
    for t in tco[1:-1]:
        assert t == -1 or lab[t] != lab[t - 1]


@pytest.mark.parametrize("seed", [41, 42, 43])
def test_parsga_equals_serial_exact_dp_and_oracle(tmp_path, seed):
    g, files = gen_graph(tmp_path, f"p{seed}", backbone_len=1500, seed=seed, vlen_min=1, vlen_max=1,
                         bubble_gap_mean=6.0, p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=2, alt_max=20)
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    off, tgt = _char_csr(files)
    prefix = str(tmp_path / f"par{seed}")
    pf.write_inputs(prefix, labels, off, tgt, threads=(1, 2, 4))
    # cut graphs: exactly the edges whose head label differs from the base
    for b in pf.BASES:
        toks = open(f"{prefix}-{b}.csr").read().split()
        assert int(toks[1]) == int(np.sum(np.frombuffer(labels, np.uint8)[tgt] != ord(b)))
    reads = g.gen_reads(10, seed, 20, 90, sub_rate=0.05, indel_rate=0.04, n_rate=0.02).to_list()
    want = orc.RefHarness(files).exact_scores(reads)
    np.testing.assert_array_equal(orc.Oracle(files).scores(reads), want)
    for T in (1, 2, 4):
        got = pf.run(prefix, reads, T, str(tmp_path))
        np.testing.assert_array_equal(got, want, err_msg=f"{T} threads")


@pytest.mark.skipif(not pf.traceback_available(), reason="the reference's ParSGA traceback driver is not built")
@pytest.mark.parametrize("seed,k", [(44, 500), (45, 16)])
def test_parsga_traceback_paths_score_the_optimum(tmp_path, seed, k):
    """The reference's ParSGA traceback (par_csr_align_reads_with_traceback,
    src/csr_traceback.hpp:825-1072, checkpointed every k rows; k = 16 makes
    every read of 40+ bases recompute several segments): every path's score
    equals the ConSGA oracle's optimum, the driver's own checks pass (path
    score = its forward pass, path ends on the read's last row), and the
    CIGAR consumes every read base."""
    g, files = gen_graph(tmp_path, f"t{seed}", backbone_len=1200, seed=seed, vlen_min=1, vlen_max=1,
                         bubble_gap_mean=6.0, p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=2, alt_max=20)
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    off, tgt = _char_csr(files)
    prefix = str(tmp_path / f"tb{seed}")
    pf.write_inputs(prefix, labels, off, tgt, threads=(2,))
    reads = g.gen_reads(10, seed, 40, 120, sub_rate=0.05, indel_rate=0.04, n_rate=0.02).to_list()
    want = orc.Oracle(files).scores(reads)
    got = pf.run_traceback(prefix, reads, 2, str(tmp_path), k=k)
    assert [r["read"] for r in got] == reads
    np.testing.assert_array_equal([r["path_score"] for r in got], want)
    np.testing.assert_array_equal([r["forward_score"] for r in got], want)
    assert all(r["score_ok"] and r["row_ok"] for r in got)
    assert [pf.cigar_read_length(r["cigar"]) for r in got] == [len(r) for r in reads]


@pytest.mark.gpu
@pytest.mark.skipif(not pf.traceback_available(), reason="the reference's ParSGA traceback driver is not built")
def test_gpu_traceback_matches_parsga_traceback_scores(tmp_path):
    """The GPU traceback (one read, checkpointed every 16 rows, and batched)
    on a single-char graph: every path scores what the reference's ParSGA
    traceback's path scores, and ends on the read's last row. The two walks
    break ties differently (ConSGA's and ParSGA's op orders), so the paths
    themselves may differ."""
    import chsga_b200 as cb
    g, files = gen_graph(tmp_path, "tg", backbone_len=1200, seed=46, vlen_min=1, vlen_max=1,
                         bubble_gap_mean=6.0, p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=2, alt_max=20)
    labels_raw = open(files[3], "rb").read().replace(b"\n", b"")
    off, tgt = _char_csr(files)
    prefix = str(tmp_path / "tbg")
    pf.write_inputs(prefix, labels_raw, off, tgt, threads=(2,))
    reads = g.gen_reads(10, 46, 40, 120, sub_rate=0.05, indel_rate=0.04, n_rate=0.02).to_list()
    par = pf.run_traceback(prefix, reads, 2, str(tmp_path), k=16)
    want = [r["path_score"] for r in par]
    labels = labels_raw
    ctx = cb.Context(0).load(g)
    try:
        for rd, w in zip(reads, want):
            ops, score, _ = ctx.align_traceback(rd, k=16)
            assert score == w and orc.rescore(ops, rd, labels) == (w, len(rd) - 1)
        for rd, w, (ops, score, _) in zip(reads, want, ctx.align_traceback_batched(reads, slots=8)):
            assert score == w and orc.rescore(ops, rd, labels) == (w, len(rd) - 1)
    finally:
        ctx.close()
