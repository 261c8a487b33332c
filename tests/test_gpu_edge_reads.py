"""The GPU paths on reads at the edges of the input domain (conftest.edge_reads:
one base, a lone N, all N, longer than any path of the graph, a
homopolymer, lower case and bytes outside the alphabet, a NUL byte, the empty
read): plain, batched at 8 and 128 slots (16-bit rows and delta rows) and
served scores equal the oracle's, which equal the reference's own code on
these reads (tests/test_oracle.py), and every non-empty read's traceback
rescores to its score."""
import os

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc
from conftest import edge_reads, gen_graph

pytestmark = pytest.mark.gpu


def test_gpu_paths_on_edge_reads(tmp_path):
    g, files = gen_graph(tmp_path, "edge", backbone_len=600, seed=71, vlen_max=8, bubble_gap_mean=10.0,
                         p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=3, alt_max=30)
    reads = edge_reads(g, 71)
    want = orc.Oracle(files).scores(reads)
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    ctx = cb.Context(0).load(g)
    try:
        np.testing.assert_array_equal(ctx.align_scores(reads), want)
        for slots in (8, 128):
            np.testing.assert_array_equal(ctx.align_scores_batched(reads, slots=slots), want,
                                          err_msg=f"{slots} slots")
        srv = cb.Server(ctx, slots=128, queue_capacity=64, arena_bytes=1 << 20)
        try:
            tickets = [srv.submit(r) for r in reads if r]
            res = srv.collect()
        finally:
            srv.close()
        assert all(res[t]["status"] == cb.OK for t in tickets)
        np.testing.assert_array_equal([res[t]["score"] for t in tickets], [w for r, w in zip(reads, want) if r])
        for rd, w in zip(reads, want):
            if not rd:
                continue
            ops, score, _ = ctx.align_traceback(rd)
            assert score == w and orc.rescore(ops, rd, labels) == (w, len(rd) - 1)
    finally:
        ctx.close()


def test_gpu_checkpoints_of_edge_reads_equal_the_oracles(tmp_path):
    """Checkpointed GPU tracebacks (every 11 rows; a byte cap of 15 int32
    rows, below the 16-bit matrix of a 40-base read and above a 12-row
    segment) of the edge-case reads of 40 or more bases: the checkpoint files
    are byte-identical to the oracle's (which equal the reference's,
    tests/test_oracle.py), and the paths rescore to the optimum."""
    g, files = gen_graph(tmp_path, "ke", backbone_len=600, seed=73, vlen_max=8, bubble_gap_mean=10.0,
                         p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=3, alt_max=30)
    reads = [r for r in edge_reads(g, 73) if len(r) >= 40]
    assert len(reads) == 3
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    o = orc.Oracle(files)
    n = o.num_chars
    ctx = cb.Context(0).load(g)
    try:
        for i, rd in enumerate(reads):
            a, b = tmp_path / f"gpu{i}", tmp_path / f"orc{i}"
            ops, score, ck = ctx.align_traceback(rd, k=11, ckpt_dir=str(a), keep_files=True,
                                                 cap_bytes=15 * n * 4)
            _, want, _ = o.traceback(rd, k=11, fast_cap_bytes=0, ckpt_dir=str(b), cleanup=False)
            assert ck and score == want
            assert orc.rescore(ops, rd, labels) == (want, len(rd) - 1)
            names = sorted(os.listdir(b))
            assert names and set(names) <= set(os.listdir(a))
            for nm in names:
                assert (a / nm).read_bytes() == (b / nm).read_bytes(), (i, nm)
    finally:
        ctx.close()


@pytest.mark.parametrize("name", ["one_segment", "one_char", "bubble"])
def test_gpu_paths_on_tiny_graphs(tmp_path, name):
    """Graphs of two to eight string vertices (conftest.TINY_GFA): a single
    run of vertices, a hierarchy of one or two levels all in the top region.
    Plain, batched at 8 and 128 slots, and the traceback of every non-empty
    read equal the oracle (which equals the reference's code on these graphs,
    tests/test_oracle.py)."""
    from conftest import TINY_READS, tiny_graph
    g, files = tiny_graph(tmp_path, name)
    want = orc.Oracle(files).scores(TINY_READS)
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    ctx = cb.Context(0).load(g)
    try:
        np.testing.assert_array_equal(ctx.align_scores(TINY_READS), want)
        for slots in (8, 128):
            np.testing.assert_array_equal(ctx.align_scores_batched(TINY_READS, slots=slots), want,
                                          err_msg=f"{slots} slots")
        for rd, w in zip(TINY_READS, want):
            if rd:
                ops, score, _ = ctx.align_traceback(rd)
                assert score == w and orc.rescore(ops, rd, labels) == (w, len(rd) - 1)
    finally:
        ctx.close()
