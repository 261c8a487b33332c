"""The GPU paths on reads at the edges of the input domain (conftest.edge_reads:
one base, a lone N, all N, longer than any path of the graph, a
homopolymer, lower case and bytes outside the alphabet, a NUL byte, the empty
read): plain, batched at 8 and 128 slots (16-bit rows and delta rows) and
served scores equal the oracle's, which equal the reference's own code on
these reads (tests/test_oracle.py), and every non-empty read's traceback
rescores to its score."""
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
