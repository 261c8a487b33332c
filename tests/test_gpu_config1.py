"""Config 1 in full on the GPU: the 100 kbp variant-bubble DAG (SNP bubble
every ~100 bp, 1-10 bp indel bubble every ~1 kbp, string vertices of 1-32
chars, seed 1) and 200 reads of 150 bp at 1% substitutions, 0.3% 1-3 bp
indels and 0.1% N.

Every GPU entry point that scores reads must give the scores of the
reference's own align_combo (src/align.hpp:470-531, compiled in oracle/_ref;
the restatement when that build is absent) for all 200 reads, and two reads
must give the reference's every DP row (the rows align_read_combo leaves,
src/align.hpp:430-463). Integer DP: every comparison is exact."""
import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg1(tmp_path_factory):
    d = tmp_path_factory.mktemp("cfg1")
    g = cb.HostGraph.generate(**cb.GRAPH_CONFIGS["cfg1"])
    g.build_pch()
    files = g.write_files(str(d / "cfg1"))
    reads = g.gen_reads(200, 101, 150, 150, sub_rate=0.01, indel_rate=0.003, n_rate=0.001,
                        indel_len_max=3).to_list()
    if orc.ref_available():
        ref = orc.RefHarness(files)
    else:
        ref = orc.Oracle(files)
    want = ref.scores(reads)
    ctx = cb.Context(0).load(g)
    yield g, files, reads, ref, want, ctx
    ctx.close()


def test_config1_graph_shape(cfg1):
    g, files, reads, ref, want, ctx = cfg1
    st = g.stats()
    # ~101.5 k chars over ~8-9 k string vertices (the recipe's expectation)
    assert 100_000 < st["num_chars"] < 103_000
    assert 5_000 < st["num_strings"] < 12_000
    assert len(reads) == 200 and all(len(r) == 150 for r in reads)
    assert any(b"N" in r for r in reads)


def test_config1_plain_equals_reference(cfg1):
    g, files, reads, ref, want, ctx = cfg1
    np.testing.assert_array_equal(ctx.align_scores(reads), want)


@pytest.mark.parametrize("slots", [8, 128])
def test_config1_batched_equals_reference(cfg1, slots):
    g, files, reads, ref, want, ctx = cfg1
    np.testing.assert_array_equal(ctx.align_scores_batched(reads, slots=slots), want)


def test_config1_served_equals_reference(cfg1):
    g, files, reads, ref, want, ctx = cfg1
    srv = cb.Server(ctx, slots=128, queue_capacity=256, arena_bytes=1 << 20)
    try:
        tickets = [srv.submit(r) for r in reads]
        res = srv.collect()
    finally:
        srv.close()
    assert all(res[t]["status"] == cb.OK for t in tickets)
    np.testing.assert_array_equal([res[t]["score"] for t in tickets], want)


def test_config1_noalloc_equals_reference(cfg1):
    g, files, reads, ref, want, ctx = cfg1
    np.testing.assert_array_equal(ctx.align_scores_noalloc(reads), want)


def test_config1_every_row_equals_reference(cfg1):
    g, files, reads, ref, want, ctx = cfg1
    n = g.stats()["num_chars"]
    for rd in (reads[0], reads[117]):
        if isinstance(ref, orc.RefHarness):
            rows = ref.rows(rd, n)
        else:
            rows = ref.rows(rd)
        np.testing.assert_array_equal(ctx.align_rows(rd, n), rows)
