"""GPU parity: the CUDA path (through the C-ABI) against the CPU oracle.

Integer DP, so every comparison is exact (bit-for-bit int32)."""
import os

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc
from conftest import gen_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx_small(small_graph):
    g, files, reads = small_graph
    ctx = cb.Context(0)
    ctx.load(g)
    yield ctx
    ctx.close()


def test_scores_plain_match_oracle(small_graph, ctx_small, oracle_small):
    g, files, reads = small_graph
    want = oracle_small.scores(reads)
    got = ctx_small.align_scores(reads)
    np.testing.assert_array_equal(got, want)


def test_every_row_matches_oracle(small_graph, ctx_small, oracle_small):
    g, files, reads = small_graph
    for rd in reads[:3]:
        want = oracle_small.rows(rd)
        got = ctx_small.align_rows(rd, oracle_small.num_chars)
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("slots", [2, 8, 32, 64, 128])
@pytest.mark.parametrize("row_bits", [16, 32])
def test_batched_matches_plain(small_graph, ctx_small, oracle_small, slots, row_bits):
    g, files, reads = small_graph
    want = oracle_small.scores(reads)
    got = ctx_small.align_scores_batched(reads, slots=slots, row_bits=row_bits)
    np.testing.assert_array_equal(got, want)
    assert ctx_small.profile()["row_bits"] == row_bits


def test_row_width_follows_the_read_length(tmp_path):
    # rows of a read longer than 65000 bases do not fit 16 bits: the engine
    # must fall back to 32-bit rows (and refuse a forced 16)
    g, files = gen_graph(tmp_path, "long", backbone_len=600, seed=81)
    rd = g.gen_reads(1, 82, 40).to_list()[0] * 1700  # 68000 bases
    o = orc.Oracle(files)
    want = o.scores([rd, rd[:300]])
    ctx = cb.Context(0).load(g)
    np.testing.assert_array_equal(ctx.align_scores_batched([rd, rd[:300]], slots=2), want)
    assert ctx.profile()["row_bits"] == 32
    with pytest.raises(cb.ChsgaError) as e:
        ctx.align_scores_batched([rd], slots=2, row_bits=16)
    assert e.value.status == cb.ERR_INVALID_ARG
    ctx.close()


def test_batched_uneven_lengths(small_graph, ctx_small, oracle_small):
    g, files, _ = small_graph
    reads = g.gen_reads(40, 9, 1, 400, sub_rate=0.03, indel_rate=0.02).to_list()
    want = oracle_small.scores(reads)
    for slots, graphs in ((16, True), (64, False)):
        got = ctx_small.align_scores_batched(reads, slots=slots, use_graphs=graphs)
        np.testing.assert_array_equal(got, want)


def test_traceback_full_matrix(small_graph, ctx_small, oracle_small):
    g, files, reads = small_graph
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    want = oracle_small.scores(reads[:6])
    edges = orc.char_edges(files)
    for rd, w in zip(reads[:6], want):
        ops, score, ck = ctx_small.align_traceback(rd)
        assert not ck
        assert score == w
        ps, last = orc.rescore(ops, rd, labels)
        assert ps == w and last == len(rd) - 1
        assert orc.check_path(ops, edges) == []  # every step follows the char graph


def test_traceback_checkpointed(small_graph, ctx_small, oracle_small, tmp_path):
    g, files, reads = small_graph
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    rd = reads[0]
    want = int(oracle_small.scores([rd])[0])
    n = oracle_small.num_chars
    # cap below the full matrix forces checkpoints; k=40 gives 4 segments
    ops, score, ck = ctx_small.align_traceback(rd, k=40, ckpt_dir=str(tmp_path / "ck"),
                                               keep_files=True, cap_bytes=60 * n * 4)
    assert ck and score == want
    ps, last = orc.rescore(ops, rd, labels)
    assert ps == want and last == len(rd) - 1
    assert orc.check_path(ops, orc.char_edges(files)) == []
    rows = oracle_small.rows(rd)
    for i in range(0, len(rd), 40):
        got = np.fromfile(str(tmp_path / "ck" / f"row_{i}.bin"), dtype=np.int32)
        np.testing.assert_array_equal(got, rows[i])


def test_traceback_two_level(small_graph, ctx_small, oracle_small):
    g, files, reads = small_graph
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    rd = reads[1]
    want = int(oracle_small.scores([rd])[0])
    n = oracle_small.num_chars
    full_ops, full_score, full_ck = ctx_small.align_traceback(rd)
    assert not full_ck and full_score == want
    # device budgets of 40 and 23 rows: a segment of 100 rows does not fit,
    # so it runs as sub-segments (a few dozen rows) from sub-checkpoints,
    # the last one walked straight from the first pass; the path is the
    # full-matrix one, op for op
    for rows in (40, 23):
        ctx = cb.Context(0, hbm_cap_bytes=rows * n * 4).load(g)
        ops, score, ck = ctx.align_traceback(rd, k=100)
        ctx.close()
        assert ck and score == want
        np.testing.assert_array_equal(ops, full_ops)
        ps, last = orc.rescore(ops, rd, labels)
        assert ps == want and last == len(rd) - 1


@pytest.mark.parametrize("seed,vmax", [(21, 1), (22, 3), (23, 32)])
def test_random_graphs(tmp_path, seed, vmax):
    g, files = gen_graph(tmp_path, f"r{seed}", backbone_len=3000, seed=seed, vlen_max=vmax,
                         bubble_gap_mean=8.0, p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=2,
                         alt_max=40)
    reads = g.gen_reads(12, seed, 20, 120, sub_rate=0.05, indel_rate=0.05, n_rate=0.01).to_list()
    o = orc.Oracle(files)
    want = o.scores(reads)
    ctx = cb.Context(0).load(g)
    np.testing.assert_array_equal(ctx.align_scores(reads), want)
    np.testing.assert_array_equal(ctx.align_scores_batched(reads, slots=4), want)
    for slots in (1, 4, 64):
        np.testing.assert_array_equal(
            ctx.align_scores_batched(reads, slots=slots, use_graphs=cb.LAUNCH_PERSISTENT), want)
    ctx.close()


@pytest.mark.parametrize("slots", [16, 64])
def test_traceback_batched_equals_one_by_one(small_graph, ctx_small, oracle_small, slots):
    g, files, reads = small_graph
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    mix = list(reads[:10]) + g.gen_reads(30, 17, 10, 700, sub_rate=0.03, indel_rate=0.02,
                                          n_rate=0.005).to_list()
    n = oracle_small.num_chars
    want = oracle_small.scores(mix)
    # a cap that sends the longer reads to the checkpointed path
    cap = 400 * n * 4
    got = ctx_small.align_traceback_batched(mix, slots=slots, k=60, cap_bytes=cap)
    for rd, w, (ops, score, ck) in zip(mix, want, got):
        one = ctx_small.align_traceback(rd, k=60, cap_bytes=cap)
        assert score == w == one[1] and ck == one[2] == (len(rd) > 400)
        np.testing.assert_array_equal(ops, one[0])
        assert orc.rescore(ops, rd, labels) == (w, len(rd) - 1)


@pytest.mark.parametrize("slots", [1, 2, 8, 32, 64, 128])
@pytest.mark.parametrize("top_vertices", [0, 300])
def test_persistent_kernel_matches_oracle(small_graph, ctx_small, oracle_small, slots, top_vertices):
    # one cooperative launch per 16 row-steps: row, levels and advance as
    # phases separated by grid barriers; uneven lengths refill slots mid-launch
    g, files, reads = small_graph
    mix = list(reads) + g.gen_reads(20, 19, 1, 400, sub_rate=0.03, indel_rate=0.02,
                                    n_rate=0.005).to_list()
    want = oracle_small.scores(mix)
    got = ctx_small.align_scores_batched(mix, slots=slots, steps_per_graph=16,
                                         use_graphs=cb.LAUNCH_PERSISTENT, top_vertices=top_vertices)
    np.testing.assert_array_equal(got, want)
    p = ctx_small.profile()
    assert p["launch_mode"] == cb.LAUNCH_PERSISTENT
    assert p["launches"] == 1 + p["row_launches"] // 16


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_plain_path_every_launch_mode(small_graph, ctx_small, oracle_small, mode):
    # one slot: the tile row kernel (a warp per tile of whole vertices, a
    # lane per 8 chars) in launches, in CUDA graphs and in the persistent kernel
    g, files, reads = small_graph
    want = oracle_small.scores(reads)
    got = ctx_small.align_scores_batched(reads, slots=1, use_graphs=mode)
    np.testing.assert_array_equal(got, want)
    assert ctx_small.profile()["launch_mode"] == mode
    # the one-thread-per-vertex row kernel gives the same scores
    got_d = ctx_small.align_scores_batched(reads, slots=1, use_graphs=mode, row_kernel=cb.ROW_DIRECT)
    np.testing.assert_array_equal(got_d, want)


def test_programmatic_dependent_launch_matches_oracle(small_graph, oracle_small, monkeypatch):
    # CHSGA_PDL=1: each row-step kernel may launch while the one before it
    # drains and waits on griddepcontrol.wait before reading its results
    g, files, reads = small_graph
    monkeypatch.setenv("CHSGA_PDL", "1")
    ctx = cb.Context(0).load(g)
    try:
        want = oracle_small.scores(reads)
        np.testing.assert_array_equal(ctx.align_scores(reads), want)
        for slots in (8, 64, 128):
            np.testing.assert_array_equal(ctx.align_scores_batched(reads, slots=slots), want)
        labels = open(files[3], "rb").read().replace(b"\n", b"")
        ops, score, _ = ctx.align_traceback(reads[0])
        assert score == want[0] and orc.rescore(ops, reads[0], labels) == (want[0], len(reads[0]) - 1)
    finally:
        ctx.close()


@pytest.mark.parametrize("top_vertices", [0, 300])
def test_cooperative_pull_matches_oracle(small_graph, oracle_small, monkeypatch, top_vertices):
    # CHSGA_PULL_COOP=1: upward levels load each target's edge list across its
    # lane group and shuffle it to every lane (64 and 128 slots)
    g, files, reads = small_graph
    monkeypatch.setenv("CHSGA_PULL_COOP", "1")
    ctx = cb.Context(0).load(g)
    try:
        mix = list(reads) + g.gen_reads(30, 23, 1, 500, sub_rate=0.03, indel_rate=0.02).to_list()
        want = oracle_small.scores(mix)
        for slots in (64, 128):
            got = ctx.align_scores_batched(mix, slots=slots, top_vertices=top_vertices)
            np.testing.assert_array_equal(got, want)
    finally:
        ctx.close()


@pytest.mark.parametrize("top_vertices", [0, 300])
def test_delta_rows_equal_oracle_and_16bit_rows(small_graph, ctx_small, oracle_small, top_vertices):
    # ROW_DELTA: 128 slots store rows as 2-bit within-vertex deltas
    # (k_row_delta); uneven lengths refill slots while others run, so a
    # slot's new read starts on rows another read left behind
    g, files, reads = small_graph
    mix = list(reads) + g.gen_reads(150, 29, 1, 2500, sub_rate=0.04, indel_rate=0.03,
                                    n_rate=0.01).to_list()
    want = oracle_small.scores(mix)
    got = ctx_small.align_scores_batched(mix, slots=128, top_vertices=top_vertices,
                                         row_kernel=cb.ROW_DELTA)
    np.testing.assert_array_equal(got, want)
    got16 = ctx_small.align_scores_batched(mix, slots=128, top_vertices=top_vertices)
    np.testing.assert_array_equal(got16, want)
