"""The CPU oracle (oracle/consga_oracle.cpp) pinned against the reference.

Three pins, all on CPU:
  * golden fixtures made by the reference's own code (tests/golden/),
  * the reference's align.hpp / traceback.hpp compiled in oracle/_ref, run
    here on fresh random graphs (scores, every DP row, traceback, checkpoint
    rows byte for byte),
  * the reference's exact DP serial_align_CSR: equal to the hierarchy result
    when every string vertex is a single char (the closure is then exact), and
    never above it otherwise.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc
from conftest import edge_reads, gen_graph

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not orc.ref_available(), reason="oracle/_ref not built")


def golden_files(name):
    return cb.files_for(os.path.join(GOLD, name))


def test_hand_dag_known_answers():
    exp = json.load(open(os.path.join(GOLD, "hand.expected.json")))
    o = orc.Oracle(golden_files("hand"))
    reads = [r.encode() for r in exp["reads"]]
    assert o.scores(reads).tolist() == [0, 0, 1, 1] == exp["scores"]
    assert o.exact_scores(reads).tolist() == exp["exact"]


def test_golden_scores_rows_and_checkpoints(tmp_path):
    exp = json.load(open(os.path.join(GOLD, "g1.expected.json")))
    o = orc.Oracle(golden_files("g1"))
    reads = [r.encode() for r in exp["reads"]]
    assert o.scores(reads).tolist() == exp["scores"]
    assert o.exact_scores(reads).tolist() == exp["exact"]
    rows = np.load(os.path.join(GOLD, "g1.rows0.npz"))["rows"].astype(np.int32)
    np.testing.assert_array_equal(o.rows(reads[0]), rows)
    d = tmp_path / "ck"
    ops, score, ck = o.traceback(reads[0], k=exp["ckpt_k"], fast_cap_bytes=0, ckpt_dir=str(d),
                                 cleanup=False)
    assert ck and score == exp["scores"][0]
    for i, h in exp["ckpt_rows_sha256"].items():
        assert hashlib.sha256((d / f"row_{i}.bin").read_bytes()).hexdigest() == h
    labels = open(golden_files("g1")[3], "rb").read()
    assert orc.rescore(ops, reads[0], labels) == (exp["scores"][0], len(reads[0]) - 1)


@needs_ref
@pytest.mark.parametrize("seed,vmax", [(31, 1), (32, 4), (33, 32), (34, 12)])
def test_oracle_matches_reference_code(tmp_path, seed, vmax):
    g, files = gen_graph(tmp_path, f"r{seed}", backbone_len=2500, seed=seed, vlen_max=vmax,
                         bubble_gap_mean=10.0, p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=3,
                         alt_max=50)
    reads = g.gen_reads(10, seed, 10, 120, sub_rate=0.05, indel_rate=0.05, n_rate=0.02).to_list()
    o, r = orc.Oracle(files), orc.RefHarness(files)
    np.testing.assert_array_equal(o.scores(reads), r.scores(reads))
    for rd in reads[:2]:
        np.testing.assert_array_equal(o.rows(rd), r.rows(rd, o.num_chars))


@needs_ref
def test_single_char_graphs_are_exact(tmp_path):
    # with one char per string vertex the hierarchy sweeps are an exact
    # shortest-path closure, so the reference's own CH result equals its
    # exact DP; the oracle must agree with both
    for seed in (41, 42, 43):
        g, files = gen_graph(tmp_path, f"s{seed}", backbone_len=1500, seed=seed, vlen_max=1,
                             bubble_gap_mean=6.0, p_snp=0.4, p_indel=0.4, p_alt=0.2, alt_min=2,
                             alt_max=20)
        reads = g.gen_reads(10, seed, 20, 90, sub_rate=0.06, indel_rate=0.06).to_list()
        r = orc.RefHarness(files)
        exact = r.exact_scores(reads)
        np.testing.assert_array_equal(r.scores(reads), exact)
        np.testing.assert_array_equal(orc.Oracle(files).scores(reads), exact)


@needs_ref
def test_multi_char_never_below_exact(tmp_path):
    g, files = gen_graph(tmp_path, "m", backbone_len=4000, seed=51, bubble_gap_mean=12.0,
                         p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=5, alt_max=80)
    reads = g.gen_reads(30, 52, 30, 150, sub_rate=0.05, indel_rate=0.05).to_list()
    ch = orc.Oracle(files).scores(reads)
    exact = orc.RefHarness(files).exact_scores(reads)
    assert (ch >= exact).all()


@needs_ref
def test_traceback_paths_rescore(tmp_path):
    g, files = gen_graph(tmp_path, "t", backbone_len=3000, seed=61, bubble_gap_mean=15.0,
                         p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=4, alt_max=40)
    reads = g.gen_reads(6, 62, 40, 140, sub_rate=0.04, indel_rate=0.04, n_rate=0.01).to_list()
    labels = open(files[3], "rb").read()
    o, fast, slow = orc.Oracle(files), orc.RefHarness(files), orc.RefHarness(files, True)
    want = o.scores(reads)
    edges = orc.char_edges(files)
    kinds = set()
    for i, rd in enumerate(reads):
        for ops in (fast.traceback(rd), slow.traceback(rd, k=25, ckpt_dir=str(tmp_path / f"c{i}")),
                    o.traceback(rd)[0], o.traceback(rd, k=25, fast_cap_bytes=0,
                                                    ckpt_dir=str(tmp_path / f"o{i}"))[0]):
            assert orc.rescore(ops, rd, labels) == (want[i], len(rd) - 1)
            # every step follows the graph: the reference's paths and the oracle's
            assert orc.check_path(ops, edges) == []
            kinds |= {int(op) for op in ops[:, 2]}
    assert kinds == {0, 1, 2}
    # a path with one step off the graph is caught
    ops = o.traceback(reads[0])[0].copy()
    j = int(np.nonzero(ops[:, 2] == 1)[0][-1])
    ops[j, 1] = (ops[j, 1] + 7) % len(labels.replace(b"\n", b""))
    assert orc.check_path(ops, edges) != []


@needs_ref
def test_checkpoint_rows_byte_identical_to_reference(tmp_path):
    g, files = gen_graph(tmp_path, "k", backbone_len=2000, seed=71, bubble_gap_mean=15.0,
                         p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=4, alt_max=40)
    rd = g.gen_reads(1, 72, 130, sub_rate=0.04, indel_rate=0.04).to_list()[0]
    a, b = tmp_path / "ref", tmp_path / "orc"
    orc.RefHarness(files, True).traceback(rd, k=20, ckpt_dir=str(a), cleanup=False)
    orc.Oracle(files).traceback(rd, k=20, fast_cap_bytes=0, ckpt_dir=str(b), cleanup=False)
    names = sorted(os.listdir(a))
    assert names == sorted(os.listdir(b)) and len(names) == 7  # rows 0, 20, ..., 120
    for n in names:
        assert (a / n).read_bytes() == (b / n).read_bytes()


needs_ref_matchn = pytest.mark.skipif(not orc.ref_available(match_n=True),
                                      reason="oracle/_ref matchN builds not built")


@needs_ref_matchn
@pytest.mark.parametrize("seed,vmax", [(51, 1), (52, 12), (53, 32)])
def test_matchn_oracle_matches_reference_code(tmp_path, seed, vmax):
    # matchN (ALPHABET_SIZE=4): 'N' in labels and reads matches every base
    from conftest import sprinkle_n
    g, files = gen_graph(tmp_path, f"m{seed}", backbone_len=2500, seed=seed, vlen_max=vmax,
                         bubble_gap_mean=10.0, p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=3,
                         alt_max=50)
    g = sprinkle_n(files, 0.03, seed)
    reads = g.gen_reads(10, seed, 10, 120, sub_rate=0.05, indel_rate=0.05, n_rate=0.05).to_list()
    o, r = orc.Oracle(files, match_n=True), orc.RefHarness(files, match_n=True)
    want = r.scores(reads)
    np.testing.assert_array_equal(o.scores(reads), want)
    # the scheme matters on these inputs
    assert (orc.Oracle(files).scores(reads) > want).any()
    for rd in reads[:2]:
        np.testing.assert_array_equal(o.rows(rd), r.rows(rd, o.num_chars))
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    for rd, w in zip(reads[:3], want):
        ops, score, _ = o.traceback(rd)
        assert score == w and orc.rescore(ops, rd, labels, match_n=True) == (w, len(rd) - 1)


@pytest.mark.skipif(not orc.ref_available(), reason="reference build absent")
def test_reference_rows_at_equals_every_row(tmp_path):
    # the two-row harness entry used for the config-4 byte-compare returns
    # the same rows as the all-rows one
    g, files = gen_graph(tmp_path, "ra", backbone_len=4000, seed=71)
    n = g.stats()["num_chars"]
    rd = g.gen_reads(1, 72, 130, sub_rate=0.03, indel_rate=0.02).to_list()[0]
    h = orc.RefHarness(files)
    every = h.rows(rd, n)
    np.testing.assert_array_equal(h.rows_at(rd, n, [0, 64, 129]), every[[0, 64, 129]])


@pytest.mark.parametrize("seed,vmax,gap", [(61, 32, 20.0), (62, 3, 6.0), (63, 32, 6.0)])
def test_rows_change_by_at_most_one_within_a_vertex(tmp_path, seed, vmax, gap):
    # the premise of the 2-bit delta rows (k_row_delta): in every DP row two
    # consecutive chars of one string vertex differ by at most 1
    g, files = gen_graph(tmp_path, f"d{seed}", backbone_len=3000, seed=seed, vlen_max=vmax,
                         bubble_gap_mean=gap, p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=2, alt_max=60)
    o = orc.Oracle(files)
    off = np.array(open(files[4]).read().split(), dtype=np.int64)
    heads = np.zeros(o.num_chars, dtype=bool)
    heads[off[:-1]] = True
    reads = g.gen_reads(6, seed, 40, 300, sub_rate=0.08, indel_rate=0.06, n_rate=0.02).to_list()
    for rd in reads:
        rows = o.rows(rd)
        diff = np.diff(rows, axis=1)
        chain = ~heads[1:]  # char c (c >= 1) continues the vertex of c - 1
        assert np.abs(diff[:, chain]).max() <= 1


@needs_ref
def test_edge_reads_match_reference_code(tmp_path):
    g, files = gen_graph(tmp_path, "edge", backbone_len=600, seed=71, vlen_max=8, bubble_gap_mean=10.0,
                         p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=3, alt_max=30)
    reads = edge_reads(g, 71)
    o, r = orc.Oracle(files), orc.RefHarness(files)
    want = r.scores(reads)
    np.testing.assert_array_equal(o.scores(reads), want)
    assert want[-1] == 1 and want[3] == 40  # empty read, 40 N (every base costs one)


@needs_ref
def test_edge_reads_match_reference_code_matchn(tmp_path):
    """The edge-case reads under matchN scoring ('N' in a read or label
    matches every base): the matchN restatement equals the reference's
    ALPHABET_SIZE=4 build; a read of N costs nothing there."""
    from conftest import sprinkle_n
    g, files = gen_graph(tmp_path, "edgen", backbone_len=600, seed=72, vlen_max=8, bubble_gap_mean=10.0,
                         p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=3, alt_max=30)
    g = sprinkle_n(files, 0.03, 72)  # N in the labels too
    reads = edge_reads(g, 72)
    want = orc.RefHarness(files, match_n=True).scores(reads)
    np.testing.assert_array_equal(orc.Oracle(files, match_n=True).scores(reads), want)
    assert want[1] == 0 and want[3] == 0  # a lone N and 40 N match anywhere


@needs_ref
def test_checkpoint_rows_of_edge_reads_byte_identical_to_reference(tmp_path):
    """Checkpoint files of edge-case reads (all N; longer than any path; odd
    bytes) from the reference's checkpointed traceback and from the oracle's
    are byte-identical, and both paths have the same score."""
    g, files = gen_graph(tmp_path, "ke", backbone_len=600, seed=73, vlen_max=8, bubble_gap_mean=10.0,
                         p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=3, alt_max=30)
    reads = [r for r in edge_reads(g, 73) if len(r) >= 12]
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    for i, rd in enumerate(reads):
        a, b = tmp_path / f"ref{i}", tmp_path / f"orc{i}"
        ref_ops = orc.RefHarness(files, True).traceback(rd, k=11, ckpt_dir=str(a), cleanup=False)
        _, so, ck = orc.Oracle(files).traceback(rd, k=11, fast_cap_bytes=0, ckpt_dir=str(b), cleanup=False)
        assert ck and orc.rescore(ref_ops, rd, labels) == (so, len(rd) - 1)
        names = sorted(os.listdir(a))
        assert names == sorted(os.listdir(b)) and len(names) == (len(rd) - 1) // 11 + 1
        for n in names:
            assert (a / n).read_bytes() == (b / n).read_bytes(), (i, n)


@needs_ref
@pytest.mark.parametrize("name", ["one_segment", "one_char", "bubble"])
def test_tiny_graphs_match_reference_code(tmp_path, name):
    """Graphs of two to eight string vertices (a single GFA segment, a single
    base, a bubble; both orientations): the oracle equals the reference's
    code on scores and every row."""
    from conftest import TINY_READS, tiny_graph
    g, files = tiny_graph(tmp_path, name)
    o, r = orc.Oracle(files), orc.RefHarness(files)
    np.testing.assert_array_equal(o.scores(TINY_READS), r.scores(TINY_READS))
    for rd in TINY_READS[:4]:
        np.testing.assert_array_equal(o.rows(rd), r.rows(rd, o.num_chars))
