"""Graph ingest (the reference's handlegraph_to_csr -> csr_to_adj pipeline,
with GFA v1 standing in for libbdsg's PackedGraph), on CPU: a hand-worked
graph with an inversion, csr_to_adj byte for byte against the reference's
own converter, and the alignment of a converted graph against the
reference's code."""
import os
import subprocess

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc
from conftest import gen_graph

HAND_GFA = """H\tVN:Z:1.0
S\t1\tACG
S\t3\tga
S\t2\tT
L\t1\t+\t2\t+\t0M
L\t1\t+\t3\t-\t0M
L\t2\t+\t3\t+\t*
L\t3\t-\t2\t-\t0M
P\tp\t1+,2+\t*
"""


def _csr_text(path):
    toks = open(path).read().split()
    n, m = int(toks[0]), int(toks[1])
    labels = toks[2:2 + n]
    offs = [int(x) for x in toks[2 + n:3 + 2 * n]]
    adj = [int(x) for x in toks[3 + 2 * n:3 + 2 * n + m]]
    return n, m, labels, offs, adj


def test_hand_gfa_known_answer(tmp_path):
    gfa = tmp_path / "h.gfa"
    gfa.write_text(HAND_GFA)
    s, c = str(tmp_path / "s.csr"), str(tmp_path / "c.csr")
    cb.gfa_to_csr_text(str(gfa), s, c)
    # nodes by id 1, 2, 3 -> vertices (0 fwd, 1 rev), (2, 3), (4, 5); lower
    # case upper-cased; "3 - 2 -" repeats 2+ -> 3+ in reverse form (kept once)
    n, m, labels, offs, adj = _csr_text(s)
    assert labels == ["ACG", "CGT", "T", "A", "GA", "TC"]
    assert offs == [0, 2, 2, 3, 4, 5, 6] and adj == [2, 5, 4, 1, 1, 3] and m == 6
    n, m, labels, offs, adj = _csr_text(c)
    assert "".join(labels) == "ACGCGTTAGATC" and n == 12
    assert offs == [0, 1, 2, 4, 5, 6, 6, 7, 8, 9, 10, 11, 12]
    assert adj == [1, 2, 6, 10, 4, 5, 8, 3, 9, 3, 11, 7]
    # the exact bytes of write_csr: every list ends with " \\n"
    assert open(s).read() == "6\n6\nACG CGT T A GA TC \n0 2 2 3 4 5 6 \n2 5 4 1 1 3 \n"
    g = cb.HostGraph.from_gfa(str(gfa))
    st = g.stats()
    assert st["num_strings"] == 6 and st["num_chars"] == 12 and st["num_char_edges"] == 12


def test_rejections(tmp_path):
    bad = tmp_path / "b.gfa"
    bad.write_text("S\tx\tACGT\n")
    with pytest.raises(cb.ChsgaError):
        cb.HostGraph.from_gfa(str(bad))
    bad.write_text("S\t1\tACGT\nS\t2\tAC\nL\t1\t+\t2\t+\t3M\n")
    with pytest.raises(cb.ChsgaError) as e:
        cb.HostGraph.from_gfa(str(bad))
    assert e.value.status == cb.ERR_UNSUPPORTED


def _to_gfa(g, path):
    """GFA v1 of a generated graph: one segment per string vertex (id + 1),
    one forward link per string edge."""
    v = g.view()
    S = v.string_graph.n
    offs = np.ctypeslib.as_array(v.label_offsets, (S + 1,))
    lab = C_bytes(v.labels, v.num_chars)
    so = np.ctypeslib.as_array(v.string_graph.offset, (S + 1,))
    st = np.ctypeslib.as_array(v.string_graph.target, (v.string_graph.m,))
    with open(path, "w") as f:
        f.write("H\tVN:Z:1.0\n")
        for s in range(S):
            f.write(f"S\t{s + 1}\t{lab[offs[s]:offs[s + 1]].decode()}\n")
        for s in range(S):
            for e in range(so[s], so[s + 1]):
                f.write(f"L\t{s + 1}\t+\t{int(st[e]) + 1}\t+\t0M\n")


def C_bytes(ptr, n):
    import ctypes
    return ctypes.string_at(ptr, n)


@pytest.mark.skipif(not os.path.exists(orc.REF_CSR_TO_ADJ), reason="reference csr_to_adj not built")
def test_csr_to_adj_matches_reference_bytes(tmp_path):
    g, _ = gen_graph(tmp_path, "src", backbone_len=3000, seed=71)
    gfa = str(tmp_path / "g.gfa")
    _to_gfa(g, gfa)
    s, c = str(tmp_path / "s.csr"), str(tmp_path / "c.csr")
    cb.gfa_to_csr_text(gfa, s, c)
    for src in (s, c):
        ours = [str(tmp_path / f"o{i}") for i in range(3)]
        ref = [str(tmp_path / f"r{i}") for i in range(3)]
        subprocess.run([os.path.join(os.path.dirname(cb.LIB_PATH), "..", "bin", "csr_to_adj"), src] + ours,
                       check=True)
        subprocess.run([orc.REF_CSR_TO_ADJ, src] + ref, check=True)
        for a, b in zip(ours, ref):
            assert open(a, "rb").read() == open(b, "rb").read()


@pytest.mark.skipif(not orc.ref_available(), reason="oracle/_ref not built")
def test_ingested_graph_aligns_like_the_reference(tmp_path):
    g0, _ = gen_graph(tmp_path, "src", backbone_len=2500, seed=72, vlen_max=12)
    gfa = str(tmp_path / "g.gfa")
    _to_gfa(g0, gfa)
    g = cb.HostGraph.from_gfa(gfa)
    g.build_pch()
    files = g.write_files(str(tmp_path / "ing"))
    st = g.stats()
    assert st["num_strings"] == 2 * g0.stats()["num_strings"]
    # reads from both strands (random source-to-sink paths of either copy)
    reads = g.gen_reads(12, 73, 20, 150, sub_rate=0.03, indel_rate=0.02).to_list()
    rc = {ord("A"): "T", ord("C"): "G", ord("G"): "C", ord("T"): "A"}
    reads += [r.decode().translate(rc)[::-1].encode() for r in reads[:4]]
    o, r = orc.Oracle(files), orc.RefHarness(files)
    np.testing.assert_array_equal(o.scores(reads), r.scores(reads))
    # the string CSR text round trip gives the same host graph
    s, c = str(tmp_path / "s.csr"), str(tmp_path / "c.csr")
    cb.gfa_to_csr_text(gfa, s, c)
    h = cb.HostGraph.from_csr_text(s, c)
    assert h.stats()["num_char_edges"] == st["num_char_edges"]


@pytest.mark.gpu
def test_ingested_graph_on_gpu(tmp_path):
    g0, _ = gen_graph(tmp_path, "src", backbone_len=6000, seed=74)
    gfa = str(tmp_path / "g.gfa")
    _to_gfa(g0, gfa)
    g = cb.HostGraph.from_gfa(gfa)
    g.build_pch()
    files = g.write_files(str(tmp_path / "ing"))
    reads = g.gen_reads(30, 75, 30, 400, sub_rate=0.03, indel_rate=0.02).to_list()
    want = orc.Oracle(files).scores(reads)
    ctx = cb.Context(0).load(g)
    np.testing.assert_array_equal(ctx.align_scores(reads), want)
    np.testing.assert_array_equal(ctx.align_scores_batched(reads, slots=64), want)
    ops, score, _ = ctx.align_traceback(reads[0])
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    assert score == want[0] and orc.rescore(ops, reads[0], labels) == (score, len(reads[0]) - 1)
    ctx.close()


def test_csr_text_reader_errors(tmp_path):
    """Malformed CSR text fails with a format status naming the problem."""
    gfa = tmp_path / "h.gfa"
    gfa.write_text(HAND_GFA)
    s, c = str(tmp_path / "s.csr"), str(tmp_path / "c.csr")
    cb.gfa_to_csr_text(str(gfa), s, c)
    good = open(s).read()
    assert cb.HostGraph.from_csr_text(s, c).stats()["num_strings"] == 6
    cases = [
        ("6\n", "x6\n", "expected the vertex count"),
        ("0 2 2 3 4 5 6 \n", "0 2 1 3 4 5 6 \n", "offsets not non-decreasing"),
        ("2 5 4 1 1 3 \n", "2 5 4 1 1 9 \n", "adjacency entry out of range"),
    ]
    for good_line, bad_line, msg in cases:
        assert good_line in good
        p = tmp_path / "bad.csr"
        p.write_text(good.replace(good_line, bad_line, 1))
        with pytest.raises(cb.ChsgaError) as e:
            cb.HostGraph.from_csr_text(str(p), c)
        assert e.value.status == cb.ERR_FORMAT and msg in str(e.value), str(e.value)
