"""matchN scoring (CHSGA_FLAG_MATCH_N, the reference's ALPHABET_SIZE=4
builds) on the GPU: graphs and reads with 'N', every device path against the
matchN oracle, and the matchN drop-in drivers against the reference's own
ConSGA_matchN_dag / ConSGA_traceback_matchN_dag."""
import os
import re
import subprocess

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc
from conftest import ROOT, gen_graph, sprinkle_n

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "chsga_b200", "bin")


@pytest.fixture(scope="module")
def mgraph(tmp_path_factory):
    d = tmp_path_factory.mktemp("mn")
    g, files = gen_graph(d, "mn", backbone_len=8000, seed=61, vlen_max=32, bubble_gap_mean=20.0,
                         p_snp=0.5, p_indel=0.3, p_alt=0.2, alt_min=3, alt_max=60)
    g = sprinkle_n(files, 0.02, 61)
    reads = g.gen_reads(40, 62, 20, 600, sub_rate=0.03, indel_rate=0.02, n_rate=0.03).to_list()
    return g, files, reads


@pytest.fixture(scope="module")
def mctx(mgraph):
    c = cb.Context(0, flags=cb.FLAG_MATCH_N).load(mgraph[0])
    yield c
    c.close()


def test_matchn_scores_every_path(mgraph, mctx):
    g, files, reads = mgraph
    want = orc.Oracle(files, match_n=True).scores(reads)
    mis = orc.Oracle(files).scores(reads)
    assert (mis > want).any()  # the scheme matters here
    np.testing.assert_array_equal(mctx.align_scores(reads), want)
    for slots, kernels in ((2, [cb.ROW_AUTO, cb.ROW_DIRECT]),
                           (32, [cb.ROW_AUTO, cb.ROW_DIRECT, cb.ROW_TILED]),
                           (128, [cb.ROW_AUTO, cb.ROW_DPX, cb.ROW_STREAM, cb.ROW_DIRECT])):
        for rk in kernels:
            np.testing.assert_array_equal(mctx.align_scores_batched(reads, slots=slots, row_kernel=rk),
                                          want)
    np.testing.assert_array_equal(mctx.align_scores_batched(reads, slots=16, row_bits=32), want)
    np.testing.assert_array_equal(mctx.align_scores_noalloc(reads), want)
    # row 0 against '\0' of an empty read: an N label matches it
    assert mctx.align_scores([b""]).tolist() == [0]
    plain = cb.Context(0).load(g)
    np.testing.assert_array_equal(plain.align_scores(reads), mis)
    assert plain.align_scores([b""]).tolist() == [1]
    plain.close()


def test_matchn_rows_and_traceback(mgraph, mctx):
    g, files, reads = mgraph
    o = orc.Oracle(files, match_n=True)
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    np.testing.assert_array_equal(mctx.align_rows(reads[0], o.num_chars), o.rows(reads[0]))
    want = o.scores(reads[:6])
    n = o.num_chars
    for i, (rd, w) in enumerate(zip(reads[:6], want)):
        kw = dict(k=30, cap_bytes=20 * n * 4) if i % 2 else {}
        ops, score, ck = mctx.align_traceback(rd, **kw)
        assert score == w and ck == bool(i % 2 and len(rd) > 20)
        assert orc.rescore(ops, rd, labels, match_n=True) == (w, len(rd) - 1)


def test_matchn_server(mgraph, mctx):
    g, files, reads = mgraph
    want = orc.Oracle(files, match_n=True).scores(reads)
    srv = cb.Server(mctx, slots=16)
    tk = [srv.submit(r) for r in reads] + [srv.submit(reads[0], cb.REQ_TRACEBACK), srv.submit(b"")]
    res = srv.collect()
    srv.close()
    np.testing.assert_array_equal([res[t]["score"] for t in tk[:-2]], want)
    assert res[tk[-2]]["score"] == want[0] and res[tk[-1]]["score"] == 0


def _score_line(out):
    m = re.search(r"^score: (.*)$", out, re.M)
    return m.group(1).split() if m else None


@pytest.mark.skipif(not os.path.exists(orc.REF_CONSGA_MATCHN), reason="reference drivers not built")
def test_matchn_drivers_match_reference(mgraph, tmp_path):
    g, files, reads = mgraph
    fa = tmp_path / "r.fa"
    fa.write_text("".join(f">r{i}\n{r.decode()}\n" for i, r in enumerate(reads[:5])))
    args = ["-I", files[0], "-i", files[1], "-c", files[2], "-r", str(fa), "-l", files[3],
            "-o", files[4]]
    ours = subprocess.run([os.path.join(BIN, "ConSGA_matchN_dag")] + args, capture_output=True,
                          text=True, timeout=300)
    ref = subprocess.run([orc.REF_CONSGA_MATCHN] + args, capture_output=True, text=True, timeout=300)
    assert ours.returncode == 0 and ref.returncode == 0, ours.stderr
    assert _score_line(ours.stdout) == _score_line(ref.stdout)
    targs = args + ["-k", "40"]
    ours = subprocess.run([os.path.join(BIN, "ConSGA_traceback_matchN_dag")] + targs +
                          ["-d", str(tmp_path / "a")], capture_output=True, text=True, timeout=300)
    ref = subprocess.run([orc.REF_CONSGA_TB_MATCHN] + targs + ["-d", str(tmp_path / "b")],
                         capture_output=True, text=True, timeout=300)
    # same per-read scores; the verdict lines are not compared: the
    # reference's check compares bytes (an N-matched step reads as a
    # substitution) and its argmin ties are nondeterministic, so which of
    # the equal-score paths each side walks decides the verdict
    pat = r"^read\[\d+\] score=\d+$"
    assert re.findall(pat, ours.stdout, re.M) == re.findall(pat, ref.stdout, re.M)
    assert ours.stdout.count("row_ok     : YES") == 5
