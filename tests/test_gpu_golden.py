"""GPU path against the golden fixtures made by the reference's own code, and
the drop-in command-line tools against the reference's drivers compiled in
oracle/_ref (same input files, same stdout lines)."""
import hashlib
import json
import os
import re
import subprocess

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc
from conftest import ROOT

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BIN = os.path.join(ROOT, "chsga_b200", "bin")


def files(name):
    return cb.files_for(os.path.join(GOLD, name))


@pytest.fixture(scope="module")
def g1():
    exp = json.load(open(os.path.join(GOLD, "g1.expected.json")))
    ctx = cb.Context(0).load(cb.HostGraph.read_files(*files("g1")))
    yield ctx, exp, [r.encode() for r in exp["reads"]]
    ctx.close()


def test_hand_dag_on_gpu():
    ctx = cb.Context(0).load(cb.HostGraph.read_files(*files("hand")))
    reads = [b"ACG", b"ATG", b"AG", b"ANG"]
    assert ctx.align_scores(reads).tolist() == [0, 0, 1, 1]
    assert ctx.align_scores_batched(reads, slots=4).tolist() == [0, 0, 1, 1]
    ctx.close()


def test_golden_scores(g1):
    ctx, exp, reads = g1
    assert ctx.align_scores(reads).tolist() == exp["scores"]
    for slots in (2, 16, 128):
        assert ctx.align_scores_batched(reads, slots=slots).tolist() == exp["scores"]


def test_golden_rows(g1):
    ctx, exp, reads = g1
    rows = np.load(os.path.join(GOLD, "g1.rows0.npz"))["rows"].astype(np.int32)
    np.testing.assert_array_equal(ctx.align_rows(reads[0], exp["num_chars"]), rows)


def test_golden_checkpoint_rows(g1, tmp_path):
    ctx, exp, reads = g1
    k = exp["ckpt_k"]
    d = tmp_path / "ck"
    ops, score, ck = ctx.align_traceback(reads[0], k=k, ckpt_dir=str(d), keep_files=True,
                                         cap_bytes=4 * exp["num_chars"] * 8)
    assert ck and score == exp["scores"][0]
    for i, h in exp["ckpt_rows_sha256"].items():
        assert hashlib.sha256((d / f"row_{i}.bin").read_bytes()).hexdigest() == h
    labels = open(files("g1")[3], "rb").read()
    assert orc.rescore(ops, reads[0], labels) == (exp["scores"][0], len(reads[0]) - 1)


def _score_line(out):
    m = re.search(r"^score: (.*)$", out, re.M)
    return m.group(1).split() if m else None


needs_ref_bins = pytest.mark.skipif(not os.path.exists(orc.REF_CONSGA),
                                    reason="reference drivers not built")


@needs_ref_bins
def test_cli_score_only_matches_reference_driver():
    f = files("g1")
    args = ["-I", f[0], "-i", f[1], "-c", f[2], "-r", os.path.join(GOLD, "g1.reads.fa"), "-l", f[3],
            "-o", f[4]]
    ours = subprocess.run([os.path.join(BIN, "ConSGA_mismatchN_dag")] + args, capture_output=True,
                          text=True, timeout=300)
    ref = subprocess.run([orc.REF_CONSGA] + args, capture_output=True, text=True, timeout=300)
    assert ours.returncode == 0 and ref.returncode == 0, ours.stderr
    assert _score_line(ours.stdout) == _score_line(ref.stdout)
    assert len(_score_line(ours.stdout)) == 5  # load_reads' cap
    assert re.search(r"^\[total over 5 reads\] : ", ours.stdout, re.M)
    env = dict(os.environ, CHSGA_MAX_READS="0", CHSGA_SLOTS="8")
    allr = subprocess.run([os.path.join(BIN, "ConSGA_mismatchN_dag")] + args, capture_output=True,
                          text=True, timeout=300, env=env)
    exp = json.load(open(os.path.join(GOLD, "g1.expected.json")))
    assert [int(x) for x in _score_line(allr.stdout)] == exp["scores"]


@needs_ref_bins
def test_cli_traceback_verification_matches_reference_driver(tmp_path):
    f = files("g1")
    args = ["-I", f[0], "-i", f[1], "-c", f[2], "-r", os.path.join(GOLD, "g1.reads.fa"), "-l", f[3],
            "-o", f[4], "-k", "16"]
    ours = subprocess.run([os.path.join(BIN, "ConSGA_traceback_mismatchN_dag")] + args +
                          ["-d", str(tmp_path / "a")], capture_output=True, text=True, timeout=300)
    ref = subprocess.run([orc.REF_CONSGA_TB] + args + ["-d", str(tmp_path / "b")],
                         capture_output=True, text=True, timeout=300)
    assert ours.returncode == 0, ours.stdout + ours.stderr
    assert ref.returncode == 0
    pat = r"^read\[\d+\] score=\d+$"
    assert re.findall(pat, ours.stdout, re.M) == re.findall(pat, ref.stdout, re.M)
    assert "[RESULT] ALL CHECKS PASSED" in ours.stdout
    assert ours.stdout.count("score_ok   : YES") == 5
    # all reads through the batched traceback: the same lines
    batched = subprocess.run([os.path.join(BIN, "ConSGA_traceback_mismatchN_dag")] + args +
                             ["-d", str(tmp_path / "c")], capture_output=True, text=True, timeout=300,
                             env=dict(os.environ, CHSGA_SLOTS="8"))
    assert batched.returncode == 0, batched.stdout + batched.stderr
    for line in (pat, r"^  CIGAR      : .*$", r"score_ok   : \w+"):
        assert re.findall(line, batched.stdout, re.M) == re.findall(line, ours.stdout, re.M)
    # -b benchmark mode prints the reference's summary lines
    b = subprocess.run([os.path.join(BIN, "ConSGA_traceback_mismatchN_dag"), "-b"] + args,
                       capture_output=True, text=True, timeout=300)
    assert b.returncode == 0 and "[total over 5 reads]" in b.stdout and "Insertions:" in b.stdout
