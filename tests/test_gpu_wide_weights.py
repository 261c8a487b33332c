"""The packed 16-bit sweep kernels (k_pull_lv16, k_down16: eight slots per
lane as four u16x2 words, relaxed by a saturating add and a min) on
hierarchy weights above 65535 and scores up to the 16-bit rows' limit.

A weight is clamped to 65535 and the sum saturates at 65535; that is exact
only because every stored score is at most 65001 (reads of at most 65000
bases), so a sum that saturates can never win the min. The graph is a GFA
chain with three 66,000-base segments among short bubbled ones, whose
contraction leaves upward and downward shortcuts heavier than 65535. The
reads cross the long segments, and one 64,000-base read of N (no label is
N) drives every score to its row index + 1, up to 64,000."""
import os

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc
from conftest import pch_arrays

pytestmark = pytest.mark.gpu


def _gfa(path, seed=3):
    rng = np.random.default_rng(seed)

    def seq(n):
        return "".join("ACGT"[i] for i in rng.integers(0, 4, n))

    lines, nid, prev = [], 1, []
    for i in range(120):
        n = 66_000 if i in (30, 60, 90) else int(rng.integers(5, 30))
        a = nid
        nid += 1
        lines.append(f"S\t{a}\t{seq(n)}")
        cur = [a]
        if i % 3 == 1 and n < 100:
            b = nid
            nid += 1
            lines.append(f"S\t{b}\t{seq(n)}")
            cur.append(b)
        lines += [f"L\t{u}\t+\t{v}\t+\t0M" for u in prev for v in cur]
        prev = cur
    with open(path, "w") as f:
        f.write("H\tVN:Z:1.0\n" + "\n".join(lines) + "\n")


def test_packed_sweeps_with_weights_above_65535(tmp_path):
    _gfa(str(tmp_path / "wide.gfa"))
    g = cb.HostGraph.from_gfa(str(tmp_path / "wide.gfa"))
    g.build_pch()
    a = pch_arrays(g)
    assert (a["up_w"] > 65535).any() and (a["down_w"] > 65535).any()
    files = g.write_files(str(tmp_path / "wide"))
    reads = g.gen_reads(6, 7, 2000, 4000, sub_rate=0.02, indel_rate=0.02).to_list()
    reads.append(b"N" * 64_000)
    o = orc.Oracle(files)
    want = o.scores(reads)
    assert want.max() >= 64_000
    ctx = cb.Context(0).load(g)
    try:
        for slots in (8, 128):
            got = ctx.align_scores_batched(reads, slots=slots)
            assert ctx.profile()["row_bits"] == 16
            np.testing.assert_array_equal(got, want, err_msg=f"{slots} slots")
    finally:
        ctx.close()
