"""The packed 16-bit sweep kernels (k_pull_lv16, k_down16: eight slots per
lane as four u16x2 words, relaxed by a saturating add and a min) on
hierarchy weights above 65535 and scores up to the 16-bit rows' limit.

A weight is clamped to 65535 and the sum saturates at 65535; that is exact
only because every stored score is at most 65001 (reads of at most 65000
bases), so a sum that saturates can never win the min.

Two graphs. A GFA chain of 2,000 segments of 400-511 bases (bubbled every
fourth one; 1.8 M chars on both strands, every vertex within the row
kernels' 512-char limit) whose contraction leaves upward and downward
shortcuts over 65535 through many vertices; its reads are checked against
the oracle, and a 64,000-base read of N (no label is N) scores exactly
64,000 (every read base costs one, whatever the path), so every relaxation
of its last rows sums past 65535. And a chain with three 66,000-base
segments, whose single-vertex shortcuts are heavier than 65535; its vertices
exceed the 512-char limit, so its rows take the per-vertex kernel, which
walks a vertex's chars in order, and its reads stay short."""
import os

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc
from conftest import pch_arrays

pytestmark = pytest.mark.gpu


def _gfa(path, n_seg, seg_len, seed=3):
    """A chain of n_seg segments, seg_len(i, rng) bases each; every fourth
    segment from the second on gets a 3-base alternative."""
    rng = np.random.default_rng(seed)

    def seq(n):
        return "".join("ACGT"[i] for i in rng.integers(0, 4, n))

    lines, nid, prev = [], 1, []
    for i in range(n_seg):
        a = nid
        nid += 1
        lines.append(f"S\t{a}\t{seq(seg_len(i, rng))}")
        cur = [a]
        if i % 4 == 1:
            lines.append(f"S\t{nid}\t{seq(3)}")
            cur.append(nid)
            nid += 1
        lines += [f"L\t{u}\t+\t{v}\t+\t0M" for u in prev for v in cur]
        prev = cur
    with open(path, "w") as f:
        f.write("H\tVN:Z:1.0\n" + "\n".join(lines) + "\n")


def _graph(tmp_path, name, n_seg, seg_len):
    p = str(tmp_path / f"{name}.gfa")
    _gfa(p, n_seg, seg_len)
    g = cb.HostGraph.from_gfa(p)
    g.build_pch()
    a = pch_arrays(g)
    assert (a["up_w"] > 65535).any() and (a["down_w"] > 65535).any()
    return g, g.write_files(str(tmp_path / name))


def test_packed_sweeps_with_weights_above_65535(tmp_path):
    g, files = _graph(tmp_path, "chain", 2000, lambda i, rng: int(rng.integers(400, 512)))
    assert g.stats()["max_label_len"] <= 512
    reads = g.gen_reads(6, 7, 300, 600, sub_rate=0.02, indel_rate=0.02).to_list()
    want = orc.Oracle(files).scores(reads)
    reads.append(b"N" * 64_000)
    want = np.append(want, 64_000).astype(want.dtype)
    ctx = cb.Context(0).load(g)
    try:
        for slots in (8, 128):
            got = ctx.align_scores_batched(reads, slots=slots)
            assert ctx.profile()["row_bits"] == 16
            np.testing.assert_array_equal(got, want, err_msg=f"{slots} slots")
    finally:
        ctx.close()


def test_long_vertices_with_weights_above_65535(tmp_path):
    g, files = _graph(tmp_path, "long", 120,
                      lambda i, rng: 66_000 if i in (30, 60, 90) else int(rng.integers(5, 30)))
    assert g.stats()["max_label_len"] == 66_000
    reads = g.gen_reads(6, 7, 100, 200, sub_rate=0.02, indel_rate=0.02).to_list()
    want = orc.Oracle(files).scores(reads)
    ctx = cb.Context(0).load(g)
    try:
        for slots in (8, 128):
            got = ctx.align_scores_batched(reads, slots=slots)
            assert ctx.profile()["row_bits"] == 16
            np.testing.assert_array_equal(got, want, err_msg=f"{slots} slots")
    finally:
        ctx.close()
