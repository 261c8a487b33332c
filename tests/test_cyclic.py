"""Cyclic graphs: the reference's DAG=0 builds of ConSGA.

DAG only switches code in ParSGA (csr_align.hpp:319, 436 and
csr_traceback.hpp:206, 698); ConSGA's align.hpp and traceback.hpp never read
it, so ConSGA_mismatchN / ConSGA_matchN (DAG=0) compute what the _dag builds
compute, on graphs with cycles too. These tests take a generated bubble
graph, add back links that close cycles of 2 to 8 string vertices, ingest it
as GFA (both orientations), build its hierarchy and check: the oracle equals
the reference's own code (CPU), and the GPU paths equal the oracle (B200).
"""
import os

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc
from conftest import ROOT, gen_graph


def cyclic_graph(tmpdir, backbone_len, seed, back_links):
    g0, _ = gen_graph(tmpdir, "acyclic", backbone_len=backbone_len, seed=seed, vlen_max=12)
    v = g0.view()
    S = v.string_graph.n
    offs = np.ctypeslib.as_array(v.label_offsets, (S + 1,))
    import ctypes
    lab = ctypes.string_at(v.labels, v.num_chars)
    so = np.ctypeslib.as_array(v.string_graph.offset, (S + 1,))
    st = np.ctypeslib.as_array(v.string_graph.target, (v.string_graph.m,))
    rng = np.random.default_rng(seed)
    gfa = os.path.join(str(tmpdir), "cyclic.gfa")
    with open(gfa, "w") as f:
        f.write("H\tVN:Z:1.0\n")
        for s in range(S):
            f.write(f"S\t{s + 1}\t{lab[offs[s]:offs[s + 1]].decode()}\n")
        for s in range(S):
            for e in range(so[s], so[s + 1]):
                f.write(f"L\t{s + 1}\t+\t{int(st[e]) + 1}\t+\t0M\n")
        for _ in range(back_links):
            s = int(rng.integers(10, S))
            f.write(f"L\t{s + 1}\t+\t{s - int(rng.integers(2, 8)) + 1}\t+\t0M\n")
    g = cb.HostGraph.from_gfa(gfa)
    g.build_pch()
    files = g.write_files(os.path.join(str(tmpdir), "cyclic"))
    reads = g0.gen_reads(24, seed + 1, 30, 200, sub_rate=0.03, indel_rate=0.02).to_list()
    return g, files, reads


def test_dag0_drop_in_names_are_built():
    for name in ("ConSGA_mismatchN", "ConSGA_matchN", "ConSGA_traceback_mismatchN",
                 "ConSGA_traceback_matchN"):
        assert os.access(os.path.join(ROOT, "chsga_b200", "bin", name), os.X_OK)


@pytest.mark.skipif(not orc.ref_available(), reason="oracle/_ref not built")
def test_oracle_equals_reference_code_on_a_cyclic_graph(tmp_path):
    g, files, reads = cyclic_graph(tmp_path, 4000, 81, 40)
    assert g.stats()["num_strings"] > 1000
    o, r = orc.Oracle(files), orc.RefHarness(files)
    np.testing.assert_array_equal(o.scores(reads), r.scores(reads))
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    for rd in reads[:4]:
        ops, score, _ = o.traceback(rd, k=40, fast_cap_bytes=0, ckpt_dir=str(tmp_path / "ck"))
        assert orc.rescore(ops, rd, labels) == (score, len(rd) - 1)


@pytest.mark.gpu
def test_gpu_paths_on_a_cyclic_graph(tmp_path):
    g, files, reads = cyclic_graph(tmp_path, 40_000, 83, 400)
    want = orc.Oracle(files).scores(reads)
    ctx = cb.Context(0).load(g)
    np.testing.assert_array_equal(ctx.align_scores(reads), want)
    for slots in (8, 64):
        np.testing.assert_array_equal(ctx.align_scores_batched(reads, slots=slots), want)
    # a top region of 2000 vertices: the lower levels run in the sweep kernels
    np.testing.assert_array_equal(ctx.align_scores_batched(reads, slots=64, top_vertices=2000), want)
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    for rd, w in zip(reads[:3], want[:3]):
        ops, score, _ = ctx.align_traceback(rd)
        assert score == w and orc.rescore(ops, rd, labels) == (w, len(rd) - 1)
    ctx.close()
