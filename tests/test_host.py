"""Host-side logic of libchsga: no GPU needed.

The C-ABI library loads and exports every entry point include/chsga.h
declares; file formats round-trip; the read loader follows kseq's record
rules and load_reads' upper-casing and 5-read cap; the generator is
deterministic; hierarchies satisfy the level invariants the GPU sweeps rely
on; malformed inputs fail with the documented status codes; the drop-in
tools keep the reference drivers' argument errors.
"""
import ctypes
import gzip
import os
import subprocess

import numpy as np
import pytest

import chsga_b200 as cb
from conftest import ROOT, gen_graph

BIN = os.path.join(ROOT, "chsga_b200", "bin")


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(cb.LIB_PATH)
    names = cb.exported_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_file_round_trip(tmp_path):
    g, files = gen_graph(tmp_path, "a", backbone_len=4000, seed=3)
    h = cb.HostGraph.read_files(*files)
    a, b = g.view(), h.view()
    assert a.num_chars == b.num_chars
    for attr in ("char_graph", "string_graph"):
        x, y = getattr(a, attr), getattr(b, attr)
        assert x.n == y.n and x.m == y.m
        assert np.array_equal(np.ctypeslib.as_array(x.offset, (x.n + 1,)),
                              np.ctypeslib.as_array(y.offset, (y.n + 1,)))
        assert np.array_equal(np.ctypeslib.as_array(x.target, (x.m,)),
                              np.ctypeslib.as_array(y.target, (y.m,)))
    assert a.pch.n == b.pch.n and a.pch.m == b.pch.m and a.pch.rm == b.pch.rm
    # writing the re-read graph reproduces every file byte for byte
    files2 = h.write_files(str(tmp_path / "b"))
    for f1, f2 in zip(files, files2):
        assert open(f1, "rb").read() == open(f2, "rb").read()


def test_generator_is_deterministic(tmp_path):
    _, f1 = gen_graph(tmp_path, "x", backbone_len=3000, seed=9)
    _, f2 = gen_graph(tmp_path, "y", backbone_len=3000, seed=9)
    for a, b in zip(f1, f2):
        assert open(a, "rb").read() == open(b, "rb").read()


def test_char_graph_is_the_string_expansion():
    g = cb.HostGraph.generate(**dict(cb.GRAPH_CONFIGS["cfg1"], backbone_len=3000))
    v = g.view()
    S, N = v.string_graph.n, v.num_chars
    offs = np.ctypeslib.as_array(v.label_offsets, (S + 1,))
    so = np.ctypeslib.as_array(v.string_graph.offset, (S + 1,))
    st = np.ctypeslib.as_array(v.string_graph.target, (v.string_graph.m,))
    co = np.ctypeslib.as_array(v.char_graph.offset, (N + 1,))
    ct = np.ctypeslib.as_array(v.char_graph.target, (v.char_graph.m,))
    for s in range(S):
        for c in range(offs[s], offs[s + 1] - 1):
            assert list(ct[co[c]:co[c + 1]]) == [c + 1]
        last = offs[s + 1] - 1
        assert list(ct[co[last]:co[last + 1]]) == [offs[t] for t in st[so[s]:so[s + 1]]]
    # char ids are topologically ordered (the exact DP relies on it)
    for u in range(N):
        assert all(t > u for t in ct[co[u]:co[u + 1]])


def test_hierarchy_invariants():
    g = cb.HostGraph.generate(**dict(cb.GRAPH_CONFIGS["cfg2"], backbone_len=200_000))
    g.build_pch()
    p = g.view().pch
    n = p.n
    rank = np.ctypeslib.as_array(p.rank, (n,))
    level = np.ctypeslib.as_array(p.level, (n,))
    assert sorted(rank.tolist()) == list(range(n))
    lo = np.ctypeslib.as_array(p.layer_offset, (p.num_layers + 1,))
    assert lo[0] == 0 and lo[-1] == n and (np.diff(lo) > 0).all()
    for off, v, what in ((p.up_offset, p.up_v, "up"), (p.down_offset, p.down_v, "down")):
        o = np.ctypeslib.as_array(off, (n + 1,))
        t = np.ctypeslib.as_array(v, (int(o[-1]),))
        src = np.repeat(np.arange(n), np.diff(o).astype(np.int64))
        # every edge joins a lower level to a strictly higher one
        assert (level[t] > level[src]).all(), what
    st = g.stats()
    assert st["pch_levels"] >= 10 and st["pch_up_edges"] > 0


def test_reads_loader_rules(tmp_path):
    fa = tmp_path / "r.fa"
    fa.write_text(">a x\nacgt\nNNac\n\n>b\nTTT\n>c\nG\n>d\nAA\n>e\nC\n>f\nGG\n")
    assert cb.Reads.load(str(fa)).to_list() == [b"ACGTNNAC", b"TTT", b"G", b"AA", b"C"]
    assert len(cb.Reads.load(str(fa), max_reads=0)) == 6
    fq = tmp_path / "r.fq.gz"
    with gzip.open(fq, "wt") as f:
        f.write("@r1\nACGTA\n+\nIIIII\n@r2\nGG\n+r2\n!!\n")
    assert cb.Reads.load(str(fq), max_reads=0).to_list() == [b"ACGTA", b"GG"]
    with pytest.raises(cb.ChsgaError) as e:
        cb.Reads.load(str(tmp_path / "missing.fa"))
    assert e.value.status == cb.ERR_IO


def test_malformed_inputs_fail_with_status(tmp_path):
    _, files = gen_graph(tmp_path, "m", backbone_len=2000, seed=5)
    bad = list(files)
    bad[2] = str(tmp_path / "nope.out")
    with pytest.raises(cb.ChsgaError) as e:
        cb.HostGraph.read_files(*bad)
    assert e.value.status == cb.ERR_IO
    trunc = tmp_path / "t.out"
    trunc.write_bytes(open(files[2], "rb").read()[:100])
    bad[2] = str(trunc)
    with pytest.raises(cb.ChsgaError) as e:
        cb.HostGraph.read_files(*bad)
    assert e.value.status == cb.ERR_FORMAT
    offs = tmp_path / "o.txt"
    offs.write_text("0 1 2\n")
    bad = list(files)
    bad[4] = str(offs)
    with pytest.raises(cb.ChsgaError) as e:
        cb.HostGraph.read_files(*bad)
    assert e.value.status == cb.ERR_FORMAT


def test_cli_argument_errors(tmp_path):
    for tool in ("ConSGA_mismatchN_dag", "ConSGA_traceback_mismatchN_dag"):
        r = subprocess.run([os.path.join(BIN, tool), "-I", "x"], capture_output=True, text=True)
        assert r.returncode == 1 and "Error: missing required arguments" in r.stderr
        r = subprocess.run([os.path.join(BIN, tool), "-Z"], capture_output=True, text=True)
        assert r.returncode == 1 and "Usage:" in r.stderr
    r = subprocess.run([os.path.join(BIN, "build_pch")], capture_output=True, text=True)
    assert r.returncode == 0 and "Usage" in r.stderr


def test_build_pch_and_gen_tools(tmp_path):
    p = str(tmp_path / "w")
    r = subprocess.run([os.path.join(BIN, "chsga_gen"), "-o", p, "-B", "3000", "-n", "4", "-L", "60"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = str(tmp_path / "again.out")
    r = subprocess.run([os.path.join(BIN, "build_pch"), "-i", p + ".string.adj", "-o", out, "-v",
                        p + ".string.label_offsets"], capture_output=True, text=True)
    assert r.returncode == 0 and "[ build time ]" in r.stdout
    # the tool and the library build the same hierarchy for the same seed
    assert open(out, "rb").read() == open(p + ".string.out", "rb").read()
    assert len(cb.Reads.load(p + ".reads.fa", 0)) == 4


@pytest.mark.parametrize("slots", [32, 64, 128])
@pytest.mark.parametrize("row_bits", [16, 32])
def test_device_layout_preflight(slots, row_bits):
    # builds the kernels' layout and the row kernel's shared-memory tiles on
    # the host and checks every copy bound, alignment and record index the
    # tiled row kernel relies on (chsga_check_layout raises on a violation)
    for cfg in (dict(cb.GRAPH_CONFIGS["cfg2"], backbone_len=300_000),
                dict(cb.GRAPH_CONFIGS["cfg1"], backbone_len=20_000, vlen_max=100)):
        g = cb.HostGraph.generate(**cfg).build_pch()
        st = g.check_layout(slots, row_bits)
        assert st["num_levels"] > 5 and st["top_vertices"] > 0
        if st["tiled"]:
            assert st["tiles"] > 0 and st["smem_bytes"] <= 232448
            assert 2 <= st["slots_per_block"] <= 16


_PCH_DIGESTS = [
    (dict(backbone_len=200_000, seed=9), dict(max_pop_count=3),
     "e578670d7c98789ec0c7aeb7d0b377f4d687bd8bbf35bad64c9d90e8899813f2"),
    (dict(backbone_len=200_000, seed=10, vlen_max=4), dict(use_label_lengths=False),
     "1eb43f61965cf588a840781f44ed73c62b59e3e8c1339c4d78700c5acf812b4c"),
    (dict(backbone_len=200_000, seed=11), dict(weight_bound=40),
     "d71f94094b09880cc3039dfa8f3ebc6bb0a101dde35283644065fedabb6da788"),
    (dict(backbone_len=200_000, seed=12), {},
     "6ac29ab9c2a483e687ee19ae467c6a980a6bbb2fa7e7dd92ddbc7509a4d20356"),
]


@pytest.mark.parametrize("over,opts,digest", _PCH_DIGESTS)
def test_hierarchy_builder_is_deterministic(over, opts, digest):
    """The builder's result depends on neither the thread count nor the
    order its parallel stages finish in; the digests pin the hierarchy of
    each case (pop limit, no label lengths, weight bound, defaults)."""
    from conftest import pch_arrays, pch_digest
    cfg = dict(cb.GRAPH_CONFIGS["cfg2"])
    cfg.update(over)
    many = pch_digest(pch_arrays(cb.HostGraph.generate(**cfg).build_pch(**opts)))
    one = pch_digest(pch_arrays(cb.HostGraph.generate(**cfg).build_pch(threads=1, **opts)))
    assert many == one == digest


def test_gpu_hierarchy_builder_fails_with_a_status_or_matches():
    """build_pch(gpu_device=0) either builds the host builder's hierarchy or,
    without a usable CUDA device, returns an error status; the graph stays
    usable for the host builder."""
    from conftest import assert_same, pch_arrays
    cfg = dict(cb.GRAPH_CONFIGS["cfg1"], backbone_len=3000, seed=44)
    host = pch_arrays(cb.HostGraph.generate(**cfg).build_pch())
    g = cb.HostGraph.generate(**cfg)
    try:
        g.build_pch(gpu_device=0)
    except cb.ChsgaError as e:
        assert "hierarchy builder" in str(e)
        g.build_pch()
    assert_same(pch_arrays(g), host)


def test_layout_rejects_a_second_special_byte(tmp_path):
    """The device layout codes A, C, G, T and one other byte: a labels file
    with 'N' bytes and, later, an 'R' is rejected, naming the two bytes in
    the order they first occur."""
    _, files = gen_graph(tmp_path, "sp", backbone_len=20_000, seed=6)
    lab = bytearray(open(files[3], "rb").read())
    pos = [i for i, b in enumerate(lab) if b in b"ACGT"]
    for i in pos[100:200:7]:
        lab[i] = ord("N")
    lab[pos[5000]] = ord("R")
    bad = list(files)
    bad[3] = str(tmp_path / "two.labels")
    open(bad[3], "wb").write(bytes(lab))
    g = cb.HostGraph.read_files(*bad)
    with pytest.raises(cb.ChsgaError) as e:
        g.check_layout(64, 16)
    assert e.value.status == cb.ERR_UNSUPPORTED
    assert "'N' and 'R'" in str(e.value)
    # one special byte alone is accepted
    lab[pos[5000]] = ord("N")
    open(bad[3], "wb").write(bytes(lab))
    assert cb.HostGraph.read_files(*bad).check_layout(64, 16)["num_levels"] > 0


def test_large_adjacency_file_errors(tmp_path):
    """Adjacency files large enough for the parallel reader still fail with
    the sequential reader's status and message: a target out of range, a
    weight that is not an integer, a weight that is not a number."""
    g, files = gen_graph(tmp_path, "big", backbone_len=600_000, seed=8)
    text = open(files[0]).read()
    assert len(text) > (4 << 20)
    lines = text.split("\n")
    n, m = int(lines[1]), int(lines[2])
    first_target, first_weight = 3 + n, 3 + n + m
    assert lines[first_weight] == "1.0"

    def read_with(line_no, value):
        bad = list(lines)
        bad[line_no] = value
        p = tmp_path / f"bad{line_no}_{value}.adj"
        p.write_text("\n".join(bad))
        return cb.HostGraph.read_files(str(p), *files[1:])

    for line_no, value, status, msg in [
        (first_target + m // 2, str(n), cb.ERR_FORMAT, "edge target out of range"),
        (first_weight + m // 3, "1.5", cb.ERR_UNSUPPORTED, "non-negative integers"),
        (first_weight + m // 3, "x1", cb.ERR_FORMAT, "malformed edge weight"),
    ]:
        with pytest.raises(cb.ChsgaError) as e:
            read_with(line_no, value)
        assert e.value.status == status and msg in str(e.value)
    # a weight of 2 is kept as a weight, not dropped with the all-one case
    h = read_with(first_weight + 5, "2")
    w = np.ctypeslib.as_array(h.view().char_graph.weight, (m,))
    assert w[5] == 2 and (np.delete(w, 5) == 1).all()


def test_packed_u16_relaxation_is_exact():
    """The packed sweep kernels (k_pull_lv16, k_down16) relax 16-bit scores
    as min(f, sat16(x + min(w, 65535))) and derive a last score as
    min(raw, sat16(f + min(len - 1, 65535))). For 16-bit f, x, raw and
    weights in [1, 2^30] that equals the int form (x + w < f ? x + w : f;
    min(raw, f + len - 1)), including scores at 65535 and sums past it."""
    rng = np.random.default_rng(9)
    n = 200_000
    edge = np.array([0, 1, 65533, 65534, 65535], dtype=np.int64)
    f = np.concatenate([rng.integers(0, 65536, n), np.repeat(edge, 5)])
    x = np.concatenate([rng.integers(0, 65536, n), np.tile(edge, 5)])
    w = np.concatenate([rng.integers(1, 1 << 30, n // 2), rng.integers(1, 70000, n - n // 2),
                        np.full(25, 1)])
    sat = lambda a: np.minimum(a, 65535)
    packed = np.minimum(f, sat(x + np.minimum(w, 65535)))
    exact = np.where(x + w < f, x + w, f)
    np.testing.assert_array_equal(packed, exact)
    raw, ln = x, rng.integers(1, 1 << 29, f.size)
    np.testing.assert_array_equal(np.minimum(raw, sat(f + np.minimum(ln - 1, 65535))),
                                  np.minimum(raw, f + ln - 1))


def test_default_top_region_is_the_8000_vertex_region():
    """top_vertices = 0 selects the 8000-vertex region (the levels from the
    highest down while they fit), and larger caps take lower levels."""
    g = cb.HostGraph.generate(**dict(cb.GRAPH_CONFIGS["cfg2"], backbone_len=200_000, seed=5))
    g.build_pch()
    d, k8 = g.check_layout(128, 16, 0), g.check_layout(128, 16, 8000)
    assert (d["top_first_level"], d["top_vertices"]) == (k8["top_first_level"], k8["top_vertices"])
    assert 0 < d["top_vertices"] <= 8000
    big = g.check_layout(128, 16, 23000)
    assert big["top_first_level"] <= d["top_first_level"] and big["top_vertices"] >= d["top_vertices"]
    with pytest.raises(cb.ChsgaError):
        g.check_layout(128, 16, 23001)
