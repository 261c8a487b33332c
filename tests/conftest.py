"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on CPU.

Small graphs are generated with the library's seeded generator and written
to a temporary directory in the reference's file formats, so the CPU oracle
(oracle/), the reference's own code compiled against its stand-in interfaces
(oracle/_ref) and the GPU path all read the same five input files.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    lib = os.path.join(ROOT, "chsga_b200", "lib", "libchsga.so")
    orc = os.path.join(ROOT, "oracle", "bin", "libconsga_oracle.so")
    if not (os.path.exists(lib) and os.path.exists(orc)):
        import __graft_entry__
        __graft_entry__.build()


_ensure_built()

import chsga_b200 as cb  # noqa: E402
import oracle as orc  # noqa: E402


def gen_graph(tmpdir, name, **over):
    cfg = dict(cb.GRAPH_CONFIGS["cfg1"])
    cfg.update(over)
    g = cb.HostGraph.generate(**cfg)
    g.build_pch()
    files = g.write_files(os.path.join(str(tmpdir), name))
    return g, files


def sprinkle_n(files, rate, seed):
    """Replaces a fraction `rate` of the label bytes with 'N' in the labels
    file of `files` (the hierarchy does not depend on label bytes) and
    returns the graph read back from the files."""
    import numpy as np
    path = files[3]
    raw = bytearray(open(path, "rb").read())
    rng = np.random.default_rng(seed)
    pos = [i for i, b in enumerate(raw) if b in b"ACGT"]
    for i in rng.choice(pos, max(1, int(rate * len(pos))), replace=False):
        raw[int(i)] = ord("N")
    open(path, "wb").write(bytes(raw))
    return cb.HostGraph.read_files(*files)


@pytest.fixture(scope="session")
def small_graph(tmp_path_factory):
    """cfg1 mix on a 20 kbp backbone: ~20k chars, ~1.7k string vertices."""
    d = tmp_path_factory.mktemp("small")
    g, files = gen_graph(d, "g", backbone_len=20_000, seed=11)
    reads = g.gen_reads(24, 5, 150, sub_rate=0.01, indel_rate=0.003, n_rate=0.001).to_list()
    return g, files, reads


@pytest.fixture(scope="session")
def oracle_small(small_graph):
    return orc.Oracle(small_graph[1])


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pch_arrays(g):
    """Every array of the graph's hierarchy (numpy copies), by name."""
    import numpy as np
    p = g.view().pch
    out = {"n": p.n, "m": p.m, "rm": p.rm}
    n, L, K = p.n, p.num_layers, p.num_cc
    sizes = {"rank": n, "level": n, "layer_offset": L + 1, "cc_offset": K + 1,
             "up_offset": n + 1, "down_offset": n + 1, "up_v": p.m, "up_w": p.m,
             "down_v": p.rm, "down_w": p.rm}
    for k, c in sizes.items():
        out[k] = np.ctypeslib.as_array(getattr(p, k), shape=(int(c),)).copy() if c else np.zeros(0)
    return out


def assert_same(a, b):
    import numpy as np
    assert a.keys() == b.keys()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def pch_digest(a):
    """sha256 over the hierarchy arrays of pch_arrays, in name order."""
    import hashlib
    h = hashlib.sha256()
    for k in sorted(a):
        v = a[k]
        h.update(k.encode())
        h.update(v.tobytes() if hasattr(v, "tobytes") else str(v).encode())
    return h.hexdigest()


def edge_reads(g, seed):
    """Reads at the edges of the input domain: one base, a lone N, all N,
    longer than any path of the graph (insertions), a homopolymer, lower
    case and bytes outside the alphabet (compared byte for byte, so they
    mismatch every label), a NUL byte, and the empty read (scored as row 0
    against '\\0', i.e. 1)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n = g.stats()["num_chars"]
    long_read = bytes(rng.choice(np.frombuffer(b"ACGT", np.uint8), 3 * n).astype(np.uint8))
    return [b"A", b"N", b"ACGT", b"N" * 40, long_read, b"T" * 200, b"acgtXYZ-ACGT", b"\x00ACGT", b""]



TINY_GFA = {
    "one_segment": "H\tVN:Z:1.0\nS\t1\tACGTTGCA\n",
    "one_char": "H\tVN:Z:1.0\nS\t1\tA\n",
    "bubble": ("H\tVN:Z:1.0\nS\t1\tACG\nS\t2\tT\nS\t3\tC\nS\t4\tGGA\n"
               "L\t1\t+\t2\t+\t0M\nL\t1\t+\t3\t+\t0M\nL\t2\t+\t4\t+\t0M\nL\t3\t+\t4\t+\t0M\n"),
}
TINY_READS = [b"A", b"ACGT", b"TTTT", b"ACGTTGCAACGT", b"N" * 5, b""]


def tiny_graph(tmpdir, name):
    """A GFA graph of one segment, one base, or a four-segment bubble (both
    orientations), its hierarchy and files."""
    p = os.path.join(str(tmpdir), name + ".gfa")
    with open(p, "w") as f:
        f.write(TINY_GFA[name])
    g = cb.HostGraph.from_gfa(p)
    g.build_pch()
    return g, g.write_files(os.path.join(str(tmpdir), name))
