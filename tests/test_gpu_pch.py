"""Hierarchy builder with its witness searches on the GPU.

Each round's bounded Dijkstra searches run on the device (pch_gpu.cu) and
must give the very same hierarchy as the host builder: ranks, levels,
layer and component offsets, and both hierarchy CSRs, array for array.
Cases cover label-length weights on and off, a pop limit small enough to
stop searches early (the tie order of the pops then matters), a weight
bound, and a hub vertex of out-degree above the device mask width, whose
searches are redone on the host.
"""
import os
import subprocess

import numpy as np
import pytest

import chsga_b200 as cb
from conftest import ROOT, assert_same, pch_arrays

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "chsga_b200", "bin")


def both(cfg, **opts):
    cpu = cb.HostGraph.generate(**cfg).build_pch(**opts)
    gpu = cb.HostGraph.generate(**cfg).build_pch(gpu_device=0, **opts)
    return pch_arrays(cpu), pch_arrays(gpu)


@pytest.mark.parametrize("over,opts", [
    (dict(backbone_len=60_000, seed=31), {}),
    (dict(backbone_len=60_000, seed=32, vlen_max=4), dict(use_label_lengths=False)),
    (dict(backbone_len=40_000, seed=33), dict(max_pop_count=3)),
    (dict(backbone_len=40_000, seed=34, vlen_min=1, vlen_max=1), dict(max_pop_count=7)),
    (dict(backbone_len=40_000, seed=35), dict(weight_bound=40)),
])
def test_gpu_witness_searches_give_the_same_hierarchy(over, opts):
    cfg = dict(cb.GRAPH_CONFIGS["cfg2"])
    cfg.update(over)
    a, b = both(cfg, **opts)
    assert a["n"] > 1000
    assert_same(a, b)


def test_gpu_builder_on_a_large_graph():
    cfg = dict(cb.GRAPH_CONFIGS["cfg2"])
    cfg.update(backbone_len=1_000_000, seed=36)
    a, b = both(cfg)
    assert a["n"] > 100_000
    assert_same(a, b)


def _hub_gfa(path, spokes=80):
    # a source links to segment 1, which links to every spoke, and every
    # spoke to the sink: the hub has an in-arc and out-degree `spokes`, above
    # what one device mask holds, so its score searches are done on the host
    rng = np.random.default_rng(7)
    seq = lambda n: "".join(rng.choice(list("ACGT"), n))
    lines = ["H\tVN:Z:1.0"]
    sink, src = spokes + 2, spokes + 3
    for i in range(1, src + 1):
        lines.append(f"S\t{i}\t{seq(int(rng.integers(1, 6)))}")
    lines.append(f"L\t{src}\t+\t1\t+\t0M")
    for k in range(2, spokes + 2):
        lines.append(f"L\t1\t+\t{k}\t+\t0M")
        lines.append(f"L\t{k}\t+\t{sink}\t+\t0M")
    open(path, "w").write("\n".join(lines) + "\n")


def test_gpu_builder_hub_searches_fall_back_to_the_host(tmp_path, capfd):
    gfa = str(tmp_path / "hub.gfa")
    _hub_gfa(gfa)
    cpu = cb.HostGraph.from_gfa(gfa).build_pch()
    gpu = cb.HostGraph.from_gfa(gfa).build_pch(gpu_device=0, print_detail=True)
    out = capfd.readouterr().out
    host = [int(l.rsplit(" ", 1)[1].rstrip(")")) for l in out.splitlines()
            if l.startswith("Device witness searches")]
    assert host and sum(host) > 0
    assert_same(pch_arrays(cpu), pch_arrays(gpu))


def test_build_pch_cli_gpu_flag_writes_the_same_file(tmp_path):
    cfg = dict(cb.GRAPH_CONFIGS["cfg2"])
    cfg.update(backbone_len=50_000, seed=37)
    g = cb.HostGraph.generate(**cfg)
    files = g.write_files(str(tmp_path / "g"))
    outs = []
    for extra in ([], ["-g", "0"]):
        out = str(tmp_path / ("h%d.out" % len(extra)))
        r = subprocess.run([os.path.join(BIN, "build_pch"), "-i", files[1], "-o", out, "-v", files[4]]
                           + extra, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        outs.append(open(out, "rb").read())
    assert outs[0] == outs[1]
