"""Child process of tests/test_gpu_checked.py: loads the checked build of
the library (CHSGA_LIBRARY, device index checks in every kernel) and runs
every GPU path on one graph; each call fails with CHSGA_ERR_INTERNAL if a
kernel met an index out of range. Prints "checked ok" when every result
also equals the oracle's."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import chsga_b200 as cb  # noqa: E402
import oracle as orc  # noqa: E402


def main(workdir):
    assert cb.LIB_PATH.endswith(os.path.join("lib_checked", "libchsga.so")), cb.LIB_PATH
    cfg = dict(cb.GRAPH_CONFIGS["cfg1"])
    cfg.update(backbone_len=20_000, seed=11)
    g = cb.HostGraph.generate(**cfg)
    g.build_pch()
    files = g.write_files(os.path.join(workdir, "g"))
    reads = g.gen_reads(16, 5, 30, 300, sub_rate=0.02, indel_rate=0.01, n_rate=0.005).to_list()
    o = orc.Oracle(files)
    want = o.scores(reads)
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    ctx = cb.Context(0).load(g)
    np.testing.assert_array_equal(ctx.align_scores(reads), want)
    for slots in (1, 2, 8, 32, 64, 128):
        for rk in (cb.ROW_AUTO, cb.ROW_DIRECT, cb.ROW_DPX, cb.ROW_STREAM, cb.ROW_TILED, cb.ROW_DELTA):
            got = ctx.align_scores_batched(reads, slots=slots, row_kernel=rk)
            np.testing.assert_array_equal(got, want, err_msg=f"slots {slots} row kernel {rk}")
        got = ctx.align_scores_batched(reads, slots=slots, use_graphs=cb.LAUNCH_PERSISTENT)
        np.testing.assert_array_equal(got, want, err_msg=f"persistent, slots {slots}")
        for rb in (32,):
            got = ctx.align_scores_batched(reads, slots=slots, row_bits=rb)
            np.testing.assert_array_equal(got, want, err_msg=f"32-bit rows, slots {slots}")
    np.testing.assert_array_equal(ctx.align_scores_noalloc(reads), want)
    n = o.num_chars
    for rd, w in zip(reads[:4], want[:4]):
        for cap in (0, 40 * n * 4):
            ops, score, ck = ctx.align_traceback(rd, k=30, cap_bytes=cap)
            assert score == w and orc.rescore(ops, rd, labels) == (w, len(rd) - 1)
    got = ctx.align_traceback_batched(reads, slots=16, k=30, cap_bytes=60 * n * 4)
    assert [s for _, s, _ in got] == list(want)
    srv = cb.Server(ctx, slots=8, queue_capacity=64, arena_bytes=1 << 20)
    tk = [srv.submit(r) for r in reads]
    res = srv.collect()
    srv.close()
    assert [res[t]["score"] for t in tk] == list(want)
    ctx.close()
    print("checked ok")


if __name__ == "__main__":
    main(sys.argv[1])
