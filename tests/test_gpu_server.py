"""Serving loop (chsga_server_*): score requests through the continuously
refilled batched engine, traceback requests on workers admitted by their
projected device footprint. Every result must equal what the one-shot entry
points give for the same read, alone or in a mix, however the requests
arrive."""
import threading
import time

import numpy as np
import pytest

import chsga_b200 as cb
import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(small_graph):
    c = cb.Context(0).load(small_graph[0])
    yield c
    c.close()


def _mix(g, seed, n, lo, hi):
    return g.gen_reads(n, seed, lo, hi, sub_rate=0.03, indel_rate=0.02, n_rate=0.005).to_list()


@pytest.mark.parametrize("order", [cb.ORDER_FIFO, cb.ORDER_LONGEST])
def test_server_scores_equal_plain_and_oracle(small_graph, ctx, oracle_small, order):
    g, files, reads = small_graph
    mix = list(reads) + _mix(g, 41, 60, 20, 1500) + [b""]
    want = ctx.align_scores(mix)
    np.testing.assert_array_equal(want[:-1], oracle_small.scores(mix[:-1]))
    # fewer result slots than reads: ids and queue entries are reused
    srv = cb.Server(ctx, slots=32, queue_capacity=64, arena_bytes=1 << 20, order=order)
    tickets = [srv.submit(r) for r in mix]
    res = srv.collect()
    st = srv.stats()
    srv.close()
    assert all(res[t]["status"] == cb.OK for t in tickets)
    np.testing.assert_array_equal([res[t]["score"] for t in tickets], want)
    assert st["completed"] == len(mix) and st["failed"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"] and st["gcups"] > 0 and st["gpu_launches"] > 0
    for t in tickets:
        r = res[t]
        assert r["submit_ns"] <= r["start_ns"] <= r["done_ns"]


def test_server_small_arena_and_waves(small_graph, ctx):
    g, files, reads = small_graph
    waves = [_mix(g, 50 + i, 25, 30, 900) for i in range(4)]
    want = [ctx.align_scores(w) for w in waves]
    # an 8 KiB arena holds a few reads at a time: admission waits for space
    srv = cb.Server(ctx, slots=8, queue_capacity=16, arena_bytes=8 << 10, steps_per_graph=4)
    tickets = []

    def producer():
        for w in waves:
            tickets.append([srv.submit(r) for r in w])
            time.sleep(0.02)  # the next wave arrives while the last one runs

    th = threading.Thread(target=producer)
    th.start()
    seen = {}
    while th.is_alive() or len(seen) < sum(map(len, waves)):
        for d in srv.poll(64, 50):
            seen[d["ticket"]] = d
    th.join()
    srv.close()
    for tk, w in zip(tickets, want):
        np.testing.assert_array_equal([seen[t]["score"] for t in tk], w)


def _tb_footprint(n_chars, length):
    # full matrix of 16-bit rows (reads of at most 65000 bases) plus the read
    pitch = (n_chars + 15) // 16 * 16
    return (length + 1) * pitch * 2 + (length + 255) // 256 * 256


def test_same_result_alone_and_in_the_mix(small_graph, ctx):
    g, files, reads = small_graph
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    x = _mix(g, 61, 1, 700, 700)[0]
    y = _mix(g, 62, 1, 400, 400)[0]
    alone = cb.Server(ctx, slots=16)
    tx = alone.submit(x)
    ty = alone.submit(y, cb.REQ_TRACEBACK)
    a = alone.collect()
    alone.close()
    scores = _mix(g, 63, 120, 50, 2000)
    tbs = _mix(g, 64, 6, 100, 500)
    mixed = cb.Server(ctx, slots=16, queue_capacity=32, tb_workers=3)
    out = {}

    def submit_many(items, key):
        out[key] = [mixed.submit(r, m) for r, m in items]

    half = len(scores) // 2
    t1 = threading.Thread(target=submit_many,
                          args=([(r, cb.REQ_SCORE) for r in scores[:half]] + [(x, cb.REQ_SCORE)], "a"))
    t2 = threading.Thread(target=submit_many,
                          args=([(r, cb.REQ_TRACEBACK) for r in tbs[:3]] + [(y, cb.REQ_TRACEBACK)] +
                                [(r, cb.REQ_SCORE) for r in scores[half:]] +
                                [(r, cb.REQ_TRACEBACK) for r in tbs[3:]], "b"))
    t1.start(), t2.start()
    t1.join(), t2.join()
    m = mixed.collect()
    mixed.close()
    rx, ry = m[out["a"][-1]], m[out["b"][3]]
    assert rx["score"] == a[tx]["score"] and rx["vertex"] == a[tx]["vertex"]
    assert ry["score"] == a[ty]["score"]
    np.testing.assert_array_equal(ry["ops"], a[ty]["ops"])
    ops, score, _ = ctx.align_traceback(y)
    np.testing.assert_array_equal(ry["ops"], ops)
    assert orc.rescore(ry["ops"], y, labels) == (score, len(y) - 1)
    np.testing.assert_array_equal([m[t]["score"] for t in out["a"][:-1]], ctx.align_scores(scores[:half]))


def test_traceback_admission_by_footprint(small_graph, ctx):
    g, files, reads = small_graph
    n = ctx_n = small_graph[0].view().num_chars
    tbs = _mix(g, 71, 8, 300, 300)
    fp = _tb_footprint(n, 300)
    # room for one running traceback at a time, whatever the worker count
    srv = cb.Server(ctx, tb_workers=4, hbm_budget_bytes=int(fp * 1.5))
    tickets = [srv.submit(r, cb.REQ_TRACEBACK) for r in tbs]
    res = srv.collect()
    st = srv.stats()
    srv.close()
    assert st["peak_tb_bytes"] == fp
    for t, r in zip(tickets, tbs):
        ops, score, _ = ctx.align_traceback(r)
        assert res[t]["status"] == cb.OK and res[t]["score"] == score
        np.testing.assert_array_equal(res[t]["ops"], ops)
    with pytest.raises(cb.ChsgaError) as e:
        cb.Server(ctx, hbm_budget_bytes=fp // 2).submit(tbs[0], cb.REQ_TRACEBACK)
    assert e.value.status == cb.ERR_OOM
    assert ctx_n == n


def test_checkpointed_traceback_request(small_graph, ctx):
    g, files, reads = small_graph
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    n = small_graph[0].view().num_chars
    r = _mix(g, 81, 1, 500, 500)[0]
    srv = cb.Server(ctx, tb_k=40, tb_cap_bytes=10 * n * 4)
    t = srv.submit(r, cb.REQ_TRACEBACK)
    res = srv.collect()[t]
    srv.close()
    ops, score, ck = ctx.align_traceback(r, k=40, cap_bytes=10 * n * 4)
    assert ck and res["checkpointed"] and res["score"] == score
    np.testing.assert_array_equal(res["ops"], ops)
    assert orc.rescore(res["ops"], r, labels) == (score, len(r) - 1)


def test_busy_and_rejections(small_graph, ctx):
    g, files, reads = small_graph
    srv = cb.Server(ctx, tb_workers=1, max_pending=4)
    long_reads = _mix(g, 91, 40, 600, 600)
    got = [srv.try_submit(r, cb.REQ_TRACEBACK) for r in long_reads]
    assert any(t is None for t in got)
    res = srv.collect()
    assert all(res[t]["status"] == cb.OK for t in got if t is not None)
    with pytest.raises(cb.ChsgaError) as e:
        srv.submit(b"A" * 65001)
    assert e.value.status == cb.ERR_UNSUPPORTED
    with pytest.raises(cb.ChsgaError) as e:
        srv.submit(b"", cb.REQ_TRACEBACK)
    assert e.value.status == cb.ERR_INVALID_ARG
    srv.close()


def test_lane_failure_fails_waiting_and_running_requests(small_graph, ctx):
    # a bounded device wait that runs out inside the running score lane: every
    # request not yet finished completes with ERR_TIMEOUT, finished ones keep
    # their exact scores, later score submissions are refused, and a new
    # server on the same context aligns exactly
    g, files, reads = small_graph
    mix = _mix(g, 61, 160, 300, 1500)
    want = ctx.align_scores(mix)
    srv = cb.Server(ctx, slots=8, queue_capacity=64, arena_bytes=1 << 20, steps_per_graph=4)
    try:
        tickets = [srv.submit(r) for r in mix]
        srv.selftest_fail()
        res = srv.collect()
        st = srv.stats()
        failed = [t for t in tickets if res[t]["status"] != cb.OK]
        assert failed and all(res[t]["status"] == cb.ERR_TIMEOUT for t in failed)
        for t, w in zip(tickets, want):
            if res[t]["status"] == cb.OK:
                assert res[t]["score"] == w
        assert st["failed"] == len(failed) and st["completed"] == len(mix) - len(failed)
        # the last submitted reads were still waiting when the lane failed
        assert res[tickets[-1]]["status"] == cb.ERR_TIMEOUT
        with pytest.raises(cb.ChsgaError) as e:
            srv.submit(mix[0])
        assert e.value.status == cb.ERR_TIMEOUT
    finally:
        srv.close()
    srv2 = cb.Server(ctx, slots=8, queue_capacity=64, arena_bytes=1 << 20, steps_per_graph=4)
    try:
        tk = [srv2.submit(r) for r in mix[:40]]
        res2 = srv2.collect()
    finally:
        srv2.close()
    assert all(res2[t]["status"] == cb.OK for t in tk)
    np.testing.assert_array_equal([res2[t]["score"] for t in tk], want[:40])
