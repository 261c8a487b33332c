"""The FP32 MLP cost model on the GPU: its loss and gradient kernels against
the float64 CPU oracle, training, and what the trained network gains over
the analytic |V| x |read| fallback on logs of the library's own runs."""
import numpy as np
import pytest

import chsga_b200 as cb
import cost_model_oracle as cmo

pytestmark = pytest.mark.gpu


def _random_case(seed, n):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 2, (n, 8)).astype(np.float32)
    y = np.exp(rng.normal(1, 2, (n, 2))).astype(np.float32)
    return x, y


def test_gradient_matches_cpu_oracle():
    m = cb.CostModel(0, seed=5)
    x, y = _random_case(7, 300)
    m.train(x, y, epochs=3, batch=64, lr=1e-3, seed=1)  # fits the normalisation, moves the weights
    p, norm = m.params()
    loss, g = m.loss_grad(x, y)
    want_loss, want_g = cmo.loss_and_grad(p.astype(np.float64), norm, x, y)
    # FP32 kernels against float64: relative 1e-4 on the loss, and on every
    # gradient entry relative 2e-3 of the gradient's largest magnitude
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss)
    scale = np.abs(want_g).max()
    np.testing.assert_allclose(g, want_g, rtol=0, atol=2e-3 * scale)
    # the same network predicts the same values on both sides
    np.testing.assert_allclose(m.predict(x[:50]), cmo.predict(p, norm, x[:50]), rtol=2e-4)
    m.close()


def test_training_fits_a_known_function():
    rng = np.random.default_rng(11)
    x = rng.uniform(-2, 2, (4000, 8)).astype(np.float32)
    t = np.stack([np.exp(0.5 * x[:, 0] + np.abs(x[:, 1])), np.exp(1.0 + x[:, 2] * x[:, 3] / 2)], 1)
    m = cb.CostModel(0, seed=3)
    before, _ = m.loss_grad(x, t)
    after = m.train(x, t.astype(np.float32), epochs=150, batch=256, lr=3e-3, seed=2)
    assert after < 0.05 * before and after < 0.02
    m.close()


def _logs(ctx, g, n_chars):
    """(features, targets) of traceback and score requests run through the
    server: full-matrix and checkpointed tracebacks at several k."""
    feats, targ = [], []
    lens = np.unique(np.geomspace(40, 1500, 36).astype(int))
    cases = [(0, 500), (12 * n_chars * 4, 16), (12 * n_chars * 4, 48), (30 * n_chars * 4, 120)]
    for ci, (cap, k) in enumerate(cases):
        srv = cb.Server(ctx, tb_workers=1, tb_k=k, tb_cap_bytes=cap, slots=16)
        reads = [g.gen_reads(1, 1000 * ci + int(L), int(L), sub_rate=0.03).to_list()[0] for L in lens]
        tk = [srv.submit(r, cb.REQ_TRACEBACK) for r in reads]
        res = srv.collect()
        srv.close()
        for t, r in zip(tk, reads):
            d = res[t]
            assert d["status"] == cb.OK
            feats.append(cb.cm_features(ctx, len(r), cb.REQ_TRACEBACK, 1, k, cap))
            targ.append([(d["done_ns"] - d["start_ns"]) / 1e6, d["peak_bytes"]])
    return np.array(feats, np.float32), np.array(targ, np.float32)


def test_trained_model_beats_analytic_fallback(small_graph):
    g = small_graph[0]
    n = g.view().num_chars
    ctx = cb.Context(0).load(g)
    warm = cb.Server(ctx, tb_workers=1)  # first-use costs stay out of the logs
    warm.submit(g.gen_reads(1, 5, 200).to_list()[0], cb.REQ_TRACEBACK)
    warm.collect()
    warm.close()
    x, y = _logs(ctx, g, n)
    rng = np.random.default_rng(0)
    order = rng.permutation(len(x))
    tr, te = order[: len(x) * 3 // 4], order[len(x) * 3 // 4:]
    m = cb.CostModel(0, seed=9)
    m.train(x[tr], y[tr], epochs=400, batch=32, lr=3e-3, seed=4)
    pred = m.predict(x[te])
    cells = n * (2 ** x[:, 0] - 1)
    # analytic fallback: time = a * |V| * |read| with a fitted on the
    # training logs (geometric mean), bytes = 4 * |V| * |read|
    a = np.exp(np.mean(np.log(y[tr, 0] / cells[tr])))
    ana = np.stack([a * cells[te], 4 * cells[te]], 1)
    err_mlp = np.mean(np.abs(np.log(pred / y[te])), 0)
    err_ana = np.mean(np.abs(np.log(ana / y[te])), 0)
    assert err_mlp[0] < err_ana[0] and err_mlp[1] < err_ana[1], (err_mlp, err_ana)
    assert err_mlp[1] < 0.25  # footprints within ~25 % on held-out requests

    # admission: with the analytic footprint a checkpointed request looks
    # like a full matrix and is refused under a budget that the model (and
    # the request's real peak) fits
    k, cap = 16, 12 * n * 4
    big = g.gen_reads(3, 77, 1400, sub_rate=0.03).to_list()
    budget = int(2.5 * 4 * n * 17 + (1 << 20))
    srv_a = cb.Server(ctx, tb_workers=2, tb_k=k, tb_cap_bytes=cap, hbm_budget_bytes=budget,
                      footprint=cb.FP_ANALYTIC)
    with pytest.raises(cb.ChsgaError) as e:
        srv_a.submit(big[0], cb.REQ_TRACEBACK)
    assert e.value.status == cb.ERR_OOM
    srv_a.close()
    srv_m = cb.Server(ctx, cost_model=m, tb_workers=2, tb_k=k, tb_cap_bytes=cap,
                      hbm_budget_bytes=budget, footprint=cb.FP_MODEL)
    tk = [srv_m.submit(r, cb.REQ_TRACEBACK) for r in big]
    res = srv_m.collect()
    srv_m.close()
    for t, r in zip(tk, big):
        ops, score, ck = ctx.align_traceback(r, k=k, cap_bytes=cap)
        assert ck and res[t]["status"] == cb.OK and res[t]["score"] == score
        np.testing.assert_array_equal(res[t]["ops"], ops)
        assert res[t]["peak_bytes"] <= budget and res[t]["predicted_ms"] > 0
    ctx.close()


def _server_logs(ctx, g, n_chars, reads, mode, slots, k=500, cap=0):
    # a server's score lane has at least 2 slots; traceback requests run one
    # read at a time whatever it has
    srv = cb.Server(ctx, slots=max(2, slots), tb_workers=1, tb_k=k, tb_cap_bytes=cap)
    tk = [srv.submit(r, mode) for r in reads]
    res = srv.collect()
    srv.close()
    x, y = [], []
    for t, r in zip(tk, reads):
        d = res[t]
        assert d["status"] == cb.OK
        x.append(cb.cm_features(ctx, len(r), mode, slots if mode == cb.REQ_SCORE else 1, k, cap))
        by = d["peak_bytes"] if mode == cb.REQ_TRACEBACK else 4.0 * (n_chars + 32) + len(r)
        y.append([max(1e-3, (d["done_ns"] - d["start_ns"]) / 1e6), by])
    return x, y


def test_gain_on_config2_size_graph_logs():
    # logs of the library's own runs on the 5 Mbp config-2 graph: score
    # requests at two slot counts, full-matrix and checkpointed tracebacks;
    # the network trained on 3/4 of them predicts the held-out quarter's
    # device time and bytes better than the analytic |V| x |read| model
    g = cb.HostGraph.generate(**cb.GRAPH_CONFIGS["cfg2"])
    g.build_pch()
    n = g.stats()["num_chars"]
    ctx = cb.Context(0).load(g)
    try:
        def mk(count, seed, lo, hi):
            return g.gen_reads(count, seed, lo, hi, sub_rate=0.02, indel_rate=0.03).to_list()
        x, y = [], []
        for slots, seed in ((16, 1), (64, 2)):
            a, b = _server_logs(ctx, g, n, mk(48, seed, 150, 3000), cb.REQ_SCORE, slots)
            x += a
            y += b
        a, b = _server_logs(ctx, g, n, mk(24, 3, 100, 1500), cb.REQ_TRACEBACK, 1)
        x += a
        y += b
        for k, seed in ((64, 4), (200, 5)):
            a, b = _server_logs(ctx, g, n, mk(8, seed, 300, 1500), cb.REQ_TRACEBACK, 1, k=k,
                                cap=12 * n * 4)
            x += a
            y += b
    finally:
        ctx.close()
    x, y = np.array(x, np.float32), np.array(y, np.float32)
    order = np.random.default_rng(1).permutation(len(x))
    tr, te = order[: len(x) * 3 // 4], order[len(x) * 3 // 4:]
    m = cb.CostModel(0, seed=9)
    m.train(x[tr], y[tr], epochs=1500, batch=32, lr=2e-3, seed=4)
    pred = m.predict(x[te])
    m.close()
    cells = n * (2 ** x[:, 0] - 1)
    a = np.exp(np.mean(np.log(y[tr, 0] / cells[tr])))
    ana = np.stack([a * cells[te], 4 * cells[te]], 1)
    err_mlp = np.mean(np.abs(np.log(pred / y[te])), 0)
    err_ana = np.mean(np.abs(np.log(ana / y[te])), 0)
    assert err_mlp[0] < err_ana[0] and err_mlp[1] < err_ana[1], (err_mlp, err_ana)
