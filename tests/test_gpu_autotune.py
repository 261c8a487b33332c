"""Autotuner and the batched engine's knobs: every row kernel and level
grouping returns the plain path's scores, and the tuned options do too."""
import numpy as np
import pytest

import chsga_b200 as cb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(small_graph):
    c = cb.Context(0).load(small_graph[0])
    yield c
    c.close()


def _mix(g, seed, n):
    rng = np.random.default_rng(seed)
    lens = np.exp(rng.uniform(np.log(30), np.log(1200), n)).astype(int)
    return [g.gen_reads(1, int(seed * 1000 + i), int(L), sub_rate=0.03, indel_rate=0.02).to_list()[0]
            for i, L in enumerate(lens)]


@pytest.mark.parametrize("row_kernel", [cb.ROW_AUTO, cb.ROW_DIRECT, cb.ROW_TILED, cb.ROW_DPX,
                                        cb.ROW_STREAM])
@pytest.mark.parametrize("top_vertices", [0, 300])
@pytest.mark.parametrize("slots", [32, 128])
def test_knobs_keep_scores(small_graph, ctx, row_kernel, top_vertices, slots):
    g = small_graph[0]
    reads = _mix(g, 3, 40)
    want = ctx.align_scores(reads)
    got = ctx.align_scores_batched(reads, slots=slots, row_kernel=row_kernel,
                                   top_vertices=top_vertices)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("row_kernel", [cb.ROW_DPX, cb.ROW_STREAM])
def test_row_kernels_on_long_vertices(tmp_path, row_kernel):
    # vertices up to 300 chars (several prefetch blocks), N in the reads
    from conftest import gen_graph
    g, files = gen_graph(tmp_path, "lv", backbone_len=6000, seed=17, vlen_min=40, vlen_max=300,
                         bubble_gap_mean=30.0, p_snp=0.3, p_indel=0.3, p_alt=0.4, alt_min=20,
                         alt_max=200)
    reads = g.gen_reads(64, 18, 20, 800, sub_rate=0.04, indel_rate=0.03, n_rate=0.01).to_list()
    c = cb.Context(0).load(g)
    want = c.align_scores(reads)
    for slots in (64, 128):
        got = c.align_scores_batched(reads, slots=slots, row_kernel=row_kernel)
        np.testing.assert_array_equal(got, want)
    c.close()


def test_autotune_picks_a_correct_config(small_graph, ctx):
    g = small_graph[0]
    reads = _mix(g, 5, 48)
    best, trials = ctx.autotune(reads, repeats=1)
    assert len(trials) >= 9 and all(t["measured_gcups"] > 0 for t in trials)
    fastest = max(trials, key=lambda t: t["measured_gcups"])
    assert best["slots"] == fastest["slots"] and best["top_vertices"] == fastest["top_vertices"]
    got = ctx.align_scores_batched(reads, slots=best["slots"], steps_per_graph=best["steps_per_graph"],
                                   row_kernel=best["row_kernel"], top_vertices=best["top_vertices"])
    np.testing.assert_array_equal(got, ctx.align_scores(reads))


def test_autotune_with_cost_model_measures_fewer(small_graph, ctx):
    g = small_graph[0]
    n = g.view().num_chars
    feats, targ = [], []
    for R in (16, 32, 64, 128):
        reads = _mix(g, 10 + R, 64)
        ctx.align_scores_batched(reads, slots=R)
        a, d = ctx.read_times(len(reads))
        for r, t0, t1 in zip(reads, a, d):
            feats.append(cb.cm_features(ctx, len(r), cb.REQ_SCORE, R))
            targ.append([max((int(t1) - int(t0)) / 1e6, 1e-3), 4.0 * (n + 32) + len(r)])
    m = cb.CostModel(0, seed=1)
    m.train(np.array(feats), np.array(targ), epochs=300, batch=32, seed=3)
    reads = _mix(g, 99, 48)
    best, trials = ctx.autotune(reads, cost_model=m, measure_top=2, repeats=1)
    slot_trials = trials[:4]
    assert sum(t["measured_gcups"] > 0 for t in slot_trials) == 2
    assert all(t["predicted_gcups"] > 0 for t in slot_trials)
    got = ctx.align_scores_batched(reads, slots=best["slots"], steps_per_graph=best["steps_per_graph"],
                                   row_kernel=best["row_kernel"], top_vertices=best["top_vertices"])
    np.testing.assert_array_equal(got, ctx.align_scores(reads))
    m.close()
