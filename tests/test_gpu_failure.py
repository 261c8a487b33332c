"""Failure detection without a GPU fault: a device-side bounded wait that
cannot succeed (nothing completes its mbarrier) gives up, the host reads the
flag and the call fails with CHSGA_ERR_TIMEOUT; the context is still usable
afterwards."""
import time

import numpy as np
import pytest

import chsga_b200 as cb

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_survives(small_graph, oracle_small):
    g, files, reads = small_graph
    ctx = cb.Context(0).load(g)
    t = time.perf_counter()
    with pytest.raises(cb.ChsgaError) as e:
        ctx.selftest_wait(4096)
    assert e.value.status == cb.ERR_TIMEOUT and "wait" in str(e.value)
    assert time.perf_counter() - t < 30
    # same context, same stream: alignments still run and are exact
    np.testing.assert_array_equal(ctx.align_scores(reads[:4]), oracle_small.scores(reads[:4]))
    np.testing.assert_array_equal(ctx.align_scores_batched(reads, slots=32), oracle_small.scores(reads))
    ctx.close()


def test_grid_barrier_wait_runs_out_and_context_survives(small_graph, oracle_small):
    # the persistent kernel's grid barrier with one block that never arrives:
    # the waiting block gives up after 2 ms of device time and flags the call
    g, files, reads = small_graph
    ctx = cb.Context(0).load(g)
    t = time.perf_counter()
    with pytest.raises(cb.ChsgaError) as e:
        ctx.selftest_grid_wait(2000)
    assert e.value.status == cb.ERR_TIMEOUT and "code 4" in str(e.value)
    assert time.perf_counter() - t < 30
    # the next persistent launch starts from a reset barrier and is exact
    np.testing.assert_array_equal(
        ctx.align_scores_batched(reads, slots=8, use_graphs=cb.LAUNCH_PERSISTENT),
        oracle_small.scores(reads))
    np.testing.assert_array_equal(ctx.align_scores(reads[:4]), oracle_small.scores(reads[:4]))
    ctx.close()
