"""chsga_align_scores_noalloc: the score-only entry point whose working memory
is a fixed device array inside the library instead of cudaMalloc.

Checked through the C-ABI against chsga_align_scores on two calls in a row
(the second smaller than the first, so state left in the shared array by the
first call would show), plus its size limits. The file name makes pytest
collect it last; it passes alone in a fresh process too, where its first call
does the per-device set-up."""
import numpy as np
import pytest

import chsga_b200 as cb

pytestmark = pytest.mark.gpu


def _free_bytes():
    import torch
    return torch.cuda.mem_get_info(0)[0]


def test_noalloc_matches_align_scores_on_two_calls(small_graph):
    g, files, reads = small_graph
    first = list(reads) + [b""] + g.gen_reads(6, 31, 200, 900, sub_rate=0.02,
                                                 indel_rate=0.01).to_list()
    second = g.gen_reads(5, 32, 20, 90, sub_rate=0.05, indel_rate=0.02,
                         n_rate=0.01).to_list() + [b"", b"A"]
    ctx = cb.Context(0).load(g)
    try:
        want1 = ctx.align_scores(first)
        want2 = ctx.align_scores(second)
        got1 = ctx.align_scores_noalloc(first)
        got2 = ctx.align_scores_noalloc(second)
        np.testing.assert_array_equal(got1, want1)
        np.testing.assert_array_equal(got2, want2)
        # once set up, calls leave the device's free memory unchanged
        before = _free_bytes()
        again1 = ctx.align_scores_noalloc(first)
        again2 = ctx.align_scores_noalloc(second)
        assert _free_bytes() == before
        np.testing.assert_array_equal(again1, want1)
        np.testing.assert_array_equal(again2, want2)
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_array(small_graph):
    g, files, reads = small_graph
    ctx = cb.Context(0).load(g)
    try:
        with pytest.raises(cb.ChsgaError) as e:
            ctx.align_scores_noalloc([b"A" * 65001])
        assert e.value.status == cb.ERR_UNSUPPORTED and "65000" in str(e.value)
        big = [b"ACGT" * 15000] * (cb.NOALLOC_SCRATCH_BYTES // 60000 + 1)
        with pytest.raises(cb.ChsgaError) as e:
            ctx.align_scores_noalloc(big)
        assert e.value.status == cb.ERR_OOM and "CHSGA_NOALLOC_SCRATCH_BYTES" in str(e.value)
        # the rejected calls ran nothing: the next one is still exact
        np.testing.assert_array_equal(ctx.align_scores_noalloc(reads[:4]),
                                      ctx.align_scores(reads[:4]))
    finally:
        ctx.close()
