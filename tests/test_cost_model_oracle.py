"""The cost model's CPU oracle (oracle/cost_model_oracle.py) pinned by
finite differences of its own loss: the back-propagated gradient must match
central differences in float64."""
import numpy as np

import cost_model_oracle as cmo


def _case(seed, n=12):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, cmo.NUM_PARAMS)
    norm = np.concatenate([rng.normal(0, 1, 8), rng.uniform(0.5, 2, 8), rng.normal(0, 1, 2),
                           rng.uniform(0.5, 2, 2)])
    x = rng.normal(0, 1.5, (n, 8))
    y = np.exp(rng.normal(0, 2, (n, 2)))
    return p, norm, x, y


def test_oracle_gradient_matches_finite_differences():
    p, norm, x, y = _case(1)
    _, g = cmo.loss_and_grad(p, norm, x, y)
    rng = np.random.default_rng(2)
    idx = rng.choice(cmo.NUM_PARAMS, 300, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (cmo.loss_only(p + e, norm, x, y) - cmo.loss_only(p - e, norm, x, y)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_oracle_layout_and_prediction():
    assert cmo.NUM_PARAMS == 4866
    p, norm, x, y = _case(3, 5)
    w = cmo.unpack(p)
    assert np.array_equal(cmo.pack(w), p)
    # a network of zeros predicts exp(ym) for every input
    z = np.zeros(cmo.NUM_PARAMS)
    out = cmo.predict(z, norm, x)
    np.testing.assert_allclose(out, np.broadcast_to(np.exp(norm[16:18]), out.shape))
