"""ORACLE — test infrastructure, not product code.

A float64 numpy restatement of the library's FP32 cost-model MLP
(chsga_b200/csrc/cost_model.cu): standardised features -> 64 ReLU -> 64
ReLU -> 2 outputs, loss 1/(2n) * sum (o - t)^2 over standardised log
targets t, and its gradient by back-propagation. The MLP has no reference
counterpart, so this oracle is pinned by finite differences of its own loss
(tests/test_cost_model.py), and the GPU kernels' loss and gradient are
checked against it. Only tests/ use it.

Parameter layout (one flat array, as the C-ABI's chsga_cm_get_params):
  W1[8][64] b1[64] W2[64][64] b2[64] W3[64][2] b3[2]
normalisation: x mean[8], x std[8], log-target mean[2], log-target std[2].
"""
from __future__ import annotations

import numpy as np

F, H, O = 8, 64, 2
SIZES = [("W1", (F, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, O)), ("b3", (O,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p: np.ndarray) -> dict:
    out, off = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[off:off + n], dtype=np.float64).reshape(shape)
        off += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([d[name].reshape(-1) for name, _ in SIZES])


def loss_and_grad(params, norm, x, y):
    """Loss and flat gradient (float64) of the batch (x: n x 8, y: n x 2 raw)."""
    w = unpack(params)
    norm = np.asarray(norm, dtype=np.float64)
    xm, xs, ym, ys = norm[:F], norm[F:2 * F], norm[2 * F:2 * F + O], norm[2 * F + O:]
    n = x.shape[0]
    xn = (np.asarray(x, np.float64) - xm) / xs
    t = (np.log(np.asarray(y, np.float64)) - ym) / ys
    z1 = xn @ w["W1"] + w["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w["W2"] + w["b2"]
    h2 = np.maximum(z2, 0)
    o = h2 @ w["W3"] + w["b3"]
    loss = 0.5 / n * np.sum((o - t) ** 2)
    d = (o - t) / n
    g = {"W3": h2.T @ d, "b3": d.sum(0)}
    dz2 = (d @ w["W3"].T) * (h2 > 0)
    g["W2"], g["b2"] = h1.T @ dz2, dz2.sum(0)
    dz1 = (dz2 @ w["W2"].T) * (h1 > 0)
    g["W1"], g["b1"] = xn.T @ dz1, dz1.sum(0)
    return loss, pack(g)


def predict(params, norm, x):
    """Predictions in raw units (time ms, bytes), n x 2."""
    w = unpack(params)
    norm = np.asarray(norm, dtype=np.float64)
    xm, xs, ym, ys = norm[:F], norm[F:2 * F], norm[2 * F:2 * F + O], norm[2 * F + O:]
    xn = (np.asarray(x, np.float64) - xm) / xs
    h1 = np.maximum(xn @ w["W1"] + w["b1"], 0)
    h2 = np.maximum(h1 @ w["W2"] + w["b2"], 0)
    return np.exp((h2 @ w["W3"] + w["b3"]) * ys + ym)


def loss_only(params, norm, x, y):
    return loss_and_grad(params, norm, x, y)[0]
