"""The CPU oracle of the warm-start network: its hand-derived gradient against
central finite differences (CPU-only; the network has no reference
counterpart, so this pins the oracle the GPU kernels are checked against)."""
from __future__ import annotations

import numpy as np

import gnn_oracle as G
from mcpdlp import generators


def tiny_instance():
    m = generators.transport(11, 4, 5)
    rng = np.random.default_rng(0)
    return m, rng.uniform(0, 50, m.num_cols), rng.normal(0, 0.3, m.num_rows), 0.4


def test_layout_size():
    L = G.layout(3)
    assert L["_total"][0] == 6 * 64 + 64 + 5 * 64 + 64 + 3 * (4 * 64 * 64 + 2 * 64) + 4 * 64 + 3


def test_gradient_matches_finite_differences():
    model, x, y, lw = tiny_instance()
    rng = np.random.default_rng(1)
    theta = rng.normal(0, 0.1, G.layout(3)["_total"][0])
    loss, grad, _ = G.loss_and_grad(theta, model, x, y, lw)
    idx = rng.choice(theta.size, 60, replace=False)
    L = G.layout(3)
    idx = np.concatenate([idx, [L["bx"][0], L["bw"][0], L["uv"][0], L["Wve"][0] + 3, L["Wcn0"][0] + 7]])
    eps = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += eps
        tm[i] -= eps
        fd = (G.loss_and_grad(tp, model, x, y, lw)[0] - G.loss_and_grad(tm, model, x, y, lw)[0]) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, grad[i])


def test_predict_shapes_and_units():
    model, _, _, _ = tiny_instance()
    theta = np.zeros(G.layout(3)["_total"][0])
    x, y, lw = G.predict(theta, model)
    assert x.shape == (model.num_cols,) and y.shape == (model.num_rows,) and np.isscalar(lw)
    assert np.all(x == 0) and np.all(y == 0) and lw == 0
