"""The network oracle's backward pass against central finite differences (CPU, FP64)."""
import numpy as np

import mpnn_oracle as mo


def small_graph(n=60, seed=0):
    rng = np.random.default_rng(seed)
    rows = [0]
    cols, vals = [], []
    for i in range(n):
        nb = rng.choice(n, size=5, replace=False)
        nb = nb[nb != i][:4]
        w = rng.uniform(0.2, 1.0, len(nb))
        cols += list(nb) + [i]
        vals += list(-w) + [w.sum() * 1.1]
        rows.append(len(cols))
    row, col, val = np.array(rows), np.array(cols), np.array(vals)
    return mo.graph_from_csr(row, col, val, rng.random(n) < 0.2)


import pytest


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_oracle_gradient_finite_differences(kind):
    rng = np.random.default_rng(1)
    G = small_graph()
    w = rng.normal(0, 0.3, mo.NPARAM)
    r = rng.normal(size=G["U"])
    r /= np.linalg.norm(r)
    t = rng.normal(size=G["U"]) * 0.1
    loss, g, _ = mo.loss_and_grad(w, G, r, t, round_bf16=False, kind=kind)
    idx = np.concatenate([rng.choice(np.arange(0, 320), 12, replace=False),
                          rng.choice(np.arange(320, mo.OFF_WD), 24, replace=False),
                          np.arange(mo.OFF_WD, mo.NPARAM)[::9]])
    eps = 1e-6
    for k in idx:
        wp, wm = w.copy(), w.copy()
        wp[k] += eps
        wm[k] -= eps
        fd = (mo.loss_and_grad(wp, G, r, t, False, kind)[0] - mo.loss_and_grad(wm, G, r, t, False, kind)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(fd)), (k, fd, g[k])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-20])
    y = mo.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0  # ties to even
    assert y[2] == 1.0078125
    assert abs(y[3] + 3.140625) < 1e-12
