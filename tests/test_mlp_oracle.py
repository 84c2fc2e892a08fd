"""The CPU backpropagation of the surrogate (oracle/mlp_oracle.py) against
central finite differences in FP64."""
import numpy as np

from oracle import mlp_oracle as mo


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(0)
    width = 16
    _, n = mo.layout(width)
    p = rng.normal(0, 0.3, n)
    p[mo.layout(width)[0][6][0]:] *= 1.0
    xy = np.stack([rng.uniform(5, 20, 40), rng.uniform(0, 200, 40)], 1)
    T = rng.normal(0, 1, (40, 3))
    dom = (5.0, 20.0, 0.0, 200.0)
    tm, ts = np.array([0.1, -0.2, 0.3]), np.array([1.5, 0.7, 2.0])
    loss, g = mo.loss_and_grad(p, width, xy, T, tm, ts, dom, round_weights=False)
    idx = rng.choice(n, 60, replace=False)
    for i in idx:
        e = np.zeros(n)
        e[i] = 1e-6
        lp, _ = mo.loss_and_grad(p + e, width, xy, T, tm, ts, dom, round_weights=False)
        lm, _ = mo.loss_and_grad(p - e, width, xy, T, tm, ts, dom, round_weights=False)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0])
    r = mo.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
