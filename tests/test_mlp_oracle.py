"""The proposal network's CPU restatement pinned by central finite
differences (float64, no BF16 rounding): the hand-written backward of
oracle/mlp_oracle.py must be the derivative of its own loss.  Tolerance:
relative 1e-5 per checked parameter (eps 1e-5; the loss has ReLU and
asymmetric-weight kinks, so the difference quotient is not exact)."""

import numpy as np

from oracle import mlp_oracle as mo


def rays(n, seed):
    rng = np.random.default_rng(seed)
    o = rng.standard_normal((n, 3))
    o = 3.0 * o / np.linalg.norm(o, axis=1, keepdims=True)
    d = -o / 3.0 + 0.4 * rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = rng.uniform(1.0, 4.0, n)
    t[rng.uniform(size=n) < 0.3] = -1.0
    flag = (t >= 0) & (rng.uniform(size=n) < 0.25)  # no-hit rays labelled where they leave the box
    return np.concatenate([o, d, t[:, None], flag[:, None]], 1).astype(np.float32)


def test_backward_matches_finite_differences():
    p = mo.init_params(3).astype(np.float64)
    r = rays(200, 4)
    batch = 64
    g, _, idx, safe = mo.train_grad(p, r, batch, 5, 11, exact=True)
    rng = np.random.default_rng(5)
    # every layer's data and bias columns, rows that matter
    picks = []
    o = 0
    for li, out in enumerate(mo.OUTS):
        rows = out if li < 3 else 2
        for _ in range(6):
            row = rng.integers(0, rows)
            col = rng.choice([rng.integers(0, 78 if li == 0 else 64), mo.ONES[li]])
            picks.append(o + row * mo.K_IN + col)
        o += out * mo.K_IN
    eps = 1e-5
    for i in picks:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (mo.loss_value(pp, r, idx, safe=safe)[0] - mo.loss_value(pm, r, idx, safe=safe)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(fd), 1e-3), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e38], np.float32)
    y = mo.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0 and y[2] == np.float32(1.0 + 2 ** -6) and y[3] == -2.5
