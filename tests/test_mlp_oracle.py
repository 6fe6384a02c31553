"""CPU checks of the predictor's oracle (no GPU).

The oracle's backward pass must be the derivative of its loss (central finite
differences in FP64), and its BF16 rounding must be round-to-nearest-even.
"""

import numpy as np

from oracle import mlp_oracle as mo


def _problem(seed=0, n=48):
    rng = np.random.default_rng(seed)
    p = np.zeros(mo.N_PARAMS)
    p[mo.W1:mo.B1] = rng.normal(0, np.sqrt(2 / mo.N_IN), mo.B1 - mo.W1)
    p[mo.B1:mo.W2] = rng.normal(0, 0.1, mo.W2 - mo.B1)
    p[mo.W2:mo.B2] = rng.normal(0, np.sqrt(2 / 64), mo.B2 - mo.W2)
    p[mo.B2:mo.W3] = rng.normal(0, 0.1, mo.W3 - mo.B2)
    p[mo.W3:mo.B3] = rng.normal(0, 0.3, mo.B3 - mo.W3)
    p[mo.B3] = 0.1
    X = rng.uniform(-1, 1, (n, mo.N_IN))
    y = (rng.uniform(size=n) < 0.3).astype(np.uint8)
    return p, X, y


def test_gradient_matches_finite_differences():
    p, X, y = _problem()
    g, loss = mo.gradients(p, X, y, pos_weight=2.5, bf16_operands=False)
    assert abs(loss - mo.loss(p, X, y, 2.5)) < 1e-12
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(mo.N_PARAMS - 1, 60, replace=False), [mo.B3, mo.B1, mo.B2, mo.W3]])
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (mo.loss(p + e, X, y, 2.5) - mo.loss(p - e, X, y, 2.5)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounds_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0, 3.0e38], dtype=np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                # tie -> even (mantissa 0)
    assert r[2] == 1.0 + 4 * 2 ** -8  # tie -> even (mantissa 2)
    assert r[3] == 1.0
    assert r[4] == -2.5 and r[5] == 0.0
    assert np.all(mo.from_bf16_bits(mo.bf16_bits(r)) == r)


def test_features_are_signed_log_differences():
    rng = np.random.default_rng(2)
    w = rng.uniform(0.5, 1.5, (5, 10, 12))
    f = mo.features(w, (0, 1, 2, 4), ranges=np.ones(4), ghosts=2)
    assert f.shape == (6 * 8, mo.N_IN)
    # centre offset (0, 0) is always zero; antisymmetry of opposite offsets on a linear field
    assert np.all(f[:, 12] == 0) and np.all(f[:, 25 + 12] == 0)
    lin = np.broadcast_to(np.arange(10.0)[:, None], (10, 12))
    w2 = np.stack([lin] * 5)
    f2 = mo.features(w2, (0, 1, 2, 4), ranges=np.ones(4), ghosts=2)
    assert np.allclose(f2[:, 0 * 5 + 2], -f2[:, 4 * 5 + 2])
    assert np.all(np.abs(f2) <= np.log1p(4 / mo.EPS) / np.log1p(1 / mo.EPS) + 1e-12)
