"""CPU checks of the proposer's oracle and feature encoding."""
import numpy as np

from oracle import np_mlp as O
from kalnajs_log_spirals_b200 import proposer as P


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    width, depth = 16, 3
    n = sum(di * do + do for di, do in O.layer_shapes(width, depth))
    p = rng.normal(scale=0.4, size=n)
    X = rng.normal(size=(7, 5))
    T = rng.normal(size=(7, 3))
    _, _, g = O.forward_backward(p, X, T, width, depth, bf16_ops=False)
    idx = rng.choice(n, 40, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = O.forward_backward(pp, X, T, width, depth, bf16_ops=False)[1]
        lm = O.forward_backward(pm, X, T, width, depth, bf16_ops=False)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159], dtype=np.float32)
    b = O.bf16(x)
    assert b[0] == 1.0 and b[1] == 1.0          # tie to even
    assert b[2] == np.float32(1.0078125)        # rounds up
    assert abs(b[3] + 3.140625) < 1e-6


def test_features_and_targets():
    x = P.features(4, 8.0, 2, [0.5, 0.2], [0.155, 0.3])
    assert x.shape == (2, 5) and x.dtype == np.float32
    assert np.allclose(x[0], [0, 0, -1, 0, 0])
    t = P.targets(np.array([np.exp(-5.0) * np.exp(1j * 0.3)]))
    assert np.allclose(t[0], [-0.5, np.sin(0.3), np.cos(0.3)], atol=1e-6)


def test_random_models_are_seeded():
    a = P.random_models(5, 3)
    b = P.random_models(5, 3)
    assert a == b
    assert all(2 <= s.n_zang <= 6 and 4 <= s.q1 <= 12 and s.m in (2, 3) for s in a)
