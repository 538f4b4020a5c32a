"""CPU checks of the proposer's oracle and feature encoding."""
import numpy as np
import pytest

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


class _StubNet:
    """Stands in for the device network: predicted log|det| = distance to a point."""

    def __init__(self, Op, g):
        self.Op, self.g = Op, g

    def forward(self, X):
        Op = X[:, 3] * 0.3 + 0.5               # undo features() for Omega_p, gamma
        g = X[:, 4] * 0.145 + 0.155
        d = np.hypot(Op - self.Op, g - self.g)
        return np.stack([d, np.zeros_like(d), np.ones_like(d)], axis=1).astype(np.float32)


def test_shortlist_takes_the_lowest_predictions_in_column_major_order():
    spec = P.ModelSpec(4, 7.0, 2)
    net = _StubNet(0.41, 0.07)
    Op, g, idx = P.shortlist(net, spec, k=6)
    assert list(idx) == sorted(idx) and len(idx) == 6
    grid_Op = np.linspace(0.2, 0.6, 41)
    grid_g = np.linspace(0.01, 0.2, 20)
    # column-major index q -> (Op column q // n_gamma, gamma row q % n_gamma)
    assert np.allclose(Op, grid_Op[idx // 20]) and np.allclose(g, grid_g[idx % 20])
    # every shortlisted prediction is at most every prediction left out
    y = net.forward(P.features(4, 7.0, 2, np.repeat(grid_Op, 20), np.tile(grid_g, 41)))[:, 0]
    rest = np.setdiff1d(np.arange(41 * 20), idx)
    assert y[idx].max() <= y[rest].min()


def test_propose_picks_the_smallest_true_determinant_of_the_shortlist():
    spec = P.ModelSpec(4, 7.0, 2)
    net = _StubNet(0.41, 0.07)
    calls = []

    def det_fn(om):                                # a true root at Omega_p 0.42, gamma 0.06
        calls.append(len(om))
        return (om.real / 2 - 0.42) + 1j * (om.imag - 0.06)

    Op, g, used = P.propose(net, spec, det_fn, k=12, descend=0, edge_rows=0)
    assert calls == [12] and used == 12
    Ops, gs, _ = P.shortlist(net, spec, k=12)
    best = np.argmin(np.abs((Ops - 0.42) + 1j * (gs - 0.06)))
    assert (Op, g) == (float(Ops[best]), float(gs[best]))


def test_propose_descends_to_the_grid_minimum():
    """The grid descent after the shortlist reaches the grid point of least
    |det| when the shortlist only lands near it."""
    spec = P.ModelSpec(4, 7.0, 2)
    net = _StubNet(0.36, 0.12)                     # shortlist around a point 3 columns away
    calls = []

    def det_fn(om):
        calls.append(len(om))
        return (om.real / 2 - 0.42) + 1j * (om.imag - 0.06)

    Op, g, used = P.propose(net, spec, det_fn, k=6, edge_rows=0)
    grid_Op = np.linspace(0.2, 0.6, 41)
    grid_g = np.linspace(0.01, 0.2, 20)
    d = np.abs((grid_Op[:, None] - 0.42) + 1j * (grid_g[None, :] - 0.06))
    i, j = np.unravel_index(np.argmin(d), d.shape)
    assert (Op, g) == (float(grid_Op[i]), float(grid_g[j]))
    assert calls[0] == 6 and used == sum(calls) and len(calls) > 1


def test_propose_includes_the_lowest_gamma_row():
    """A deep minimum on the grid row next to the real axis, far from the
    network's shortlist, is found through the edge row."""
    spec = P.ModelSpec(4, 7.0, 2)
    net = _StubNet(0.25, 0.15)
    calls = []

    def det_fn(om):                                # a root just below the grid at Omega_p 0.52
        calls.append(len(om))
        return (om.real / 2 - 0.52) + 1j * (om.imag - 0.005)

    Op, g, used = P.propose(net, spec, det_fn, k=12)
    assert (Op, g) == (float(np.linspace(0.2, 0.6, 41)[32]), 0.01)
    assert calls[0] == 12 + 41 - len(set(range(0, 41 * 20, 20)) & set(P.shortlist(net, spec, k=12)[2]))


def test_propose_ties_go_to_the_first_point_in_column_major_order():
    """|det| constant on the grid: find_minimum (GridScan.jl:234-246) takes
    grid index 0, and so does the proposal."""
    spec = P.ModelSpec(4, 7.0, 2)
    net = _StubNet(0.4, 0.1)
    Op, g, _ = P.propose(net, spec, lambda om: np.ones(len(om)), k=12)
    assert (Op, g) == (0.2, 0.01)


def test_network_inputs_are_shape_checked_before_the_library_reads_them():
    """The library reads n x 5 features and n x 3 targets: other shapes raise
    on the host instead of being read out of bounds."""
    X = P.MLP._rows(np.zeros((7, 5), dtype=np.float64), 5)
    assert X.dtype == np.float32 and X.flags.c_contiguous and X.shape == (7, 5)
    assert P.MLP._rows(np.zeros((7, 3)), 3, 7).shape == (7, 3)
    for bad, width, n in ((np.zeros((7, 4)), 5, None), (np.zeros(35), 5, None),
                          (np.zeros((6, 3)), 3, 7)):
        with pytest.raises(ValueError):
            P.MLP._rows(bad, width, n)
