"""Host logic of the learned proposer (no GPU): shortlist, edge row, descent.

``proposer.propose`` replaces grid_scan + find_minimum (GridScan.jl:25-88,
234-246) by a network shortlist plus a few true determinants.  Here the
network is a stand-in with a known prediction and the determinant a known
function of omega, so the start it returns can be checked against the
oracle's find_minimum over the whole grid.
"""
import numpy as np

from kalnajs_log_spirals_b200 import proposer as P
from oracle import np_oracle as O

GRID = dict(n_Op=41, n_gamma=20, Op_range=(0.2, 0.6), g_range=(0.01, 0.2))
SPEC = P.ModelSpec(4, 7.0, 2)


class BowlNet:
    """Predicts log|det| as a bowl around (Op_c, g_c); features 3 and 4 are
    the grid point's normalised Omega_p and gamma (proposer.features)."""

    def __init__(self, Op_c, g_c):
        self.c = (Op_c, g_c)

    def forward(self, X):
        X = np.asarray(X)
        Op = X[:, 3].astype(np.float64) * 0.3 + 0.5
        g = X[:, 4].astype(np.float64) * 0.145 + 0.155
        y = np.zeros((len(X), 3), dtype=np.float32)
        y[:, 0] = np.log((Op - self.c[0]) ** 2 + (g - self.c[1]) ** 2 + 1e-6)
        return y


def grid_points():
    Op = np.linspace(*GRID["Op_range"], GRID["n_Op"])
    g = np.linspace(*GRID["g_range"], GRID["n_gamma"])
    return Op, g


def scan_argmin(det_fn):
    """The reference workflow's start: every grid point, first minimum in
    column-major order (the oracle's find_minimum)."""
    Op, g = grid_points()
    dg = np.array([[det_fn(np.array([SPEC.m * o + 1j * gg]))[0] for o in Op] for gg in g])
    return O.find_minimum(dg, Op, g)


def counting(det_fn):
    calls = []

    def f(om):
        om = np.asarray(om)
        calls.append(len(om))
        return det_fn(om)
    return f, calls


def test_descent_reaches_the_scan_argmin():
    """The network's bowl is 3 grid cells off the true minimum: the descent
    walks to the scan's own argmin, with far fewer determinants than a scan."""
    Op, g = grid_points()
    root = complex(SPEC.m * Op[17], g[9])
    true = lambda om: (om - root) * (1.0 + 0.1 * (om - root))
    net = BowlNet(Op[20], g[12])
    det_fn, calls = counting(true)
    Op_p, g_p, used = P.propose(net, SPEC, det_fn, k=16, **GRID)
    assert (Op_p, g_p) == scan_argmin(true)
    assert used == sum(calls) < GRID["n_Op"] * GRID["n_gamma"] // 4


def test_edge_row_catches_a_minimum_next_to_the_real_axis():
    """The true minimum sits on the lowest-gamma row far from the shortlist;
    the edge row brings it in."""
    Op, g = grid_points()
    root = complex(SPEC.m * Op[3], 0.0)
    true = lambda om: om - root
    net = BowlNet(Op[35], g[15])
    Op_p, g_p, used = P.propose(net, SPEC, true, k=8, descend=0, **GRID)
    assert (Op_p, g_p) == scan_argmin(true)
    # without the edge row the shortlist alone stays near the network's bowl
    Op_n, g_n, _ = P.propose(net, SPEC, true, k=8, descend=0, edge_rows=0, **GRID)
    assert (Op_n, g_n) != scan_argmin(true)


def test_ties_go_to_the_first_point_in_column_major_order():
    """|det| constant on the grid: find_minimum takes index 0, so does propose."""
    net = BowlNet(0.4, 0.1)
    Op_p, g_p, _ = P.propose(net, SPEC, lambda om: np.ones(len(om)), k=12, **GRID)
    assert (Op_p, g_p) == scan_argmin(lambda om: np.ones(len(om)))


def test_shortlist_is_sorted_column_major_and_of_size_k():
    Op, g = grid_points()
    net = BowlNet(Op[10], g[5])
    so, sg, idx = P.shortlist(net, SPEC, k=9, **GRID)
    assert len(idx) == 9 and np.all(np.diff(idx) > 0)
    nG = GRID["n_gamma"]
    assert np.array_equal(so, Op[idx // nG]) and np.array_equal(sg, g[idx % nG])
    # the bowl's centre and its 8 neighbours are the 9 lowest predictions
    want = sorted(a * nG + b for a in range(9, 12) for b in range(4, 7))
    assert list(idx) == want


def test_network_inputs_are_shape_checked_before_the_library_reads_them():
    """The library reads n x 5 features and n x 3 targets: other shapes raise
    on the host instead of being read out of bounds."""
    import pytest
    X = P.MLP._rows(np.zeros((7, 5), dtype=np.float64), 5)
    assert X.dtype == np.float32 and X.flags.c_contiguous and X.shape == (7, 5)
    assert P.MLP._rows(np.zeros((7, 3)), 3, 7).shape == (7, 3)
    for bad, width, n in ((np.zeros((7, 4)), 5, None), (np.zeros(35), 5, None),
                          (np.zeros((6, 3)), 3, 7)):
        with pytest.raises(ValueError):
            P.MLP._rows(bad, width, n)
