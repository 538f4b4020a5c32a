"""The oracle against the reference's published results and known answers.

Pins: ``convergence_table.txt:13-14`` of the reference (MATLAB
NL_newton_search.m output, printed to 10 decimals) for ``configs/small.toml``
with ``models/kalnajs_zang4.toml``, l_max = 10 and 25.
"""
import math

import numpy as np
import pytest

from oracle import np_oracle as O

SMALL = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=61, Ne=21, Rc_min=0.01, Rc_max=10.0,
             v_min=0.01, N_alpha=101, alpha_max=10.0, l_min=-10, l_max=10, nw=10001, nwa=201)

# (l_max, Omega_p, gamma) from convergence_table.txt:13-14
GOLDEN_ROOTS = [(10, 0.4397142267, 0.1230663944), (25, 0.4401281969, 0.1245357121)]
BAND = 5e-11 + 1e-11   # 10-decimal rounding band + Newton stopping slack


@pytest.mark.parametrize("lmax,Op_ref,g_ref", GOLDEN_ROOTS)
def test_oracle_reproduces_published_root(lmax, Op_ref, g_ref):
    c = O.OracleConfig(**{**SMALL, "l_min": -lmax, "l_max": lmax})
    pc = O.precompute_all(c)
    r = O.newton_search(lambda w: O.compute_det(pc, w), c.m, 0.44, 0.13, tol=1e-12, delta=1e-6)
    assert r.converged
    assert abs(r.Omega_p - Op_ref) <= BAND
    assert abs(r.gamma - g_ref) <= BAND


def test_line_search_variant_same_root():
    c = O.OracleConfig(**SMALL)
    pc = O.precompute_all(c)
    f = lambda w: O.compute_det(pc, w)
    a = O.newton_search(f, c.m, 0.44, 0.13, tol=1e-12)
    b = O.newton_search(f, c.m, 0.44, 0.13, tol=1e-12, use_line_search=True)
    assert a.converged and b.converged
    assert abs(a.Omega_p - b.Omega_p) < 1e-11 and abs(a.gamma - b.gamma) < 1e-11


def test_quadrature_weights_sum_to_interval():
    x = np.linspace(0.3, 2.7, 11)
    assert math.isclose(O.trapezoid_coef(x).sum(), 2.4, rel_tol=1e-14)
    assert math.isclose(O.simpson_coef(x).sum(), 2.4, rel_tol=1e-14)
    xe = np.linspace(0.3, 2.7, 10)          # even length: Simpson falls back to trapezoid
    assert np.array_equal(O.simpson_coef(xe), O.trapezoid_coef(xe))
    assert O.trapezoid_coef(np.array([1.0])).tolist() == [0.0]


def test_circular_orbit_known_answer():
    c = O.OracleConfig(NR=5, Ne=3, nw=201, nwa=21, Rc_min=0.1, Rc_max=10.0, v_min=0.5)
    model = O.ToomreZang.from_config(c)
    g = O.compute_grids(c, model)
    o = O.compute_orbits(c, model, g)
    R = g.Rc[:, -1]                         # v = 1 column: e = 0
    assert np.allclose(o.Omega_1[:, -1], math.sqrt(2) / R, rtol=1e-15)
    assert np.allclose(o.Omega_2[:, -1], 1 / R, rtol=1e-15)
    assert np.all(o.jacobian[:, -1] == 0.0)
    # W_l of a circular orbit: R^{-1/2} e^{-i alpha ln R} for l = 0 (w1 spans (0, pi))
    alpha = np.linspace(-3, 3, 5)
    W = O.compute_W_l(c, o, alpha, np.array([0]))
    p = 2 + c.NR * (c.Ne - 1)
    wa = o.w1[2, -1]
    span = wa[-1] - wa[0]
    # phi = (Om2/Om1) w1 - theta = 0 on a circular orbit, so cos(m phi) = 1 and
    # the trapezoid weights sum to the w1 span
    expect = R[2] ** -0.5 * np.exp(-1j * alpha * math.log(R[2])) * span / math.pi
    assert np.allclose(W[p, :, 0], expect, rtol=1e-12)


def test_N_kernel_against_direct_gamma():
    import scipy.special as sps
    alpha = np.linspace(-30, 30, 61)
    d = O.trapezoid_coef(alpha)
    for m in (1, 2, 3):
        N = O.compute_N_kernel(m, alpha, d)
        ia = 1j * alpha
        direct = np.real(sps.gamma((m + 0.5 + ia) / 2) * sps.gamma((m + 0.5 - ia) / 2)
                         / (sps.gamma((m + 1.5 + ia) / 2) * sps.gamma((m + 1.5 - ia) / 2))) \
            * math.pi * d
        assert np.allclose(N, direct, rtol=1e-12)


def test_det_identity_when_G_zero():
    c = O.OracleConfig(NR=6, Ne=5, N_alpha=7, l_min=-2, l_max=2, nw=101, nwa=11, G=0.0)
    pc = O.precompute_all(c)
    assert O.compute_det(pc, 0.9 + 0.1j) == 1.0


def test_denominator_clamp():
    c = O.OracleConfig(NR=6, Ne=5, N_alpha=7, l_min=-2, l_max=2, nw=101, nwa=11)
    pc = O.precompute_all(c)
    om = complex(pc.Omega_res[7, 3], 0.0)     # exactly resonant
    w = O.weights(pc, om)
    assert w[7, 3] == pc.DJ[7] * pc.F0l[7, 3] / (1e-12 + 1e-12j)


def test_find_minimum_column_major_first():
    g = np.array([[3, 1, 5], [1, 4, 1]], dtype=complex)
    # minima |1| at (0,1), (1,0), (1,2); column-major first is (1,0)
    assert O.find_minimum(g, np.array([0.1, 0.2, 0.3]), np.array([0.01, 0.02])) == (0.1, 0.02)


def test_boole_rule_is_exact_to_degree_five():
    x = np.linspace(0.0, 2.0, 9)                 # n = 4k + 1
    S = O.boole_coef(x)
    for k in range(6):
        exact = 2.0 ** (k + 1) / (k + 1)
        assert abs(np.dot(S, x ** k) - exact) < 1e-13 * exact, k
    assert abs(np.dot(S, x ** 6) - 2.0 ** 7 / 7) > 1e-6   # degree 6 is not exact


def test_boole_falls_back_to_simpson_and_trapezoid():
    for n in (6, 7, 8, 4, 3, 2):
        x = np.linspace(-1.0, 3.0, n)
        assert np.array_equal(O.boole_coef(x), O.simpson_coef(x)), n
    for rule in "tsb":
        for n in (5, 9, 13, 10):
            x = np.linspace(-1.0, 3.0, n)
            assert abs(O.quad_coef(x, rule).sum() - 4.0) < 1e-13, (rule, n)


def test_quadrature_config_key(tmp_path):
    import kalnajs_log_spirals_b200 as K
    p = tmp_path / "c.toml"
    p.write_text('[grid]\nNR = 9\nquadrature = "bbs"\n')
    c = K.load_config(str(p))
    assert c.grid.quadrature == "bbs"
    K.save_config(c, str(tmp_path / "d.toml"))
    assert K.load_config(str(tmp_path / "d.toml")).grid.quadrature == "bbs"
    p.write_text('[grid]\nquadrature = "tx"\n')
    with pytest.raises(ValueError):
        K.load_config(str(p))
    from kalnajs_log_spirals_b200 import api, _lib
    k = api._kls_config(c, None)
    assert (k.quad_alpha, k.quad_rc, k.quad_v) == (_lib.KLS_QUAD_BOOLE, _lib.KLS_QUAD_BOOLE,
                                                   _lib.KLS_QUAD_SIMPSON)
