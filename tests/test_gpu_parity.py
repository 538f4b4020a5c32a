"""GPU parity: libkls.so against the oracle and the reference's published roots.

Tolerances (FP64 throughout), per element:
  |gpu - oracle| <= floor * max|oracle| + 4 * sens
with floor = 1e-12 for grids, orbit fields and the W table, 1e-13 for
N_m(alpha), 1e-11 for M(omega) entries and det(I - M); ``sens`` is the change
the oracle itself shows when ln x along the orbit integrals is perturbed by
2 ulps (stored in the fixtures by tests/golden/make_fixtures.py).  The
radial-velocity integrand cancels like 1/e^2 near the turning points of
near-circular orbits, so math libraries that differ in the last bit of ln
legitimately disagree there by up to ~1e-10 relative in Omega_1.
Newton roots: 1e-10 absolute in Omega_p and gamma.
"""
import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from oracle import np_oracle as O
from tests.conftest import load_case
from tests.golden.make_fixtures import BASE, CASES

pytestmark = pytest.mark.gpu


def kconfig(**kw) -> K.KalnajsConfig:
    c = K.KalnajsConfig()
    for f in ("m", "G"):
        if f in kw:
            setattr(c.physics, f, kw[f])
    for f in ("L0", "n_zang", "q1"):
        if f in kw:
            setattr(c.model, f, kw[f])
    for f in ("NR", "Ne", "Rc_min", "Rc_max", "v_min", "N_alpha", "alpha_max", "l_min",
              "l_max", "nw", "nwa"):
        if f in kw:
            setattr(c.grid, f, kw[f])
    if "quad" in kw:
        c.grid.quadrature = kw["quad"]
    return c


def relmax(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a - b))) / (s if s > 0 else 1.0)


def close(got, ref, key, floor):
    """Per-element check against the oracle with its own ulp sensitivity."""
    got = np.asarray(got).reshape(np.shape(ref[key]), order="F") if np.size(got) == np.size(ref[key]) else got
    r = np.asarray(ref[key])
    sens = np.asarray(ref.get("sens_" + key, np.zeros_like(np.abs(r))))
    tol = floor * float(np.max(np.abs(r))) + 4.0 * sens
    bad = np.abs(np.asarray(got) - r) > tol
    return not bad.any(), float(np.max(np.abs(np.asarray(got) - r) - tol))


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, lib_path):
    name = request.param
    over = {**BASE, **CASES[name]}
    pc = K.precompute_all(kconfig(**over))
    yield name, load_case(name), pc
    pc.close()


def test_orbits_and_grids(case):
    name, ref, pc = case
    o = pc.orbit_data
    cm = lambda a: np.asarray(a).reshape(-1, order="F")
    for k in ("Omega_1", "Omega_2", "jacobian", "F0", "FE", "FL", "w1", "ra", "pha"):
        ok, worst = close(cm(getattr(o, k)), ref, k, 1e-12)
        assert ok, (name, k, worst)
    for k in ("Rc", "e", "E", "L_m", "S_e"):
        ok, worst = close(cm(getattr(o.grids, k)), ref, "grid_" + k, 1e-12)
        assert ok, (name, k, worst)
    assert close(o.grids.S_RC, ref, "grid_S_RC", 1e-12)[0]
    assert close(pc.DJ_vec, ref, "DJ", 1e-12)[0]


def test_alpha_and_N_kernel(case):
    name, ref, pc = case
    assert relmax(pc.alpha_arr, ref["alpha"]) < 1e-15
    assert relmax(pc.d_alpha, ref["d_alpha"]) < 1e-14
    assert relmax(pc.N_kernel, ref["N_kernel"]) < 1e-13


def test_resonant_rows(case):
    name, ref, pc = case
    assert close(pc.F0l_all.reshape(-1, order="F"), ref, "F0l", 1e-12)[0]
    assert close(pc.Omega_res.reshape(-1, order="F"), ref, "Omega_res", 1e-12)[0]


def test_W_table(case):
    name, ref, pc = case
    W = pc.W_l_mat
    assert W.shape == ref["W"].shape
    ok, worst = close(W, ref, "W", 1e-12)
    assert ok, (name, worst, relmax(W, ref["W"]))


def test_M_and_det(case):
    name, ref, pc = case
    M = K.build_M_matrix(ref["omegas"][0], pc)
    ok, worst = close(M, ref, "M0", 1e-11)
    assert ok, (name, worst, relmax(M, ref["M0"]))
    d = K.compute_determinant_batched(ref["omegas"], pc)
    tol = 1e-11 * np.abs(ref["dets"]) + 4 * ref["sens_dets"]
    assert np.all(np.abs(d - ref["dets"]) <= tol), (name, np.abs(d - ref["dets"]) / np.abs(ref["dets"]))


def test_M_and_det_3m_form(case):
    """The 3M (Gauss) FP64 contraction against the oracle, same tolerances."""
    name, ref, pc = case
    pc.ctx.call("kls_set_f64_form", 1)
    try:
        M = K.build_M_matrix(ref["omegas"][0], pc)
        d = K.compute_determinant_batched(ref["omegas"], pc)
        a = K.compute_determinant_batched(ref["omegas"][:3], pc, batch_size=3)
        b = np.array([K.compute_determinant(w, pc) for w in ref["omegas"][:3]])
    finally:
        pc.ctx.call("kls_set_f64_form", 0)
    ok, worst = close(M, ref, "M0", 1e-11)
    assert ok, (name, worst, relmax(M, ref["M0"]))
    tol = 1e-11 * np.abs(ref["dets"]) + 4 * ref["sens_dets"]
    assert np.all(np.abs(d - ref["dets"]) <= tol), (name, np.abs(d - ref["dets"]) / np.abs(ref["dets"]))
    assert np.array_equal(a, b)


def test_single_omega_entry_point(case):
    """kls_det (one omega) is the batch of one: same bits, same log|det|."""
    import ctypes as C
    name, ref, pc = case
    w = complex(ref["omegas"][0])
    dr, di, la = C.c_double(), C.c_double(), C.c_double()
    pc.ctx.call("kls_det", w.real, w.imag, K.KLS_MODE_FP64, C.byref(dr), C.byref(di), C.byref(la))
    d, l = K.compute_determinant_batched(np.array([w]), pc, log_abs=True)
    assert complex(dr.value, di.value) == d[0] and la.value == l[0]


def test_batch_composition_is_bitwise_stable(case):
    name, ref, pc = case
    om = np.array([0.88 + 0.12j, 0.7 + 0.2j, 0.91 + 0.02j, 1.3 + 0.4j] * 5)
    a = K.compute_determinant_batched(om, pc, batch_size=len(om))
    b = np.array([K.compute_determinant(w, pc) for w in om[:4]])
    assert np.array_equal(a[:4], b)
    assert np.array_equal(a[:4], a[4:8])


# ---------------------------------------------------------------------------
# end-to-end roots
# ---------------------------------------------------------------------------
SMALL = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=61, Ne=21, Rc_min=0.01, Rc_max=10.0,
             v_min=0.01, N_alpha=101, alpha_max=10.0, l_min=-10, l_max=10, nw=10001, nwa=201)


def test_newton_reproduces_published_root(lib_path):
    """convergence_table.txt:13 (MATLAB, 10 decimals): 0.4397142267, 0.1230663944."""
    c = kconfig(**SMALL)
    c.newton.tol = 1e-12
    c.newton.use_line_search = False
    pc = K.precompute_all(c)
    r = K.newton_search(c, pc, None, K.GPUType.NVIDIA, "Float64", 0.44, 0.13)
    pc.close()
    assert r.converged
    assert abs(r.Omega_p - 0.4397142267) <= 6e-11
    assert abs(r.gamma - 0.1230663944) <= 6e-11
    # the oracle's root from the same start
    oc = O.OracleConfig(**SMALL)
    opc = O.precompute_all(oc)
    ro = O.newton_search(lambda w: O.compute_det(opc, w), 2, 0.44, 0.13, tol=1e-12)
    assert abs(r.Omega_p - ro.Omega_p) <= 1e-10 and abs(r.gamma - ro.gamma) <= 1e-10


def test_newton_line_search_and_history(lib_path):
    c = kconfig(**SMALL)
    c.newton.tol = 1e-12
    c.newton.use_line_search = True
    pc = K.precompute_all(c)
    r = K.newton_search(c, pc, None, K.GPUType.NVIDIA, "Float64", 0.44, 0.13)
    pc.close()
    oc = O.OracleConfig(**SMALL)
    opc = O.precompute_all(oc)
    ro = O.newton_search(lambda w: O.compute_det(opc, w), 2, 0.44, 0.13, tol=1e-12,
                         use_line_search=True)
    assert r.converged and r.iterations == ro.iterations
    assert np.allclose(r.history[:, :2], ro.history[:, :2], rtol=0, atol=1e-10)


def test_grid_scan_matches_oracle(lib_path):
    c = kconfig(**{**SMALL, "NR": 31, "Ne": 11, "N_alpha": 41, "nw": 2001, "nwa": 101})
    c.scan.n_Op, c.scan.n_gamma = 9, 5
    pc = K.precompute_all(c)
    dg, Op0, g0 = K.grid_scan(c, pc)
    oc = O.OracleConfig(**{**SMALL, "NR": 31, "Ne": 11, "N_alpha": 41, "nw": 2001, "nwa": 101})
    opc = O.precompute_all(oc)
    s = c.scan
    odg, oOp, og = O.grid_scan(lambda w: O.compute_det(opc, w), 2, s.n_Op, s.n_gamma,
                               s.Omega_p_min, s.Omega_p_max, s.gamma_min, s.gamma_max)
    pc.close()
    assert dg.shape == (5, 9)
    assert np.all(np.abs(dg - odg) <= 1e-11 * np.abs(odg))
    assert (Op0, g0) == (oOp, og)


@pytest.mark.slow
def test_size_s_newton_matches_oracle(lib_path):
    """Benchmark size S: NR=101, Ne=21, N_alpha=101 on [-30,30], l=+-25, nw=100001."""
    import os
    from tests.conftest import ROOT
    c = K.load_config(os.path.join(ROOT, "configs", "size_s.toml"))
    c = K.load_model(c, os.path.join(ROOT, "models", "kalnajs_zang4.toml"))
    ref = load_case("size_s")          # oracle outputs, tests/golden/make_size_s.py
    pc = K.precompute_all(c)
    r = K.newton_search(c, pc, None, K.GPUType.NVIDIA, "Float64")
    M = K.build_M_matrix(complex(ref["omega_root"][0]), pc)
    d = K.compute_determinant_batched(ref["omegas"], pc)
    pc.close()
    assert r.converged and r.iterations == int(ref["iterations"][0])
    assert abs(r.Omega_p - ref["root"][0]) <= 1e-10 and abs(r.gamma - ref["root"][1]) <= 1e-10
    ok, worst = close(M, ref, "M0", 1e-11)
    assert ok, (worst, relmax(M, ref["M0"]))
    tol = 1e-11 * np.abs(ref["dets"]) + 4 * ref["sens_dets"]
    assert np.all(np.abs(d - ref["dets"]) <= tol)
