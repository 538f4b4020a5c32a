"""The split-BF16 tensor-core contraction (KLS_MODE_MIXED).

1. Emulation: the device result equals a NumPy restatement of the same
   algorithm (table split error-free into BF16 hi + lo; U = w conj(W) formed
   in FP32 and split; P = hi*hi + hi*lo + lo*hi) up to FP32 accumulation and
   FP32 rounding of U: |M_gpu - M_emul| <= 2e-6 max|M|.  A layout or indexing
   error shows up as an O(1) difference.
2. Accuracy against the plain FP64 form: M entries within 5e-5 of max|M|,
   det(I - M) within 1e-3 relative, and a mixed-precision Newton root within
   1e-5 of the FP64 root.
"""
import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from tests.conftest import load_case
from tests.golden.make_fixtures import BASE, CASES
from tests.test_gpu_parity import kconfig, relmax

pytestmark = pytest.mark.gpu


def bf16(x):
    """Round float32 values to BF16 (round to nearest even), returned as float32."""
    x = np.asarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def split_fp64(v):
    hi = bf16(v.astype(np.float32))
    lo = bf16((v - hi.astype(np.float64)).astype(np.float32))
    return hi, lo


def emulate_M(W, wt, G, N):
    """W [K, Na] complex128, wt [K] complex128 -> M [Na, Na] of the split algorithm."""
    Ah, Al = split_fp64(W.real)
    Bh, Bl = split_fp64(W.imag)
    Wr = (Ah + Al).astype(np.float32)
    Wi = (Bh + Bl).astype(np.float32)
    dr = wt.real.astype(np.float32)[:, None]
    di = wt.imag.astype(np.float32)[:, None]
    Ur = dr * Wr + di * Wi
    Ui = di * Wr - dr * Wi
    Urh, Url = bf16(Ur), bf16(Ur - bf16(Ur))
    Uih, Uil = bf16(Ui), bf16(Ui - bf16(Ui))

    def prod(Xh, Xl, Yh, Yl):
        f = lambda a: a.astype(np.float64)
        return f(Xh).T @ f(Yh) + f(Xh).T @ f(Yl) + f(Xl).T @ f(Yh)

    Mr = prod(Ah, Al, Urh, Url) - prod(Bh, Bl, Uih, Uil)
    Mi = prod(Ah, Al, Uih, Uil) + prod(Bh, Bl, Urh, Url)
    return (Mr + 1j * Mi) * G * N[None, :]


def weights_np(pc, omega):
    Ores = pc.Omega_res.reshape(-1, order="F")
    G = pc.DJ_vec[np.tile(np.arange(pc.NPh), pc.n_l)] * pc.F0l_all.reshape(-1, order="F")
    den = omega - Ores
    den = np.where(np.abs(den) < 1e-12, 1e-12 + 1e-12j, den)
    return G / den


@pytest.fixture(scope="module", params=["general", "variants"])
def mixed_case(request, lib_path):
    over = {**BASE, **CASES[request.param]}
    pc = K.precompute_all(kconfig(**over))
    dev = K.to_device(pc, K.GPUType.NVIDIA, "Float32")
    yield request.param, pc, dev
    pc.close()


def test_mixed_matches_emulation(mixed_case):
    name, pc, dev = mixed_case
    omega = 0.88 + 0.12j
    M = K.build_M_matrix(omega, pc, dev)
    W = pc.W_l_mat                                   # [NPh, Na, n_l]
    Wk = np.concatenate([W[:, :, il] for il in range(pc.n_l)], axis=0)   # rows k = il*NPh + p
    Me = emulate_M(Wk, weights_np(pc, omega), pc.G, pc.N_kernel)
    assert relmax(M, Me) < 2e-6, (name, relmax(M, Me))


def test_mixed_close_to_fp64(mixed_case):
    name, pc, dev = mixed_case
    om = np.array([0.88 + 0.12j, 0.6 + 0.05j, 1.2 + 0.3j])
    M64 = K.build_M_matrix(om[0], pc)
    Mmx = K.build_M_matrix(om[0], pc, dev)
    assert relmax(Mmx, M64) < 5e-5, (name, relmax(Mmx, M64))
    d64 = K.compute_determinant_batched(om, pc)
    dmx = K.compute_determinant_batched(om, pc, dev)
    assert np.all(np.abs(dmx - d64) <= 1e-3 * np.abs(d64)), (name, np.abs(dmx - d64) / np.abs(d64))


def test_mixed_batch_composition_stable(mixed_case):
    name, pc, dev = mixed_case
    om = np.array([0.88 + 0.12j, 0.7 + 0.2j, 0.91 + 0.02j])
    a = K.compute_determinant_batched(om, pc, dev)
    b = np.array([K.compute_determinant(w, pc, dev) for w in om])
    assert np.array_equal(a, b)


SMALL = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=61, Ne=21, Rc_min=0.01, Rc_max=10.0,
             v_min=0.01, N_alpha=101, alpha_max=10.0, l_min=-10, l_max=10, nw=10001, nwa=201)


def test_mixed_and_hybrid_newton(lib_path):
    """Mixed-only Newton lands within the split form's accuracy (1e-4); the
    hybrid (split-BF16 secant phase, one FP64 anchor, anchored finish) lands on
    the FP64 root (1e-10), where the plain FP64 determinant is below tol too."""
    from kalnajs_log_spirals_b200.api import newton_search_hybrid
    c = kconfig(**SMALL)
    c.newton.tol = 1e-12
    c.newton.use_line_search = False
    pc = K.precompute_all(c)
    r64 = K.newton_search(c, pc, None, K.GPUType.NVIDIA, "Float64", 0.44, 0.13)
    rh = newton_search_hybrid(c, pc, 0.44, 0.13)
    dev = K.to_device(pc, K.GPUType.NVIDIA, "Float32")
    c2 = kconfig(**SMALL)
    c2.newton.tol = 1e-6          # the mixed form's det noise is far above 1e-12
    c2.newton.max_iter = 20
    c2.newton.use_line_search = False
    rmx = K.newton_search(c2, pc, dev, K.GPUType.NVIDIA, "Float32", 0.44, 0.13)
    d64_at_h = K.compute_determinant(rh.omega, pc, None)
    pc.close()
    assert r64.converged and rh.converged
    assert abs(rmx.Omega_p - r64.Omega_p) < 1e-4 and abs(rmx.gamma - r64.gamma) < 1e-4
    assert abs(rh.Omega_p - r64.Omega_p) <= 1e-10 and abs(rh.gamma - r64.gamma) <= 1e-10
    evals = (rh.mixed_evals, rh.fp64_evals, rh.anchored_evals)
    assert abs(rh.det_val) < 1e-12 and abs(d64_at_h) < 1e-12, (rh.det_val, d64_at_h, evals)
    assert rh.fp64_evals <= 2, evals


def test_hybrid_far_start_follows_the_fp64_path(lib_path):
    """From a start whose first Newton step is long, the hybrid's far phase
    (FP64 anchor + anchored forward difference per step) reaches the root the
    plain FP64 Newton reaches from the same start (1e-10)."""
    from kalnajs_log_spirals_b200.api import newton_search_hybrid
    c = kconfig(**SMALL)
    c.newton.tol = 1e-12
    c.newton.use_line_search = False
    pc = K.precompute_all(c)
    checked = 0
    for Op0, g0 in [(0.47, 0.16), (0.41, 0.09), (0.50, 0.20), (0.45, 0.05)]:
        r64 = K.newton_search(c, pc, None, K.GPUType.NVIDIA, "Float64", Op0, g0)
        if not (r64.converged and r64.gamma > 1e-4):
            continue
        rh = newton_search_hybrid(c, pc, Op0, g0)
        assert rh.converged, (Op0, g0)
        assert abs(rh.Omega_p - r64.Omega_p) <= 1e-10 and abs(rh.gamma - r64.gamma) <= 1e-10, \
            (Op0, g0, rh.Omega_p - r64.Omega_p, rh.gamma - r64.gamma)
        checked += 1
    pc.close()
    assert checked >= 1
