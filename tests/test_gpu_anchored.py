"""The FP64-anchored form (KLS_MODE_ANCHORED): M(omega) = M(omega_a) + dM.

M(omega_a) is the plain FP64 matrix at the anchor (kls_set_anchor); dM is the
split-BF16 contraction of the weight differences w_k(omega) - w_k(omega_a).
Checked against the plain FP64 form of the same context:

* at the anchor itself dM is exactly zero, so the determinant is bitwise the
  FP64 one;
* near the anchor the error is the split form's error scaled by |dM| / |M|
  (~|omega - omega_a| / gamma): 1e-6 from the anchor it stays below 1e-9 of
  max|M|, and at every distance it is at least 100x below the plain split
  form's own error at the same omega;
* without an anchor, with a non-finite anchor, or (for a new anchor) after
  the FP64 table is released, the calls fail with the documented codes; an
  existing anchor keeps working after the release.
"""
import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from kalnajs_log_spirals_b200 import _lib
from tests.test_gpu_parity import kconfig, relmax

pytestmark = pytest.mark.gpu

BASE = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=41, Ne=15, Rc_min=0.01, Rc_max=10.0,
            v_min=0.01, N_alpha=101, alpha_max=10.0, l_min=-8, l_max=8, nw=4001, nwa=201)
W_A = 0.88 + 0.12j


def dev(pc, mode):
    return K.api.DevicePrecomputed(pc.m, pc.G, pc.N_alpha, pc.n_l, pc.NPh, mode, pc)


@pytest.fixture(scope="module")
def pc(lib_path):
    p = K.precompute_all(kconfig(**BASE))
    K.to_device(p, K.GPUType.NVIDIA, "Float32")
    yield p
    p.close()


def test_anchor_is_bitwise_fp64(pc):
    d_a = K.set_anchor(pc, W_A)
    d64 = K.compute_determinant(W_A, pc, None)
    M64 = K.build_M_matrix(W_A, pc, None)
    Man = K.build_M_matrix(W_A, pc, dev(pc, K.KLS_MODE_ANCHORED))
    d_an = K.compute_determinant(W_A, pc, dev(pc, K.KLS_MODE_ANCHORED))
    assert np.array_equal(Man, M64), relmax(Man, M64)
    assert d_a == d64 and d_an == d64


@pytest.mark.parametrize("dist", [1e-7, 1e-6, 1e-5, 1e-4])
def test_anchored_M_error_scales_with_distance(pc, dist):
    K.set_anchor(pc, W_A)
    w = W_A + dist * np.exp(0.7j)
    M64 = K.build_M_matrix(w, pc, None)
    Man = K.build_M_matrix(w, pc, dev(pc, K.KLS_MODE_ANCHORED))
    Mmx = K.build_M_matrix(w, pc, dev(pc, K.KLS_MODE_MIXED))
    e_an, e_mx = relmax(Man, M64), relmax(Mmx, M64)
    print(f"|omega - omega_a| = {dist:.0e}: anchored {e_an:.2e}, split-BF16 {e_mx:.2e} of max|M|")
    assert e_an < e_mx / 100, (e_an, e_mx)
    if dist <= 1e-6:
        assert e_an < 1e-9, e_an


def test_anchored_batch_composition_stable(pc):
    K.set_anchor(pc, W_A)
    d = dev(pc, K.KLS_MODE_ANCHORED)
    om = W_A + np.array([0, 1e-6, -2e-6j, 3e-6 + 1e-6j])
    a = K.compute_determinant_batched(om, pc, d)
    b = np.array([K.compute_determinant(w, pc, d) for w in om])
    assert np.array_equal(a, b)


def test_anchored_errors_and_release(lib_path):
    p = K.precompute_all(kconfig(**BASE))
    d = dev(p, K.KLS_MODE_ANCHORED)
    with pytest.raises(K.KlsError) as e:
        K.compute_determinant(W_A, p, d)
    assert e.value.code == _lib.KLS_ERR_STATE
    with pytest.raises(K.KlsError) as e:
        K.set_anchor(p, complex(np.nan, 0.1))
    assert e.value.code == _lib.KLS_ERR_NONFINITE
    K.set_anchor(p, W_A)
    before = K.compute_determinant(W_A + 1e-6, p, d)
    K.release_fp64(p)
    after = K.compute_determinant(W_A + 1e-6, p, d)
    with pytest.raises(K.KlsError) as e:
        K.set_anchor(p, W_A + 1e-3)
    assert e.value.code == _lib.KLS_ERR_STATE
    p.close()
    assert before == after
