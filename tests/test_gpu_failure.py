"""Failure paths of the library on the GPU, made without faulting the GPU.

* A NaN written into one device weight row (the fault-injection hook, a plain
  memory write) makes every determinant NaN: kls_det_batch, the grid scan
  and Newton return KLS_ERR_NONFINITE in both precision forms; clearing the
  hook restores the row and the bits of the earlier result.
* G = 0: M(omega) = 0, det(I - M) = 1 everywhere, so Newton's
  finite-difference Jacobian is exactly zero: KLS_ERR_SINGULAR (the
  reference's `J \\ F` throws a SingularException there, NewtonSolver.jl:112),
  for the plain FP64 Newton and the hybrid.
* A non-finite omega is rejected before any launch (KLS_ERR_NONFINITE).
The bounded-wait path (KLS_ERR_TIMEOUT) is in tests/test_gpu_mixed_tmem.py.
"""
import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from kalnajs_log_spirals_b200 import _lib
from kalnajs_log_spirals_b200.api import newton_search_hybrid
from tests.test_gpu_parity import kconfig

pytestmark = pytest.mark.gpu

BASE = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=21, Ne=7, Rc_min=0.01, Rc_max=10.0,
            v_min=0.01, N_alpha=41, alpha_max=10.0, l_min=-6, l_max=6, nw=2001, nwa=101)
OMEGAS = np.array([0.88 + 0.12j, 0.6 + 0.05j])


def test_nan_row_reports_nonfinite_and_recovers(lib_path):
    c = kconfig(**BASE)
    pc = K.precompute_all(c)
    dev = K.to_device(pc, K.GPUType.NVIDIA, "Float32")
    good64 = K.compute_determinant_batched(OMEGAS, pc)
    goodmx = K.compute_determinant_batched(OMEGAS, pc, dev)
    pc.ctx.call("kls_set_fault_injection", _lib.KLS_FAULT_NAN_ROW)
    try:
        for d in (None, dev):
            with pytest.raises(K.KlsError) as e:
                K.compute_determinant_batched(OMEGAS, pc, d)
            assert e.value.code == _lib.KLS_ERR_NONFINITE and "NaN determinant" in str(e.value)
        with pytest.raises(K.KlsError) as e:
            K.newton_search(c, pc, None, K.GPUType.NVIDIA, "Float64", 0.44, 0.13)
        assert e.value.code == _lib.KLS_ERR_NONFINITE
        c.scan.n_Op, c.scan.n_gamma = 3, 2
        with pytest.raises(K.KlsError) as e:
            K.grid_scan(c, pc)
        assert e.value.code == _lib.KLS_ERR_NONFINITE
    finally:
        pc.ctx.call("kls_set_fault_injection", _lib.KLS_FAULT_NONE)
    assert np.array_equal(K.compute_determinant_batched(OMEGAS, pc), good64)
    assert np.array_equal(K.compute_determinant_batched(OMEGAS, pc, dev), goodmx)
    pc.close()


def test_zero_coupling_gives_singular_jacobian(lib_path):
    c = kconfig(**dict(BASE, G=0.0))
    pc = K.precompute_all(c)
    d = K.compute_determinant_batched(OMEGAS, pc)
    assert np.array_equal(d, np.ones(len(OMEGAS), dtype=complex))      # det(I - 0) = 1
    with pytest.raises(K.KlsError) as e:
        K.newton_search(c, pc, None, K.GPUType.NVIDIA, "Float64", 0.44, 0.13)
    assert e.value.code == _lib.KLS_ERR_SINGULAR
    with pytest.raises(K.KlsError) as e:
        newton_search_hybrid(c, pc, 0.44, 0.13)
    assert e.value.code == _lib.KLS_ERR_SINGULAR
    pc.close()


def test_nonfinite_omega_rejected(lib_path):
    pc = K.precompute_all(kconfig(**BASE))
    with pytest.raises(K.KlsError) as e:
        K.compute_determinant_batched(np.array([np.nan + 0.1j]), pc)
    assert e.value.code == _lib.KLS_ERR_NONFINITE
    pc.close()
