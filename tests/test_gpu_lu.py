"""Determinant stage forms on the GPU.

The cluster LU (matrix in the shared memory of an 8- or 16-CTA cluster) and
the one-CTA-per-matrix LU must return bitwise the same determinants and
log|det| for the same I - M(omega): same pivot rule, multiplier and update
arithmetic and determinant product order.  Both forms also stay within the
FP64 parity tolerance of the oracle through the parity tests (auto mode).
"""
import ctypes as C

import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from kalnajs_log_spirals_b200 import _lib
from tests.test_gpu_parity import kconfig

pytestmark = pytest.mark.gpu

BASE = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=11, Ne=5, Rc_min=0.01, Rc_max=10.0,
            v_min=0.01, alpha_max=10.0, l_min=-2, l_max=2, nw=2001, nwa=101)


def dets(pc, om, mode):
    pc.ctx.call("kls_set_lu_mode", mode)
    d, la = K.compute_determinant_batched(om, pc, None, batch_size=16, log_abs=True)
    return d, la


@pytest.mark.parametrize("Na", [201, 301, 400])
def test_cluster_lu_is_bitwise_the_cta_lu(lib_path, Na):
    pc = K.precompute_all(kconfig(**BASE, N_alpha=Na))
    rng = np.random.default_rng(Na)
    om = 2 * rng.uniform(0.3, 0.6, 5) + 1j * rng.uniform(0.02, 0.25, 5)
    d1, l1 = dets(pc, om, _lib.KLS_LU_CTA)
    try:
        d2, l2 = dets(pc, om, _lib.KLS_LU_CLUSTER)
    except K.KlsError as e:
        pc.close()
        if e.code == _lib.KLS_ERR_UNSUPPORTED:
            pytest.skip(f"no cluster form for N_alpha={Na} on this device: {e}")
        raise
    d3, l3 = dets(pc, om, _lib.KLS_LU_AUTO)
    pc.close()
    assert np.all(np.isfinite(d1)) and np.all(np.abs(d1) > 0)
    assert np.array_equal(d1, d2), np.max(np.abs(d1 - d2) / np.abs(d1))
    assert np.array_equal(l1, l2)
    assert np.array_equal(d1, d3) and np.array_equal(l1, l3)


def test_lu_mode_rejects_unknown(lib_path):
    pc = K.precompute_all(kconfig(**BASE, N_alpha=41))
    lib = pc.ctx.lib
    assert lib.kls_set_lu_mode(pc.ctx.h, 7) == _lib.KLS_ERR_CONFIG
    pc.close()


def test_contexts_of_different_sizes_interleave(lib_path):
    """Kernel launch limits (dynamic shared memory) are per kernel, shared by
    all contexts: a larger context created first and used after a smaller one
    still launches, in the cluster LU and the TMEM-operand contraction."""
    big = K.precompute_all(kconfig(**BASE, N_alpha=301))
    small = K.precompute_all(kconfig(**BASE, N_alpha=161))
    om = np.array([0.88 + 0.12j, 0.7 + 0.05j])
    devs = [K.to_device(p, K.GPUType.NVIDIA, "Float32") for p in (big, small)]
    for p in (big, small):
        p.ctx.call("kls_set_mixed_form", _lib.KLS_MIXED_TMEM)
    first = [dets(p, om, _lib.KLS_LU_CLUSTER)[0] for p in (big, small)]
    mixed = [K.compute_determinant_batched(om, p, d) for p, d in zip((big, small), devs)]
    again = [dets(p, om, _lib.KLS_LU_CLUSTER)[0] for p in (big, small)]
    mixed2 = [K.compute_determinant_batched(om, p, d) for p, d in zip((big, small), devs)]
    big.close()
    small.close()
    for a, b in zip(first + mixed, again + mixed2):
        assert np.array_equal(a, b)
