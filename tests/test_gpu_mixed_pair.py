"""The CTA-pair split-BF16 contraction (KLS_MIXED_PAIR, tcgen05 cta_group::2).

Against the one-CTA kernel on the same table, the same weights and the same K
splits, M(omega) and det(I - M) are bitwise equal (both kernels sum the same
products per MMA in the same chunks and flush order), and the pair form
passes the same emulation bound as the one-CTA form.  Sizes cover 2 N_pad = 128 (one pair whose
odd CTA has no rows), 256 (one full pair) and 384 (one and a half pairs), with
an odd number of omegas (one pair tile with a single omega).
"""
import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from kalnajs_log_spirals_b200 import _lib
from tests.test_gpu_mixed import emulate_M, weights_np
from tests.test_gpu_parity import kconfig, relmax

pytestmark = pytest.mark.gpu

BASE = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=21, Ne=7, Rc_min=0.01, Rc_max=10.0,
            v_min=0.01, alpha_max=10.0, l_min=-6, l_max=6, nw=2001, nwa=101)


@pytest.fixture(scope="module", params=[41, 101, 161])
def pc(request, lib_path):
    p = K.precompute_all(kconfig(**BASE, N_alpha=request.param))
    K.to_device(p, K.GPUType.NVIDIA, "Float32")
    yield p
    p.close()


def with_form(pc, form, fn):
    pc.ctx.call("kls_set_mixed_form", form)
    try:
        return fn()
    finally:
        pc.ctx.call("kls_set_mixed_form", _lib.KLS_MIXED_ONE_CTA)


def test_pair_matches_one_cta(pc):
    dev = K.api.DevicePrecomputed(pc.m, pc.G, pc.N_alpha, pc.n_l, pc.NPh, K.KLS_MODE_MIXED, pc)
    om = np.array([0.88 + 0.12j, 0.6 + 0.05j, 1.2 + 0.3j])
    M1 = with_form(pc, _lib.KLS_MIXED_ONE_CTA, lambda: K.build_M_matrix(om[0], pc, dev))
    M2 = with_form(pc, _lib.KLS_MIXED_PAIR, lambda: K.build_M_matrix(om[0], pc, dev))
    d1 = with_form(pc, _lib.KLS_MIXED_ONE_CTA, lambda: K.compute_determinant_batched(om, pc, dev))
    d2 = with_form(pc, _lib.KLS_MIXED_PAIR, lambda: K.compute_determinant_batched(om, pc, dev))
    assert np.array_equal(M2, M1), relmax(M2, M1)
    assert np.array_equal(d2, d1), np.abs(d2 - d1) / np.abs(d1)


def test_pair_matches_emulation(pc):
    dev = K.api.DevicePrecomputed(pc.m, pc.G, pc.N_alpha, pc.n_l, pc.NPh, K.KLS_MODE_MIXED, pc)
    omega = 0.88 + 0.12j
    M = with_form(pc, _lib.KLS_MIXED_PAIR, lambda: K.build_M_matrix(omega, pc, dev))
    W = pc.W_l_mat
    Wk = np.concatenate([W[:, :, il] for il in range(pc.n_l)], axis=0)
    Me = emulate_M(Wk, weights_np(pc, omega), pc.G, pc.N_kernel)
    assert relmax(M, Me) < 2e-6, relmax(M, Me)
