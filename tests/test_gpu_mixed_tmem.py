"""The TMEM-operand split-BF16 contraction (KLS_MIXED_TMEM).

* Emulation: M(omega) equals the NumPy restatement of the split algorithm
  (tests/test_gpu_mixed.py: table split error-free into BF16 hi + lo, U =
  w conj(W) in FP32 split the same way, hi*hi + hi*lo + lo*hi) to 2e-6 of
  max|M|; an operand layout or indexing error is an O(1) difference.  Sizes:
  N_alpha_pad = 64, 128, 192, 320 and 384 (one or two MMAs along N), 1 to 4
  omegas (odd tile counts leave the last CTA pair with a padding CTA).
* Accumulation chunks: one K split long enough for several FP32 chunk
  flushes into the FP64 partial loses or repeats no chunk.
* It agrees with the one-CTA form (another summation order) to 2e-6 of
  max|M| and its determinants do not depend on the batch they are in.
* Failure path: with a short wait limit and the fault-injection hook one
  producer arrival is skipped, the MMA warp's bounded wait runs out and the
  call returns KLS_ERR_TIMEOUT (no trap, no hang); the next call on the same
  context returns the same bits as before.
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
OMEGAS = np.array([0.88 + 0.12j, 0.6 + 0.05j, 1.2 + 0.3j, 0.95 + 0.2j])


def mixed_dev(pc):
    return K.api.DevicePrecomputed(pc.m, pc.G, pc.N_alpha, pc.n_l, pc.NPh, K.KLS_MODE_MIXED, pc)


def emulated(pc, omega):
    W = pc.W_l_mat
    Wk = np.concatenate([W[:, :, il] for il in range(pc.n_l)], axis=0)
    return emulate_M(Wk, weights_np(pc, omega), pc.G, pc.N_kernel)


@pytest.fixture(scope="module", params=[41, 101, 161, 301, 381])
def pc(request, lib_path):
    p = K.precompute_all(kconfig(**BASE, N_alpha=request.param))
    K.to_device(p, K.GPUType.NVIDIA, "Float32")
    p.ctx.call("kls_set_mixed_form", _lib.KLS_MIXED_TMEM)
    yield p
    p.close()


def test_tmem_matches_emulation(pc):
    dev = mixed_dev(pc)
    for omega in OMEGAS[:2]:
        M = K.build_M_matrix(omega, pc, dev)
        Me = emulated(pc, omega)
        assert relmax(M, Me) < 2e-6, (pc.N_alpha, omega, relmax(M, Me))


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_tmem_batch_composition_stable(pc, n):
    dev = mixed_dev(pc)
    a = K.compute_determinant_batched(OMEGAS[:n], pc, dev)
    b = np.array([K.compute_determinant(w, pc, dev) for w in OMEGAS[:n]])
    assert np.array_equal(a, b), (pc.N_alpha, n)


def test_tmem_close_to_one_cta_form(pc):
    dev = mixed_dev(pc)
    M3 = K.build_M_matrix(OMEGAS[0], pc, dev)
    pc.ctx.call("kls_set_mixed_form", _lib.KLS_MIXED_ONE_CTA)
    try:
        M1 = K.build_M_matrix(OMEGAS[0], pc, dev)
    finally:
        pc.ctx.call("kls_set_mixed_form", _lib.KLS_MIXED_TMEM)
    assert relmax(M3, M1) < 2e-6, (pc.N_alpha, relmax(M3, M1))


@pytest.mark.parametrize("chunk", [16, 128])
def test_tmem_chunk_flushes(lib_path, chunk):
    """One K split of 13,125 complex k (412 stages of 32): the FP32
    accumulator is flushed into the FP64 partial every `chunk` stages.  A
    lost or repeated chunk would be an O(1e-1) error; what remains is FP32
    accumulation over each chunk (measured on a B200: 1.9e-5 of max|M| at
    128 stages per chunk here, where the terms cancel strongly), printed
    beside the one-CTA form's on the same split (2048 k per chunk)."""
    p = K.precompute_all(kconfig(**dict(BASE, NR=75, Ne=25, l_min=-3, l_max=3), N_alpha=101))
    dev = K.to_device(p, K.GPUType.NVIDIA, "Float32")
    Me = emulated(p, OMEGAS[0])
    p.ctx.call("kls_set_mixed_form", _lib.KLS_MIXED_ONE_CTA)
    p.ctx.call("kls_set_splits", K.KLS_MODE_MIXED, 1)
    err_one = relmax(K.build_M_matrix(OMEGAS[0], p, dev), Me)
    p.ctx.call("kls_set_mixed_form", _lib.KLS_MIXED_TMEM)
    p.ctx.call("kls_set_splits", K.KLS_MODE_MIXED, 1)
    p.ctx.call("kls_set_mixed_chunk", chunk)
    err = relmax(K.build_M_matrix(OMEGAS[0], p, dev), Me)
    p.close()
    print(f"chunk {chunk}: TMEM form {err:.2e}, one-CTA form {err_one:.2e} of max|M|")
    assert err < 1e-4 and err_one < 1e-4, (err, err_one)


def test_tmem_timeout_returns_error_and_context_recovers(lib_path):
    p = K.precompute_all(kconfig(**BASE, N_alpha=101))
    dev = K.to_device(p, K.GPUType.NVIDIA, "Float32")
    p.ctx.call("kls_set_mixed_form", _lib.KLS_MIXED_TMEM)
    good = K.compute_determinant_batched(OMEGAS[:3], p, dev)
    p.ctx.call("kls_set_wait_limit", 0.05)
    p.ctx.call("kls_set_fault_injection", _lib.KLS_FAULT_SKIP_ARRIVAL)
    with pytest.raises(K.KlsError) as e:
        K.compute_determinant_batched(OMEGAS[:3], p, dev)
    assert e.value.code == _lib.KLS_ERR_TIMEOUT, str(e.value)
    p.ctx.call("kls_set_wait_limit", 2.0)
    again = K.compute_determinant_batched(OMEGAS[:3], p, dev)     # injection was one-shot
    p.close()
    assert np.array_equal(again, good)


def test_wait_limit_and_injection_reject_bad_arguments(lib_path):
    p = K.precompute_all(kconfig(**BASE, N_alpha=41))
    for fn, arg in [("kls_set_wait_limit", 0.0), ("kls_set_wait_limit", 100.0),
                    ("kls_set_fault_injection", 3)]:
        with pytest.raises(K.KlsError) as e:
            p.ctx.call(fn, arg)
        assert e.value.code == _lib.KLS_ERR_CONFIG
    p.close()
