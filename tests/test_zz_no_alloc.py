"""kls_det_lu_static: determinants without any device allocation by the library.

Callers that must not allocate device memory (a host whose pool allocator owns
the whole GPU, or a loop that cannot take cudaMalloc's implicit device
synchronisation) pass their own device input and output buffers; the library
works in a fixed scratch array of its own image.  This test allocates its
buffers with torch (standing in for such a caller's pool), calls the entry
point through the C ABI twice in a row and compares each result with the
existing path, kls_det_batch, for the same matrices I - M(omega): relative
difference <= 1e-11 (the tolerance of the other determinant tests).

The file name makes pytest collect it after every other test file.
"""
import ctypes as C

import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from kalnajs_log_spirals_b200 import _lib
from tests.golden.make_fixtures import BASE
from tests.test_gpu_parity import kconfig

pytestmark = pytest.mark.gpu

SMALL = dict(BASE, NR=12, Ne=7, N_alpha=33, l_min=-4, l_max=4, nw=401, nwa=41)


def test_det_lu_static_matches_det_batch(lib_path):
    import torch
    torch.cuda.init()
    lib = _lib.load(lib_path)
    pc = K.precompute_all(kconfig(**SMALL))
    omegas = np.array([0.88 + 0.12j, 0.6 + 0.05j, 1.2 + 0.3j])
    ref = K.compute_determinant_batched(omegas, pc)            # existing entry point
    N = pc.N_alpha
    # I - M(omega), row-major [beta][alpha] as the library factors it
    mats = np.stack([np.eye(N) - K.build_M_matrix(w, pc) for w in omegas])
    pc.close()
    a = torch.tensor(np.ascontiguousarray(mats).view(np.float64), dtype=torch.float64,
                     device="cuda")
    for call in range(2):
        det = torch.zeros((len(omegas), 2), dtype=torch.float64, device="cuda")
        la = torch.zeros(len(omegas), dtype=torch.float64, device="cuda")
        code = lib.kls_det_lu_static(C.c_void_p(a.data_ptr()), len(omegas), N,
                                     C.c_void_p(det.data_ptr()), C.c_void_p(la.data_ptr()), None)
        assert code == 0, lib.kls_create_error()
        torch.cuda.synchronize()
        d = det.cpu().numpy()
        got = d[:, 0] + 1j * d[:, 1]
        rel = np.abs(got - ref) / np.abs(ref)
        assert np.all(rel <= 1e-11), (call, rel)
        assert np.allclose(la.cpu().numpy(), np.log(np.abs(ref)), rtol=0, atol=1e-11)
    # the input was not modified
    assert np.array_equal(a.cpu().numpy(), np.ascontiguousarray(mats).view(np.float64))


def test_det_lu_static_at_the_scratch_limit(lib_path):
    """16 matrices of N = 256 fill the 2^20-element scratch exactly (the last
    CTA's block ends at the array's end); results equal numpy's LAPACK det."""
    import torch
    lib = _lib.load(lib_path)
    n, N = 16, 256
    rng = np.random.default_rng(3)
    mats = np.eye(N)[None] + (rng.standard_normal((n, N, N))
                              + 1j * rng.standard_normal((n, N, N))) * (0.3 / N ** 0.5)
    ref = np.linalg.det(mats)
    a = torch.tensor(np.ascontiguousarray(mats).view(np.float64), dtype=torch.float64,
                     device="cuda")
    det = torch.zeros((n, 2), dtype=torch.float64, device="cuda")
    code = lib.kls_det_lu_static(C.c_void_p(a.data_ptr()), n, N, C.c_void_p(det.data_ptr()),
                                 None, None)
    assert code == 0, lib.kls_create_error()
    torch.cuda.synchronize()
    d = det.cpu().numpy()
    got = d[:, 0] + 1j * d[:, 1]
    assert np.max(np.abs(got - ref) / np.abs(ref)) <= 1e-11


def test_det_lu_static_rejects_oversize(lib_path):
    lib = _lib.load(lib_path)
    dummy = C.c_void_p(1)
    code = lib.kls_det_lu_static(dummy, 12, 301, dummy, None, None)   # 12 * 301^2 > 2^20
    assert code == _lib.KLS_ERR_CONFIG
    assert b"exceeds the fixed scratch" in lib.kls_create_error()
    code = lib.kls_det_lu_static(dummy, 1, 1025, dummy, None, None)   # one matrix > 2^20
    assert code == _lib.KLS_ERR_CONFIG
    assert b"1025 > 1024" in lib.kls_create_error()
