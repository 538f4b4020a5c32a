"""CPU-side checks: the C ABI library, the config layer and host logic."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from kalnajs_log_spirals_b200 import _lib
from kalnajs_log_spirals_b200.api import column_ranges, find_minimum
from tests.conftest import ROOT


def header_symbols():
    src = open(os.path.join(ROOT, "include", "kls.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(kls_\w+)\s*\(", src, re.M)))


def test_library_exports_every_header_symbol(lib_path):
    lib = C.CDLL(lib_path)
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    # the ctypes binding declares every header symbol
    assert set(syms) == set(_lib.SIGNATURES)


def test_library_links_no_torch(lib_path):
    import subprocess
    out = subprocess.run(["ldd", lib_path], capture_output=True, text=True).stdout
    assert "torch" not in out and "libcudart.so" not in out   # static cudart, no torch


def test_create_without_gpu_reports_error(lib_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load(lib_path)
    cfg = _lib.kls_config(m=2, G=1.0, L0=1.0, n_zang=4, q1=7.0, NR=4, Ne=3, Rc_min=0.1,
                          Rc_max=1.0, v_min=0.01, N_alpha=5, alpha_max=1.0, l_min=-1, l_max=1,
                          nw=101, nwa=11)
    h = C.c_void_p()
    code = lib.kls_create(C.byref(cfg), 0, C.byref(h))
    assert code != 0 and not h.value
    assert len(lib.kls_create_error()) > 0


def test_invalid_config_rejected_before_device(lib_path):
    lib = _lib.load(lib_path)
    cfg = _lib.kls_config(m=2, G=1.0, L0=1.0, n_zang=4, q1=7.0, NR=4, Ne=3, Rc_min=0.1,
                          Rc_max=1.0, v_min=0.01, N_alpha=5, alpha_max=1.0, l_min=-1, l_max=1,
                          nw=102, nwa=11)   # length(1:10:102) = 11 ok? (101/10 = 10 -> 11)
    cfg.nw, cfg.nwa = 100, 12             # length(1:9:100) = 12 -> valid; make it invalid:
    cfg.nw, cfg.nwa = 105, 12             # nwai = 104 // 11 = 9, length(1:9:105) = 12 ok
    cfg.nw, cfg.nwa = 110, 12             # nwai = 109 // 11 = 9, length(1:9:110) = 13 != 12
    h = C.c_void_p()
    assert lib.kls_create(C.byref(cfg), 0, C.byref(h)) == _lib.KLS_ERR_CONFIG
    assert b"DimensionMismatch" in lib.kls_create_error()
    cfg.nw, cfg.nwa = 101, 11
    cfg.l_max = -5
    assert lib.kls_create(C.byref(cfg), 0, C.byref(h)) == _lib.KLS_ERR_CONFIG
    cfg.l_max = 1
    cfg.NR, cfg.Ne = 50000, 50000          # 2.5e9 orbits: past the int32 orbit index
    assert lib.kls_create(C.byref(cfg), 0, C.byref(h)) == _lib.KLS_ERR_CONFIG
    assert b"2^31" in lib.kls_create_error()
    cfg.NR, cfg.Ne, cfg.N_alpha = 4, 3, 8000   # LU rows beyond one CTA's shared memory
    assert lib.kls_create(C.byref(cfg), 0, C.byref(h)) == _lib.KLS_ERR_CONFIG
    assert b"N_alpha" in lib.kls_create_error()


def test_null_context_calls_fail_cleanly(lib_path):
    lib = _lib.load(lib_path)
    out = np.zeros(2)
    assert lib.kls_det_batch(None, _lib.dptr(out), 1, 0, _lib.dptr(out), None) != 0
    assert lib.kls_last_error(None) == b"NULL context"
    assert lib.kls_launch_count(None) == 0


def test_load_config_and_model_roundtrip(tmp_path):
    c = K.load_config(os.path.join(ROOT, "configs", "default.toml"))
    c = K.load_model(c, os.path.join(ROOT, "models", "kalnajs_zang4.toml"))
    assert (c.grid.NR, c.grid.Ne, c.grid.N_alpha, c.grid.l_min, c.grid.l_max) == (501, 51, 301, -100, 100)
    assert c.newton.tol == 1e-12 and c.newton.use_line_search is False
    assert c.gpu.precision_double and c.cpu.precision_double
    assert (c.physics.m, c.physics.G, c.model.n_zang, c.model.q1) == (2, 1.0, 4, 7)
    assert c.reference.Omega_p == 0.4397142267
    assert K.get_n_l(c) == 201 and K.get_NPh(c) == 25551
    assert K.get_float_type(c) == "Float64" and K.get_complex_type(c, False) == "ComplexF64"
    p = tmp_path / "saved.toml"
    K.save_config(c, str(p))
    d = K.load_config(str(p))
    assert d.grid == c.grid and d.physics == c.physics and d.model == c.model
    assert d.scan == c.scan


def test_config_defaults_match_reference():
    c = K.KalnajsConfig()
    assert (c.grid.NR, c.grid.Ne, c.grid.Rc_min, c.grid.nw, c.grid.nwa) == (201, 21, 1e-3, 10001, 201)
    assert (c.scan.n_Op, c.scan.n_gamma, c.scan.Omega_p_min, c.scan.gamma_max) == (41, 20, 0.2, 0.2)
    assert (c.newton.max_iter, c.newton.tol, c.newton.delta) == (50, 1e-10, 1e-6)
    assert c.newton.use_line_search is True and c.gpu.precision_double is False


def test_missing_files_raise():
    with pytest.raises(FileNotFoundError, match="Configuration file not found"):
        K.load_config("/nonexistent.toml")
    with pytest.raises(FileNotFoundError, match="Model file not found"):
        K.load_model(K.KalnajsConfig(), "/nonexistent.toml")


def test_column_ranges_like_scan_multi_gpu():
    r = column_ranges(41, 3)
    assert [(s.start, s.stop) for s in r] == [(0, 14), (14, 28), (28, 41)]
    assert sum(s.stop - s.start for s in column_ranges(7, 8)) == 7


def test_find_minimum_matches_oracle():
    from oracle import np_oracle as O
    rng = np.random.default_rng(3)
    g = rng.normal(size=(20, 41)) + 1j * rng.normal(size=(20, 41))
    Op = np.linspace(0.2, 0.6, 41)
    gm = np.linspace(0.01, 0.2, 20)
    assert find_minimum(g, Op, gm) == O.find_minimum(g, Op, gm)


def test_model_constants():
    c = K.KalnajsConfig()
    m = K.create_toomre_zang_model(c)
    from oracle import np_oracle as O
    o = O.ToomreZang.from_config(O.OracleConfig())
    assert m.DF_const == pytest.approx(o.DF_const, rel=1e-15)
    assert m.sigma_r0 == 1 / np.sqrt(7) and m.q_zang == 6


def test_dptr_accepts_only_contiguous_doubles():
    """The ctypes helper hands the library double* buffers: float64 or
    complex128, contiguous in C or Fortran order; other arrays raise."""
    import numpy as np
    assert _lib.dptr(np.zeros(4)) is not None
    assert _lib.dptr(np.zeros((3, 2), order="F")) is not None
    assert _lib.dptr(np.zeros(2, dtype=np.complex128)) is not None
    for bad in (np.zeros(4, dtype=np.float32), np.zeros(4, dtype=np.int64),
                np.zeros((4, 4))[:, 1]):
        with pytest.raises(TypeError):
            _lib.dptr(bad)


def test_bounds_checked_build_loads_and_reports(lib_path):
    """libkls_checked.so (the same sources with KLS_CHECKED: guarded global
    accesses, a device log per translation unit) is built beside libkls.so,
    exports the same symbols, and answers kls_bounds_report; the default
    library answers KLS_ERR_UNSUPPORTED and names the checked one."""
    import torch
    lib = _lib.load(lib_path)
    v = C.c_int64(-1)
    assert lib.kls_bounds_report(C.byref(v), None, None, None, 0) == _lib.KLS_ERR_UNSUPPORTED
    assert b"libkls_checked.so" in lib.kls_create_error()
    assert v.value == -1
    checked = _lib.load_checked()
    for s in header_symbols():
        assert hasattr(checked, s), s
    out = subprocess_ldd(_lib.CHECKED_LIB_PATH)
    assert "torch" not in out and "libcudart.so" not in out
    site, idx, ext = C.c_int32(-1), C.c_int64(-1), C.c_int64(-1)
    code = checked.kls_bounds_report(C.byref(v), C.byref(site), C.byref(idx), C.byref(ext), 1)
    if torch.cuda.is_available():
        assert code == _lib.KLS_OK and v.value == 0
    else:
        # no device: the logs cannot be read, and the call says so
        assert code == _lib.KLS_ERR_CUDA and b"device log" in checked.kls_create_error()


def subprocess_ldd(path):
    import subprocess
    return subprocess.run(["ldd", path], capture_output=True, text=True).stdout
