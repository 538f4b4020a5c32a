"""Uneven batch over models (kls_multi) and the autotuner on the GPU.

* A batch of models of different NR, Ne, N_alpha, l range and m gives, in one
  persistent launch per pass, bitwise the determinants each model's own
  context gives (FP64 and split-BF16 forms), including a partial last pass.
* kls_scan_multi returns each model's grid_scan grid and argmin.
* The passes replay one captured CUDA graph.
* kls_autotune picks one of its candidates, caches it, and the determinant
  after tuning agrees with the untuned one to FP64 rounding (a different
  split count only regroups the FP64 sum).
"""
import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from kalnajs_log_spirals_b200 import _lib
from tests.test_gpu_parity import kconfig

pytestmark = pytest.mark.gpu

BASE = dict(G=1.0, L0=1.0, Rc_min=0.01, Rc_max=10.0, v_min=0.01, alpha_max=10.0, nw=2001,
            nwa=101)
# (m, n_zang, q1, NR, Ne, N_alpha, l_max): three sizes, both m
MODELS = [(2, 4, 7.0, 41, 11, 41, 10), (3, 3, 9.5, 31, 9, 97, 6), (2, 6, 5.2, 61, 13, 63, 16),
          (3, 5, 11.0, 21, 7, 33, 4)]


def configs():
    return [kconfig(**BASE, m=m, n_zang=nz, q1=q, NR=nr, Ne=ne, N_alpha=na, l_min=-lm, l_max=lm)
            for m, nz, q, nr, ne, na, lm in MODELS]


def omegas(n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.3, 0.6, n) * 2 + 1j * rng.uniform(0.02, 0.25, n)


@pytest.fixture(scope="module")
def pcs(lib_path):
    p = [K.precompute_all(c) for c in configs()]
    yield p
    for x in p:
        x.close()


@pytest.mark.parametrize("Tgpu,form", [("Float64", None), ("Float64", "3m"),
                                       ("Float32", _lib.KLS_MIXED_ONE_CTA),
                                       ("Float32", _lib.KLS_MIXED_TMEM),
                                       ("Float32", "mixed forms")])
def test_batch_is_bitwise_the_single_model_result(pcs, Tgpu, form):
    n = 7                                  # passes of 3: 3 + 3 + 1
    om = np.stack([omegas(n, 10 + i) * (m / 2) for i, (m, *_) in enumerate(MODELS)])
    singles = []
    for pc, o in zip(pcs, om):
        dev = K.to_device(pc, K.GPUType.NVIDIA, Tgpu)
        if form == "3m":
            pc.ctx.call("kls_set_f64_form", _lib.KLS_F64_3M)
        elif form == "mixed forms":
            # TMEM-operand form and the older forms side by side in one batch
            pc.ctx.call("kls_set_mixed_form",
                        [_lib.KLS_MIXED_TMEM, _lib.KLS_MIXED_ONE_CTA, _lib.KLS_MIXED_TMEM,
                         _lib.KLS_MIXED_PAIR][len(singles)])
        elif form is not None:
            # the batch runs this form's kernel body when it is every model's form
            pc.ctx.call("kls_set_mixed_form", form)
        singles.append(K.compute_determinant_batched(o, pc, dev, batch_size=16, log_abs=True))
    mb = K.ModelBatch(pcs, Tgpu, batch=3)
    d, la = mb.det(om)
    info = mb.info()
    mb.close()
    if form == "3m":
        for pc in pcs:
            pc.ctx.call("kls_set_f64_form", _lib.KLS_F64_4M)
    for i, (ds, ls) in enumerate(singles):
        assert np.array_equal(d[i], ds), (i, np.max(np.abs(d[i] - ds) / np.abs(ds)))
        assert np.array_equal(la[i], ls), i
    assert info["graph"] == 1 and info["replays"] == 3 and info["n_models"] == len(MODELS)
    assert info["launches_per_replay"] >= 4 and info["n_items"] > 0 and info["grid"] > 0
    if form == _lib.KLS_MIXED_TMEM:
        assert info["grid"] == 2 * info["n_items"]            # one CTA pair per item
    elif form != "mixed forms":
        assert info["n_items"] >= info["grid"]
    if Tgpu == "Float32":
        assert info["schedule"] in ((1, 2) if form == _lib.KLS_MIXED_TMEM else (0, 1))
        assert min(info["schedule_ms"]) > 0


def test_mixed_batch_close_to_fp64_batch(pcs):
    om = np.stack([omegas(4, 20 + i) * (m / 2) for i, (m, *_) in enumerate(MODELS)])
    a = K.ModelBatch(pcs, "Float64", batch=4)
    b = K.ModelBatch(pcs, "Float32", batch=4)
    d64, _ = a.det(om)
    d32, _ = b.det(om)
    a.close()
    b.close()
    assert np.max(np.abs(d32 - d64) / np.abs(d64)) < 1e-3


def test_scan_multi_matches_grid_scan(pcs):
    mb = K.ModelBatch(pcs, "Float64", batch=16)
    dg, la, Op0, g0 = mb.scan(n_Op=9, n_gamma=5, Omega_p_range=(0.2, 0.6), gamma_range=(0.01, 0.2))
    mb.close()
    for i, pc in enumerate(pcs):
        cfg = pc.config
        cfg.scan.n_Op, cfg.scan.n_gamma = 9, 5
        cfg.scan.Omega_p_min, cfg.scan.Omega_p_max = 0.2, 0.6
        cfg.scan.gamma_min, cfg.scan.gamma_max = 0.01, 0.2
        ref, o0, gg0 = K.grid_scan(cfg, pc)
        assert dg[i].shape == ref.shape
        assert np.array_equal(dg[i], ref)
        assert np.allclose(la[i], np.log(np.abs(ref)), rtol=0, atol=1e-12)
        assert (Op0[i], g0[i]) == (o0, gg0)


@pytest.mark.parametrize("Tgpu", ["Float64", "Float32"])
def test_autotune(lib_path, Tgpu):
    c = configs()[2]
    pc = K.precompute_all(c)
    dev = K.to_device(pc, K.GPUType.NVIDIA, Tgpu)
    om = omegas(3, 5)
    before = K.compute_determinant_batched(om, pc, dev)
    t = K.autotune(pc, Tgpu, batch=2)
    assert t.candidates >= 2 and t.splits >= 1 and t.default_splits >= 1
    assert 0 < t.ms_per_omega <= t.default_ms_per_omega * 1.0001
    after = K.compute_determinant_batched(om, pc, dev)
    # FP64: a split count only regroups the FP64 sum; split-BF16: tuning may
    # also change the kernel, whose summation orders differ by their FP32
    # accumulation error (~2e-5 of the scale at this size)
    tol = 1e-12 if Tgpu == "Float64" else 1e-4
    assert np.max(np.abs(after - before) / np.abs(before)) < tol
    again = K.autotune(pc, Tgpu, batch=2)          # process cache
    assert again.candidates == 0 and again.splits == t.splits
    # a batch built after tuning keeps the tuned split count: bitwise the
    # context's own result in the forms whose kernel body the batch runs
    mb = K.ModelBatch([pc], Tgpu, batch=3)
    d, _ = mb.det(om[None, :])
    mb.close()
    if Tgpu == "Float64" or t.form != _lib.KLS_MIXED_TMEM:
        assert np.array_equal(d[0], after)
    else:
        assert np.max(np.abs(d[0] - after) / np.abs(after)) < 1e-5
    pc.close()


def test_multi_rejects_bad_input(pcs):
    with pytest.raises(K.KlsError):
        K.ModelBatch(pcs, "Float64", batch=0)
    mb = K.ModelBatch(pcs[:1], "Float64", batch=2)
    with pytest.raises(K.KlsError):
        mb.det(np.array([[np.nan + 0j, 1.0 + 0.1j]]))
    mb.close()


def test_release_fp64_keeps_mixed(lib_path):
    c = configs()[1]
    pc = K.precompute_all(c)
    dev = K.to_device(pc, K.GPUType.NVIDIA, "Float32")
    pc.ctx.call("kls_set_mixed_form", _lib.KLS_MIXED_ONE_CTA)   # the batch's kernel body
    om = omegas(3, 8) * 1.5
    before = K.compute_determinant_batched(om, pc, dev)
    K.release_fp64(pc)
    after = K.compute_determinant_batched(om, pc, dev)
    assert np.array_equal(before, after)
    with pytest.raises(K.KlsError):
        K.compute_determinant_batched(om, pc, None)
    with pytest.raises(K.KlsError):
        K.ModelBatch([pc], "Float64", batch=2)
    mb = K.ModelBatch([pc], "Float32", batch=3)
    d, _ = mb.det(om[None, :])
    mb.close()
    assert np.array_equal(d[0], after)
    pc.close()


def test_ksharded_path_on_one_rank(lib_path):
    """The K-sharded determinant path (partial M per rank, all_reduce, device
    LU) on a single rank equals the one-context determinant."""
    import datetime
    import os
    import socket
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=0, world_size=1, timeout=datetime.timedelta(seconds=30))
    try:
        c = configs()[0]
        pc = K.precompute_ksharded(c, device=0)
        om = omegas(3, 31)
        d = K.compute_determinant_ksharded(om, c, pc)
        ref = K.compute_determinant_batched(om, pc)
        pc.close()
    finally:
        dist.destroy_process_group()
    assert np.max(np.abs(d - ref) / np.abs(ref)) < 1e-12, np.abs(d - ref) / np.abs(ref)


def test_ksharded_lu_batch_larger_than_one_chunk(lib_path):
    """13 matrices of N = 301 need two kls_det_lu_static calls (11 fit its
    scratch); the chunked path equals numpy's LAPACK determinant."""
    import datetime
    import os
    import socket
    import torch.distributed as dist
    N, n = 301, 13
    assert K.api.static_lu_chunks(n, N) == [(0, 11), (11, 13)]
    rng = np.random.default_rng(5)
    mats = (rng.standard_normal((n, N, N)) + 1j * rng.standard_normal((n, N, N))) * (0.3 / N ** 0.5)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=0, world_size=1, timeout=datetime.timedelta(seconds=30))
    try:
        d = K.compute_determinant_ksharded(np.arange(n) * (1 + 0.1j), None,
                                           M_fn=lambda w: mats[int(round(w.real))])
    finally:
        dist.destroy_process_group()
    ref = np.linalg.det(np.eye(N)[None] - mats)
    assert np.max(np.abs(d - ref) / np.abs(ref)) < 1e-11


def test_batched_m3_real_q1_model_matches_oracle(pcs):
    """Model 1 of the batch (m = 3, n_zang = 3, q1 = 9.5, NR = 31, Ne = 9,
    N_alpha = 97, l = +-6) evaluated inside the uneven batch against the
    oracle directly: FP64 within 1e-11 relative + 4x the oracle's own 2-ulp-ln
    sensitivity, split-BF16 within 1e-3 relative."""
    from oracle import np_oracle as O
    m, nz, q, nr, ne, na, lm = MODELS[1]
    over = dict(BASE, m=m, n_zang=nz, q1=q, NR=nr, Ne=ne, N_alpha=na, l_min=-lm, l_max=lm)
    om = np.stack([omegas(5, 40 + i) * (mm / 2) for i, (mm, *_) in enumerate(MODELS)])
    mb64 = K.ModelBatch(pcs, "Float64", batch=5)
    d64, _ = mb64.det(om)
    mb64.close()
    mb32 = K.ModelBatch(pcs, "Float32", batch=5)
    d32, _ = mb32.det(om)
    mb32.close()

    def oracle_dets():
        pc = O.precompute_all(O.OracleConfig(**over))
        return np.array([O.compute_det(pc, w) for w in om[1]])

    ref = oracle_dets()
    orig = O.orbit_log
    O.orbit_log = lambda x: orig(x) * (1.0 + 4.440892098500626e-16)
    try:
        sens = np.abs(oracle_dets() - ref)
    finally:
        O.orbit_log = orig
    assert np.all(np.abs(d64[1] - ref) <= 1e-11 * np.abs(ref) + 4 * sens), \
        np.abs(d64[1] - ref) / np.abs(ref)
    assert np.max(np.abs(d32[1] - ref) / np.abs(ref)) < 1e-3


def test_batch_needs_one_fp64_form(pcs):
    pcs[1].ctx.call("kls_set_f64_form", _lib.KLS_F64_3M)
    try:
        with pytest.raises(K.KlsError) as e:
            K.ModelBatch(pcs, "Float64", batch=2)
        assert e.value.code == _lib.KLS_ERR_CONFIG
        with pytest.raises(K.KlsError) as e:
            pcs[0].ctx.call("kls_set_f64_form", 2)
        assert e.value.code == _lib.KLS_ERR_CONFIG
    finally:
        pcs[1].ctx.call("kls_set_f64_form", _lib.KLS_F64_4M)


def test_batch_matches_the_oracle(pcs):
    """Each model of the uneven batch (real-valued q1, m = 2 and 3, four sizes)
    against the oracle's own determinants (oracle/np_oracle.py, the reference's
    per-harmonic form) at 3 omegas: 1e-9 relative in FP64 (no per-element
    sensitivity is stored for these models; the fixture-based parity tests
    hold 1e-11 plus the 2-ulp-ln sensitivity), 1e-3 in the split-BF16 form."""
    from oracle import np_oracle as O
    om = np.stack([omegas(3, 40 + i) * (m / 2) for i, (m, *_) in enumerate(MODELS)])
    got = {}
    for Tgpu in ("Float64", "Float32"):
        mb = K.ModelBatch(pcs, Tgpu, batch=3)
        got[Tgpu], _ = mb.det(om)
        mb.close()
    for i, c in enumerate(configs()):
        g, md = c.grid, c.model
        oc = O.OracleConfig(m=int(c.physics.m), G=float(c.physics.G), L0=float(md.L0),
                            n_zang=int(md.n_zang), q1=float(md.q1), NR=g.NR, Ne=g.Ne,
                            Rc_min=g.Rc_min, Rc_max=g.Rc_max, v_min=g.v_min,
                            N_alpha=g.N_alpha, alpha_max=g.alpha_max, l_min=g.l_min,
                            l_max=g.l_max, nw=g.nw, nwa=g.nwa)
        opc = O.precompute_all(oc)
        ref = np.array([O.compute_det(opc, w) for w in om[i]])
        r64 = np.abs(got["Float64"][i] - ref) / np.abs(ref)
        rmx = np.abs(got["Float32"][i] - ref) / np.abs(ref)
        print(f"model {i} (m={oc.m}, q1={oc.q1}): FP64 {r64.max():.1e}, split-BF16 {rmx.max():.1e}")
        assert r64.max() < 1e-9, (i, r64)
        assert rmx.max() < 1e-3, (i, rmx)
