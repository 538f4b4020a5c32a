"""Parity at the default size (config [1]) against the oracle.

Fixture: tests/golden/size_d.npz, made by tests/golden/make_size_d.py (the
oracle at configs/default.toml + models/kalnajs_zang4.toml: NR=501, Ne=51,
N_alpha=301 on [-30, 30], l = +-100, nw=100001, nwa=2001; determinant in the
reference script's form, one ZGEMM per harmonic + LAPACK zgetrf).

Tolerances, FP64 (as in tests/test_gpu_parity.py): per element
|gpu - oracle| <= 1e-11 * scale + 4 * sens, sens being the oracle's own change
under a 2-ulp perturbation of ln along the orbit integrals (stored in the
fixture); Newton roots 1e-10 absolute plus the oracle root's own 2-ulp shift.
Split-BF16: the relative det error against the oracle on the seeded accuracy
points stays below 1e-3, and the hybrid Newton (split-BF16 phase, FP64
anchor, anchored finish) lands within 1e-10 of the oracle's root, where the
plain FP64 determinant is below tol as well.
"""
import os

import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from kalnajs_log_spirals_b200.api import newton_search_hybrid
from tests.conftest import GOLDEN, ROOT

FIXTURE = os.path.join(GOLDEN, "size_d.npz")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(FIXTURE),
                                 reason="tests/golden/size_d.npz not generated")]


@pytest.fixture(scope="module")
def ref():
    d = np.load(FIXTURE)
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="module")
def default_model(lib_path):
    cfg = K.load_model(K.load_config(os.path.join(ROOT, "configs", "default.toml")),
                       os.path.join(ROOT, "models", "kalnajs_zang4.toml"))
    pc = K.precompute_all(cfg)
    yield cfg, pc
    pc.close()


def sens(ref, key, like):
    return ref.get("sens_" + key, np.zeros(np.shape(like)))


def test_fp64_root_matches_oracle(default_model, ref):
    cfg, pc = default_model
    r = K.newton_search(cfg, pc, None, K.GPUType.NVIDIA, "Float64")
    tol = 1e-10 + 4 * sens(ref, "root", ref["root"])
    assert r.converged and abs(r.det_val) < cfg.newton.tol
    assert abs(r.Omega_p - ref["root"][0]) <= tol[0], (r.Omega_p, ref["root"])
    assert abs(r.gamma - ref["root"][1]) <= tol[1], (r.gamma, ref["root"])


def test_fp64_M_at_root_matches_oracle(default_model, ref):
    _, pc = default_model
    M = K.build_M_matrix(complex(ref["omega_root"][0]), pc)
    M0 = ref["M0"]
    tol = 1e-11 * np.abs(M0).max() + 4 * sens(ref, "M0", M0)
    err = np.abs(M - M0)
    assert np.all(err <= tol), float(np.max(err - tol))


def test_fp64_dets_match_oracle(default_model, ref):
    _, pc = default_model
    d = K.compute_determinant_batched(ref["omegas"], pc, None, batch_size=16)
    d0 = ref["dets"]
    tol = 1e-11 * np.abs(d0) + 4 * sens(ref, "dets", d0)
    assert np.all(np.abs(d - d0) <= tol), np.abs(d - d0) / np.abs(d0)


def test_mixed_against_oracle(default_model, ref):
    cfg, pc = default_model
    dev = K.to_device(pc, K.GPUType.NVIDIA, "Float32")
    om, d0 = ref["omegas"], ref["dets"]
    n_fixed = int(ref["n_fixed"][0])
    dmx = K.compute_determinant_batched(om[n_fixed:], pc, dev, batch_size=16)
    rel = np.abs(dmx - d0[n_fixed:]) / np.abs(d0[n_fixed:])
    print(f"split-BF16 det error vs oracle: median {np.median(rel):.2e}, max {rel.max():.2e}")
    assert rel.max() < 1e-3, rel
    rh = newton_search_hybrid(cfg, pc)
    d64 = K.compute_determinant(rh.omega, pc, None)
    print(f"hybrid: {rh.mixed_evals} split-BF16, {rh.fp64_evals} FP64, {rh.anchored_evals} "
          f"anchored determinants; |det| {abs(rh.det_val):.2e}, plain FP64 there {abs(d64):.2e}")
    assert rh.converged and abs(d64) < cfg.newton.tol
    assert abs(rh.Omega_p - ref["root"][0]) <= 1e-10 and abs(rh.gamma - ref["root"][1]) <= 1e-10, \
        (rh.Omega_p - ref["root"][0], rh.gamma - ref["root"][1])
