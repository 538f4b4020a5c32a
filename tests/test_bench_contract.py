"""bench.py's reference arm (CPU only): one JSON line with the driver's keys.

The reference arm times the reference algorithm's CPU form (the oracle's BLAS
restatement) on the host cores; it must print the same metric and unit as the
GPU arm, ``impl: reference``, a ``cpu_baseline`` describing the run and an
``e2e`` block with no host<->device bytes.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    # at the small size S: the default size builds a 24.7 GB table on the host
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1", "--config",
                          os.path.join(ROOT, "configs", "size_s.toml")], capture_output=True,
                         text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "det_evals/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["NR"] == 101 and d["ms_per_step"] > 0
    import bench
    assert d["metric"] == bench.METRIC


def test_small_size_cpu_figures_on_a_host_table(monkeypatch):
    """bench.cpu_small_size (the naive-loop and BLAS-form CPU figures) on a
    stand-in context whose exports come from the oracle at a tiny size: every
    figure is present, the three determinant forms agree, and the CPU Newton
    reaches the stand-in GPU's root."""
    import types
    import numpy as np
    import bench
    import kalnajs_log_spirals_b200 as K
    from oracle import np_oracle as O

    real_load = K.load_config

    def tiny(path):
        c = real_load(path)
        for k, v in dict(NR=12, Ne=7, N_alpha=17, l_min=-4, l_max=4, nw=401, nwa=41).items():
            setattr(c.grid, k, v)
        return c

    class Ctx:
        def __init__(self, opc):
            self.opc, self.dims = opc, types.SimpleNamespace(NPh=opc.NPh)

        def call(self, name, il, nl, ptr):
            # kls_export_W: one harmonic, [N_alpha][NPh] interleaved complex
            assert name == "kls_export_W" and nl == 1
            Wl = np.ascontiguousarray(self.opc.W[:, :, il].T)
            np.ctypeslib.as_array(ptr, shape=(2 * Wl.size,))[:] = Wl.view(np.float64).ravel()

    class PC:
        def __init__(self, cfg):
            o = self.opc = O.precompute_all(bench.oracle_config(cfg))
            self.ctx = Ctx(o)
            self.alpha_arr, self.d_alpha, self.N_kernel, self.DJ_vec = (o.alpha, o.d_alpha,
                                                                         o.N_kernel, o.DJ)
            self.F0l_all = o.F0l.reshape(-1, order="F")
            self.Omega_res = o.Omega_res.reshape(-1, order="F")
            self.closed = False

        def close(self):
            self.closed = True

    made = []

    def precompute(cfg, device=0):
        made.append(PC(cfg))
        return made[-1]

    def newton(cfg, pc, dev, gpu, T):
        r = O.newton_search(lambda w: O.compute_det(pc.opc, w), cfg.physics.m,
                            cfg.reference.Omega_p, cfg.reference.gamma, tol=cfg.newton.tol)
        r.det_evals = 3 * r.iterations
        return r

    monkeypatch.setattr(K, "load_config", tiny)
    monkeypatch.setattr(K, "precompute_all", precompute)
    monkeypatch.setattr(K, "compute_determinant", lambda w, pc: O.compute_det(pc.opc, w))
    monkeypatch.setattr(K, "newton_search", newton)
    args = types.SimpleNamespace(model=os.path.join(ROOT, "models", "kalnajs_zang4.toml"))
    out = bench.cpu_small_size(args, K, 0)
    assert made and made[0].closed
    assert out["naive_loops"]["s_per_det"] > 0
    assert out["naive_loops"]["det_rel_diff_vs_gpu"] < 1e-13
    for leg in ("blas_all_threads", "blas_4_threads"):
        b = out[leg]
        assert b["det_rel_diff_vs_gpu"] < 1e-13 and b["newton_converged"]
        assert np.allclose(b["newton_root"], out["gpu_fp64_newton"]["root"], rtol=0, atol=1e-12)
    assert out["blas_4_threads"]["threads"] <= 4
