#!/usr/bin/env python
"""Benchmark of the det(I - M(omega)) hot path at the default size.

Workload: Toomre-Zang n_zang=4, q1=7, m=2 disk, NR=501, Ne=51, N_alpha=301 on
[-30, 30], l in [-100, 100] (K = 5,135,751 orbit x l terms), complex128 M,
plain FP64 form.  One step = one Newton finite-difference triple
(omega, omega + m*delta, omega + i*delta) evaluated as one batch.

  value : det evaluations / s with the W table resident in HBM and omegas /
          dets in device buffers (CUDA events on the launching stream)
  e2e   : the same through the C ABI with host buffers (kls_det_batch: H2D of
          omegas, D2H of dets and log|det| inside the timed region)

Also reported: roofline of the contraction kernel (algorithmic FLOPs
8 N_alpha^2 K per determinant against an in-run cuBLAS DGEMM peak, and the
DMMA work the chosen 4M or 3M form issues), the split-BF16 form, Newton
time-to-root from the reference start (plain FP64 against the hybrid: split-
BF16 secant steps, one FP64 anchor, anchored finish), parity against the
default-size oracle fixture, precompute time, the CPU baseline (the oracle's
BLAS form, one whole determinant on the host cores) and SM clocks sampled
during the timed region.

--impl reference times the reference algorithm's CPU form (oracle port: the
oracle builds its own table, then one ZGEMM per harmonic + LAPACK LU per
whole determinant, all host threads) on the same metric.
Multi-GPU (torchrun): independent replicas, each rank evaluating its own
omegas ("replicas only"; the path needs no collective).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Newton time-to-root & det(I−M) evals/s at |Δω|≤1e-10, mixed vs plain FP64"
UNIT = "det_evals/s"
def workload(cfg) -> str:
    """The benchmark workload named by what it is, with its sizes."""
    g, md = cfg.grid, cfg.model
    return (f"plain FP64 det(I-M(omega)): Toomre-Zang n={md.n_zang} m={cfg.physics.m} "
            f"q1={md.q1:g}, NR={g.NR} Ne={g.Ne} N_alpha={g.N_alpha} alpha_max={g.alpha_max:g} "
            f"l=[{g.l_min},{g.l_max}]")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default=os.path.join(ROOT, "configs", "default.toml"))
    ap.add_argument("--model", default=os.path.join(ROOT, "models", "kalnajs_zang4.toml"))
    ap.add_argument("--no-newton", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--accuracy-points", type=int, default=200)
    ap.add_argument("--no-proposer", action="store_true",
                    help="skip the learned-proposal time-to-root block")
    ap.add_argument("--scan-columns", type=int, default=0,
                    help="time only this many columns of the FP64 41x20 scan and scale "
                         "(0: the whole scan, measured)")
    ap.add_argument("--no-uneven", action="store_true",
                    help="skip the 16-model uneven batched scan block")
    ap.add_argument("--no-refgpu", action="store_true",
                    help="skip the reference GPU algorithm (cuBLAS ZGEMM per harmonic) arm")
    ap.add_argument("--heldout", type=int, default=0,
                    help="also evaluate the proposer on N held-out models at the default size")
    ap.add_argument("--heldout-save", default="",
                    help="save the held-out network's parameters (.npy) after training")
    ap.add_argument("--heldout-far", type=float, default=2e-3,
                    help="far_step of the held-out evaluation's second hybrid refinement")
    ap.add_argument("--heldout-params", default="",
                    help="load the held-out network's parameters (.npy) instead of training")
    ap.add_argument("--uneven-columns", type=int, default=1,
                    help="whole Omega_p columns (128 gammas) of the 256 x 128 grid per model")
    ap.add_argument("--uneven-batch", type=int, default=16)
    ap.add_argument("--uneven-out", default="",
                    help="save the evaluated log|det| / arg det maps of the 16 models (.npz)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


# ---------------------------------------------------------------------------
# CPU reference: the oracle's restatement of the reference CPU algorithm
# (NL_julia_direct.jl:177-310: orbits, W_l table, then per determinant one
# weighted copy + one ZGEMM per harmonic and LAPACK zgetrf), on the real model
# at the benchmark's own size, on all host threads
# ---------------------------------------------------------------------------
def oracle_config(cfg):
    from oracle import np_oracle as O
    g, md = cfg.grid, cfg.model
    return O.OracleConfig(m=int(cfg.physics.m), G=float(cfg.physics.G), L0=float(md.L0),
                          n_zang=int(md.n_zang), q1=float(md.q1), NR=g.NR, Ne=g.Ne,
                          Rc_min=g.Rc_min, Rc_max=g.Rc_max, v_min=g.v_min, N_alpha=g.N_alpha,
                          alpha_max=g.alpha_max, l_min=g.l_min, l_max=g.l_max, nw=g.nw,
                          nwa=g.nwa, quad=g.quadrature)


def blas_threads() -> int:
    try:
        from threadpoolctl import threadpool_info
        return max([i.get("num_threads", 1) for i in threadpool_info()
                    if i.get("internal_api") == "openblas"] or [os.cpu_count() or 1])
    except Exception:
        return os.cpu_count() or 1


def table_storage(nbytes: float):
    """Shared memory when /dev/shm holds the table with room to spare, else a
    file in the temporary directory (None: shared memory)."""
    import shutil
    try:
        if shutil.disk_usage("/dev/shm").free > 1.2 * nbytes:
            return None
    except OSError:
        pass
    return os.path.join(tempfile.mkdtemp(prefix="kls_ref_"), "W.c128")


def fixture_check(dets_fn, m: int):
    """The oracle's det at the default-size fixture's first omega against the
    committed value (tests/golden/size_d.npz), when the run is at that size."""
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "size_d.npz")
    if not os.path.exists(path):
        return None
    f = np.load(path)
    w = complex(f["omegas"][0])
    d = dets_fn(w)
    ref = complex(f["dets"][0])
    return {"omega": [w.real, w.imag], "det": [d.real, d.imag],
            "rel_diff_vs_fixture": abs(d - ref) / abs(ref)}


def reference_arm(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    import numpy as np
    import kalnajs_log_spirals_b200 as K
    from oracle import np_oracle_large as L
    cfg = K.load_model(K.load_config(args.config), args.model)
    oc = oracle_config(cfg)
    threads = blas_threads()
    nbytes = 16.0 * oc.NPh * oc.N_alpha * oc.n_l
    path = table_storage(nbytes)
    t0 = time.perf_counter()
    pc = L.precompute_large(oc, workers=os.cpu_count() or 1, table_path=path)
    t_pre = time.perf_counter() - t0
    try:
        m = oc.m
        # one determinant per step, the omegas of the GPU arm's Newton triples
        n_steps = args.warmup + args.steps
        oms = [omegas_for_step(s // 3, 0, m, cfg.reference.Omega_p, cfg.reference.gamma,
                               cfg.newton.delta)[s % 3] for s in range(n_steps)]
        for s in range(args.warmup):
            L.compute_det_large(pc, oms[s])
        dets = []
        t0 = time.perf_counter()
        for s in range(args.warmup, n_steps):
            dets.append(L.compute_det_large(pc, oms[s]))
        t = time.perf_counter() - t0
        same_size = (oc.NR, oc.Ne, oc.N_alpha, oc.l_min, oc.l_max) == (501, 51, 301, -100, 100)
        check = fixture_check(lambda w: L.compute_det_large(pc, w), m) if same_size else None
    finally:
        pc.close()
        if path:
            import shutil
            shutil.rmtree(os.path.dirname(path), ignore_errors=True)
    rate = args.steps / t
    sample = (f"whole determinants at {oc.NR}x{oc.Ne} orbits, N_alpha={oc.N_alpha}, "
              f"l=[{oc.l_min},{oc.l_max}] ({oc.n_l} ZGEMMs {oc.N_alpha}x{oc.NPh}x{oc.N_alpha} "
              f"+ zgetrf per det), one det per step; table precompute {t_pre:.0f} s untimed")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the model's own grids)",
            "config": {"workload": workload(cfg), "NR": oc.NR, "Ne": oc.Ne, "N_alpha": oc.N_alpha,
                       "l": [oc.l_min, oc.l_max], "omegas_per_step": 1,
                       "step": "one whole determinant (the omegas of the GPU arm's Newton "
                               "triples, in order)"},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "precompute_s": t_pre, "host_cores": os.cpu_count(),
            "dets": [[d.real, d.imag] for d in dets[:3]], "oracle_fixture_check": check}
    print(json.dumps(line), flush=True)
    return 0


def oracle_parity(K, cfg, pc, newton, mixed: bool):
    """FP64 and split-BF16 results against the oracle at the default size
    (tests/golden/size_d.npz, made by tests/golden/make_size_d.py: the
    oracle's Newton root, M at that root and dets at 23 omegas).  FP64
    tolerances as in the parity tests: 1e-11 of the scale plus 4x the oracle's
    own 2-ulp-ln sensitivity; roots 1e-10."""
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "size_d.npz")
    g = cfg.grid
    if not os.path.exists(path) or (g.NR, g.Ne, g.N_alpha, g.l_min, g.l_max) != \
            (501, 51, 301, -100, 100):
        return None
    f = np.load(path)
    om, d_or = f["omegas"], f["dets"]
    sens = f["sens_dets"] if "sens_dets" in f.files else np.zeros(len(om))
    d64 = K.compute_determinant_batched(om, pc, None, batch_size=16)
    err64 = np.abs(d64 - d_or)
    M = K.build_M_matrix(complex(f["omega_root"][0]), pc)
    M0 = f["M0"]
    sM = f["sens_M0"] if "sens_M0" in f.files else np.zeros(M0.shape)
    errM = np.abs(M - M0)
    root = f["root"]
    out = {"fixture": "tests/golden/size_d.npz (oracle, NL_julia_direct.jl BLAS form)",
           "omegas": int(len(om)),
           "fp64": {"det_rel_err_max": float(np.max(err64 / np.abs(d_or))),
                    "det_within_tol": bool(np.all(err64 <= 1e-11 * np.abs(d_or) + 4 * sens)),
                    "M_at_root_err_over_max": float(errM.max() / np.abs(M0).max()),
                    "M_within_tol": bool(np.all(errM <= 1e-11 * np.abs(M0).max() + 4 * sM))},
           "oracle_root": [float(root[0]), float(root[1])]}
    if newton:
        r = newton["plain_fp64"]
        out["fp64"]["root_abs_diff"] = [abs(r["Omega_p"] - root[0]), abs(r["gamma"] - root[1])]
        h = newton.get("mixed_fp64_finish")
        if h:
            out["hybrid_root_abs_diff"] = [abs(h["Omega_p"] - root[0]), abs(h["gamma"] - root[1])]
    if mixed:
        try:
            dev = K.to_device(pc, K.GPUType.NVIDIA, "Float32")
            dmx = K.compute_determinant_batched(om, pc, dev, batch_size=16)
            rel = np.abs(dmx - d_or) / np.abs(d_or)
            out["mixed"] = {"det_rel_err_vs_oracle": {"median": float(np.median(rel)),
                                                      "max": float(rel.max())}}
        except K.KlsError as e:
            out["mixed"] = {"unavailable": str(e)}
    return out


def cpu_det_baseline(pc, cfg, omega: complex):
    """The oracle's BLAS-form determinant (one ZGEMM per harmonic + zgetrf) on
    the host cores, timed on one whole determinant of the benchmark model; the
    table is the device's own, exported harmonic by harmonic (the oracle's
    table build is timed by --impl reference).  Returns (det/s, det, note)."""
    import numpy as np
    from oracle import np_oracle_large as L
    oc = oracle_config(cfg)
    dims = pc.ctx.dims
    W = np.empty((oc.n_l, dims.NPh, oc.N_alpha), dtype=np.complex128)
    buf = np.empty(dims.NPh * oc.N_alpha, dtype=np.complex128)
    for il in range(oc.n_l):
        pc.ctx.call("kls_export_W", il, 1, buf.view(np.float64).ctypes.data_as(
            C.POINTER(C.c_double)))
        W[il] = buf.reshape(oc.N_alpha, dims.NPh).T
    DJ = pc.DJ_vec
    F0l = pc.F0l_all.reshape(dims.NPh, oc.n_l, order="F")
    Ores = pc.Omega_res.reshape(dims.NPh, oc.n_l, order="F")

    class _T:
        arr = W

        @staticmethod
        def close(unlink=False):
            pass

    lp = L.LargePrecomputed(oc, pc.alpha_arr, pc.d_alpha, pc.N_kernel, None, None, DJ, F0l,
                            Ores, _T())
    L.compute_det_large(lp, omega + 1e-3)            # warm the BLAS pool
    t0 = time.perf_counter()
    d = L.compute_det_large(lp, omega)
    t = time.perf_counter() - t0
    del W
    return 1.0 / t, d, (f"one whole determinant (all {oc.n_l} harmonics, ZGEMM "
                        f"{oc.N_alpha}x{dims.NPh}x{oc.N_alpha} each, + zgetrf) on the device's "
                        f"exported table")


def cpu_small_size(args, K, local):
    """Secondary CPU figures at the small size (NR=101, Ne=21, N_alpha=101,
    l in [-25, 25], Newton tol 1e-10) on the device's exported table:
    the reference module's naive loops (MatrixBuilder.jl:37-87, its --gpu=CPU
    path) as one whole determinant, and the BLAS form (NL_julia_direct.jl:
    299-310) on all host threads and on the reference's configured 4 threads
    (max_threads), each as one whole determinant and as a whole FP64 Newton
    solve from the reference start; the GPU's FP64 Newton on the same model
    beside them."""
    import numpy as np
    from threadpoolctl import threadpool_limits
    from oracle import np_oracle as O
    cfg = K.load_model(K.load_config(os.path.join(ROOT, "configs", "size_s.toml")), args.model)
    pc = K.precompute_all(cfg, device=local)
    try:
        oc = oracle_config(cfg)
        NPh, Na, nl = pc.ctx.dims.NPh, oc.N_alpha, oc.n_l
        W = np.empty((NPh, Na, nl), dtype=np.complex128, order="F")
        buf = np.empty(NPh * Na, dtype=np.complex128)
        for il in range(nl):
            pc.ctx.call("kls_export_W", il, 1, buf.view(np.float64).ctypes.data_as(
                C.POINTER(C.c_double)))
            W[:, :, il] = buf.reshape(Na, NPh).T
        opc = O.Precomputed(oc, oc.m, float(oc.G), Na, nl, np.arange(oc.l_min, oc.l_max + 1),
                            NPh, pc.alpha_arr, pc.d_alpha, None, pc.DJ_vec,
                            pc.F0l_all.reshape(NPh, nl, order="F"),
                            pc.Omega_res.reshape(NPh, nl, order="F"), W, pc.N_kernel)
        m = oc.m
        Op0, g0 = float(cfg.reference.Omega_p), float(cfg.reference.gamma)
        nc = cfg.newton
        w0 = complex(m * Op0, g0)
        out = {"size": f"NR={oc.NR} Ne={oc.Ne} N_alpha={Na} l=[{oc.l_min},{oc.l_max}] "
                       f"(K = {NPh * nl})", "host_cores": os.cpu_count(),
               "start": [Op0, g0], "tol": float(nc.tol)}
        t0 = time.perf_counter()
        d_naive = O.compute_det_naive(opc, w0)
        t_naive = time.perf_counter() - t0
        d_gpu = K.compute_determinant(w0, pc)
        out["naive_loops"] = {"s_per_det": t_naive, "det_evals_per_s": 1.0 / t_naive,
                              "threads": 1, "det_rel_diff_vs_gpu": abs(d_naive - d_gpu) / abs(d_gpu)}
        for label, nthr in (("blas_all_threads", None), ("blas_4_threads", 4)):
            with threadpool_limits(nthr, user_api="blas"):
                O.compute_det(opc, w0 + 1e-3)                    # warm the BLAS pool
                t0 = time.perf_counter()
                d_blas = O.compute_det(opc, w0)
                t_det = time.perf_counter() - t0
                t0 = time.perf_counter()
                r = O.newton_search(lambda w: O.compute_det(opc, w), m, Op0, g0,
                                    max_iter=int(nc.max_iter), tol=float(nc.tol),
                                    delta=float(nc.delta))
                t_newton = time.perf_counter() - t0
                out[label] = {"threads": blas_threads(), "s_per_det": t_det,
                              "det_evals_per_s": 1.0 / t_det,
                              "det_rel_diff_vs_gpu": abs(d_blas - d_gpu) / abs(d_gpu),
                              "newton_s": t_newton, "newton_root": [r.Omega_p, r.gamma],
                              "newton_iterations": int(r.iterations),
                              "newton_converged": bool(r.converged)}
        t0 = time.perf_counter()
        rg = K.newton_search(cfg, pc, None, K.GPUType.NVIDIA, "Float64")
        t_gpu = time.perf_counter() - t0
        out["gpu_fp64_newton"] = {"newton_s": t_gpu, "root": [rg.Omega_p, rg.gamma],
                                  "iterations": int(rg.iterations), "det_evals": int(rg.det_evals)}
        return out
    finally:
        pc.close()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv",
                                       "-lms", "200", "-i", str(gpu_index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.strip() for r in self.f.read().splitlines()[1:] if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            parts = [x.strip() for x in r.split(",")]
            try:
                sm.append(float(parts[1].split()[0]))
                mx = float(parts[2].split()[0])
            except Exception:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dgemm_peak_tflops(torch) -> float:
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def read_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the data file beside the ncu
    summaries (profiles/traffic.json): (bytes, scaled from a smaller case)."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))[kernel]
        return float(d["bytes_per_launch"]), bool(d.get("scaled", False))
    except (OSError, KeyError, ValueError):
        return None, None


def precompute_roofline(cfg, dims, pre_ms, peak64: float, peaks: dict):
    """Orbit integration and W_l quadrature kernels against the FP64 and HBM
    peaks (CUDA-event times of the precompute in this run)."""
    NPh, Na, n_l, nwa, nw = dims.NPh, dims.N_alpha, dims.n_l, dims.nwa, cfg.grid.nw
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    hbm_note = "of measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else \
        "of fallback (6.65 TB/s)"
    t_orb, t_wl = pre_ms[0] * 1e-3, pre_ms[1] * 1e-3
    out = {}
    if t_orb > 0:
        orb_bytes = 3.0 * nwa * NPh * 8 + 17.0 * NPh * 8 + 2.0 * nw * 8
        out["orbit_kernel"] = {
            "ms": pre_ms[0], "point_evaluations_per_s": 2.0 * nw * NPh / t_orb,
            "algorithmic_bytes": orb_bytes, "hbm_gbs": orb_bytes / t_orb / 1e9,
            "hbm_frac": orb_bytes / t_orb / 1e9 / hbm, "hbm_peak_note": hbm_note,
            "bound": "FP64 + transcendentals (2 nw point evaluations per orbit)"}
    if t_wl > 0:
        wl_bytes = float(NPh) * Na * n_l * 16 + 3.0 * nwa * NPh * 8
        wl_flops = 4.0 * n_l * nwa * Na * NPh
        out["wl_kernel"] = {
            "ms": pre_ms[1], "algorithmic_bytes": wl_bytes, "hbm_gbs": wl_bytes / t_wl / 1e9,
            "hbm_frac": wl_bytes / t_wl / 1e9 / hbm, "hbm_peak_note": hbm_note,
            "algorithmic_flops": wl_flops, "tflops": wl_flops / t_wl / 1e12,
            "fp64_frac": wl_flops / t_wl / 1e12 / peak64,
            "fp64_peak_note": "of measured: cuBLAS DGEMM in this run",
            "bound": "FP64 tensor pipe (DMMA); output 16 B per table entry"}
    return out


def omegas_for_step(step: int, rank: int, m: int, Op: float, g: float, delta: float):
    # a Newton FD triple around a point that moves with the step (distinct omegas)
    Op_s = Op + 1e-4 * ((step * 7 + rank * 131) % 97) / 97.0
    g_s = g + 1e-4 * ((step * 13 + rank * 71) % 89) / 89.0
    return [complex(m * Op_s, g_s), complex(m * (Op_s + delta), g_s), complex(m * Op_s, g_s + delta)]


# ---------------------------------------------------------------------------
# the reference's GPU algorithm on this B200 (NL_julia_direct_gpu.jl:277-288,
# MatrixBuilder.jl:100-185): per harmonic l a weighted copy w .* conj(W_l) and
# one ZGEMM W_l^T (.) (cuBLAS through torch), then M to the host and LAPACK det
# ---------------------------------------------------------------------------
def reference_algorithm_gpu(torch, K, pc, cfg, reps: int = 2):
    """The reference's own GPU algorithm on the benchmark model: the device's
    W table exported harmonic by harmonic into the reference layout
    [n_l][NPh][N_alpha] complex128 on the device, then per determinant one
    weighted copy w .* conj(W_l) and one ZGEMM W_l^T (.) per harmonic (cuBLAS
    through torch), M to the host and LAPACK det.  Its determinant is also an
    independent library check of the FP64 kernels' result at this size."""
    import numpy as np
    dims = pc.ctx.dims
    NPh, Na, n_l = dims.NPh, dims.N_alpha, dims.n_l
    W = torch.empty((n_l, NPh, Na), dtype=torch.complex128, device="cuda")
    buf = np.empty(NPh * Na, dtype=np.complex128)
    for il in range(n_l):
        pc.ctx.call("kls_export_W", il, 1, buf.view(np.float64).ctypes.data_as(
            C.POINTER(C.c_double)))
        W[il] = torch.from_numpy(buf.reshape(Na, NPh).T.copy()).to("cuda")
    F0l = torch.tensor(pc.F0l_all.reshape(NPh, n_l, order="F").T.copy(), device="cuda")
    Ores = torch.tensor(pc.Omega_res.reshape(NPh, n_l, order="F").T.copy(), device="cuda")
    DJ = torch.tensor(pc.DJ_vec, device="cuda")
    Nk = pc.N_kernel
    G = float(cfg.physics.G)
    eye = np.eye(Na)

    def one(omega):
        M = torch.zeros((Na, Na), dtype=torch.complex128, device="cuda")
        for l in range(n_l):
            den = omega - Ores[l]
            den = torch.where(den.abs() < 1e-12, torch.full_like(den, 1e-12 + 1e-12j), den)
            M += W[l].transpose(0, 1) @ (((DJ * F0l[l]) / den)[:, None] * W[l].conj())
        Mh = M.cpu().numpy() * G * Nk[None, :]
        return complex(np.linalg.det(eye - Mh))

    w0 = complex(2 * cfg.reference.Omega_p, cfg.reference.gamma)
    one(w0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dets = [one(w0 + 1e-3 * r) for r in range(reps)]
    t = (time.perf_counter() - t0) / reps
    ours = K.compute_determinant_batched(np.array([w0 + 1e-3 * r for r in range(reps)]), pc)
    del W
    torch.cuda.empty_cache()
    return {"det_evals_per_s": 1.0 / t, "s_per_det": t, "reps": reps,
            "form": "per-harmonic weighted copy + cuBLAS ZGEMM (torch.matmul complex128), "
                    "M to the host, numpy LAPACK det; the benchmark model's own table",
            "det_rel_diff_vs_ours_fp64": float(np.max(np.abs(np.array(dets) - ours)
                                                      / np.abs(ours)))}


# ---------------------------------------------------------------------------
# time-to-root: the reference workflow (41 x 20 grid scan, argmin, Newton) in
# plain FP64 against a learned proposal + mixed/FP64 hybrid Newton
# ---------------------------------------------------------------------------
def time_to_root(args, K, P, cfg, pc, local, sync):
    import numpy as np
    from kalnajs_log_spirals_b200.api import newton_search_hybrid
    out = {}
    # proposer: trained on 2^17 samples of one batched scan over 64 seeded
    # random models (small size), by the library's own BF16 kernels
    base = K.load_model(K.load_config(os.path.join(ROOT, "configs", "size_s.toml")), args.model)
    t0 = time.perf_counter()
    specs = P.random_models(64, seed=2024)
    X, T = P.scan_samples(base, specs, n_Op=64, n_gamma=32, batch=16, device=local)
    t_gen = time.perf_counter() - t0
    mlp = P.MLP(256, 4, seed=0, device=local)
    t0 = time.perf_counter()
    hist = mlp.train(X, T, epochs=150, batch=1024, lr=1e-3, seed=0)
    t_train = time.perf_counter() - t0
    out["proposer_training"] = {
        "samples": int(X.shape[0]), "models": len(specs), "model_seed": 2024,
        "sample_grid": "64 x 32 over Omega_p [0.2, 0.8], gamma [0.01, 0.30] per model",
        "model_size": "NR=101 Ne=21 N_alpha=101 l=[-25,25]", "network": "5-256-256-256-3 GELU",
        "epochs": 150, "sample_gen_s": t_gen, "train_s": t_train,
        "loss_first_last": [float(hist[0]), float(hist[-1])]}
    s = cfg.scan
    Op_grid = np.linspace(s.Omega_p_min, s.Omega_p_max, s.n_Op)
    g_grid = np.linspace(s.gamma_min, s.gamma_max, s.n_gamma)
    m = cfg.physics.m
    devmx = K.to_device(pc, K.GPUType.NVIDIA, "Float32")
    spec = P.ModelSpec(int(cfg.model.n_zang), float(cfg.model.q1), int(m))

    # learned proposal + hybrid Newton
    sync()
    t0 = time.perf_counter()
    Op_p, g_p, used = P.propose(mlp, spec, lambda om: K.compute_determinant_batched(
        om, pc, devmx, batch_size=16), k=48, n_Op=s.n_Op, n_gamma=s.n_gamma,
        Op_range=(s.Omega_p_min, s.Omega_p_max), g_range=(s.gamma_min, s.gamma_max))
    t_prop = time.perf_counter() - t0
    t0 = time.perf_counter()
    rh = newton_search_hybrid(cfg, pc, Op_p, g_p)
    t_hyb = time.perf_counter() - t0

    # plain FP64 reference workflow
    sync()
    t0 = time.perf_counter()
    dgm, Op_m, g_m = K.grid_scan(cfg, pc, devmx)
    t_scan_mx = time.perf_counter() - t0
    if args.scan_columns <= 0:
        t0 = time.perf_counter()
        dg64, Op64, g64 = K.grid_scan(cfg, pc, None)
        t_scan64 = time.perf_counter() - t0
        scan_note = "measured: whole 41 x 20 FP64 scan"
    else:
        # whole columns of the FP64 scan (the mixed argmin's and its
        # neighbours), the same batches of 16 the scan launches, scaled
        j = int(np.argmin(np.abs(Op_grid - Op_m)))
        cols = sorted({min(max(j + d, 0), s.n_Op - 1) for d in range(args.scan_columns)})
        om = np.array([m * Op_grid[c] + 1j * g for c in cols for g in g_grid])
        t0 = time.perf_counter()
        d64 = K.compute_determinant_batched(om, pc, None, batch_size=16)
        t_cols = time.perf_counter() - t0
        t_scan64 = t_cols * s.n_Op / len(cols)
        q = int(np.argmin(np.abs(d64)))
        Op64, g64 = float(Op_grid[cols[q // s.n_gamma]]), float(g_grid[q % s.n_gamma])
        scan_note = (f"extrapolated: columns {cols} of {s.n_Op} ({len(om)} FP64 dets in "
                     f"{t_cols:.2f} s) x {s.n_Op}/{len(cols)}")
    sync()
    t0 = time.perf_counter()
    r64 = K.newton_search(cfg, pc, None, K.GPUType.NVIDIA, "Float64", Op64, g64)
    t_n64 = time.perf_counter() - t0
    dOp, dg = abs(rh.Omega_p - r64.Omega_p), abs(rh.gamma - r64.gamma)
    plain_total = t_scan64 + t_n64
    mlp.close()
    learned_total = t_prop + t_hyb
    out.update({
        "workflow": "grid_scan 41x20 -> argmin -> Newton (tol %g)" % cfg.newton.tol,
        "plain_fp64": {"scan_s": t_scan64, "scan": scan_note, "newton_s": t_n64,
                       "total_s": plain_total, "start": [Op64, g64],
                       "Omega_p": r64.Omega_p, "gamma": r64.gamma, "converged": r64.converged,
                       "det_evals": s.n_Op * s.n_gamma + r64.det_evals},
        "mixed_scan_then_hybrid": {"scan_s": t_scan_mx, "start": [float(Op_m), float(g_m)],
                                   "total_s": t_scan_mx + t_hyb,
                                   "note": "hybrid Newton time of the proposal row (same start)"
                                   if (Op_m, g_m) == (Op_p, g_p) else "start differs from proposal"},
        "learned_proposal_then_hybrid": {
            "propose_s": t_prop, "mixed_dets_for_proposal": used, "start": [Op_p, g_p],
            "newton_s": t_hyb, "total_s": learned_total, "Omega_p": rh.Omega_p,
            "gamma": rh.gamma, "converged": rh.converged, "mixed_evals": rh.mixed_evals,
            "fp64_evals": rh.fp64_evals},
        "abs_dOmega_p": dOp, "abs_dgamma": dg,
        "same_root_within_1e-10": bool(rh.converged and r64.converged and dOp <= 1e-10
                                       and dg <= 1e-10),
        "speedup_learned_vs_plain": plain_total / learned_total,
        "learned_total_with_training_s": learned_total + t_gen + t_train,
        "speedup_learned_with_training_vs_plain": plain_total / (learned_total + t_gen + t_train),
        "timing": "host wall clock around synchronous library calls"})
    return out


# ---------------------------------------------------------------------------
# proposer on held-out models at the default size: the learned start + hybrid
# Newton against the scan-started FP64 Newton (the scan argmin taken from the
# split-BF16 scan and confirmed by FP64 determinants of its 5 best points)
# ---------------------------------------------------------------------------
def polish(K, cfg, pc, Op, g, steps: int = 2):
    """FP64 Newton steps from (Op, g) past the |det| < tol test: the stopping
    rule pins a root only to tol / |det'|, which for flat determinants is far
    above 1e-10; two more steps pin it to the FP64 noise."""
    c = K.config.copy_config(cfg)
    c.newton.tol = 0.0
    c.newton.max_iter = steps
    r = K.newton_search(c, pc, None, K.GPUType.NVIDIA, "Float64", Op, g)
    return r.Omega_p, r.gamma


def heldout_eval(args, K, P, base_cfg, n_models: int, t_fp64_det: float, local, sync):
    import numpy as np
    from kalnajs_log_spirals_b200.api import newton_search_hybrid
    mlp = P.MLP(256, 4, seed=0, device=local)
    if args.heldout_params:
        # parameters of an earlier training run of the same recipe
        params = np.load(args.heldout_params)
        mlp.set_params(params)
        n_samples, t_gen, t_train, hist = None, 0.0, 0.0, [float("nan"), float("nan")]
    else:
        # the network for this size: trained on batched split-BF16 scans of 64
        # seeded models at the default size (6 mixed-only models per batch)
        t0 = time.perf_counter()
        X, T = P.scan_samples(base_cfg, P.random_models(64, seed=2024), n_Op=32, n_gamma=16,
                              batch=16, chunk=6, device=local)
        t_gen = time.perf_counter() - t0
        n_samples = int(X.shape[0])
        t0 = time.perf_counter()
        hist = mlp.train(X, T, epochs=300, batch=1024, lr=1e-3, seed=0)
        t_train = time.perf_counter() - t0
        if args.heldout_save:
            np.save(args.heldout_save, mlp.params())
    specs = P.random_models(n_models, seed=7)
    rows = []
    for sp in specs:
        cfg = P.model_config(base_cfg, sp)
        s = cfg.scan
        pc = K.precompute_all(cfg, device=local)
        devmx = K.to_device(pc, K.GPUType.NVIDIA, "Float32")
        sync()
        t0 = time.perf_counter()
        dgm, _, _ = K.grid_scan(cfg, pc, devmx)
        t_scan_mx = time.perf_counter() - t0
        Op_grid = np.linspace(s.Omega_p_min, s.Omega_p_max, s.n_Op)
        g_grid = np.linspace(s.gamma_min, s.gamma_max, s.n_gamma)
        flat = np.abs(dgm).ravel(order="F")
        top = np.argsort(flat, kind="stable")[:5]
        om = np.array([sp.m * Op_grid[q // s.n_gamma] + 1j * g_grid[q % s.n_gamma] for q in top])
        d64 = np.abs(K.compute_determinant_batched(om, pc, None, batch_size=16))
        q = int(top[int(np.argmin(d64))])
        Op0, g0 = float(Op_grid[q // s.n_gamma]), float(g_grid[q % s.n_gamma])
        t0 = time.perf_counter()
        r64 = K.newton_search(cfg, pc, None, K.GPUType.NVIDIA, "Float64", Op0, g0)
        t_n64 = time.perf_counter() - t0
        sync()
        t0 = time.perf_counter()
        Op_p, g_p, used = P.propose(mlp, sp, lambda w: K.compute_determinant_batched(
            w, pc, devmx, batch_size=16), k=48, n_Op=s.n_Op, n_gamma=s.n_gamma,
            Op_range=(s.Omega_p_min, s.Omega_p_max), g_range=(s.gamma_min, s.gamma_max))
        t_prop = time.perf_counter() - t0
        # the proposal refined three ways: FP64 Newton (the workload's own
        # refinement), the hybrid with its defaults, and the hybrid with far
        # steps of FP64 accuracy down to --heldout-far (grid starts are coarse)
        t0 = time.perf_counter()
        rp = K.newton_search(cfg, pc, None, K.GPUType.NVIDIA, "Float64", Op_p, g_p)
        t_rp = time.perf_counter() - t0
        t0 = time.perf_counter()
        rh = newton_search_hybrid(cfg, pc, Op_p, g_p)
        t_h = time.perf_counter() - t0
        t0 = time.perf_counter()
        rh2 = newton_search_hybrid(cfg, pc, Op_p, g_p, K.api.HybridConfig(far_step=args.heldout_far))
        t_h2 = time.perf_counter() - t0
        growing = bool(r64.converged and r64.gamma > 1e-4)
        a = polish(K, cfg, pc, r64.Omega_p, r64.gamma) if growing else None

        def same_as_scan(r):
            if not (growing and r.converged):
                return False, None
            b = polish(K, cfg, pc, r.Omega_p, r.gamma)
            return abs(a[0] - b[0]) <= 1e-10 and abs(a[1] - b[1]) <= 1e-10, b

        same, _ = same_as_scan(rp)
        same_h, b = same_as_scan(rh)
        same_h2, _ = same_as_scan(rh2)
        pc.close()
        rows.append({"n_zang": sp.n_zang, "q1": sp.q1, "m": sp.m, "growing_mode": growing,
                     "same_root": same, "same_root_hybrid": same_h,
                     "same_root_hybrid_far": same_h2,
                     "start_equals_scan_argmin": (Op_p, g_p) == (Op0, g0),
                     "proposal_dets": used,
                     "plain_fp64_s": s.n_Op * s.n_gamma * t_fp64_det + t_n64,
                     "mixed_scan_s": t_scan_mx, "learned_s": t_prop + t_rp,
                     "learned_hybrid_s": t_prop + t_h, "learned_hybrid_far_s": t_prop + t_h2,
                     "Omega_p": r64.Omega_p, "gamma": r64.gamma,
                     "scan_start": [Op0, g0], "proposal_start": [Op_p, g_p],
                     "fp64_from_proposal": [rp.Omega_p, rp.gamma, bool(rp.converged)],
                     "hybrid": [rh.Omega_p, rh.gamma, bool(rh.converged), rh.mixed_evals,
                                rh.fp64_evals, rh.anchored_evals],
                     "hybrid_far": [rh2.Omega_p, rh2.gamma, bool(rh2.converged),
                                         rh2.mixed_evals, rh2.fp64_evals, rh2.anchored_evals],
                     "polished_scan_root": a, "polished_hybrid_root": b})
    grow = [r for r in rows if r["growing_mode"]]
    ok = [r for r in grow if r["same_root"]]
    rate = lambda key: (len([r for r in grow if r[key]]) / len(grow)) if grow else None
    mean = lambda k, rs: float(np.mean([r[k] for r in rs])) if rs else None
    mlp.close()
    return {"models": n_models, "model_seed": 7, "size": "default (NR=501 Ne=51 N_alpha=301 l=+-100)",
            "training": {"samples": n_samples, "models": 64, "model_seed": 2024,
                         "from_file": bool(args.heldout_params),
                         "grid": "32 x 16 over Omega_p [0.2, 0.8], gamma [0.01, 0.30]",
                         "size": "default", "sample_gen_s": t_gen, "train_s": t_train,
                         "epochs": 300, "loss_first_last": [float(hist[0]), float(hist[-1])]},
            "same_root_rule": "both roots polished by 2 FP64 Newton steps, then |dOmega_p|, "
                              "|dgamma| <= 1e-10",
            "refinement": "success_rate: proposal refined by FP64 Newton (the workload's "
                          "refinement); also by the hybrid Newton (defaults) and by the hybrid "
                          "with far_step --heldout-far",
            "with_growing_mode": len(grow), "same_root_within_1e-10": len(ok),
            "success_rate": len(ok) / len(grow) if grow else None,
            "success_rate_hybrid": rate("same_root_hybrid"),
            "success_rate_hybrid_far": rate("same_root_hybrid_far"),
            "far_step": args.heldout_far,
            "mean_time_to_root_s": {"plain_fp64 (scan at the measured FP64 det time)":
                                    mean("plain_fp64_s", grow),
                                    "learned_proposal_then_fp64_newton": mean("learned_s", grow),
                                    "learned_proposal_then_hybrid": mean("learned_hybrid_s", grow),
                                    "learned_proposal_then_hybrid_far":
                                        mean("learned_hybrid_far_s", grow)},
            "per_model": rows}


# ---------------------------------------------------------------------------
# uneven batched scan: 16 seeded models of three sizes, one persistent launch
# per pass, split-BF16 form, autotuned K splits
# ---------------------------------------------------------------------------
def uneven_batch(args, K, P, local, sync):
    """Config [3]: 16 seeded models of three sizes on the 256 x 128 grid over
    Omega_p [0.2, 0.8], gamma [0.01, 0.30], split-BF16; the first
    `--uneven-columns` whole Omega_p columns (128 gammas each) of every model
    are evaluated (one graph replay per pass of `--uneven-batch` omegas per
    model) and the full grid's time is projected from them.  With
    `--uneven-out` the log|det| and arg det maps are saved (.npz)."""
    import numpy as np
    base = K.load_model(K.load_config(args.config), args.model)
    specs = P.random_models(16, seed=0, sizes=P.SIZES)
    t0 = time.perf_counter()
    pcs, tunes = [], []
    for sp in specs:
        pc = K.precompute_all(P.model_config(base, sp), device=local)
        pc.ctx.call("kls_prepare_mixed")
        tunes.append(K.autotune(pc, "Float32", batch=args.uneven_batch))
        K.release_fp64(pc)
        pcs.append(pc)
    sync()
    t_setup = time.perf_counter() - t0
    B, cols = args.uneven_batch, args.uneven_columns
    nO, nG = 256, 128
    Op = np.linspace(0.2, 0.8, nO)
    gm = np.linspace(0.01, 0.30, nG)
    n_pts = cols * nG                                   # column-major: whole columns
    q = np.arange(n_pts)
    pts = Op[q // nG], gm[q % nG]
    om = np.stack([sp.m * pts[0] + 1j * pts[1] for sp in specs])
    mb = K.ModelBatch(pcs, "Float32", batch=B)
    mb.det(om[:, :B])                                   # warm-up pass
    sync()
    dets = np.empty(om.shape, dtype=np.complex128)
    la = np.empty(om.shape)
    t0 = time.perf_counter()
    dev_ms = 0.0
    npass = 0
    for p0 in range(0, n_pts, B):
        d, l = mb.det(om[:, p0:p0 + B])
        dets[:, p0:p0 + B], la[:, p0:p0 + B] = d, l
        dev_ms += mb.info()["last_ms"]
        npass += 1
    t_wall = time.perf_counter() - t0
    info = mb.info()
    mb.close()
    n_det = len(specs) * n_pts
    # one column model by model through each context's own batch call; each
    # context is released after its column (a context's own split-BF16
    # partials for B omegas are GBs at the default size, 16 would not fit
    # beside the tables)
    t_seq = 0.0
    for pc, o in zip(pcs, om):
        dev = K.to_device(pc, K.GPUType.NVIDIA, "Float32")
        sync()
        t0 = time.perf_counter()
        K.compute_determinant_batched(o[:nG], pc, dev, batch_size=B)
        sync()
        t_seq += time.perf_counter() - t0
        pc.close()
    rate = n_det / (dev_ms * 1e-3)
    # the smallest batched model against the oracle (its own table, built on
    # the host cores) at 3 of the evaluated points: split-BF16 det error
    oracle_check = None
    small = [i for i, sp in enumerate(specs) if sp.size == P.SIZES[0]]
    if small:
        from oracle import np_oracle_large as L
        i = small[0]
        oc = oracle_config(P.model_config(base, specs[i]))
        t0 = time.perf_counter()
        lp = L.precompute_large(oc, workers=os.cpu_count() or 1)
        try:
            pick = [0, nG // 3, (2 * nG) // 3]
            ref = np.array([L.compute_det_large(lp, om[i, q]) for q in pick])
        finally:
            lp.close()
        rel = np.abs(dets[i, pick] - ref) / np.abs(ref)
        oracle_check = {"model": i, "spec": [specs[i].n_zang, specs[i].q1, specs[i].m,
                                             *specs[i].size],
                        "omegas": [[complex(om[i, q]).real, complex(om[i, q]).imag] for q in pick],
                        "split_bf16_rel_det_err_vs_oracle": [float(x) for x in rel],
                        "oracle_s": time.perf_counter() - t0}
    if args.uneven_out:
        np.savez_compressed(args.uneven_out, log_abs=la.reshape(len(specs), cols, nG),
                            arg=np.angle(dets).reshape(len(specs), cols, nG),
                            Omega_p=Op[:cols], gamma=gm,
                            models=np.array([[sp.n_zang, sp.q1, sp.m, *sp.size] for sp in specs]))
    sizes = [sp.size for sp in specs]
    return {
        "models": len(specs), "model_seed": 0, "sizes": {str(sz): sizes.count(sz) for sz in P.SIZES},
        "grid": "256 x 128 over Omega_p [0.2, 0.8], gamma [0.01, 0.30]",
        "evaluated": f"{cols} whole Omega_p column(s) x 128 gammas per model ({n_det} dets)",
        "omegas_per_model_per_pass": B, "passes": npass,
        "det_evals_per_s": rate, "ms_per_pass_device": dev_ms / npass,
        "wall_det_evals_per_s": n_det / t_wall,
        "one_model_at_a_time_det_evals_per_s": len(specs) * nG / t_seq,
        "projected_full_grid_s": len(specs) * nO * nG / rate,
        "maps_saved": args.uneven_out or None,
        "oracle_check": oracle_check,
        "batch_launch": {"items": info["n_items"], "ctas": info["grid"],
                         "schedule": ["persistent round robin", "one CTA (pair) per item",
                                      "one launch per model"][info["schedule"]],
                         "schedule_pass_ms": info["schedule_ms"],
                         "graph_replay": bool(info["graph"]),
                         "kernels_per_pass": info["launches_per_replay"]},
        # a model whose sizes were tuned before in the process reuses the
        # cached choice without timing it (candidates 0, no times)
        "autotune": [{"splits": t.splits, "default": t.default_splits, "form": t.form,
                      "cached": t.candidates == 0,
                      "ms_per_omega": t.ms_per_omega if t.candidates else None,
                      "default_ms_per_omega": t.default_ms_per_omega if t.candidates else None}
                     for t in tunes],
        "setup_s": t_setup,
        "form": "split-BF16 (FP64 tables released after the split)"}


def ours(args):
    import numpy as np
    import torch
    import kalnajs_log_spirals_b200 as K
    from kalnajs_log_spirals_b200 import _lib
    from kalnajs_log_spirals_b200.api import newton_search_hybrid

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    cfg = K.load_model(K.load_config(args.config), args.model)
    m = cfg.physics.m

    peak64 = dgemm_peak_tflops(torch)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak_bf16 = float(peaks.get("bf16_tflops", 1590.0))
    peak_bf16_note = "of measured (MEASURED_PEAKS.json bf16_tflops, burst)" if "bf16_tflops" in peaks \
        else "of fallback (1.59 PFLOP/s)"

    t0 = time.perf_counter()
    pc = K.api.PrecomputedData(cfg, K.create_toomre_zang_model(cfg), local)
    lib, h = pc.ctx.lib, pc.ctx.h
    _lib.check(h, lib.kls_enable_timing(h, 1))
    pc.ctx.call("kls_precompute")
    _lib.check(h, lib.kls_enable_timing(h, 0))
    torch.cuda.synchronize()
    t_pre = time.perf_counter() - t0
    pre_ms = (C.c_float * 2)()
    _lib.check(h, lib.kls_get_precompute_ms(h, pre_ms))
    dims = pc.ctx.dims
    # a dedicated stream: the library launches on it and the events are
    # recorded on it (the legacy default stream has handle 0, which the
    # C ABI reads as "the context's own stream")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    _lib.check(h, lib.kls_set_stream(h, C.c_void_p(stream.cuda_stream)))

    nb = 3
    flops_per_det = 8.0 * dims.N_alpha ** 2 * dims.K
    # tensor flops of the 3-product split GEMM per determinant (unpadded)
    mixed_flops_per_det = 3 * 2.0 * (2 * dims.N_alpha) ** 2 * dims.K
    d_det = torch.empty((nb, 2), dtype=torch.float64, device="cuda")
    d_la = torch.empty((nb,), dtype=torch.float64, device="cuda")
    n_steps = args.warmup + args.steps
    all_om = np.array([[[w.real, w.imag] for w in omegas_for_step(
        s, rank, m, cfg.reference.Omega_p, cfg.reference.gamma, cfg.newton.delta)]
        for s in range(n_steps)])
    d_all = torch.tensor(all_om, dtype=torch.float64, device="cuda")

    def dev_step(s, mode):
        _lib.check(h, lib.kls_det_batch_device(h, C.c_void_p(d_all[s % n_steps].data_ptr()), nb,
                                               mode, C.c_void_p(d_det.data_ptr()),
                                               C.c_void_p(d_la.data_ptr())))

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def time_device(mode, sample_clocks=False):
        for s in range(args.warmup):
            dev_step(s, mode)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local) if sample_clocks else None
        l0 = lib.kls_launch_count(h)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for s in range(args.warmup, n_steps):
            dev_step(s, mode)
        ev1.record(stream)
        torch.cuda.synchronize()
        launches = lib.kls_launch_count(h) - l0
        clk = clocks.stop() if clocks else None
        barrier()
        return max_over_ranks(ev0.elapsed_time(ev1)), launches, clk

    def stage_times(mode):
        _lib.check(h, lib.kls_enable_timing(h, 1))
        stage = np.zeros(4)
        reps = max(1, min(args.steps, 4))
        for s in range(reps):
            dev_step(args.warmup + s, mode)
            torch.cuda.synchronize()
            buf = (C.c_float * 4)()
            _lib.check(h, lib.kls_get_stage_ms(h, buf))
            stage += np.array(buf[:])
        _lib.check(h, lib.kls_enable_timing(h, 0))
        return stage / reps

    # K split counts chosen by the library's autotuner at this batch size
    tunes = {"fp64": K.autotune(pc, "Float64", batch=nb)}

    # ---- plain FP64: device-resident timing (headline) ----------------------
    ms, launches, clk = time_device(_lib.KLS_MODE_FP64, sample_clocks=True)
    ms_per_step = ms / args.steps
    value = world * nb * args.steps / (ms * 1e-3)
    stage = stage_times(_lib.KLS_MODE_FP64)
    achieved = nb * flops_per_det / (stage[1] * 1e-3) / 1e12
    # real DMMA flops the kernel issues (padded tiles): 4 or 3 real products
    f64_3m = tunes["fp64"].form == _lib.KLS_F64_3M
    issued_per_det = (6.0 if f64_3m else 8.0) * dims.N_alpha_pad ** 2 * dims.K_pad
    issued = nb * issued_per_det / (stage[1] * 1e-3) / 1e12

    # ---- end to end through the C ABI with host buffers -----------------------
    h_om = np.ascontiguousarray(all_om)
    det_h = np.empty((nb, 2))
    la_h = np.empty(nb)
    for s in range(args.warmup):
        _lib.check(h, lib.kls_det_batch(h, _lib.dptr(h_om[s]), nb, _lib.KLS_MODE_FP64,
                                        _lib.dptr(det_h), _lib.dptr(la_h)))
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in range(args.warmup, n_steps):
        _lib.check(h, lib.kls_det_batch(h, _lib.dptr(h_om[s]), nb, _lib.KLS_MODE_FP64,
                                        _lib.dptr(det_h), _lib.dptr(la_h)))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e = world * nb * args.steps / (e2e_ms * 1e-3)

    # ---- mixed form: split-BF16 tensor-core contraction ------------------------
    mixed = None
    if not args.no_mixed:
        t0 = time.perf_counter()
        _lib.check(h, lib.kls_prepare_mixed(h))
        t_split = time.perf_counter() - t0
        tunes["mixed"] = K.autotune(pc, "Float32", batch=nb)
        mixed_kernel = {_lib.KLS_MIXED_TMEM: "mixed_tm_kernel",
                        _lib.KLS_MIXED_PAIR: "mixed_pair_kernel"}.get(tunes["mixed"].form,
                                                                    "mixed_contract_kernel")
        ms_mx, launches_mx, _ = time_device(_lib.KLS_MODE_MIXED)
        stage_mx = stage_times(_lib.KLS_MODE_MIXED)
        ach_mx = nb * mixed_flops_per_det / (stage_mx[1] * 1e-3) / 1e12
        # accuracy against the plain FP64 form on 200 seeded omegas:
        # Omega_p ~ U[0.3, 0.6], gamma ~ U[0.02, 0.25], omega = m Omega_p + i gamma
        rng = np.random.default_rng(0)
        om = m * rng.uniform(0.3, 0.6, args.accuracy_points) + \
            1j * rng.uniform(0.02, 0.25, args.accuracy_points)
        d64 = K.compute_determinant_batched(om, pc, None, batch_size=16)
        dmx = np.empty_like(d64)
        _lib.check(h, lib.kls_det_batch(h, _lib.dptr(om.view(np.float64)), len(om),
                                        _lib.KLS_MODE_MIXED, _lib.dptr(dmx.view(np.float64)),
                                        C.cast(None, C.POINTER(C.c_double))))
        rel = np.abs(dmx - d64) / np.abs(d64)
        # accumulation chunk of the TMEM-operand form: time and accuracy
        chunk_sweep = []
        if tunes["mixed"].form == _lib.KLS_MIXED_TMEM:
            for ch in (32, 64, 128, 256):
                _lib.check(h, lib.kls_set_mixed_chunk(h, ch))
                ms_c, _, _ = time_device(_lib.KLS_MODE_MIXED)
                dc = np.empty_like(d64[:40])
                _lib.check(h, lib.kls_det_batch(h, _lib.dptr(om[:40].view(np.float64)), 40,
                                                _lib.KLS_MODE_MIXED, _lib.dptr(dc.view(np.float64)),
                                                C.cast(None, C.POINTER(C.c_double))))
                rc = np.abs(dc - d64[:40]) / np.abs(d64[:40])
                chunk_sweep.append({"k_blocks": ch, "ms_per_step": ms_c / args.steps,
                                    "rel_det_err_median": float(np.median(rc)),
                                    "rel_det_err_max": float(rc.max())})
            _lib.check(h, lib.kls_set_mixed_chunk(h, 128))
        mixed = {"det_evals_per_s": world * nb * args.steps / (ms_mx * 1e-3),
                 "ms_per_step": ms_mx / args.steps, "gpu_launches": int(launches_mx),
                 "split_table_s": t_split,
                 "roofline": {"bound": "tensor", "kernel": mixed_kernel + " (tcgen05 kind::f16, TMEM)",
                              "achieved": ach_mx, "peak": peak_bf16, "unit": "TFLOP/s",
                              "frac": ach_mx / peak_bf16, "peak_note": peak_bf16_note,
                              "algorithmic_flops_per_launch": nb * mixed_flops_per_det,
                              "traffic": read_traffic(mixed_kernel)[0],
                              "traffic_scaled": read_traffic(mixed_kernel)[1],
                              "stage_ms": {"weights": stage_mx[0], "contract": stage_mx[1],
                                           "reduce": stage_mx[2], "lu": stage_mx[3]}},
                 "chunk_sweep": chunk_sweep,
                 "rel_det_err_vs_fp64": {"points": int(len(om)), "seed": 0,
                                         "median": float(np.median(rel)),
                                         "p90": float(np.quantile(rel, 0.9)),
                                         "max": float(rel.max())}}

    # ---- Newton time-to-root from the reference start -------------------------
    newton = None
    if not args.no_newton:
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = K.newton_search(cfg, pc, None, K.GPUType.NVIDIA, "Float64")
        t_plain = time.perf_counter() - t0
        newton = {"plain_fp64": {"time_to_root_s": t_plain, "Omega_p": r.Omega_p, "gamma": r.gamma,
                                 "abs_det": abs(r.det_val), "iterations": r.iterations,
                                 "det_evals": r.det_evals, "converged": r.converged},
                  "tol": cfg.newton.tol}
        if not args.no_mixed:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rh = newton_search_hybrid(cfg, pc)
            t_h = time.perf_counter() - t0
            d64_h = K.compute_determinant(rh.omega, pc, None)     # outside the timed region
            newton["mixed_fp64_finish"] = {
                "time_to_root_s": t_h, "Omega_p": rh.Omega_p, "gamma": rh.gamma,
                "abs_det": abs(rh.det_val), "abs_det_plain_fp64_at_result": abs(d64_h),
                "converged": rh.converged,
                "mixed_evals": rh.mixed_evals, "fp64_evals": rh.fp64_evals,
                "anchored_evals": rh.anchored_evals,
                "history": [[float(x) for x in row] for row in rh.history],
                "abs_dOmega_p_vs_plain": abs(rh.Omega_p - r.Omega_p),
                "abs_dgamma_vs_plain": abs(rh.gamma - r.gamma)}
            newton["speedup_hybrid_vs_plain"] = t_plain / t_h
            # conditioning at the FP64 root: |det'| (complex derivative,
            # forward difference) and the split form's residual there, whose
            # ratio is the split form's own root error
            w_r = complex(m * r.Omega_p, r.gamma)
            d_pair = K.compute_determinant_batched(np.array([w_r, w_r + 1e-7]), pc, None)
            dprime = abs((d_pair[1] - d_pair[0]) / 1e-7)
            d_mx = K.compute_determinant(w_r, pc, K.to_device(pc, K.GPUType.NVIDIA, "Float32"))
            # anchored form 1e-6 and 1e-5 from the root: M error against the
            # FP64 M there, and its determinant residual at the root
            M64 = K.build_M_matrix(w_r, pc, None)
            dev_an = K.api.DevicePrecomputed(pc.m, pc.G, pc.N_alpha, pc.n_l, pc.NPh,
                                             K.KLS_MODE_ANCHORED, pc)
            anch = {}
            for dist in (1e-6, 1e-5):
                K.set_anchor(pc, w_r + dist * np.exp(0.7j))
                Man = K.build_M_matrix(w_r, pc, dev_an)
                d_an = K.compute_determinant(w_r, pc, dev_an)
                anch[f"{dist:.0e}"] = {
                    "M_err_over_max": float(np.abs(Man - M64).max() / np.abs(M64).max()),
                    "abs_det_at_fp64_root": abs(d_an),
                    "root_error_estimate": abs(d_an) / dprime}
            newton["at_fp64_root"] = {"abs_det_prime": dprime, "abs_mixed_det": abs(d_mx),
                                      "mixed_root_error_estimate": abs(d_mx) / dprime,
                                      "anchored_at_distance": anch}

    # ---- parity against the oracle's default-size fixture ----------------------
    parity = None
    if rank == 0:
        parity = oracle_parity(K, cfg, pc, newton, not args.no_mixed)

    # ---- CPU baseline: the oracle's BLAS-form determinant on the host cores ---
    cpu = None
    if rank == 0 and not args.no_cpu:
        w0 = complex(*all_om[args.warmup][0])
        rate, d_cpu, sample = cpu_det_baseline(pc, cfg, w0)
        d_gpu = K.compute_determinant(w0, pc)
        cpu = {"value": rate, "unit": UNIT, "cores": blas_threads(), "kind": "port",
               "sample": sample, "host_cores": os.cpu_count(),
               "det_rel_diff_vs_gpu_fp64": abs(d_cpu - d_gpu) / abs(d_gpu)}
        if world == 1:
            try:
                cpu["small_size"] = cpu_small_size(args, K, local)
            except Exception as e:             # a secondary figure never fails the run
                cpu["small_size"] = {"unavailable": f"{type(e).__name__}: {e}"}

    refgpu = None
    if world == 1 and not args.no_refgpu:
        refgpu = reference_algorithm_gpu(torch, K, pc, cfg)
    # the two workflow blocks run at N = 1 only (the scaling run times the
    # headline step alone)
    ttr = None
    if world == 1 and not args.no_proposer and not args.no_mixed:
        from kalnajs_log_spirals_b200 import proposer as P
        ttr = time_to_root(args, K, P, cfg, pc, local, torch.cuda.synchronize)
    pc.close()
    if ttr is not None and args.heldout > 0:
        # after the benchmark's own context is released (memory for the scans)
        n_grid = cfg.scan.n_Op * cfg.scan.n_gamma
        ttr["heldout"] = heldout_eval(args, K, P, cfg, args.heldout,
                                      ttr["plain_fp64"]["scan_s"] / n_grid, local,
                                      torch.cuda.synchronize)
    uneven = None
    if world == 1 and not args.no_uneven:
        from kalnajs_log_spirals_b200 import proposer as P
        uneven = uneven_batch(args, K, P, local, torch.cuda.synchronize)

    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return 0
    traffic, traffic_scaled = read_traffic("contract3m_kernel" if f64_3m else "contract_kernel")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (no dataset: the workload is the model's own grids)",
        "config": {"workload": workload(cfg), "step": "one Newton finite-difference triple "
                   "(omega, omega + m delta, omega + i delta) in one batch",
                   "NR": cfg.grid.NR, "Ne": cfg.grid.Ne,
                   "N_alpha": cfg.grid.N_alpha, "l": [cfg.grid.l_min, cfg.grid.l_max],
                   "K": dims.K, "omegas_per_step": nb, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (W table %.1f GB in HBM)" % (
                       2 * 8 * dims.K_pad * dims.N_alpha_pad / 1e9)},
        "roofline": {"bound": "tensor",
                     "kernel": ("contract3m_kernel (FP64 DMMA m8n8k4, 3 real products per "
                                "complex one)" if f64_3m else
                                "contract_kernel (FP64 DMMA m8n8k4, 4 real products)"),
                     "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                     "frac": achieved / peak64,
                     "peak_note": "of measured: cuBLAS DGEMM 8192^3 best-of-5 in this run",
                     "algorithmic_flops_per_launch": nb * flops_per_det,
                     "algorithmic_note": "8 N_alpha^2 K per determinant (a complex MAC as 4 "
                                         "real ones); the 3M form issues 3, so its frac can "
                                         "exceed the DMMA pipe's",
                     "dmma_issued_tflops": issued, "dmma_issued_frac": issued / peak64,
                     "traffic": traffic, "traffic_scaled": traffic_scaled, "stage_ms": {"weights": stage[0], "contract": stage[1],
                                                      "reduce": stage[2], "lu": stage[3]}},
        "cpu_baseline": cpu,
        "parity_vs_oracle": parity,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": nb * 16,
                "d2h_bytes_per_step": nb * 24},
        "gpu_launches": int(launches),
        "clocks": clk,
        "autotune": {k: {"splits": t.splits, "default_splits": t.default_splits,
                         "form": ({0: "FP64 4M", 1: "FP64 3M"} if k == "fp64" else
                                  {1: "one CTA", 2: "CTA pair",
                                   3: "TMEM-operand CTA pair"}).get(t.form, t.form),
                         "candidates": t.candidates, "ms_per_omega": t.ms_per_omega,
                         "default_ms_per_omega": t.default_ms_per_omega}
                     for k, t in tunes.items()},
        "precompute_s": t_pre,
        "precompute": precompute_roofline(cfg, dims, pre_ms, peak64, peaks),
        "mixed": mixed,
        "newton": newton,
        "reference_algorithm_gpu": refgpu,
        "time_to_root": ttr,
        "uneven_batch": uneven,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
