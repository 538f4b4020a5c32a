"""Golden data at the default size D, from the oracle.

    python tests/golden/make_size_d.py     (about 45 minutes on 8 cores, 26 GB RAM)

Size D (configs/default.toml + models/kalnajs_zang4.toml): Toomre-Zang
n_zang=4, q1=7, m=2; NR=501, Ne=51, N_alpha=301 on [-30, 30], l in
[-100, 100], Rc in [1e-4, 100], v_min=0.01, nw=100001, nwa=2001
(K = 5,135,751 orbit x l terms).  The table is built by the oracle's
per-orbit arithmetic in a process pool (oracle/np_oracle_large.py) and the
determinant is the reference's CPU script form, one ZGEMM per harmonic
(NL_julia_direct.jl:299-310).  Stored:

* the oracle's Newton root from the reference start (0.4397142267,
  0.1230663944), tol 1e-12, delta 1e-6, no line search (NewtonSolver.jl:36-172),
  with its iteration history;
* M(omega) at that root;
* det(I - M) at three fixed omegas and at the first 20 of the 200 seeded
  mixed-precision accuracy points (Omega_p ~ U[0.3, 0.6], gamma ~
  U[0.02, 0.25], omega = 2 Omega_p + i gamma, NumPy PCG64 seed 0);
* the change of the root, of M at the root and of every det when ln x along
  the orbit integrals is perturbed by 2 ulps (the conditioning of the
  reference algorithm at this size).
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import np_oracle as O  # noqa: E402
from oracle import np_oracle_large as L  # noqa: E402

CFG = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=501, Ne=51, Rc_min=1e-4, Rc_max=100.0,
           v_min=0.01, N_alpha=301, alpha_max=30.0, l_min=-100, l_max=100, nw=100001, nwa=2001)
START = (0.4397142267, 0.1230663944)
TOL, DELTA = 1e-12, 1e-6
OMEGAS = [0.88 + 0.12j, 0.87 + 0.14j, 0.9 + 0.1j]
N_SEEDED = 20


def seeded_omegas(n_total: int = 200, m: int = 2) -> np.ndarray:
    """The accuracy points of the mixed-precision workload (PCG64 seed 0)."""
    rng = np.random.default_rng(0)
    return m * rng.uniform(0.3, 0.6, n_total) + 1j * rng.uniform(0.02, 0.25, n_total)


def log(msg: str) -> None:
    print(f"[{time.strftime('%H:%M:%S')}] {msg}", flush=True)


def run(perturb: float, omega_root=None):
    t0 = time.time()
    pc = L.precompute_large(O.OracleConfig(**CFG), perturb=perturb)
    log(f"precompute (perturb {perturb:g}): {time.time() - t0:.0f} s")
    try:
        f = lambda w: L.compute_det_large(pc, w)
        t0 = time.time()
        r = O.newton_search(f, CFG["m"], *START, tol=TOL, delta=DELTA)
        log(f"newton: {r.iterations} it, root {r.Omega_p:.13f} {r.gamma:.13f}, "
            f"|det| {abs(r.det_val):.2e}, {time.time() - t0:.0f} s")
        M = L.build_M_large(pc, r.omega if omega_root is None else omega_root)
        om = np.concatenate([np.array(OMEGAS), seeded_omegas()[:N_SEEDED]])
        t0 = time.time()
        dets = np.array([f(w) for w in om])
        log(f"{len(om)} dets: {time.time() - t0:.0f} s")
    finally:
        pc.close()
    return r, M, om, dets


def main() -> None:
    r, M, om, dets = run(0.0)
    out = dict(root=np.array([r.Omega_p, r.gamma]), iterations=np.array([r.iterations]),
               converged=np.array([r.converged]), history=r.history,
               det_root=np.array([r.det_val]), omega_root=np.array([r.omega]), M0=M,
               omegas=om, dets=dets, n_fixed=np.array([len(OMEGAS)]))
    path = os.path.join(HERE, "size_d.npz")
    np.savez_compressed(path, **out)           # usable before the sensitivity run ends
    log(f"wrote {path} (without sensitivities)")
    rp, Mp, _, detsp = run(L.ULP2, omega_root=r.omega)
    out.update(root_sens=np.abs(np.array([rp.Omega_p - r.Omega_p, rp.gamma - r.gamma])),
               sens_M0=np.abs(Mp - M), sens_dets=np.abs(detsp - dets))
    np.savez_compressed(path, **out)
    log(f"wrote {path}: root {r.Omega_p:.13f} {r.gamma:.13f} ({r.iterations} it), "
        f"root shift under 2-ulp ln {out['root_sens']}, "
        f"max sens_M0/max|M| {out['sens_M0'].max() / np.abs(M).max():.2e}, "
        f"max sens_det/|det| {np.max(out['sens_dets'] / np.abs(dets)):.2e}")


if __name__ == "__main__":
    main()
