"""Golden data at the small benchmark size S, from the oracle.

    python tests/golden/make_size_s.py     (about a minute on 8 cores)

Size S: Toomre-Zang n_zang=4, q1=7, m=2; NR=101, Ne=21, N_alpha=101 on
[-30, 30], l in [-25, 25], Rc in [1e-4, 100], v_min=0.01, nw=100001,
nwa=2001.  Stored: the oracle's Newton root from the reference start
(tol 1e-10, delta 1e-6, no line search), M(omega) at that root, det(I - M)
at three omegas, and the change of each when ln x along the orbit integrals
is perturbed by 2 ulps (the conditioning of the reference algorithm).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import np_oracle as O  # noqa: E402

CFG = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=101, Ne=21, Rc_min=1e-4, Rc_max=100.0,
           v_min=0.01, N_alpha=101, alpha_max=30.0, l_min=-25, l_max=25, nw=100001, nwa=2001)
START = (0.4397142267, 0.1230663944)
OMEGAS = [0.88 + 0.12j, 0.87 + 0.14j, 0.9 + 0.1j]


def run():
    pc = O.precompute_all(O.OracleConfig(**CFG))
    r = O.newton_search(lambda w: O.compute_det(pc, w), CFG["m"], *START, tol=1e-10, delta=1e-6)
    M = O.build_M(pc, r.omega)
    dets = np.array([O.compute_det(pc, w) for w in OMEGAS])
    return r, M, dets


def main() -> None:
    r, M, dets = run()
    orig = O.orbit_log
    O.orbit_log = lambda x: orig(x) * (1.0 + 4.440892098500626e-16)
    try:
        rp, Mp, detsp = run()
    finally:
        O.orbit_log = orig
    Mp_at_root = Mp  # M at the perturbed root differs by the root shift; recompute at r.omega
    O.orbit_log = lambda x: orig(x) * (1.0 + 4.440892098500626e-16)
    try:
        pcp = O.precompute_all(O.OracleConfig(**CFG))
        Mp_at_root = O.build_M(pcp, r.omega)
    finally:
        O.orbit_log = orig
    out = dict(root=np.array([r.Omega_p, r.gamma]), iterations=np.array([r.iterations]),
               root_sens=np.abs(np.array([rp.Omega_p - r.Omega_p, rp.gamma - r.gamma])),
               omega_root=np.array([r.omega]), M0=M, sens_M0=np.abs(Mp_at_root - M),
               omegas=np.array(OMEGAS), dets=dets, sens_dets=np.abs(detsp - dets))
    path = os.path.join(HERE, "size_s.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: root {r.Omega_p:.12f} {r.gamma:.12f} ({r.iterations} it), "
          f"root shift under 2-ulp ln {out['root_sens']}, "
          f"max sens_M0/max|M| {out['sens_M0'].max() / np.abs(M).max():.2e}")


if __name__ == "__main__":
    main()
