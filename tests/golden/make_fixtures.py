"""Generate the committed golden fixtures of tests/golden/*.npz from the oracle.

    python tests/golden/make_fixtures.py

Each case is a tiny grid chosen to exercise one branch of the reference's
orbit integration (OrbitIntegration.jl:222-302) and of the DF / Jacobian
guards; every array the path produces is stored, plus M(omega) and
det(I - M(omega)) at fixed omegas.  The oracle itself is pinned to the
reference's published roots by tests/test_oracle_golden.py.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import np_oracle as O  # noqa: E402

BASE = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=8, Ne=5, Rc_min=0.01, Rc_max=10.0,
            v_min=0.01, N_alpha=9, alpha_max=10.0, l_min=-3, l_max=3, nw=201, nwa=21)

CASES = {
    # general orbits + the circular v = 1 column
    "general": dict(),
    # near-circular epicyclic branch (e < 0.01)
    "epicyclic": dict(v_min=0.95, Ne=7),
    # radial orbit (v -> 1e-12, L = 0) and retrograde orbits (v < 0)
    "radial_retro": dict(v_min=-1.0, Ne=9),
    # odd/even quadrature fallbacks, other m, n_zang, real q1
    "variants": dict(m=3, n_zang=2, q1=5.5, Ne=6, NR=7, N_alpha=8, l_min=-2, l_max=4,
                     alpha_max=5.0, nw=301, nwa=31),
    # Boole rule on all three grids (n = 4k + 1), NL_julia_boole.jl --quad=bbb
    "boole": dict(quad="bbb", NR=9, Ne=9, N_alpha=9),
    # Simpson on alpha and ln Rc, Boole falling back to Simpson/trapezoid on v
    "quad_mixed": dict(quad="ssb", NR=9, Ne=8, N_alpha=11),
}

OMEGAS = [0.88 + 0.12j, 0.6 + 0.05j, 1.2 + 0.3j]


def make(name: str, over: dict) -> dict:
    c = O.OracleConfig(**{**BASE, **over})
    pc = O.precompute_all(c)
    o = pc.orbits
    out = {"config": np.array([repr(sorted({**BASE, **over}.items()))])}
    cm = lambda a: np.asarray(a).reshape(-1, order="F")
    for k in ("Omega_1", "Omega_2", "jacobian", "F0", "FE", "FL"):
        out[k] = cm(getattr(o, k))
    g = o.grids
    for k in ("Rc", "e", "E", "L_m", "S_e"):
        out["grid_" + k] = cm(getattr(g, k))
    out["grid_S_RC"] = g.S_RC
    # [NR, Ne, nwa] -> reference layout [nwa, NR, Ne] flattened column-major
    for k in ("w1", "ra", "pha"):
        a = getattr(o, k)
        out[k] = np.transpose(a, (2, 0, 1)).reshape(-1, order="F")
    out["DJ"] = pc.DJ
    out["alpha"] = pc.alpha
    out["d_alpha"] = pc.d_alpha
    out["N_kernel"] = pc.N_kernel
    out["F0l"] = pc.F0l.reshape(-1, order="F")
    out["Omega_res"] = pc.Omega_res.reshape(-1, order="F")
    out["W"] = pc.W
    out["omegas"] = np.array(OMEGAS)
    out["M0"] = O.build_M(pc, OMEGAS[0])
    out["dets"] = np.array([O.compute_det(pc, w) for w in OMEGAS])
    return out


def sensitivity(name: str, over: dict, base: dict) -> dict:
    """|change| of every array when ln x along the orbits is off by 2 ulps.

    The radial-velocity integrand 1/v_r with v_r^2 = 2(E - ln x) x^2 - L^2
    cancels like 1/e^2 near the turning points of near-circular orbits, so
    math libraries that differ in the last bit of ln give visibly different
    Omega_1, Omega_2, w1 and theta.  The GPU tests allow a small multiple of
    this change on top of a fixed FP64 floor.
    """
    orig = O.orbit_log
    O.orbit_log = lambda x: orig(x) * (1.0 + 4.440892098500626e-16)
    try:
        pert = make(name, over)
    finally:
        O.orbit_log = orig
    return {"sens_" + k: np.abs(np.asarray(pert[k]) - np.asarray(v))
            for k, v in base.items() if k not in ("config", "omegas")}


def main(names=None) -> None:
    for name, over in CASES.items():
        if names and name not in names:
            continue
        d = make(name, over)
        d.update(sensitivity(name, over, d))
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **d)
        print(f"wrote {path}: W {d['W'].shape}, dets {d['dets']}")


if __name__ == "__main__":
    main(sys.argv[1:])
