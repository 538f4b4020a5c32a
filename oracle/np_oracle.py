"""CPU oracle for the Kalnajs log-spiral matrix-method path (TEST INFRASTRUCTURE).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` import it.  The library in ``kalnajs_log_spirals_b200``
never calls it and has no CPU fallback.

It restates, in plain FP64 NumPy, the reference's Julia package
``src/KalnajsLogSpiral`` (file:line cited per function):

* Models.jl:40-169            -> ToomreZang, taper, df, df_E, df_L
* OrbitIntegration.jl:63-95   -> trapezoid_coef, simpson_coef
* OrbitIntegration.jl:102-170 -> compute_grids
* OrbitIntegration.jl:181-336 -> compute_orbits (three branches, endpoint
  extrapolation, subsampling, NaN->0 of the DF)
* OrbitIntegration.jl:341-382 -> compute_jacobian
* BasisFunctions.jl:73-165    -> precompute_all (DJ, F0l, Omega_res)
* BasisFunctions.jl:199-266   -> compute_W_l (skip of non-finite orbits,
  zeroing of non-finite integrands)
* BasisFunctions.jl:281-304   -> compute_N_kernel
* MatrixBuilder.jl:27-87      -> build_M / compute_det (denominator clamp,
  G and N scaling, det(I - M))
* GridScan.jl:25-88,234-246   -> grid_scan, find_minimum
* NewtonSolver.jl:36-172      -> newton_search

Third-party arithmetic the reference relies on and which is restated here by
library calls rather than copied: the complex Gamma function used for
N_m(alpha) (the package's Lanczos routine, BasisFunctions.jl:309-366, and
``SpecialFunctions.gamma`` in NL_julia_direct.jl:284-286) is evaluated with
``scipy.special.loggamma``; ``LinearAlgebra.det`` (LAPACK zgetrf) is
``numpy.linalg.det`` / ``slogdet`` (OpenBLAS/LAPACK zgetrf as shipped with
NumPy).

Parity pin: the end-to-end roots printed by the reference's MATLAB original
(``convergence_table.txt:13-14``) for ``configs/small.toml`` are reproduced by
this oracle (tests/test_oracle_golden.py).

The W_l quadrature is evaluated per orbit as the matrix product
C[l,k] @ E[k,alpha] with C = Sw1_k cos(l w1_k + m phi_k) and
E = exp(-i alpha ln r_k) / sqrt(r_k); this is the same sum as the reference's
``sum(Sw1 .* integrand) / pi`` in a different association order.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Optional, Sequence

import numpy as np
import scipy.special as sps


# --------------------------------------------------------------------------
# configuration (plain dataclass, fields named after Configuration.jl)
# --------------------------------------------------------------------------
@dataclasses.dataclass
class OracleConfig:
    m: int = 2
    G: float = 1.0
    L0: float = 1.0
    n_zang: int = 4
    q1: float = 7.0
    NR: int = 201
    Ne: int = 21
    Rc_min: float = 1e-3
    Rc_max: float = 100.0
    v_min: float = 1e-2
    N_alpha: int = 101
    alpha_max: float = 10.0
    l_min: int = -25
    l_max: int = 25
    nw: int = 10001
    nwa: int = 201
    # quadrature rules of the alpha, ln Rc and v grids, one of t / s / b each
    # (NL_julia_boole.jl:14-16, 221-249); "tts" is the package's choice
    quad: str = "tts"

    @property
    def n_l(self) -> int:
        return self.l_max - self.l_min + 1

    @property
    def NPh(self) -> int:
        return self.NR * self.Ne


# ln x along the orbit integrals; the fixture generator swaps in a perturbed
# version to measure how sensitive the reference algorithm is to last-ulp
# differences between math libraries
orbit_log: Callable[[np.ndarray], np.ndarray] = np.log


def _ln(x):
    """ln of the potential V = ln r along grids, orbits and Jacobian."""
    return orbit_log(x)


def linspace(a: float, b: float, n: int) -> np.ndarray:
    """``range(a, b, length=n)``: a + i*step with the last point exactly b."""
    return np.linspace(a, b, n)


# --------------------------------------------------------------------------
# Models.jl:24-169
# --------------------------------------------------------------------------
@dataclasses.dataclass
class ToomreZang:
    L0: float
    n_zang: int
    q1: float
    q_zang: float
    sigma_r0: float
    G: float
    DF_const: float

    @staticmethod
    def from_config(c: OracleConfig) -> "ToomreZang":
        # Models.jl:40-57; q1 generalised to real values (Gamma of a real)
        q1 = float(c.q1)
        sigma_r0 = 1.0 / math.sqrt(q1)
        q = q1 - 1.0
        DF_const = 1.0 / (2.0 * math.pi * 2.0 ** (q / 2.0) * math.sqrt(math.pi)
                          * math.gamma((q + 1.0) / 2.0) * sigma_r0 ** (q + 2.0))
        return ToomreZang(float(c.L0), int(c.n_zang), q1, q, sigma_r0, float(c.G), DF_const)

    # potential V = ln r and derivatives (Models.jl:64-76)
    @staticmethod
    def V(r):
        return np.log(r)

    @staticmethod
    def dV(r):
        return 1.0 / r

    @staticmethod
    def Omega(r):
        return 1.0 / r

    @staticmethod
    def kappa(r):
        return math.sqrt(2.0) / r

    def taper(self, L: float) -> float:
        # Models.jl:91-102
        if self.n_zang == 0:
            return 1.0
        La = abs(L)
        if La < 1e-12:
            return 0.0
        return 1.0 / (1.0 + (self.L0 / La) ** self.n_zang)

    def df(self, E: float, L: float) -> float:
        # Models.jl:137-150
        La = abs(L)
        if La < 1e-12:
            return 0.0
        with np.errstate(all="ignore"):
            r = self.DF_const * math.exp(-E / self.sigma_r0 ** 2) * La ** self.q_zang * self.taper(L)
        return r if math.isfinite(r) else 0.0

    def df_E(self, E: float, L: float) -> float:
        # Models.jl:153-155
        return -self.df(E, L) / self.sigma_r0 ** 2

    def df_L(self, E: float, L: float) -> float:
        # Models.jl:158-169
        La = abs(L)
        if La < 1e-12:
            return 0.0
        f0 = self.df(E, L)
        t = self.taper(L)
        return f0 * (self.q_zang + self.n_zang - self.n_zang * t) / La


# --------------------------------------------------------------------------
# quadrature weights: OrbitIntegration.jl:63-95, BasisFunctions.jl:174-188
# --------------------------------------------------------------------------
def trapezoid_coef(x: np.ndarray) -> np.ndarray:
    n = len(x)
    S = np.zeros(n)
    if n >= 2:
        S[0] = (x[1] - x[0]) / 2
        S[-1] = (x[-1] - x[-2]) / 2
        S[1:-1] = (x[2:] - x[:-2]) / 2
    return S


def simpson_coef(x: np.ndarray) -> np.ndarray:
    n = len(x)
    if n < 3 or n % 2 == 0:
        return trapezoid_coef(x)
    dx = x[1] - x[0]
    S = np.zeros(n)
    S[0] = dx / 3
    S[-1] = dx / 3
    S[1:-1:2] = 4 * dx / 3   # Julia indices 2:2:n-1
    S[2:-1:2] = 2 * dx / 3   # Julia indices 3:2:n-2
    return S


def boole_coef(x: np.ndarray) -> np.ndarray:
    """Composite Boole weights 2h/45 (7, 32, 12, 32, 14, ..., 7) for n = 4k + 1
    points, else the Simpson rule (NL_julia_boole.jl:186-217; n < 5 also
    falls back, where the script has no defined result)."""
    n = len(x)
    if n < 5 or (n - 1) % 4 != 0:
        return simpson_coef(x)
    dx = x[1] - x[0]
    f = 2 * dx / 45
    S = np.empty(n)
    for i in range(n):
        r = i % 4
        S[i] = 14 * f if r == 0 else (12 * f if r == 2 else 32 * f)
    S[0] = 7 * f
    S[-1] = 7 * f
    return S


def quad_coef(x: np.ndarray, rule: str) -> np.ndarray:
    """GetCoefs (NL_julia_boole.jl:221-232): t trapezoid, s Simpson, b Boole."""
    return {"t": trapezoid_coef, "s": simpson_coef, "b": boole_coef}[rule](x)


# --------------------------------------------------------------------------
# OrbitIntegration.jl:102-170
# --------------------------------------------------------------------------
@dataclasses.dataclass
class Grids:
    Rc: np.ndarray
    e: np.ndarray
    v: np.ndarray
    R1: np.ndarray
    R2: np.ndarray
    E: np.ndarray
    L_m: np.ndarray
    L2_m: np.ndarray
    SGNL: np.ndarray
    S_RC: np.ndarray
    S_e: np.ndarray


def compute_grids(c: OracleConfig, model: ToomreZang) -> Grids:
    NR, Ne = c.NR, c.Ne
    # the C library's pow and log (the device uses the same host-computed grid)
    Rc_1d = np.array([10.0 ** float(x) for x in linspace(math.log10(c.Rc_min),
                                                          math.log10(c.Rc_max), NR)])
    uRc = np.array([math.log(x) for x in Rc_1d])
    S_RC = Rc_1d * quad_coef(uRc, c.quad[1])
    v_arr = linspace(c.v_min, 1.0, Ne)
    S_e = np.tile(quad_coef(v_arr, c.quad[2]), (NR, 1))
    v = np.tile(v_arr, (NR, 1))
    Rc = np.tile(Rc_1d[:, None], (1, Ne))
    v = np.where(np.abs(v) < 1e-14, 1e-12, v)
    SGNL = np.sign(v)
    e = 1.0 - np.abs(v)
    R1 = Rc * (1.0 - e)
    R2 = Rc * (1.0 + e)
    E = np.zeros((NR, Ne))
    for iR in range(NR):
        for ie in range(Ne):
            r1, r2 = R1[iR, ie], R2[iR, ie]
            V1, V2 = _ln(r1), _ln(r2)
            if abs(r2 ** 2 - r1 ** 2) > 1e-14:
                E[iR, ie] = (V2 * r2 ** 2 - V1 * r1 ** 2) / (r2 ** 2 - r1 ** 2)
            else:
                r = Rc[iR, ie]
                E[iR, ie] = r * (1.0 / r) / 2 + _ln(r)
            if not math.isfinite(E[iR, ie]):
                E[iR, ie] = _ln(R2[iR, ie])
    L2_m = 2.0 * (E - _ln(R2)) * R2 ** 2
    L2_m[L2_m < 1e-14] = 0.0
    L_m = np.sqrt(L2_m) * SGNL
    return Grids(Rc, e, v, R1, R2, E, L_m, L2_m, SGNL, S_RC, S_e)


# --------------------------------------------------------------------------
# OrbitIntegration.jl:181-336 and :341-382
# --------------------------------------------------------------------------
@dataclasses.dataclass
class Orbits:
    grids: Grids
    Omega_1: np.ndarray    # [NR, Ne]
    Omega_2: np.ndarray    # [NR, Ne]
    w1: np.ndarray         # [NR, Ne, nwa]  (orbit-major; the reference stores [nwa, NR, Ne])
    ra: np.ndarray
    pha: np.ndarray
    jacobian: np.ndarray
    F0: np.ndarray
    FE: np.ndarray
    FL: np.ndarray


def orbit_grid(c: OracleConfig):
    """The w grid of the orbit integrals and its subsampling
    (OrbitIntegration.jl:188-197): (w, dw, cos w, sin w, Ia, w[Ia])."""
    eps_w = 1e-8
    w = linspace(eps_w, math.pi - eps_w, c.nw)
    dw = w[1] - w[0]
    nwai = (c.nw - 1) // (c.nwa - 1)
    Ia = np.arange(0, c.nw, nwai)
    return w, dw, np.cos(w), np.sin(w), Ia, w[Ia]


def orbit_samples(g: Grids, iR: int, ie: int, wg):
    """One orbit (OrbitIntegration.jl:222-302): Omega_1, Omega_2 and the
    subsampled w1, r, theta along it (three branches, endpoint extrapolation)."""
    w, dw, cosw, sinw, Ia, wa = wg
    nw = len(w)
    R_i = g.Rc[iR, 0]
    kap = math.sqrt(2.0) / R_i
    Om = 1.0 / R_i
    E_i = g.E[iR, ie]
    L_j = g.L_m[iR, ie]
    L2_j = g.L2_m[iR, ie]
    ecc = g.e[iR, ie]
    r1, r2 = g.R1[iR, ie], g.R2[iR, ie]
    sg = g.SGNL[iR, ie]
    if abs(ecc) < 1e-10:                    # :222-229
        om1, om2 = kap, Om * sg
        return om1, om2, wa.copy(), np.full(len(Ia), R_i), wa * om2 / om1
    if ecc < 0.01:                          # :232-241
        a_j = (r2 - r1) / 2
        om1, om2 = kap, Om * sg
        return (om1, om2, wa.copy(), R_i - a_j * cosw[Ia],
                wa * om2 / om1 + 2 * Om / kap * a_j / R_i * sinw[Ia] * sg)
    rs = (r1 + r2) / 2                      # :244-302
    drs = (r2 - r1) / 2
    xs = rs - drs * cosw
    if L2_j > 1e-12:
        vr_sq = 2.0 * (E_i - _ln(xs)) * xs ** 2 - L2_j
        rvr = np.sqrt(np.maximum(0.0, vr_sq))
        svr = sinw * xs / rvr
        svr[0] = 2.0 * svr[1] - svr[2]
        svr[-1] = 2.0 * svr[-2] - svr[-3]
    else:
        vr_sq = 2.0 * (E_i - _ln(xs))
        rvr = np.sqrt(np.maximum(0.0, vr_sq))
        svr = sinw / rvr
        svr[-1] = 2.0 * svr[-2] - svr[-3]
    dt1 = drs * dw * svr
    dt2 = np.zeros(nw)
    dt2[1:] = (dt1[:-1] + dt1[1:]) / 2
    t = np.cumsum(dt2)
    om1 = math.pi / t[-1]
    w1 = t[Ia] * om1
    ra = xs[Ia]
    if abs(1.0 - ecc) > 1e-10 and L2_j > 1e-12:
        sp = sinw / rvr
        sp[0] = 2.0 * sp[1] - sp[2]
        sp[-1] = 2.0 * sp[-2] - sp[-3]
        dt3 = drs * dw * sp / xs
        dt4 = np.zeros(nw)
        dt4[1:] = (dt3[:-1] + dt3[1:]) / 2
        ph = L_j * np.cumsum(dt4)[Ia]
    else:
        ph = math.pi / 2 * np.ones(len(Ia)) * sg
        ph[0] = 0.0
    om2 = om1 * ph[-1] / math.pi
    return om1, om2, w1, ra, ph


def df_fields(model: ToomreZang, g: Grids):
    """F0, FE, FL on the grid with non-finite values set to 0
    (OrbitIntegration.jl:315-333)."""
    NR, Ne = g.E.shape
    F0 = np.zeros((NR, Ne))
    FE = np.zeros((NR, Ne))
    FL = np.zeros((NR, Ne))
    for iR in range(NR):
        for ie in range(Ne):
            E, L = g.E[iR, ie], g.L_m[iR, ie]
            F0[iR, ie] = model.df(E, L)
            FE[iR, ie] = model.df_E(E, L)
            FL[iR, ie] = model.df_L(E, L)
    for a in (F0, FE, FL):
        a[~np.isfinite(a)] = 0.0
    return F0, FE, FL


def compute_orbits(c: OracleConfig, model: ToomreZang, g: Grids) -> Orbits:
    NR, Ne = c.NR, c.Ne
    wg = orbit_grid(c)
    na = len(wg[4])
    Om1 = np.zeros((NR, Ne))
    Om2 = np.zeros((NR, Ne))
    w1 = np.full((NR, Ne, na), np.nan)
    ra = np.full((NR, Ne, na), np.nan)
    pha = np.full((NR, Ne, na), np.nan)
    with np.errstate(all="ignore"):
        for iR in range(NR):
            for ie in range(Ne):
                Om1[iR, ie], Om2[iR, ie], w1[iR, ie], ra[iR, ie], pha[iR, ie] = \
                    orbit_samples(g, iR, ie, wg)
    jac = compute_jacobian(g, Om1)
    F0, FE, FL = df_fields(model, g)
    return Orbits(g, Om1, Om2, w1, ra, pha, jac, F0, FE, FL)


def compute_jacobian(g: Grids, Om1: np.ndarray) -> np.ndarray:
    NR, Ne = Om1.shape
    jac = np.zeros((NR, Ne))
    for iR in range(NR):
        for ie in range(Ne):
            r1, r2, rc = g.R1[iR, ie], g.R2[iR, ie], g.Rc[iR, ie]
            E_val, L_val, om1 = g.E[iR, ie], g.L_m[iR, ie], Om1[iR, ie]
            j = 0.0
            if abs(r2 - r1) > 1e-12 and abs(L_val) > 1e-12:
                V1, V2 = _ln(r1), _ln(r2)
                dV1, dV2 = 1.0 / r1, 1.0 / r2
                t1 = 2 * (E_val - V1) * r1 - dV1 * r1 ** 2
                t2 = 2 * (E_val - V2) * r2 - dV2 * r2 ** 2
                den = r2 ** 2 - r1 ** 2
                j = 2 * abs(t1 * t2 / den) * rc / om1 / abs(L_val)
            if abs(L_val) <= 1e-12:
                DelE = 2.0 * (E_val - _ln(r1))
                with np.errstate(all="ignore"):
                    j = math.sqrt(max(DelE, 0.0)) * (1.0 / r2) * 2 * rc / om1 if om1 != 0 else math.inf
                if not math.isfinite(j):
                    j = 0.0
            jac[iR, ie] = j
    return jac


# --------------------------------------------------------------------------
# BasisFunctions.jl:199-304
# --------------------------------------------------------------------------
def w_orbit(m: int, om1: float, om2: float, w1v, rv, thv, alpha, l_arr):
    """W_l(alpha) of one orbit, [n_l, N_alpha] (BasisFunctions.jl:217-252), or
    None for an orbit with non-finite samples (skipped, i.e. zero)."""
    if not (np.all(np.isfinite(rv)) and np.all(np.isfinite(thv)) and np.all(np.isfinite(w1v))):
        return None
    Sw1 = trapezoid_coef(w1v)
    ratio = om2 / om1
    phi = ratio * w1v - thv
    C = Sw1[None, :] * np.cos(l_arr[:, None] * w1v[None, :] + m * phi[None, :])
    C[~np.isfinite(C)] = 0.0
    E = np.exp(-1j * alpha[None, :] * np.log(rv)[:, None]) / np.sqrt(rv)[:, None]
    E[~np.isfinite(E)] = 0.0
    return (C @ E) / math.pi


def compute_W_l(c: OracleConfig, o: Orbits, alpha: np.ndarray, l_arr: np.ndarray) -> np.ndarray:
    """W[p, a, il] complex128 (p = iR + NR*ie, i.e. column-major orbit index)."""
    NR, Ne, m = c.NR, c.Ne, c.m
    W = np.zeros((NR, Ne, len(alpha), len(l_arr)), dtype=np.complex128)
    with np.errstate(all="ignore"):
        for iR in range(NR):
            for ie in range(Ne):
                blk = w_orbit(m, o.Omega_1[iR, ie], o.Omega_2[iR, ie], o.w1[iR, ie], o.ra[iR, ie],
                              o.pha[iR, ie], alpha, l_arr)
                if blk is not None:
                    W[iR, ie] = blk.T
    return W.reshape(NR * Ne, len(alpha), len(l_arr), order="F")


def compute_N_kernel(m: int, alpha: np.ndarray, d_alpha: np.ndarray) -> np.ndarray:
    ia = 1j * alpha
    z1 = (m + 0.5 + ia) / 2
    z2 = (m + 0.5 - ia) / 2
    z3 = (m + 1.5 + ia) / 2
    z4 = (m + 1.5 - ia) / 2
    lr = sps.loggamma(z1) + sps.loggamma(z2) - sps.loggamma(z3) - sps.loggamma(z4)
    return np.real(np.exp(lr)) * math.pi * d_alpha


# --------------------------------------------------------------------------
# BasisFunctions.jl:73-165
# --------------------------------------------------------------------------
@dataclasses.dataclass
class Precomputed:
    cfg: OracleConfig
    m: int
    G: float
    N_alpha: int
    n_l: int
    l_arr: np.ndarray
    NPh: int
    alpha: np.ndarray
    d_alpha: np.ndarray
    orbits: Orbits
    DJ: np.ndarray          # [NPh]
    F0l: np.ndarray         # [NPh, n_l]
    Omega_res: np.ndarray   # [NPh, n_l]
    W: np.ndarray           # [NPh, N_alpha, n_l] complex128
    N_kernel: np.ndarray    # [N_alpha]


def precompute_all(c: OracleConfig, with_W: bool = True) -> Precomputed:
    model = ToomreZang.from_config(c)
    g = compute_grids(c, model)
    o = compute_orbits(c, model, g)
    alpha = linspace(-c.alpha_max, c.alpha_max, c.N_alpha)
    d_alpha = quad_coef(alpha, c.quad[0])
    l_arr = np.arange(c.l_min, c.l_max + 1)
    W = compute_W_l(c, o, alpha, l_arr) if with_W else None
    N = compute_N_kernel(c.m, alpha, d_alpha)
    DJ = (g.S_RC[:, None] * g.S_e * o.jacobian).reshape(-1, order="F")
    Om1 = o.Omega_1.reshape(-1, order="F")
    Om2 = o.Omega_2.reshape(-1, order="F")
    FE = o.FE.reshape(-1, order="F")
    FL = o.FL.reshape(-1, order="F")
    F0l = (l_arr[None, :] * Om1[:, None] + c.m * Om2[:, None]) * FE[:, None] + c.m * FL[:, None]
    Ores = l_arr[None, :] * Om1[:, None] + c.m * Om2[:, None]
    return Precomputed(c, c.m, float(c.G), c.N_alpha, c.n_l, l_arr, c.NPh, alpha, d_alpha,
                       o, DJ, F0l, Ores, W, N)


# --------------------------------------------------------------------------
# MatrixBuilder.jl:27-87
# --------------------------------------------------------------------------
def weights(pc: Precomputed, omega: complex) -> np.ndarray:
    """DJ * F0l / (omega - Omega_res) with the |den| < 1e-12 clamp, [NPh, n_l]."""
    den = omega - pc.Omega_res.astype(np.complex128)
    den = np.where(np.abs(den) < 1e-12, 1e-12 + 1e-12j, den)
    return (pc.DJ[:, None] * pc.F0l) / den


def build_M(pc: Precomputed, omega: complex, l_range: Optional[Sequence[int]] = None) -> np.ndarray:
    """M[beta, alpha] = G N(alpha) sum_l W_l^T diag(w_l) conj(W_l)  (MatrixBuilder.jl:39-67)."""
    wt = weights(pc, omega)
    M = np.zeros((pc.N_alpha, pc.N_alpha), dtype=np.complex128)
    idx = range(pc.n_l) if l_range is None else l_range
    for il in idx:
        Wl = pc.W[:, :, il]
        M += Wl.T @ (wt[:, il][:, None] * np.conj(Wl))
    M *= pc.G
    M *= pc.N_kernel[None, :]
    return M


def compute_det(pc: Precomputed, omega: complex) -> complex:
    M = build_M(pc, omega)
    return complex(np.linalg.det(np.eye(pc.N_alpha) - M))


def build_M_naive(pc: Precomputed, omega: complex) -> np.ndarray:
    """M(omega) by the reference module's own CPU loops (MatrixBuilder.jl:37-67,
    the ``--gpu=CPU`` path of run_kalnajs_gpu.jl): per harmonic the weights
    with the |den| < 1e-12 clamp, then for every (alpha, beta) one elementwise
    product over the orbits, ``sum(W[:, beta] .* weight .* conj.(W[:, alpha]))``,
    and G, N(alpha) at the end.  The same sums as ``build_M`` in another order
    (agreement to rounding); kept as the reference's slow CPU form for timing."""
    M = np.zeros((pc.N_alpha, pc.N_alpha), dtype=np.complex128)
    for il in range(pc.n_l):
        W = pc.W[:, :, il]
        den = omega - pc.Omega_res[:, il].astype(np.complex128)
        den[np.abs(den) < 1e-12] = 1e-12 + 1e-12j
        weight = pc.DJ * pc.F0l[:, il] / den
        for a in range(pc.N_alpha):
            for b in range(pc.N_alpha):
                M[b, a] += np.sum(W[:, b] * weight * np.conj(W[:, a]))
    M *= pc.G
    for a in range(pc.N_alpha):
        M[:, a] *= pc.N_kernel[a]
    return M


def compute_det_naive(pc: Precomputed, omega: complex) -> complex:
    """det(I - M) with M from the naive loops (MatrixBuilder.jl:76-87)."""
    M = build_M_naive(pc, omega)
    return complex(np.linalg.det(np.eye(pc.N_alpha) - M))


# --------------------------------------------------------------------------
# GridScan.jl:25-88, 234-246
# --------------------------------------------------------------------------
def find_minimum(det_grid: np.ndarray, Op_grid: np.ndarray, g_grid: np.ndarray):
    a = np.abs(det_grid)
    idx = int(np.argmin(a.ravel(order="F")))   # first minimum in column-major order
    n_g = det_grid.shape[0]
    i_g, i_Op = idx % n_g, idx // n_g
    return float(Op_grid[i_Op]), float(g_grid[i_g])


def grid_scan(det_fn: Callable[[complex], complex], m: int, n_Op: int, n_gamma: int,
              Op_min: float, Op_max: float, g_min: float, g_max: float):
    Op_grid = linspace(Op_min, Op_max, n_Op)
    g_grid = linspace(g_min, g_max, n_gamma)
    det_grid = np.empty((n_gamma, n_Op), dtype=np.complex128)
    for j, Op in enumerate(Op_grid):
        for i, gm in enumerate(g_grid):
            det_grid[i, j] = det_fn(complex(m * Op, gm))
    Op0, g0 = find_minimum(det_grid, Op_grid, g_grid)
    return det_grid, Op0, g0


# --------------------------------------------------------------------------
# NewtonSolver.jl:19-172
# --------------------------------------------------------------------------
@dataclasses.dataclass
class NewtonResult:
    Omega_p: float
    gamma: float
    omega: complex
    det_val: complex
    iterations: int
    converged: bool
    history: np.ndarray


def newton_search(det_fn: Callable[[complex], complex], m: int, Op0: float, g0: float, *,
                  max_iter: int = 50, tol: float = 1e-10, delta: float = 1e-6,
                  use_line_search: bool = False, max_line_search: int = 10) -> NewtonResult:
    Op, gm = float(Op0), float(g0)
    hist = np.zeros((max_iter + 1, 3))
    converged = False
    it = 0
    for k in range(1, max_iter + 1):
        it = k
        d = det_fn(complex(m * Op, gm))
        F = np.array([d.real, d.imag])
        res = float(np.hypot(F[0], F[1]))
        hist[k - 1] = (Op, gm, abs(d))
        if res < tol:
            converged = True
            break
        dOp = det_fn(complex(m * (Op + delta), gm))
        dg = det_fn(complex(m * Op, gm + delta))
        J = np.array([[(dOp.real - d.real) / delta, (dg.real - d.real) / delta],
                      [(dOp.imag - d.imag) / delta, (dg.imag - d.imag) / delta]])
        dx = -np.linalg.solve(J, F)
        if use_line_search:
            a = 1.0
            for ls in range(1, max_line_search + 1):
                Opn = Op + a * dx[0]
                gn = gm + a * dx[1]
                if gn < 1e-4 or Opn < 0.0 or Opn > 1.0:
                    a *= 0.5
                    continue
                dn = det_fn(complex(m * Opn, gn))
                if abs(complex(dn)) < res:
                    Op, gm = Opn, gn
                    break
                a *= 0.5
                if ls == max_line_search:
                    Op += dx[0]
                    gm += dx[1]
        else:
            Op += dx[0]
            gm += dx[1]
        gm = max(gm, 1e-4)
        Op = min(max(Op, 0.0), 1.0)
    dfin = det_fn(complex(m * Op, gm))
    return NewtonResult(Op, gm, complex(m * Op, gm), dfin, it, converged, hist[:it].copy())
