"""Large-size driver of the CPU oracle (TEST INFRASTRUCTURE).

Only ``tests/`` (fixture generation), and the ``cpu_baseline`` / ``--impl
reference`` legs of ``bench.py`` use this module; the library never calls it.

It evaluates the same per-orbit arithmetic as ``oracle/np_oracle.py``
(``orbit_samples``, ``w_orbit``: OrbitIntegration.jl:222-302,
BasisFunctions.jl:217-252) over orbit ranges in a process pool, so that the
default size (NR=501, Ne=51, N_alpha=301, l in [-100, 100], nw=100001,
nwa=2001: a 24.7 GB complex128 table) can be built on the host cores.  The
table is stored harmonic-major, ``W[il]`` = the reference's ``W_l_mat[:, :,
il]`` (NPh x N_alpha), in shared memory or in a file-backed memmap.

The determinant follows the reference's CPU script NL_julia_direct.jl:299-310
literally: for every harmonic one weighted copy ``weight .* conj(W_l)`` and one
ZGEMM ``transpose(W_l) * (...)`` accumulated into M, then ``M .*= G``,
``M .*= N(alpha)`` and LAPACK ``det(I - M)`` (numpy's OpenBLAS zgetrf).

The pool is started with the ``spawn`` method (safe in a process that has
already initialised CUDA).
"""
from __future__ import annotations

import dataclasses
import math
import multiprocessing as mp
import os
from multiprocessing import shared_memory
from typing import Optional

import numpy as np

from oracle import np_oracle as O

ULP2 = 4.440892098500626e-16      # 2 ulps of 1.0: the perturbed-ln sensitivity runs


def _set_log(perturb: float) -> None:
    if perturb:
        O.orbit_log = lambda x: np.log(x) * (1.0 + perturb)
    else:
        O.orbit_log = np.log


def _init_worker(perturb: float) -> None:
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(1)
    except Exception:
        pass
    _set_log(perturb)


def _orbit_rows(args):
    """Orbits of grid rows iR in [r0, r1): Omega_1/2 [n, Ne], samples [n, Ne, nwa]."""
    cfgd, r0, r1 = args
    c = O.OracleConfig(**cfgd)
    g = O.compute_grids(c, O.ToomreZang.from_config(c))
    wg = O.orbit_grid(c)
    na = len(wg[4])
    n = r1 - r0
    Om1 = np.zeros((n, c.Ne))
    Om2 = np.zeros((n, c.Ne))
    S = np.full((3, n, c.Ne, na), np.nan)
    with np.errstate(all="ignore"):
        for i, iR in enumerate(range(r0, r1)):
            for ie in range(c.Ne):
                Om1[i, ie], Om2[i, ie], S[0, i, ie], S[1, i, ie], S[2, i, ie] = \
                    O.orbit_samples(g, iR, ie, wg)
    return r0, Om1, Om2, S


class _Table:
    """complex128 [n_l, NPh, N_alpha] in shared memory or a file memmap."""

    def __init__(self, shape, path: Optional[str] = None, create: bool = True,
                 name: Optional[str] = None):
        self.shape = tuple(shape)
        self.path = path
        nbytes = int(np.prod(self.shape)) * 16
        if path:
            self.shm = None
            self.arr = np.memmap(path, dtype=np.complex128, mode="w+" if create else "r+",
                                 shape=self.shape)
        else:
            self.shm = shared_memory.SharedMemory(name=name, create=create, size=nbytes)
            self.arr = np.ndarray(self.shape, dtype=np.complex128, buffer=self.shm.buf)

    def spec(self):
        return (self.shape, self.path, None if self.shm is None else self.shm.name)

    @classmethod
    def attach(cls, spec):
        shape, path, name = spec
        return cls(shape, path, create=False, name=name)

    def close(self, unlink: bool = False):
        self.arr = None
        if self.shm is not None:
            self.shm.close()
            if unlink:
                self.shm.unlink()
        elif unlink and self.path and os.path.exists(self.path):
            os.unlink(self.path)


def _w_range(args):
    """W of orbits p in [p0, p1) into the shared table (zero rows stay zero)."""
    spec, m, alpha, l_arr, p0, Om1, Om2, w1, ra, pha = args
    t = _Table.attach(spec)
    W = t.arr
    with np.errstate(all="ignore"):
        for j in range(len(Om1)):
            blk = O.w_orbit(m, Om1[j], Om2[j], w1[j], ra[j], pha[j], alpha, l_arr)
            W[:, p0 + j, :] = 0.0 if blk is None else blk
    if t.shm is None:
        W.flush()
    t.close()
    return p0


@dataclasses.dataclass
class LargePrecomputed:
    cfg: O.OracleConfig
    alpha: np.ndarray
    d_alpha: np.ndarray
    N_kernel: np.ndarray
    Omega_1: np.ndarray       # [NPh] column-major orbit index p = iR + NR*ie
    Omega_2: np.ndarray
    DJ: np.ndarray            # [NPh]
    F0l: np.ndarray           # [NPh, n_l]
    Omega_res: np.ndarray     # [NPh, n_l]
    table: _Table             # W [n_l, NPh, N_alpha]

    @property
    def W(self) -> np.ndarray:
        return self.table.arr

    def close(self):
        if self.table is not None:
            self.table.close(unlink=True)
            self.table = None


def precompute_large(c: O.OracleConfig, workers: Optional[int] = None,
                     table_path: Optional[str] = None, perturb: float = 0.0,
                     orbit_rows_per_task: int = 4, orbits_per_task: int = 128) -> LargePrecomputed:
    """precompute_all (BasisFunctions.jl:73-165) over a spawn process pool."""
    workers = workers or os.cpu_count() or 1
    cfgd = dataclasses.asdict(c)
    _set_log(perturb)
    try:
        model = O.ToomreZang.from_config(c)
        g = O.compute_grids(c, model)
        NR, Ne, NPh = c.NR, c.Ne, c.NPh
        alpha = O.linspace(-c.alpha_max, c.alpha_max, c.N_alpha)
        d_alpha = O.quad_coef(alpha, c.quad[0])
        l_arr = np.arange(c.l_min, c.l_max + 1)
        na = len(O.orbit_grid(c)[4])
        Om1 = np.zeros((NR, Ne))
        Om2 = np.zeros((NR, Ne))
        S = np.empty((3, Ne, NR, na))          # [field][ie][iR] -> p order after reshape
        ctx = mp.get_context("spawn")
        table = _Table((c.n_l, NPh, c.N_alpha), table_path)
        try:
            with ctx.Pool(workers, initializer=_init_worker, initargs=(perturb,)) as pool:
                tasks = [(cfgd, r, min(NR, r + orbit_rows_per_task))
                         for r in range(0, NR, orbit_rows_per_task)]
                for r0, o1, o2, s in pool.imap_unordered(_orbit_rows, tasks):
                    n = o1.shape[0]
                    Om1[r0:r0 + n] = o1
                    Om2[r0:r0 + n] = o2
                    S[:, :, r0:r0 + n] = np.transpose(s, (0, 2, 1, 3))
                S = S.reshape(3, NPh, na)
                om1p = Om1.reshape(-1, order="F")
                om2p = Om2.reshape(-1, order="F")
                spec = table.spec()
                wtasks = [(spec, c.m, alpha, l_arr, p, om1p[p:p + orbits_per_task],
                           om2p[p:p + orbits_per_task], S[0, p:p + orbits_per_task],
                           S[1, p:p + orbits_per_task], S[2, p:p + orbits_per_task])
                          for p in range(0, NPh, orbits_per_task)]
                for _ in pool.imap_unordered(_w_range, wtasks):
                    pass
        except BaseException:
            table.close(unlink=True)
            raise
        jac = O.compute_jacobian(g, Om1)
        F0, FE, FL = O.df_fields(model, g)
    finally:
        _set_log(0.0)
    N = O.compute_N_kernel(c.m, alpha, d_alpha)
    DJ = (g.S_RC[:, None] * g.S_e * jac).reshape(-1, order="F")
    FEp = FE.reshape(-1, order="F")
    FLp = FL.reshape(-1, order="F")
    om1p = Om1.reshape(-1, order="F")
    om2p = Om2.reshape(-1, order="F")
    F0l = (l_arr[None, :] * om1p[:, None] + c.m * om2p[:, None]) * FEp[:, None] + c.m * FLp[:, None]
    Ores = l_arr[None, :] * om1p[:, None] + c.m * om2p[:, None]
    return LargePrecomputed(c, alpha, d_alpha, N, om1p, om2p, DJ, F0l, Ores, table)


def build_M_large(pc: LargePrecomputed, omega: complex) -> np.ndarray:
    """M(omega), one ZGEMM per harmonic (NL_julia_direct.jl:299-308;
    denominator clamp MatrixBuilder.jl:45-51)."""
    c = pc.cfg
    Na = c.N_alpha
    M = np.zeros((Na, Na), dtype=np.complex128)
    G_k = pc.DJ
    for il in range(c.n_l):
        Wl = pc.W[il]
        den = omega - pc.Omega_res[:, il].astype(np.complex128)
        den = np.where(np.abs(den) < 1e-12, 1e-12 + 1e-12j, den)
        weight = G_k * pc.F0l[:, il] / den
        M += Wl.T @ (weight[:, None] * np.conj(Wl))
    M *= c.G
    M *= pc.N_kernel[None, :]
    return M


def compute_det_large(pc: LargePrecomputed, omega: complex) -> complex:
    """det(I - M(omega)) (NL_julia_direct.jl:309)."""
    M = build_M_large(pc, omega)
    return complex(np.linalg.det(np.eye(pc.cfg.N_alpha) - M))
