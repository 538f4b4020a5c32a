"""Host-side mirror of the reference's Julia package API.

Same names, argument meaning and results as ``src/KalnajsLogSpiral``
(export list ``src/KalnajsLogSpiral.jl:23-43``); every numeric step runs in
``libkls.so`` on the GPU:

=============================  ==============================================
reference (file:line)          here
=============================  ==============================================
Models.jl:24-57                ToomreZangModel, create_toomre_zang_model
BasisFunctions.jl:30-165       PrecomputedData, precompute_all  (on device)
BasisFunctions.jl:381-437      DevicePrecomputed, to_device
MatrixBuilder.jl:197-244       compute_determinant, compute_determinant_batched,
                               build_M_matrix
GridScan.jl:25-88, 234-246     grid_scan, find_minimum
GridScan.jl:125-197            ModelBatch (many models per launch), autotune
NewtonSolver.jl:19-172         NewtonResult, newton_search
GPUBackend.jl:27-31, 50-72     GPUType, detect_gpu_type
=============================  ==============================================

Differences a caller can observe, all deliberate:

* ``precompute_all`` runs on the device and leaves the W_l table there; the
  reference's host arrays (``orbit_data``, ``W_l_mat``, ...) are exported
  lazily on first attribute access.
* There is no CPU path: ``devprecomp=None`` or ``gpu_type=GPUType.NONE``
  still evaluate on the GPU (in FP64).  Without a usable GPU every call raises
  ``KlsError``.
* ``Tgpu`` selects the contraction precision: ``"Float64"`` is the plain FP64
  form; ``"Float32"`` (the reference's reduced-precision GPU setting) selects
  the split-BF16 tensor-core form with FP32 accumulation.  ``Tcpu`` is
  accepted; the determinant is always formed in FP64.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
import threading
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import KLS_MODE_FP64, KLS_MODE_MIXED, check, dptr
from .config import check_quadrature, KalnajsConfig, copy_config


# ---------------------------------------------------------------------------
# GPUBackend.jl:27-31
# ---------------------------------------------------------------------------
class GPUType(enum.Enum):
    NVIDIA = 0
    AMD = 1
    NONE = 2


def detect_gpu_type() -> GPUType:
    """NVIDIA when a CUDA device is visible, else NONE (GPUBackend.jl:50-72)."""
    try:
        import torch
        return GPUType.NVIDIA if torch.cuda.is_available() else GPUType.NONE
    except Exception:
        return GPUType.NONE


# ---------------------------------------------------------------------------
# Models.jl:24-57
# ---------------------------------------------------------------------------
@dataclass
class ToomreZangModel:
    L0: float
    n_zang: int
    q1: float
    q_zang: float
    sigma_r0: float
    G: float
    DF_const: float


def create_toomre_zang_model(config: KalnajsConfig) -> ToomreZangModel:
    L0 = float(config.model.L0)
    n_zang = int(config.model.n_zang)
    q1 = float(config.model.q1)
    G = float(config.physics.G)
    sigma_r0 = 1.0 / math.sqrt(q1)
    q = q1 - 1.0
    DF_const = 1.0 / (2.0 * math.pi * 2.0 ** (q / 2) * math.sqrt(math.pi)
                      * math.gamma((q + 1) / 2) * sigma_r0 ** (q + 2))
    return ToomreZangModel(L0, n_zang, q1, q, sigma_r0, G, DF_const)


def _kls_config(config: KalnajsConfig, model: Optional[ToomreZangModel]) -> _lib.kls_config:
    g = config.grid
    k = _lib.kls_config()
    k.m = int(config.physics.m)
    k.G = float(model.G if model is not None else config.physics.G)
    k.L0 = float(model.L0 if model is not None else config.model.L0)
    k.n_zang = int(model.n_zang if model is not None else config.model.n_zang)
    k.q1 = float(model.q1 if model is not None else config.model.q1)
    k.NR, k.Ne = int(g.NR), int(g.Ne)
    k.Rc_min, k.Rc_max, k.v_min = float(g.Rc_min), float(g.Rc_max), float(g.v_min)
    k.N_alpha, k.alpha_max = int(g.N_alpha), float(g.alpha_max)
    k.l_min, k.l_max = int(g.l_min), int(g.l_max)
    k.nw, k.nwa = int(g.nw), int(g.nwa)
    q = getattr(g, "quadrature", "tts")
    check_quadrature(q)
    k.quad_alpha, k.quad_rc, k.quad_v = (_lib.QUAD_CODES[ch] for ch in q)
    return k


# ---------------------------------------------------------------------------
# Context: one libkls context per device
# ---------------------------------------------------------------------------
class _Context:
    def __init__(self, config: KalnajsConfig, model: Optional[ToomreZangModel], device: int):
        self.lib = _lib.load()
        self.kcfg = _kls_config(config, model)
        self.device = device
        h = C.c_void_p()
        check(None, self.lib.kls_create(C.byref(self.kcfg), device, C.byref(h)))
        self.h = h
        self.lock = threading.Lock()
        d = _lib.kls_dims()
        check(self.h, self.lib.kls_get_dims(self.h, C.byref(d)))
        self.dims = d

    def call(self, name: str, *args):
        with self.lock:
            check(self.h, getattr(self.lib, name)(self.h, *args))

    def close(self):
        if getattr(self, "h", None):
            self.lib.kls_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# OrbitIntegration.jl:26-54 (exported views)
# ---------------------------------------------------------------------------
@dataclass
class GridData:
    Rc: np.ndarray
    e: np.ndarray
    E: np.ndarray
    L_m: np.ndarray
    S_RC: np.ndarray
    S_e: np.ndarray


@dataclass
class OrbitData:
    grids: GridData
    Omega_1: np.ndarray
    Omega_2: np.ndarray
    w1: np.ndarray      # [nwa, NR, Ne] (column-major order as in the reference)
    ra: np.ndarray
    pha: np.ndarray
    jacobian: np.ndarray
    F0: np.ndarray
    FE: np.ndarray
    FL: np.ndarray


# ---------------------------------------------------------------------------
# BasisFunctions.jl:30-60, 73-165
# ---------------------------------------------------------------------------
class PrecomputedData:
    """All omega-independent quantities, resident on the device.

    Host copies of the reference's fields are exported on first access:
    ``alpha_arr``, ``d_alpha``, ``N_kernel``, ``DJ_vec``, ``F0l_all``,
    ``Omega_res``, ``orbit_data`` and ``W_l_mat`` ([NPh, N_alpha, n_l]
    complex; 16 * NPh * N_alpha * n_l bytes of host memory).
    """

    def __init__(self, config: KalnajsConfig, model: Optional[ToomreZangModel], device: int = 0):
        self.config = copy_config(config)
        self.model = model
        self.ctx = _Context(config, model, device)
        self.m = int(config.physics.m)
        self.G = float(model.G if model is not None else config.physics.G)
        self.N_alpha = int(config.grid.N_alpha)
        self.n_l = int(config.grid.l_max - config.grid.l_min + 1)
        self.l_arr = np.arange(config.grid.l_min, config.grid.l_max + 1)
        self.NPh = int(config.grid.NR * config.grid.Ne)
        self._cache = {}

    def close(self):
        self.ctx.close()

    # -- lazy exports --------------------------------------------------------
    def _alpha(self):
        if "alpha" not in self._cache:
            a = np.empty(self.N_alpha); d = np.empty(self.N_alpha); n = np.empty(self.N_alpha)
            self.ctx.call("kls_export_alpha", dptr(a), dptr(d), dptr(n))
            self._cache["alpha"] = (a, d, n)
        return self._cache["alpha"]

    @property
    def alpha_arr(self) -> np.ndarray:
        return self._alpha()[0]

    @property
    def d_alpha(self) -> np.ndarray:
        return self._alpha()[1]

    @property
    def N_kernel(self) -> np.ndarray:
        return self._alpha()[2]

    @property
    def orbit_data(self) -> OrbitData:
        if "orbits" not in self._cache:
            g = self.config.grid
            NR, Ne, nwa = g.NR, g.Ne, g.nwa
            f = [np.empty(NR * Ne) for _ in range(7)]
            w = [np.empty(NR * Ne * nwa) for _ in range(3)]
            self.ctx.call("kls_export_orbits", *[dptr(x) for x in f], *[dptr(x) for x in w])
            gr = [np.empty(NR * Ne) for _ in range(4)] + [np.empty(NR), np.empty(NR * Ne)]
            self.ctx.call("kls_export_grids", *[dptr(x) for x in gr])
            cm = lambda a: a.reshape(NR, Ne, order="F")
            tr = lambda a: a.reshape(nwa, NR, Ne, order="F")
            grids = GridData(cm(gr[0]), cm(gr[1]), cm(gr[2]), cm(gr[3]), gr[4], cm(gr[5]))
            self._cache["DJ"] = f[6]
            self._cache["orbits"] = OrbitData(grids, cm(f[0]), cm(f[1]), tr(w[0]), tr(w[1]),
                                              tr(w[2]), cm(f[2]), cm(f[3]), cm(f[4]), cm(f[5]))
        return self._cache["orbits"]

    @property
    def DJ_vec(self) -> np.ndarray:
        self.orbit_data
        return self._cache["DJ"]

    def _resonant(self):
        if "res" not in self._cache:
            K = self.NPh * self.n_l
            f = np.empty(K); o = np.empty(K)
            self.ctx.call("kls_export_resonant", dptr(f), dptr(o))
            self._cache["res"] = (f.reshape(self.NPh, self.n_l, order="F"),
                                  o.reshape(self.NPh, self.n_l, order="F"))
        return self._cache["res"]

    @property
    def F0l_all(self) -> np.ndarray:
        return self._resonant()[0]

    @property
    def Omega_res(self) -> np.ndarray:
        return self._resonant()[1]

    def export_W(self, il0: int = 0, nl: Optional[int] = None) -> np.ndarray:
        """W_l_mat[:, :, il0:il0+nl] as complex128 [NPh, N_alpha, nl]."""
        nl = self.n_l - il0 if nl is None else nl
        buf = np.empty(2 * self.NPh * self.N_alpha * nl)
        self.ctx.call("kls_export_W", il0, nl, dptr(buf))
        return buf.view(np.complex128).reshape(self.NPh, self.N_alpha, nl, order="F")

    @property
    def W_l_mat(self) -> np.ndarray:
        return self.export_W()


def precompute_all(config: KalnajsConfig, model: Optional[ToomreZangModel] = None,
                   backend: GPUType = GPUType.NVIDIA, verbose: bool = False,
                   device: int = 0) -> PrecomputedData:
    """BasisFunctions.jl:73-165, evaluated on the GPU."""
    if model is None:
        model = create_toomre_zang_model(config)
    if verbose:
        print("Computing grids, orbits, W_l basis functions and N_m(alpha) on the GPU...")
    pc = PrecomputedData(config, model, device)
    pc.ctx.call("kls_precompute")
    if verbose:
        print("Precomputation complete.")
    return pc


@dataclass
class DevicePrecomputed:
    """BasisFunctions.jl:381-395: the device side of the precompute."""
    m: int
    G: float
    N_alpha: int
    n_l: int
    NPh: int
    mode: int
    precomp: PrecomputedData


def _mode_for(Tgpu) -> int:
    name = getattr(Tgpu, "__name__", str(Tgpu))
    if name in ("Float64", "float64", "ComplexF64", "complex128"):
        return KLS_MODE_FP64
    if name in ("Float32", "float32", "ComplexF32", "complex64"):
        return KLS_MODE_MIXED
    raise ValueError(f"unsupported GPU precision {Tgpu!r}")


def to_device(precomp: PrecomputedData, gpu_type: GPUType = GPUType.NVIDIA,
              Tgpu="Float64") -> DevicePrecomputed:
    """BasisFunctions.jl:397-437; the table already lives on the device."""
    mode = _mode_for(Tgpu)
    if mode == KLS_MODE_MIXED:
        precomp.ctx.call("kls_prepare_mixed")
    return DevicePrecomputed(precomp.m, precomp.G, precomp.N_alpha, precomp.n_l, precomp.NPh,
                             mode, precomp)


def release_fp64(precomp: PrecomputedData) -> None:
    """Keep only the split-BF16 table (kls_release_fp64): FP64 evaluations of
    this precompute raise KlsError afterwards."""
    precomp.ctx.call("kls_release_fp64")


def _mode(devprecomp: Optional[DevicePrecomputed]) -> int:
    return KLS_MODE_FP64 if devprecomp is None else devprecomp.mode


# ---------------------------------------------------------------------------
# MatrixBuilder.jl:197-244
# ---------------------------------------------------------------------------
def compute_determinant_batched(omegas: Sequence[complex], precomputed: PrecomputedData,
                                devprecomp: Optional[DevicePrecomputed] = None,
                                gpu_type: GPUType = GPUType.NVIDIA, Tcpu="Float64",
                                batch_size: int = 100, log_abs: bool = False):
    """det(I - M(omega)) for every omega; returns complex128 array (and log|det|)."""
    om = np.ascontiguousarray(np.asarray(omegas, dtype=np.complex128).reshape(-1))
    n = om.size
    out = np.empty(n, dtype=np.complex128)
    la = np.empty(n)
    ri = om.view(np.float64)
    for s in range(0, n, max(1, int(batch_size))):
        e = min(n, s + max(1, int(batch_size)))
        o = out[s:e]
        l = la[s:e]
        precomputed.ctx.call("kls_det_batch", dptr(ri[2 * s:2 * e]), e - s, _mode(devprecomp),
                             dptr(o.view(np.float64)), dptr(l))
    return (out, la) if log_abs else out


def compute_determinant(omega: complex, precomputed: PrecomputedData,
                        devprecomp: Optional[DevicePrecomputed] = None,
                        gpu_type: GPUType = GPUType.NVIDIA, Tcpu="Float64") -> complex:
    return complex(compute_determinant_batched([omega], precomputed, devprecomp, gpu_type, Tcpu)[0])


def build_M_matrix(omega: complex, precomputed: PrecomputedData,
                   devprecomp: Optional[DevicePrecomputed] = None) -> np.ndarray:
    """M(omega) [N_alpha, N_alpha] complex128 (MatrixBuilder.jl:242-244)."""
    N = precomputed.N_alpha
    buf = np.empty(2 * N * N)
    precomputed.ctx.call("kls_build_M", float(np.real(omega)), float(np.imag(omega)),
                         _mode(devprecomp), dptr(buf))
    return buf.view(np.complex128).reshape(N, N, order="F")


# ---------------------------------------------------------------------------
# GridScan.jl:25-246
# ---------------------------------------------------------------------------
def _linspace(a: float, b: float, n: int) -> np.ndarray:
    return np.linspace(a, b, n)


def find_minimum(det_grid: np.ndarray, Omega_p_grid, gamma_grid) -> Tuple[float, float]:
    """argmin |det| in column-major order, first occurrence (GridScan.jl:234-246)."""
    a = np.abs(np.asarray(det_grid))
    idx = int(np.argmin(a.ravel(order="F")))
    n_g = a.shape[0]
    return float(np.asarray(Omega_p_grid)[idx // n_g]), float(np.asarray(gamma_grid)[idx % n_g])


def _scan_columns(pc: PrecomputedData, mode: int, Op_cols: np.ndarray, g_grid: np.ndarray,
                  m: int) -> np.ndarray:
    # omega = Complex(m * Op, gamma) in column-major grid order (GridScan.jl:101-104)
    om = np.empty((len(g_grid), len(Op_cols)), dtype=np.complex128, order="F")
    om.real[...] = (m * Op_cols)[None, :]
    om.imag[...] = g_grid[:, None]
    om = np.ascontiguousarray(om.ravel(order="F"))
    d = np.empty_like(om)
    pc.ctx.call("kls_det_batch", dptr(om.view(np.float64)), len(om), mode,
                dptr(d.view(np.float64)), C.cast(None, C.POINTER(C.c_double)))
    return d.reshape(len(g_grid), len(Op_cols), order="F")


def grid_scan(config: KalnajsConfig, precomputed: PrecomputedData,
              devprecomp: Optional[DevicePrecomputed] = None,
              gpu_type: GPUType = GPUType.NVIDIA, Tcpu="Float64", verbose: bool = False,
              gpu_devices: Sequence[int] = ()):
    """Returns (det_grid [n_gamma, n_Op], Omega_p_init, gamma_init) (GridScan.jl:25-88).

    With several ``gpu_devices`` the Omega_p columns are split across devices
    exactly as ``scan_multi_gpu!`` does (GridScan.jl:125-197), each device
    holding its own replica of the precompute.
    """
    s = config.scan
    m = int(config.physics.m)
    Op_grid = _linspace(s.Omega_p_min, s.Omega_p_max, s.n_Op)
    g_grid = _linspace(s.gamma_min, s.gamma_max, s.n_gamma)
    mode = _mode(devprecomp)
    if verbose:
        print(f"Scanning (Ω_p, γ) grid: {s.n_Op} × {s.n_gamma} = {s.n_Op * s.n_gamma} points")
    devs = list(gpu_devices)
    if len(devs) > 1:
        ranges = column_ranges(s.n_Op, len(devs))
        det_grid = np.empty((s.n_gamma, s.n_Op), dtype=np.complex128)
        errs: List[BaseException] = []

        def work(dev, cols):
            try:
                if dev == precomputed.ctx.device:
                    pc = precomputed
                else:
                    pc = precompute_all(precomputed.config, precomputed.model, device=dev)
                    if mode == KLS_MODE_MIXED:
                        pc.ctx.call("kls_prepare_mixed")
                det_grid[:, cols] = _scan_columns(pc, mode, Op_grid[cols], g_grid, m)
                if pc is not precomputed:
                    pc.close()
            except BaseException as e:   # re-raised on the calling thread
                errs.append(e)

        th = [threading.Thread(target=work, args=(d, r)) for d, r in zip(devs, ranges)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if errs:
            raise errs[0]
    else:
        det_grid = _scan_columns(precomputed, mode, Op_grid, g_grid, m)
    Op0, g0 = find_minimum(det_grid, Op_grid, g_grid)
    if verbose:
        print(f"Minimum |det| = {np.abs(det_grid).min():.2e} at Ω_p = {Op0:.6f}, γ = {g0:.6f}")
    return det_grid, Op0, g0


def grid_scan_distributed(config: KalnajsConfig, precomputed: Optional[PrecomputedData] = None,
                          devprecomp: Optional[DevicePrecomputed] = None, group=None,
                          column_fn=None):
    """grid_scan with one process per GPU (torch.distributed, e.g. under torchrun).

    Rank r of W evaluates the Omega_p columns ``column_ranges(n_Op, W)[r]``
    (the column split of scan_multi_gpu!, GridScan.jl:133-144) on its own
    replica of the precompute; one all_gather of the det blocks (16 B per
    determinant) gives every rank the same (det_grid, Omega_p_init,
    gamma_init) that grid_scan returns.  ``column_fn(Op_cols, gamma_grid, m)``
    evaluates one [n_gamma, n_cols] block; by default this rank's
    ``precomputed`` on its GPU.
    """
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    s = config.scan
    m = int(config.physics.m)
    Op_grid = _linspace(s.Omega_p_min, s.Omega_p_max, s.n_Op)
    g_grid = _linspace(s.gamma_min, s.gamma_max, s.n_gamma)
    ranges = column_ranges(s.n_Op, world)
    cols = ranges[rank]
    if column_fn is None:
        mode = _mode(devprecomp)
        column_fn = lambda Opc, gg, mm: _scan_columns(precomputed, mode, Opc, gg, mm)
    block = np.asarray(column_fn(Op_grid[cols], g_grid, m), dtype=np.complex128)
    width = max(r.stop - r.start for r in ranges)
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    buf = torch.zeros((s.n_gamma, width, 2), dtype=torch.float64, device=dev)
    if block.size:
        buf[:, :block.shape[1]] = torch.view_as_real(torch.from_numpy(block)).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    det_grid = np.empty((s.n_gamma, s.n_Op), dtype=np.complex128)
    for r, part in zip(ranges, parts):
        p = part.cpu().numpy()
        det_grid[:, r] = p[:, :r.stop - r.start, 0] + 1j * p[:, :r.stop - r.start, 1]
    Op0, g0 = find_minimum(det_grid, Op_grid, g_grid)
    return det_grid, Op0, g0


def harmonic_ranges(l_min: int, l_max: int, n_ranks: int) -> List[Tuple[int, int]]:
    """Contiguous (l_lo, l_hi) harmonic slices, inclusive; the first
    n_l % n_ranks slices one harmonic wider."""
    n_l = l_max - l_min + 1
    per, rem = divmod(n_l, n_ranks)
    out, lo = [], l_min
    for r in range(n_ranks):
        hi = lo + per + (1 if r < rem else 0) - 1
        out.append((lo, hi))
        lo = hi + 1
    return out


def precompute_ksharded(config: KalnajsConfig, group=None, device: Optional[int] = None
                        ) -> PrecomputedData:
    """This rank's slice of the W table: the harmonics harmonic_ranges(...)[rank]
    (K sharding: the contraction over k = (orbit, l) is a sum, so the slices'
    partial M(omega) add up to M(omega))."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = harmonic_ranges(config.grid.l_min, config.grid.l_max, world)[rank]
    c = copy_config(config)
    c.grid.l_min, c.grid.l_max = lo, hi
    dev = torch.cuda.current_device() if device is None else device
    return precompute_all(c, device=dev)


def compute_determinant_ksharded(omegas: Sequence[complex], config: KalnajsConfig,
                                 precomputed: Optional[PrecomputedData] = None,
                                 devprecomp: Optional[DevicePrecomputed] = None, group=None,
                                 M_fn=None, det_fn=None) -> np.ndarray:
    """det(I - M(omega)) with the W table split over the ranks by harmonic.

    Every rank forms its partial M(omega) (``M_fn``, default: build_M_matrix on
    its slice from precompute_ksharded), one all_reduce (sum) of the
    [n, N_alpha, N_alpha] complex partials gives M on every rank, and the
    determinant is taken on the device (``det_fn``, default: the library's
    LU through kls_det_lu_static).  The reference's 2-GPU split
    (NL_julia_gpu.jl:313-378) loops every GPU over all harmonics; here each
    harmonic is contracted once.
    """
    import torch
    import torch.distributed as dist
    om = np.asarray(omegas, dtype=np.complex128).reshape(-1)
    if M_fn is None:
        M_fn = lambda w: build_M_matrix(w, precomputed, devprecomp)
    M = np.stack([np.asarray(M_fn(w), dtype=np.complex128) for w in om])
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.view_as_real(torch.from_numpy(np.ascontiguousarray(M))).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    Mt = torch.view_as_complex(t.contiguous()).cpu().numpy()
    A = np.eye(M.shape[1])[None, :, :] - Mt
    if det_fn is not None:
        return np.array([det_fn(a) for a in A])
    lib = _lib.load()
    n, N = A.shape[0], A.shape[1]
    # row-major I - M on the device for the library's LU
    dA = torch.view_as_real(torch.from_numpy(np.ascontiguousarray(A))).to("cuda").contiguous()
    dd = torch.empty((n, 2), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # one call per chunk that fits the static LU's scratch; calls on one
    # stream run in order, so they do not race on the scratch
    for lo, hi in static_lu_chunks(n, N):
        check(None, lib.kls_det_lu_static(C.c_void_p(dA[lo].data_ptr()), hi - lo, N,
                                          C.c_void_p(dd[lo].data_ptr()), C.c_void_p(None),
                                          C.c_void_p(stream)))
    d = dd.cpu().numpy()
    return d[:, 0] + 1j * d[:, 1]


STATIC_LU_MAX = 1 << 20     # complex elements of kls_det_lu_static's scratch


def static_lu_chunks(n: int, N: int) -> List[Tuple[int, int]]:
    """[lo, hi) ranges of at most STATIC_LU_MAX // N^2 matrices each, the
    batches one kls_det_lu_static call accepts.  A single N x N matrix larger
    than the scratch (N > 1024) cannot be factored there: _lib.KlsError."""
    per = STATIC_LU_MAX // (N * N)
    if per < 1:
        raise _lib.KlsError(_lib.KLS_ERR_CONFIG,
                            f"N_alpha = {N} > 1024: one matrix exceeds the fixed scratch of "
                            "kls_det_lu_static; pass det_fn")
    return [(lo, min(n, lo + per)) for lo in range(0, n, per)]


def column_ranges(n_Op: int, n_gpus: int) -> List[slice]:
    """Contiguous column blocks, the first n_Op % n_gpus one wider (GridScan.jl:133-144)."""
    per, rem = divmod(n_Op, n_gpus)
    out, start = [], 0
    for g in range(n_gpus):
        end = start + per + (1 if g < rem else 0)
        out.append(slice(start, end))
        start = end
    return out


# ---------------------------------------------------------------------------
# NewtonSolver.jl:19-172
# ---------------------------------------------------------------------------
@dataclass
class NewtonResult:
    Omega_p: float
    gamma: float
    omega: complex
    det_val: complex
    iterations: int
    converged: bool
    history: np.ndarray      # [iterations, 3]: (Omega_p, gamma, |det|)
    det_evals: int = 0


def newton_search(config: KalnajsConfig, precomputed: PrecomputedData,
                  devprecomp: Optional[DevicePrecomputed] = None,
                  gpu_type: GPUType = GPUType.NVIDIA, Tcpu="Float64",
                  Omega_p_init: Optional[float] = None, gamma_init: Optional[float] = None,
                  verbose: bool = False) -> NewtonResult:
    n = config.newton
    if Omega_p_init is None:
        Omega_p_init = config.reference.Omega_p
    if gamma_init is None:
        gamma_init = config.reference.gamma
    nc = _lib.kls_newton_cfg(int(n.max_iter), float(n.tol), float(n.delta),
                             int(bool(n.use_line_search)), int(n.max_line_search),
                             _mode(devprecomp))
    res = _lib.kls_newton_result()
    hist = np.zeros((int(n.max_iter), 3))
    precomputed.ctx.call("kls_newton", float(Omega_p_init), float(gamma_init), C.byref(nc),
                         C.byref(res), dptr(hist))
    h = hist[:res.iterations].copy()
    if verbose:
        print("Newton-Raphson refinement:")
        print(f"  max_iter = {n.max_iter}, tol = {n.tol}, delta = {n.delta}\n")
        for i, (Op, g, a) in enumerate(h, 1):
            print(f"Iter {i:2d}: Ω_p={Op:.10f}  γ={g:.10f}  |det|={a:.2e}")
        if res.converged:
            print("✓ Converged!")
    return NewtonResult(res.Omega_p, res.gamma, complex(res.omega_re, res.omega_im),
                        complex(res.det_re, res.det_im), int(res.iterations),
                        bool(res.converged), h, int(res.det_evals))


@dataclass
class HybridConfig:
    """Parameters of newton_search_hybrid (kls_hybrid_cfg in include/kls.h).

    The split-BF16 determinant carries a ~5e-5 relative error, so the first
    finite-difference slope of the mixed phase uses a step of 1e-3; the mixed
    phase hands over once its next step is below 1e-5 (its root error is
    ~1e-6).  Anchored determinants stay within FP64 accuracy for ~1e-5 around
    the anchor; a step beyond anchor_radius re-anchors (one FP64
    determinant).  From a start whose first Newton step is longer than
    far_step the iteration first follows the reference's path with steps of
    FP64 accuracy (one FP64 and one anchored determinant each), so that a
    long path from a grid edge ends on the root the FP64 Newton reaches."""
    mixed_delta: float = 1e-3
    mixed_step_tol: float = 1e-5
    mixed_max_iter: int = 30
    fp64_max_iter: int = 50
    anchor_radius: float = 1e-5
    final_fp64: bool = False
    far_step: float = 2e-2


def set_anchor(precomputed: PrecomputedData, omega: complex) -> complex:
    """FP64 M(omega_a) kept on the device for KLS_MODE_ANCHORED; returns
    det(I - M(omega_a)) (no reference counterpart)."""
    out = np.zeros(2)
    precomputed.ctx.call("kls_set_anchor", float(np.real(omega)), float(np.imag(omega)),
                         dptr(out))
    return complex(out[0], out[1])


def newton_search_hybrid(config: KalnajsConfig, precomputed: PrecomputedData,
                         Omega_p_init: Optional[float] = None,
                         gamma_init: Optional[float] = None,
                         hybrid: Optional[HybridConfig] = None) -> NewtonResult:
    """Split-BF16 secant phase, then an FP64 anchor and anchored steps to the
    reference's stopping rule (kls_newton_hybrid).

    No reference counterpart: the result satisfies |det(I - M)| <
    config.newton.tol (NewtonSolver.jl:89) on an FP64-accurate determinant
    (the anchored form, or plain FP64 with ``final_fp64``); ``det_evals``
    counts every evaluation and ``history`` has one row per evaluation.
    """
    n = config.newton
    hc = hybrid or HybridConfig()
    if Omega_p_init is None:
        Omega_p_init = config.reference.Omega_p
    if gamma_init is None:
        gamma_init = config.reference.gamma
    precomputed.ctx.call("kls_prepare_mixed")
    nc = _lib.kls_newton_cfg(int(n.max_iter), float(n.tol), float(n.delta),
                             int(bool(n.use_line_search)), int(n.max_line_search), KLS_MODE_FP64)
    h = _lib.kls_hybrid_cfg(float(hc.mixed_delta), float(hc.mixed_step_tol),
                            int(hc.mixed_max_iter), int(hc.fp64_max_iter),
                            float(hc.anchor_radius), int(bool(hc.final_fp64)),
                            float(hc.far_step))
    res = _lib.kls_newton_result()
    ev = (C.c_int32 * 3)()
    hist = np.zeros((int(n.max_iter), 3))
    precomputed.ctx.call("kls_newton_hybrid", float(Omega_p_init), float(gamma_init), C.byref(nc),
                         C.byref(h), C.byref(res), ev, dptr(hist))
    r = NewtonResult(res.Omega_p, res.gamma, complex(res.omega_re, res.omega_im),
                     complex(res.det_re, res.det_im), int(res.iterations), bool(res.converged),
                     hist[:min(res.iterations, int(n.max_iter))].copy(), int(res.det_evals))
    r.mixed_evals, r.fp64_evals, r.anchored_evals = int(ev[0]), int(ev[1]), int(ev[2])
    return r


# ---------------------------------------------------------------------------
# Uneven batch over models and the autotuner (no reference counterpart)
# ---------------------------------------------------------------------------
@dataclass
class TuneResult:
    mode: int
    splits: int
    default_splits: int
    candidates: int
    ms_per_omega: float
    default_ms_per_omega: float
    form: int = 0


def autotune(precomputed: PrecomputedData, Tgpu="Float64", batch: int = 2) -> TuneResult:
    """Choose the context's K split count for `Tgpu` by timing (kls_autotune)."""
    r = _lib.kls_tune_result()
    precomputed.ctx.call("kls_autotune", _mode_for(Tgpu), int(batch), C.byref(r))
    return TuneResult(r.mode, r.splits, r.default_splits, r.candidates, r.ms_per_omega,
                      r.default_ms_per_omega, r.form)


class ModelBatch:
    """Many precomputed models of any sizes evaluated together (kls_multi).

    Each pass evaluates `batch` omegas per model: one persistent contraction
    launch for all models, replayed from a captured CUDA graph.  Results are
    bitwise those of compute_determinant_batched on each model's own context.
    """

    def __init__(self, precomputed: Sequence[PrecomputedData], Tgpu="Float64", batch: int = 16):
        self.lib = _lib.load()
        self.models = list(precomputed)
        self.mode = _mode_for(Tgpu)
        if self.mode == KLS_MODE_MIXED:
            for pc in self.models:
                pc.ctx.call("kls_prepare_mixed")
        arr = (C.c_void_p * len(self.models))(*[pc.ctx.h for pc in self.models])
        h = C.c_void_p()
        code = self.lib.kls_multi_create(arr, len(self.models), self.mode, int(batch), C.byref(h))
        if code:
            raise _lib.KlsError(code, self.lib.kls_multi_last_error(None).decode())
        self.h = h
        self.batch = int(batch)

    def _ck(self, code):
        if code:
            raise _lib.KlsError(code, self.lib.kls_multi_last_error(self.h).decode())

    def det(self, omegas) -> Tuple[np.ndarray, np.ndarray]:
        """omegas [n_models, n] complex -> (det [n_models, n], log|det| [n_models, n])."""
        om = np.ascontiguousarray(np.asarray(omegas, dtype=np.complex128))
        if om.ndim != 2 or om.shape[0] != len(self.models):
            raise ValueError(f"expected omegas of shape [{len(self.models)}, n], got {om.shape}")
        n = om.shape[1]
        d = np.empty_like(om)
        la = np.empty(om.shape)
        self._ck(self.lib.kls_multi_det(self.h, dptr(om.view(np.float64)), n,
                                        dptr(d.view(np.float64)), dptr(la)))
        return d, la

    def scan(self, n_Op: int = 41, n_gamma: int = 20, Omega_p_range=(0.2, 0.6),
             gamma_range=(0.01, 0.2)):
        """Every model's grid_scan on one grid: (det [n_models, n_gamma, n_Op],
        log|det| likewise, Omega_p0 [n_models], gamma0 [n_models])."""
        sc = _lib.kls_scan_cfg(int(n_Op), int(n_gamma), float(Omega_p_range[0]),
                               float(Omega_p_range[1]), float(gamma_range[0]),
                               float(gamma_range[1]), self.mode, self.batch)
        nm, n = len(self.models), n_Op * n_gamma
        d = np.empty(nm * n, dtype=np.complex128)
        la = np.empty(nm * n)
        Op0 = np.empty(nm)
        g0 = np.empty(nm)
        self._ck(self.lib.kls_scan_multi(self.h, C.byref(sc), dptr(d.view(np.float64)), dptr(la),
                                         dptr(Op0), dptr(g0)))
        # per model a column-major [n_gamma, n_Op] block
        return (d.reshape(nm, n_Op, n_gamma).transpose(0, 2, 1),
                la.reshape(nm, n_Op, n_gamma).transpose(0, 2, 1), Op0, g0)

    def info(self) -> dict:
        i = _lib.kls_multi_info()
        self._ck(self.lib.kls_multi_get_info(self.h, C.byref(i)))
        d = {f: getattr(i, f) for f, _ in i._fields_}
        d["schedule_ms"] = list(i.schedule_ms)
        return d

    def close(self):
        if getattr(self, "h", None):
            self.lib.kls_multi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
