"""Learned root proposer (no counterpart in the reference).

A small MLP maps (n_zang, q1, m, Omega_p, gamma) to features of
det(I - M(omega)) -- (log|det|, sin arg det, cos arg det) -- and proposes a
Newton start as the minimum of its predicted log|det| over the scan region, in
place of the reference's grid scan (GridScan.jl:25-88).  FP64 Newton on the
exact determinant refines every proposal; a proposal counts only if it
converges to the root the scan-started Newton finds.

The network is trained on the GPU by libkls.so's own BF16 forward/backward
kernels (kls_mlp_*) on samples that batched scans of seeded random models
produce.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check
from .config import KalnajsConfig, copy_config

LOG_SCALE = 10.0          # log|det| is learned as log|det| / LOG_SCALE


def features(n_zang, q1, m, Omega_p, gamma) -> np.ndarray:
    """Normalised inputs, float32 [n, 5]."""
    b = np.broadcast_arrays(*(np.asarray(v, dtype=np.float64) for v in
                              (n_zang, q1, m, Omega_p, gamma)))
    x = np.stack([(b[0] - 4.0) / 2.0, (b[1] - 8.0) / 4.0, (b[2] - 2.5) * 2.0,
                  (b[3] - 0.5) / 0.3, (b[4] - 0.155) / 0.145], axis=-1)
    return np.ascontiguousarray(x.reshape(-1, 5), dtype=np.float32)


def targets(det: np.ndarray, log_abs: Optional[np.ndarray] = None) -> np.ndarray:
    """(log|det| / LOG_SCALE, sin arg, cos arg), float32 [n, 3]."""
    d = np.asarray(det, dtype=np.complex128).reshape(-1)
    la = np.log(np.abs(d)) if log_abs is None else np.asarray(log_abs).reshape(-1)
    ph = np.angle(d)
    t = np.stack([la / LOG_SCALE, np.sin(ph), np.cos(ph)], axis=-1)
    return np.ascontiguousarray(t, dtype=np.float32)


class MLP:
    """kls_mlp handle: width-`width` GELU MLP with `depth` linear layers."""

    def __init__(self, width: int = 256, depth: int = 4, seed: int = 0, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(None, self.lib.kls_mlp_create(device, width, depth, seed, C.byref(h)))
        self.h = h
        self.width, self.depth = width, depth
        n = C.c_int64()
        self.lib.kls_mlp_num_params(self.h, C.byref(n))
        self.nparams = int(n.value)

    def close(self):
        if getattr(self, "h", None):
            self.lib.kls_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _f(a) -> C.POINTER(C.c_float):
        return a.ctypes.data_as(C.POINTER(C.c_float))

    def _ck(self, code):
        if code:
            raise _lib.KlsError(code, self.lib.kls_create_error().decode())

    def params(self) -> np.ndarray:
        p = np.empty(self.nparams, dtype=np.float32)
        self._ck(self.lib.kls_mlp_get_params(self.h, self._f(p)))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.nparams:
            raise ValueError(f"expected {self.nparams} parameters, got {p.size}")
        self._ck(self.lib.kls_mlp_set_params(self.h, self._f(p)))

    @staticmethod
    def _rows(A: np.ndarray, width: int, n: Optional[int] = None) -> np.ndarray:
        """A as contiguous float32 [n, width]; the library reads n * width
        floats, so any other shape is an error here."""
        A = np.ascontiguousarray(A, dtype=np.float32)
        if A.ndim != 2 or A.shape[1] != width or (n is not None and A.shape[0] != n):
            raise ValueError(f"expected a [{'n' if n is None else n}, {width}] array, "
                             f"got shape {A.shape}")
        return A

    def forward(self, X: np.ndarray) -> np.ndarray:
        X = self._rows(X, 5)
        Y = np.empty((X.shape[0], 3), dtype=np.float32)
        self._ck(self.lib.kls_mlp_forward(self.h, self._f(X), X.shape[0], self._f(Y)))
        return Y

    def grad(self, X: np.ndarray, T: np.ndarray) -> Tuple[np.ndarray, float]:
        X = self._rows(X, 5)
        T = self._rows(T, 3, X.shape[0])
        g = np.empty(self.nparams, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        self._ck(self.lib.kls_mlp_grad(self.h, self._f(X), self._f(T), X.shape[0], self._f(g),
                                       self._f(loss)))
        return g, float(loss[0])

    def train(self, X: np.ndarray, T: np.ndarray, epochs: int = 40, batch: int = 4096,
              lr: float = 2e-3, seed: int = 0) -> np.ndarray:
        X = self._rows(X, 5)
        T = self._rows(T, 3, X.shape[0])
        hist = np.zeros(max(epochs, 1), dtype=np.float32)
        self._ck(self.lib.kls_mlp_train(self.h, self._f(X), self._f(T), X.shape[0], epochs, batch,
                                        lr, seed, self._f(hist)))
        return hist[:epochs]


# ---------------------------------------------------------------------------
# training data from batched scans of random models
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class ModelSpec:
    n_zang: int
    q1: float
    m: int
    size: Optional[Tuple[int, int, int, int]] = None    # (NR, Ne, N_alpha, l_max)


# the three disk-model sizes of the uneven batched scan
SIZES = ((101, 21, 101, 25), (301, 31, 201, 60), (501, 51, 301, 100))


def random_models(n: int, seed: int, sizes: Optional[Sequence[Tuple[int, int, int, int]]] = None
                  ) -> List[ModelSpec]:
    """n_zang in {2..6}, q1 ~ U[4, 12] (real), m in {2, 3}; size drawn from
    `sizes` when given (else the base configuration's)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nz, q1, m = int(rng.integers(2, 7)), float(rng.uniform(4.0, 12.0)), int(rng.integers(2, 4))
        size = tuple(sizes[int(rng.integers(0, len(sizes)))]) if sizes else None
        out.append(ModelSpec(nz, q1, m, size))
    return out


def model_config(base: KalnajsConfig, spec: ModelSpec) -> KalnajsConfig:
    c = copy_config(base)
    c.model.n_zang, c.model.q1, c.physics.m = spec.n_zang, spec.q1, spec.m
    if spec.size is not None:
        NR, Ne, Na, lmax = spec.size
        c.grid.NR, c.grid.Ne, c.grid.N_alpha = NR, Ne, Na
        c.grid.l_min, c.grid.l_max = -lmax, lmax
    return c


def scan_samples(base: KalnajsConfig, specs: Sequence[ModelSpec], n_Op: int, n_gamma: int,
                 Op_range=(0.2, 0.8), g_range=(0.01, 0.30), mixed: bool = True,
                 device: int = 0, batch: int = 16, chunk: int = 0):
    """Features and targets of every (model, omega) point of batched scans
    over the models (api.ModelBatch: every pass is one launch over the uneven
    batch).  ``chunk`` > 0 scans that many models per batch, with mixed-only
    contexts (FP64 tables released), so that many large models fit one GPU."""
    from . import api
    groups = [list(specs)] if chunk <= 0 else [list(specs[i:i + chunk])
                                              for i in range(0, len(specs), chunk)]
    ds, las = [], []
    for group in groups:
        pcs = []
        try:
            for sp in group:
                pc = api.precompute_all(model_config(base, sp), device=device)
                pcs.append(pc)
                if chunk > 0 and mixed:
                    api.release_fp64(pc)
            mb = api.ModelBatch(pcs, "Float32" if mixed else "Float64", batch=batch)
            dd, ll, _, _ = mb.scan(n_Op, n_gamma, Op_range, g_range)  # [models, n_gamma, n_Op]
            mb.close()
            ds.append(dd)
            las.append(ll)
        finally:
            for pc in pcs:
                pc.close()
    d, la = np.concatenate(ds), np.concatenate(las)
    Op = np.linspace(*Op_range, n_Op)
    gm = np.linspace(*g_range, n_gamma)
    OP, GM = np.meshgrid(Op, gm, indexing="xy")                   # [n_gamma, n_Op]
    Xs, Ts = [], []
    for i, spec in enumerate(specs):
        di, li = d[i].ravel(), la[i].ravel()
        ok = np.isfinite(li) & np.isfinite(di)
        Xs.append(features(spec.n_zang, spec.q1, spec.m, OP.ravel()[ok], GM.ravel()[ok]))
        Ts.append(targets(di[ok], li[ok]))
    return np.concatenate(Xs), np.concatenate(Ts)


def shortlist(mlp: MLP, spec: ModelSpec, k: int = 48, n_Op: int = 41, n_gamma: int = 20,
              Op_range=(0.2, 0.6), g_range=(0.01, 0.2)):
    """The k points of the scan grid with the lowest predicted log|det|.

    The grid is the reference scan's (ScanConfig defaults,
    Configuration.jl:72-79); returns (Omega_p, gamma, column-major index)
    arrays sorted by that index.
    """
    Op = np.linspace(*Op_range, n_Op)
    gm = np.linspace(*g_range, n_gamma)
    OP, GM = np.meshgrid(Op, gm, indexing="xy")           # [n_gamma, n_Op]
    y = mlp.forward(features(spec.n_zang, spec.q1, spec.m, OP.ravel(order="F"),
                             GM.ravel(order="F")))
    idx = np.sort(np.argsort(y[:, 0], kind="stable")[:k])   # column-major grid indices
    return OP.ravel(order="F")[idx], GM.ravel(order="F")[idx], idx


def propose(mlp: MLP, spec: ModelSpec, det_fn, k: int = 48, descend: int = 6,
            edge_rows: int = 1, **grid) -> Tuple[float, float, int]:
    """Newton start in place of grid_scan + find_minimum (GridScan.jl:25-88, 234-246).

    ``det_fn(omegas) -> dets`` evaluates the true determinant at the k
    shortlisted grid points and at the ``edge_rows`` grid rows of lowest
    gamma (one batch): next to the real axis the resonant denominators make
    |det| vary on scales finer than the network resolves, and modes of
    small gamma put the scan's argmin on that row.  From the point of
    minimal |det| a descent on the scan grid follows: the point's unevaluated
    8 neighbours are evaluated (one batch) and the start moves to the lowest
    |det| seen, up to ``descend`` times or until it stays, so a shortlist that
    lands next to the scan's argmin still finds it.  Ties go to the first
    point in column-major order, as find_minimum takes it.  When the scan's
    own argmin is the lowest point reached this is exactly the scan's start.
    Returns (Omega_p, gamma, determinant evaluations used).
    """
    n_Op, n_gamma = grid.get("n_Op", 41), grid.get("n_gamma", 20)
    Op_g = np.linspace(*grid.get("Op_range", (0.2, 0.6)), n_Op)
    g_g = np.linspace(*grid.get("g_range", (0.01, 0.2)), n_gamma)
    _, _, idx = shortlist(mlp, spec, k=k, **grid)
    at = lambda q: (float(Op_g[q // n_gamma]), float(g_g[q % n_gamma]))
    known = {}

    def evaluate(qs):
        pts = np.array([spec.m * at(q)[0] + 1j * at(q)[1] for q in qs])
        for q, v in zip(qs, np.abs(np.asarray(det_fn(pts)))):
            known[int(q)] = float(v)

    edge = [a * n_gamma + b for a in range(n_Op) for b in range(min(edge_rows, n_gamma))]
    evaluate(sorted(set(int(q) for q in idx) | set(edge)))
    best = min(known, key=lambda q: (known[q], q))
    for _ in range(descend):
        iO, ig = best // n_gamma, best % n_gamma
        nb = [a * n_gamma + b for a in range(iO - 1, iO + 2) for b in range(ig - 1, ig + 2)
              if 0 <= a < n_Op and 0 <= b < n_gamma and a * n_gamma + b not in known]
        if not nb:
            break
        evaluate(nb)
        nxt = min(known, key=lambda q: (known[q], q))
        if nxt == best:
            break
        best = nxt
    return at(best)[0], at(best)[1], len(known)


@dataclasses.dataclass
class RootResult:
    """find_root outcome: the Newton result and how its start was found."""
    newton: object                 # api.NewtonResult of the refinement
    start: Tuple[float, float]
    source: str                    # "proposal", "proposal_fp64" or "grid_scan"
    proposal_dets: int             # determinants spent on the proposal
    scan_dets: int                 # determinants spent on the fallback scan (0 if none)


def find_root(mlp: MLP, config: KalnajsConfig, precomputed, k: int = 48,
              min_gamma: float = 1e-4, refine: str = "fp64") -> RootResult:
    """Newton root of det(I - M) with a learned start and the scan as fallback.

    The proposal (``propose`` over the config's scan grid, split-BF16
    determinants) is refined by plain FP64 Newton (``refine="fp64"``,
    newton_search: the reference's iteration, so a start equal to the scan's
    argmin gives the scan's root exactly; 28 of 29 held-out default-size
    models reach the scan's root) or by ``newton_search_hybrid`` with FP64
    far steps down to 2e-3 (``refine="hybrid"``: 2-3x faster, 22 of 29; near
    the real axis its split-BF16 steps can leave the reference's path), with
    plain FP64 Newton from the same start when the hybrid does not converge.
    If no growing mode (gamma > min_gamma) is reached, the reference workflow
    runs instead: the full grid scan (GridScan.jl:25-88) in the split-BF16
    form and the same refinement from its argmin.
    """
    from . import api
    if refine not in ("fp64", "hybrid"):
        raise ValueError(f"refine must be 'fp64' or 'hybrid', not {refine!r}")
    s = config.scan
    spec = ModelSpec(int(config.model.n_zang), float(config.model.q1), int(config.physics.m))
    dev = api.to_device(precomputed, api.GPUType.NVIDIA, "Float32")
    Op, g, used = propose(mlp, spec, lambda om: api.compute_determinant_batched(
        om, precomputed, dev, batch_size=16), k=k, n_Op=s.n_Op, n_gamma=s.n_gamma,
        Op_range=(s.Omega_p_min, s.Omega_p_max), g_range=(s.gamma_min, s.gamma_max))

    def fp64(Op0, g0):
        return api.newton_search(config, precomputed, None, api.GPUType.NVIDIA, "Float64", Op0, g0)

    def hybrid(Op0, g0):
        # a grid point is a coarse start: steps longer than 2e-3 are taken
        # with FP64 accuracy, on the reference's path
        return api.newton_search_hybrid(config, precomputed, Op0, g0,
                                        api.HybridConfig(far_step=2e-3))

    if refine == "fp64":
        r = fp64(Op, g)
        if r.converged and r.gamma > min_gamma:
            return RootResult(r, (Op, g), "proposal_fp64", used, 0)
    else:
        r = hybrid(Op, g)
        if r.converged and r.gamma > min_gamma:
            return RootResult(r, (Op, g), "proposal", used, 0)
        if not r.converged:
            # the arbiter: plain FP64 Newton from the same start
            r = fp64(Op, g)
            if r.converged and r.gamma > min_gamma:
                return RootResult(r, (Op, g), "proposal_fp64", used, 0)
    _, Op0, g0 = api.grid_scan(config, precomputed, dev)
    r = fp64(Op0, g0) if refine == "fp64" else hybrid(Op0, g0)
    return RootResult(r, (Op0, g0), "grid_scan", used, s.n_Op * s.n_gamma)
