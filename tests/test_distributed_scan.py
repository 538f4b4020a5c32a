"""Omega-sharded grid scan and K-sharded determinants over processes (gloo,
world size 2, CPU).

The host logic of api.grid_scan_distributed (column split as in
GridScan.jl:133-144, one all_gather of the det blocks, column-major argmin)
runs on CPU ranks; each rank's column block comes from the oracle, so the
gathered grid must equal the single-process oracle scan exactly.  A rank that
fails before the collective makes the other rank's all_gather end with an
error within the process-group timeout instead of waiting for ever.
"""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import kalnajs_log_spirals_b200 as K
from oracle import np_oracle as O
from tests.golden.make_fixtures import BASE

SCAN = dict(n_Op=5, n_gamma=3, Omega_p_min=0.3, Omega_p_max=0.5, gamma_min=0.05, gamma_max=0.15)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _config():
    c = K.KalnajsConfig()
    c.physics.m = BASE["m"]
    for k, v in SCAN.items():
        setattr(c.scan, k, v)
    return c


def _oracle_columns():
    pc = O.precompute_all(O.OracleConfig(**BASE))

    def cols(Op_cols, g_grid, m):
        return np.array([[O.compute_det(pc, complex(m * Op, g)) for Op in Op_cols] for g in g_grid],
                        dtype=np.complex128).reshape(len(g_grid), len(Op_cols))
    return cols


def _rank(rank, world, port, fail_rank, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=8))
    try:
        if rank == fail_rank:
            raise RuntimeError("rank failed before the collective")
        det, Op0, g0 = K.grid_scan_distributed(_config(), column_fn=_oracle_columns())
        q.put((rank, "ok", det, Op0, g0))
    except Exception as e:           # reported to the test, never swallowed
        q.put((rank, "error", repr(e), None, None))
    finally:
        if rank != fail_rank:
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def _rank_k(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=8))
    try:
        pc = O.precompute_all(O.OracleConfig(**BASE))
        lo, hi = K.harmonic_ranges(BASE["l_min"], BASE["l_max"], world)[rank]
        il = range(lo - BASE["l_min"], hi - BASE["l_min"] + 1)     # this rank's harmonics
        d = K.compute_determinant_ksharded(
            OMEGAS, _config(), M_fn=lambda w: O.build_M(pc, w, l_range=il),
            det_fn=lambda a: np.linalg.det(a))
        q.put((rank, "ok", d, None, None))
    except Exception as e:
        q.put((rank, "error", repr(e), None, None))
    finally:
        dist.destroy_process_group()


OMEGAS = [0.88 + 0.12j, 0.6 + 0.05j, 1.2 + 0.3j]


def _run(world, fail_rank=-1, target=None):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    if target is None:
        ps = [ctx.Process(target=_rank, args=(r, world, port, fail_rank, q)) for r in range(world)]
    else:
        ps = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda t: t[0])


def test_sharded_scan_equals_single_process_scan():
    res = _run(2)
    pc = O.precompute_all(O.OracleConfig(**BASE))
    ref_det, ref_Op, ref_g = O.grid_scan(
        lambda w: O.compute_det(pc, w), BASE["m"],
        SCAN["n_Op"], SCAN["n_gamma"], SCAN["Omega_p_min"], SCAN["Omega_p_max"],
        SCAN["gamma_min"], SCAN["gamma_max"])
    for rank, status, det, Op0, g0 in res:
        assert status == "ok", det
        assert np.array_equal(det, ref_det), rank
        assert (Op0, g0) == (ref_Op, ref_g)


def test_failed_rank_surfaces_as_an_error():
    res = dict((r[0], r[1:]) for r in _run(2, fail_rank=1))
    assert res[1][0] == "error"
    assert res[0][0] == "error"        # the collective ended with an error, not a hang


def test_column_ranges_split_like_the_reference():
    r = K.api.column_ranges(41, 3)
    assert [(x.start, x.stop) for x in r] == [(0, 14), (14, 28), (28, 41)]
    assert [x.stop - x.start for x in K.api.column_ranges(5, 2)] == [3, 2]


def test_k_sharded_determinant_equals_the_full_one():
    """Each rank contracts only its harmonics; the all-reduced M gives the
    full determinant (to the FP64 rounding of a regrouped sum)."""
    res = _run(2, target=_rank_k)
    pc = O.precompute_all(O.OracleConfig(**BASE))
    ref = np.array([O.compute_det(pc, w) for w in OMEGAS])
    for rank, status, d, _, _ in res:
        assert status == "ok", d
        assert np.max(np.abs(d - ref) / np.abs(ref)) < 1e-12, (rank, d, ref)


def test_harmonic_ranges_cover_each_harmonic_once():
    r = K.harmonic_ranges(-100, 100, 8)
    ls = [l for lo, hi in r for l in range(lo, hi + 1)]
    assert ls == list(range(-100, 101))
    assert [hi - lo + 1 for lo, hi in r] == [26] + [25] * 7


def test_static_lu_chunks_fit_the_scratch():
    from kalnajs_log_spirals_b200.api import STATIC_LU_MAX, static_lu_chunks
    assert static_lu_chunks(13, 301) == [(0, 11), (11, 13)]
    assert static_lu_chunks(16, 256) == [(0, 16)]
    assert static_lu_chunks(0, 301) == []
    for n, N in [(100, 301), (7, 1024), (3, 33)]:
        ch = static_lu_chunks(n, N)
        assert ch[0][0] == 0 and ch[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(ch, ch[1:]))
        assert all((hi - lo) * N * N <= STATIC_LU_MAX for lo, hi in ch)
    with pytest.raises(K.KlsError):
        static_lu_chunks(2, 1025)
