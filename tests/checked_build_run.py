"""Run the FP64 determinant path on libkls_checked.so (run as a script).

Loaded first in a fresh process, the bounds-checked build serves every call
of the package.  At three shapes the default build's parity tests use (the
smoke shape and the `general` and `radial_retro` fixtures) it evaluates three
determinants in the 4M and 3M contraction forms and with both LU forms,
compares them with the oracle (relative error <= 1e-11, the determinant
tolerance of the parity tests) and reads kls_bounds_report, which must count
no skipped access.  Prints CHECKED_OK and exits 0 when all of that holds.
"""
import ctypes as C
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from kalnajs_log_spirals_b200 import _lib  # noqa: E402

LIB = _lib.load(_lib.CHECKED_LIB_PATH)     # before any other load: the API runs on it

import kalnajs_log_spirals_b200 as K  # noqa: E402
from oracle import np_oracle as O  # noqa: E402
from tests.golden.make_fixtures import BASE, CASES  # noqa: E402
from tests.test_gpu_parity import kconfig  # noqa: E402

SMOKE = dict(m=2, G=1.0, L0=1.0, n_zang=4, q1=7, NR=12, Ne=7, Rc_min=0.01, Rc_max=10.0,
             v_min=0.01, N_alpha=17, alpha_max=10.0, l_min=-4, l_max=4, nw=401, nwa=41)


def report(reset=True):
    v, site, idx, ext = C.c_int64(), C.c_int32(), C.c_int64(), C.c_int64()
    code = LIB.kls_bounds_report(C.byref(v), C.byref(site), C.byref(idx), C.byref(ext),
                                 int(reset))
    return code, v.value, site.value, idx.value, ext.value


def main() -> int:
    ok = True
    for name, over in (("smoke", SMOKE), ("general", {**BASE, **CASES["general"]}),
                       ("radial_retro", {**BASE, **CASES["radial_retro"]})):
        pc = K.precompute_all(kconfig(**over), device=0)
        om = np.array([0.88 + 0.12j, 0.7 + 0.05j, 1.1 + 0.2j])
        d4 = K.compute_determinant_batched(om, pc)
        pc.ctx.call("kls_set_lu_mode", _lib.KLS_LU_CLUSTER)
        dcl = K.compute_determinant_batched(om, pc)
        pc.ctx.call("kls_set_lu_mode", _lib.KLS_LU_CTA)
        pc.ctx.call("kls_set_f64_form", _lib.KLS_F64_3M)
        d3 = K.compute_determinant_batched(om, pc)
        pc.close()
        opc = O.precompute_all(O.OracleConfig(**over))
        do = np.array([O.compute_det(opc, w) for w in om])
        e4 = float(np.max(np.abs(d4 - do) / np.abs(do)))
        e3 = float(np.max(np.abs(d3 - do) / np.abs(do)))
        code, n, site, idx, ext = report()
        print(f"{name}: report code {code} violations {n} (site {site}, index {idx}, extent "
              f"{ext}); 4M err {e4:.2e}, 3M err {e3:.2e}, cluster LU bitwise "
              f"{np.array_equal(d4, dcl)}", flush=True)
        ok = ok and code == 0 and n == 0 and e4 <= 1e-11 and e3 <= 1e-11
    print("CHECKED_OK" if ok else "CHECKED_FAIL", flush=True)
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
