"""Build libkls.so in-tree with nvcc for sm_100a.

``python -m kalnajs_log_spirals_b200.build`` compiles every ``csrc/*.cu`` into
``kalnajs_log_spirals_b200/libkls.so``, and again with ``-DKLS_CHECKED`` into
``kalnajs_log_spirals_b200/libkls_checked.so`` (the bounds-checked build).
Objects go to ``_build/`` (``_build/checked/``) at the repository root; a
translation unit is recompiled when it or a header is newer than its object.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libkls.so")
CHECKED_LIB = os.path.join(PKG, "libkls_checked.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
              "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]
# per-file extra flags: the orbit integrals are ill-conditioned near turning
# points, so they keep the reference's separate multiply/add roundings
EXTRA_FLAGS = {"kls_orbits.cu": ["-fmad=false"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, verbose: bool, checked: bool = False) -> str:
    out_dir = os.path.join(BUILD, "checked") if checked else BUILD
    obj = os.path.join(out_dir, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _headers_mtime()):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *(["-DKLS_CHECKED"] if checked else []),
           *EXTRA_FLAGS.get(os.path.basename(src), []), "-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(out_dir, os.path.basename(src) + ".log")
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr[-6000:]}")
    if verbose:
        print(f"compiled {os.path.basename(src)}{' (checked)' if checked else ''}")
    return obj


def build(verbose: bool = False, checked: bool = False) -> str:
    """Build libkls.so, or with ``checked`` libkls_checked.so; returns its path."""
    lib = CHECKED_LIB if checked else LIB
    os.makedirs(os.path.join(BUILD, "checked") if checked else BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, checked), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", lib, *objs, "-lrt", "-ldl", "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr[-4000:]}")
        if verbose:
            print(f"linked {lib}")
    return lib


if __name__ == "__main__":
    build(verbose="-q" not in sys.argv)
    build(verbose="-q" not in sys.argv, checked=True)
