"""The bindings' structs match include/kls.h field by field (CPU only).

The Julia module cannot run in this image, so its struct layouts and ccall
symbols are checked against the C header as text; the ctypes structs of the
Python binding are checked the same way.
"""
import ctypes as C
import os
import re

from kalnajs_log_spirals_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = open(os.path.join(ROOT, "include", "kls.h")).read()
JULIA = open(os.path.join(ROOT, "kalnajs_log_spirals_b200", "julia",
                          "KalnajsLogSpiralB200.jl")).read()

C_TYPES = {"int32_t": "i32", "double": "f64", "int64_t": "i64"}
JL_TYPES = {"Int32": "i32", "Float64": "f64", "Int64": "i64"}
CT_TYPES = {C.c_int32: "i32", C.c_double: "f64", C.c_int64: "i64"}

PAIRS = {"kls_config": "KlsConfig", "kls_newton_cfg": "KlsNewtonCfg",
         "kls_newton_result": "KlsNewtonResult", "kls_scan_cfg": "KlsScanCfg",
         "kls_hybrid_cfg": "KlsHybridCfg", "kls_tune_result": "KlsTuneResult"}


def c_fields(name):
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), HEADER, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        ctype, names = decl.split(None, 1)
        n = len([x for x in names.split(",") if x.strip()])
        out += [C_TYPES[ctype]] * n
    return out


def jl_fields(name):
    body = re.search(r"struct %s\n(.*?)\nend" % name, JULIA, re.S).group(1)
    body = re.sub(r"#.*", "", body)
    return [JL_TYPES[t] for t in re.findall(r"\w+::(\w+)", body)]


def test_julia_structs_match_header():
    for c_name, jl_name in PAIRS.items():
        assert jl_fields(jl_name) == c_fields(c_name), c_name


def test_ctypes_structs_match_header():
    for c_name in PAIRS:
        ct = getattr(_lib, c_name)
        assert [CT_TYPES[t] for _, t in ct._fields_] == c_fields(c_name), c_name


def test_julia_ccalls_name_declared_symbols():
    used = set(re.findall(r"ccall\(\(:(kls_\w+), LIBKLS\)", JULIA))
    declared = set(re.findall(r"\b(kls_\w+)\(", HEADER))
    assert used and used <= declared, used - declared


def test_julia_passes_the_grid_quadrature():
    codes = dict(re.findall(r"'(\w)' => Int32\((\d)\)", JULIA))
    hdr = {k: v for k, v in re.findall(r"#define KLS_QUAD_(\w+)\s+(\d)", HEADER)}
    assert codes == {"t": hdr["TRAPEZOID"], "s": hdr["SIMPSON"], "b": hdr["BOOLE"]}
    assert "g.nw, g.nwa, qa, qr, qv)" in JULIA
