"""TOML configuration with the reference's schema and defaults.

Mirrors ``src/KalnajsLogSpiral/Configuration.jl``: the section structs
(:31-149) with identical field names and defaults, ``load_config`` (:160-261),
``load_model`` (:269-300), ``save_config`` (:307-371) and the helpers
``get_float_type`` / ``get_complex_type`` / ``get_n_l`` / ``get_NPh``
(:380-416).  A missing file raises ``FileNotFoundError`` with the reference's
message (its ``error(...)`` at :162 and :271).

Deviation, stated: ``ModelConfig.q1`` accepts real values (the reference
types it ``Int``, :42); integer input behaves identically.
"""
from __future__ import annotations

import dataclasses
import os
import tomllib
from dataclasses import dataclass, field
from typing import Any, Dict, List


@dataclass
class PhysicsConfig:
    m: int = 2
    G: float = 1.0


@dataclass
class ModelConfig:
    L0: float = 1.0
    n_zang: int = 4
    q1: float = 7


@dataclass
class GridConfig:
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
    # alpha, ln Rc and v quadrature rules, t / s / b each (the --quad option
    # of NL_julia_boole.jl:14-16); "tts" is the package's choice
    quadrature: str = "tts"


@dataclass
class ScanConfig:
    n_Op: int = 41
    n_gamma: int = 20
    Omega_p_min: float = 0.2
    Omega_p_max: float = 0.6
    gamma_min: float = 0.01
    gamma_max: float = 0.2


@dataclass
class NewtonConfig:
    max_iter: int = 50
    tol: float = 1e-10
    delta: float = 1e-6
    use_line_search: bool = True
    max_line_search: int = 10
    use_complex_step: bool = True
    complex_step_h: float = 1e-20
    enable_convergence_study: bool = False


@dataclass
class GPUConfig:
    backend: str = "auto"
    precision_double: bool = False
    devices: List[int] = field(default_factory=list)


@dataclass
class CPUConfig:
    precision_double: bool = False
    max_threads: int = 32


@dataclass
class IOConfig:
    output_path: str = "results"
    save_intermediate: bool = False
    verbose: bool = True


@dataclass
class ReferenceConfig:
    Omega_p: float = 0.44
    gamma: float = 0.13


@dataclass
class KalnajsConfig:
    physics: PhysicsConfig = field(default_factory=PhysicsConfig)
    model: ModelConfig = field(default_factory=ModelConfig)
    grid: GridConfig = field(default_factory=GridConfig)
    scan: ScanConfig = field(default_factory=ScanConfig)
    newton: NewtonConfig = field(default_factory=NewtonConfig)
    gpu: GPUConfig = field(default_factory=GPUConfig)
    cpu: CPUConfig = field(default_factory=CPUConfig)
    io: IOConfig = field(default_factory=IOConfig)
    reference: ReferenceConfig = field(default_factory=ReferenceConfig)


def check_quadrature(q: str) -> None:
    """Three rule letters (alpha, ln Rc, v), each t / s / b."""
    if not (isinstance(q, str) and len(q) == 3 and all(ch in "tsb" for ch in q)):
        raise ValueError(f"grid.quadrature must be 3 letters of t/s/b (alpha, Rc, v), got {q!r}")


def _apply(obj: Any, data: Dict[str, Any], keys) -> None:
    for k in keys:
        if k in data:
            setattr(obj, k, data[k])


def load_config(filepath: str) -> KalnajsConfig:
    """Configuration.jl:160-261."""
    if not os.path.isfile(filepath):
        raise FileNotFoundError(f"Configuration file not found: {filepath}")
    with open(filepath, "rb") as f:
        data = tomllib.load(f)
    c = KalnajsConfig()
    if "physics" in data:
        _apply(c.physics, data["physics"], ("m", "G"))
    if "model" in data:
        _apply(c.model, data["model"], ("L0", "n_zang", "q1"))
    if "grid" in data:
        _apply(c.grid, data["grid"], ("NR", "Ne", "Rc_min", "Rc_max", "v_min", "N_alpha",
                                      "alpha_max", "l_min", "l_max", "nw", "nwa", "quadrature"))
        check_quadrature(c.grid.quadrature)
    if "scan" in data:
        _apply(c.scan, data["scan"], ("n_Op", "n_gamma", "Omega_p_min", "Omega_p_max",
                                      "gamma_min", "gamma_max"))
    if "newton" in data:
        _apply(c.newton, data["newton"], ("max_iter", "tol", "delta", "use_line_search",
                                          "max_line_search", "use_complex_step",
                                          "complex_step_h", "enable_convergence_study"))
    if "precision" in data:
        p = data["precision"]
        if "gpu_double_precision" in p:
            c.gpu.precision_double = p["gpu_double_precision"]
        if "cpu_double_precision" in p:
            c.cpu.precision_double = p["cpu_double_precision"]
    if "gpu" in data:
        g = data["gpu"]
        if "backend" in g:
            c.gpu.backend = str(g["backend"])
        if "precision_double" in g:
            c.gpu.precision_double = g["precision_double"]
        if "devices" in g:
            c.gpu.devices = list(g["devices"])
    if "cpu" in data:
        _apply(c.cpu, data["cpu"], ("precision_double", "max_threads"))
    if "io" in data:
        _apply(c.io, data["io"], ("output_path", "save_intermediate", "verbose"))
    return c


def load_model(config: KalnajsConfig, filepath: str) -> KalnajsConfig:
    """Configuration.jl:269-300: [physics], [model] (G may sit here) and [reference]."""
    if not os.path.isfile(filepath):
        raise FileNotFoundError(f"Model file not found: {filepath}")
    with open(filepath, "rb") as f:
        data = tomllib.load(f)
    if "physics" in data:
        _apply(config.physics, data["physics"], ("m", "G"))
    if "model" in data:
        m = data["model"]
        _apply(config.model, m, ("L0", "n_zang", "q1"))
        if "G" in m:
            config.physics.G = m["G"]
    if "reference" in data:
        _apply(config.reference, data["reference"], ("Omega_p", "gamma"))
    return config


def _toml_value(v: Any) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, str):
        return f'"{v}"'
    if isinstance(v, list):
        return "[" + ", ".join(_toml_value(x) for x in v) + "]"
    return repr(v)


def save_config(config: KalnajsConfig, filepath: str) -> None:
    """Configuration.jl:307-371 (same sections and keys)."""
    sections = [
        ("physics", config.physics, ("m", "G")),
        ("model", config.model, ("L0", "n_zang", "q1")),
        ("grid", config.grid, ("NR", "Ne", "Rc_min", "Rc_max", "v_min", "N_alpha", "alpha_max",
                               "l_min", "l_max", "nw", "nwa", "quadrature")),
        ("scan", config.scan, ("n_Op", "n_gamma", "Omega_p_min", "Omega_p_max", "gamma_min",
                               "gamma_max")),
        ("newton", config.newton, ("max_iter", "tol", "delta", "use_line_search",
                                   "use_complex_step", "enable_convergence_study")),
        ("gpu", config.gpu, ("backend", "precision_double", "devices")),
        ("cpu", config.cpu, ("precision_double", "max_threads")),
        ("io", config.io, ("output_path", "save_intermediate", "verbose")),
    ]
    with open(filepath, "w") as f:
        f.write("# Kalnajs Log-Spiral Configuration\n\n")
        for name, obj, keys in sections:
            f.write(f"[{name}]\n")
            for k in keys:
                f.write(f"{k} = {_toml_value(getattr(obj, k))}\n")
            f.write("\n")


def get_float_type(config: KalnajsConfig, for_gpu: bool = True) -> str:
    """'Float64' or 'Float32' (Configuration.jl:380-386)."""
    dbl = config.gpu.precision_double if for_gpu else config.cpu.precision_double
    return "Float64" if dbl else "Float32"


def get_complex_type(config: KalnajsConfig, for_gpu: bool = True) -> str:
    dbl = config.gpu.precision_double if for_gpu else config.cpu.precision_double
    return "ComplexF64" if dbl else "ComplexF32"


def get_n_l(config: KalnajsConfig) -> int:
    return config.grid.l_max - config.grid.l_min + 1


def get_NPh(config: KalnajsConfig) -> int:
    return config.grid.NR * config.grid.Ne


def precision_gpu(config: KalnajsConfig) -> str:
    return get_float_type(config, True)


def precision_cpu(config: KalnajsConfig) -> str:
    return get_float_type(config, False)


def copy_config(config: KalnajsConfig) -> KalnajsConfig:
    return dataclasses.replace(config, **{f.name: dataclasses.replace(getattr(config, f.name))
                                          for f in dataclasses.fields(config)})
