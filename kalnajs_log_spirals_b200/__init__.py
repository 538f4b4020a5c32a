"""B200 (sm_100a) implementation of the Kalnajs log-spiral matrix-method path.

The numerical work lives in ``libkls.so`` (CUDA kernels behind the C ABI in
``include/kls.h``); this package is the host-side mirror of the reference's
Julia API (``src/KalnajsLogSpiral.jl:23-43``).
"""
from .config import (CPUConfig, GPUConfig, GridConfig, IOConfig, KalnajsConfig, ModelConfig,
                     NewtonConfig, PhysicsConfig, ReferenceConfig, ScanConfig, get_complex_type,
                     get_float_type, get_n_l, get_NPh, load_config, load_model, precision_cpu,
                     precision_gpu, save_config)
from .api import (DevicePrecomputed, GPUType, NewtonResult, OrbitData, PrecomputedData,
                  ModelBatch, ToomreZangModel, TuneResult, autotune, build_M_matrix, compute_determinant,
                  compute_determinant_batched, create_toomre_zang_model, detect_gpu_type,
                  compute_determinant_ksharded, find_minimum, grid_scan, grid_scan_distributed,
                  harmonic_ranges, precompute_ksharded, newton_search, precompute_all, release_fp64,
                  set_anchor, to_device)
from ._lib import KLS_MODE_ANCHORED, KLS_MODE_FP64, KLS_MODE_MIXED, KlsError

__all__ = [
    "KalnajsConfig", "PhysicsConfig", "ModelConfig", "GridConfig", "ScanConfig", "NewtonConfig",
    "GPUConfig", "CPUConfig", "IOConfig", "ReferenceConfig", "load_config", "load_model",
    "save_config", "get_float_type", "get_complex_type", "get_n_l", "get_NPh", "precision_gpu",
    "precision_cpu", "GPUType", "detect_gpu_type", "ToomreZangModel",
    "create_toomre_zang_model", "PrecomputedData", "OrbitData", "precompute_all",
    "DevicePrecomputed", "to_device", "compute_determinant", "compute_determinant_batched",
    "build_M_matrix", "grid_scan", "find_minimum", "newton_search", "NewtonResult", "KlsError",
    "KLS_MODE_FP64", "KLS_MODE_MIXED", "KLS_MODE_ANCHORED", "set_anchor", "ModelBatch",
    "autotune", "TuneResult", "release_fp64", "grid_scan_distributed",
    "harmonic_ranges", "precompute_ksharded", "compute_determinant_ksharded",
]
