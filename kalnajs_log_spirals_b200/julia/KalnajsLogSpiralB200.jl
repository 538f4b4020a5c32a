# KalnajsLogSpiralB200.jl — Julia binding of libkls.so with the reference
# package's API (src/KalnajsLogSpiral.jl:23-43).  It reuses the reference's
# Configuration module for TOML parsing and replaces precompute_all,
# to_device, compute_determinant(_batched), grid_scan and newton_search with
# ccalls into libkls.so (include/kls.h), and adds newton_search_hybrid,
# grid_scan_multi, autotune and release_fp64.  Not exercised in this repository's
# tests (no Julia toolchain in the build image); the Python mirror in
# kalnajs_log_spirals_b200/api.py calls the same entry points.
module KalnajsLogSpiralB200

const LIBKLS = get(ENV, "LIBKLS", joinpath(@__DIR__, "..", "libkls.so"))

const KLS_MODE_FP64 = Int32(0)
const KLS_MODE_MIXED = Int32(1)
const KLS_MODE_ANCHORED = Int32(2)

# kls_config (include/kls.h), field order and C types
struct KlsConfig
    m::Int32; G::Float64; L0::Float64; n_zang::Int32; q1::Float64
    NR::Int32; Ne::Int32; Rc_min::Float64; Rc_max::Float64; v_min::Float64
    N_alpha::Int32; alpha_max::Float64; l_min::Int32; l_max::Int32
    nw::Int32; nwa::Int32
    quad_alpha::Int32; quad_rc::Int32; quad_v::Int32   # 0: the package's rules
end

struct KlsNewtonCfg
    max_iter::Int32; tol::Float64; delta::Float64
    use_line_search::Int32; max_line_search::Int32; mode::Int32
end

mutable struct KlsNewtonResult
    Omega_p::Float64; gamma::Float64; omega_re::Float64; omega_im::Float64
    det_re::Float64; det_im::Float64; iterations::Int32; converged::Int32; det_evals::Int32
end
KlsNewtonResult() = KlsNewtonResult(0, 0, 0, 0, 0, 0, 0, 0, 0)

struct KlsScanCfg
    n_Op::Int32; n_gamma::Int32; Omega_p_min::Float64; Omega_p_max::Float64
    gamma_min::Float64; gamma_max::Float64; mode::Int32; batch::Int32
end

struct NewtonResult{T<:AbstractFloat}
    Omega_p::T; gamma::T; omega::Complex{T}; det_val::Complex{T}
    iterations::Int; converged::Bool; history::Matrix{T}
end

mutable struct PrecomputedData
    handle::Ptr{Cvoid}
    m::Int; G::Float64; N_alpha::Int; n_l::Int; NPh::Int
end

struct DevicePrecomputed
    precomp::PrecomputedData
    mode::Int32
end

function check(h, code)
    code == 0 && return
    msg = h == C_NULL ? unsafe_string(ccall((:kls_create_error, LIBKLS), Cstring, ())) :
                        unsafe_string(ccall((:kls_last_error, LIBKLS), Cstring, (Ptr{Cvoid},), h))
    error("libkls status $code: $msg")
end

const QUAD_CODES = Dict('t' => Int32(1), 's' => Int32(2), 'b' => Int32(3))

"""Quadrature rules of the alpha, ln Rc and v grids: the `quadrature` field of
the grid config when it has one (three letters of t/s/b, the --quad option of
NL_julia_boole.jl:14-16), else the package's rules ("tts")."""
function quad_codes(g)
    q = hasproperty(g, :quadrature) ? String(getproperty(g, :quadrature)) : "tts"
    (length(q) == 3 && all(c -> haskey(QUAD_CODES, c), q)) ||
        error("grid quadrature must be 3 letters of t/s/b (alpha, Rc, v), got $q")
    q == "tts" && return (Int32(0), Int32(0), Int32(0))
    return (QUAD_CODES[q[1]], QUAD_CODES[q[2]], QUAD_CODES[q[3]])
end

function kls_config(config, model)
    g = config.grid
    qa, qr, qv = quad_codes(g)
    KlsConfig(config.physics.m, config.physics.G, config.model.L0, config.model.n_zang,
              Float64(config.model.q1), g.NR, g.Ne, g.Rc_min, g.Rc_max, g.v_min, g.N_alpha,
              g.alpha_max, g.l_min, g.l_max, g.nw, g.nwa, qa, qr, qv)
end

"precompute_all (BasisFunctions.jl:73): grids, orbits, W_l, N_m on the GPU."
function precompute_all(config, model, backend; verbose::Bool=false, device::Int=0)
    cfg = Ref(kls_config(config, model))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(C_NULL, ccall((:kls_create, LIBKLS), Cint, (Ref{KlsConfig}, Cint, Ref{Ptr{Cvoid}}),
                        cfg, device, h))
    check(h[], ccall((:kls_precompute, LIBKLS), Cint, (Ptr{Cvoid},), h[]))
    pc = PrecomputedData(h[], config.physics.m, config.physics.G, config.grid.N_alpha,
                         config.grid.l_max - config.grid.l_min + 1, config.grid.NR * config.grid.Ne)
    finalizer(p -> ccall((:kls_destroy, LIBKLS), Cint, (Ptr{Cvoid},), p.handle), pc)
    return pc
end

"to_device (BasisFunctions.jl:397): Float64 -> plain FP64, Float32 -> split-BF16 form."
function to_device(precomp::PrecomputedData, gpu_type, Tgpu::Type)
    mode = Tgpu === Float64 ? KLS_MODE_FP64 : KLS_MODE_MIXED
    if mode == KLS_MODE_MIXED
        check(precomp.handle, ccall((:kls_prepare_mixed, LIBKLS), Cint, (Ptr{Cvoid},), precomp.handle))
    end
    return DevicePrecomputed(precomp, mode)
end

modeof(d) = d === nothing ? KLS_MODE_FP64 : d.mode

"compute_determinant_batched (MatrixBuilder.jl:215)."
function compute_determinant_batched(omegas::Vector{ComplexF64}, precomp::PrecomputedData,
                                     devprecomp, gpu_type, Tcpu::Type; batch_size::Int=100)
    out = Vector{ComplexF64}(undef, length(omegas))
    for s in 1:batch_size:length(omegas)
        e = min(s + batch_size - 1, length(omegas))
        om = omegas[s:e]
        det = Vector{ComplexF64}(undef, length(om))
        check(precomp.handle, ccall((:kls_det_batch, LIBKLS), Cint,
              (Ptr{Cvoid}, Ptr{ComplexF64}, Cint, Cint, Ptr{ComplexF64}, Ptr{Float64}),
              precomp.handle, om, length(om), modeof(devprecomp), det, C_NULL))
        out[s:e] .= det
    end
    return out
end

"compute_determinant (MatrixBuilder.jl:197)."
compute_determinant(omega::ComplexF64, precomp::PrecomputedData, devprecomp, gpu_type, Tcpu::Type) =
    compute_determinant_batched([omega], precomp, devprecomp, gpu_type, Tcpu)[1]

"grid_scan (GridScan.jl:25) -> (det_grid, Omega_p_init, gamma_init)."
function grid_scan(config, precomp::PrecomputedData, devprecomp, gpu_type, Tcpu::Type;
                   verbose::Bool=false, gpu_devices::Vector{Int}=Int[])
    s = config.scan
    sc = Ref(KlsScanCfg(s.n_Op, s.n_gamma, s.Omega_p_min, s.Omega_p_max, s.gamma_min,
                        s.gamma_max, modeof(devprecomp), 0))
    det_grid = Matrix{ComplexF64}(undef, s.n_gamma, s.n_Op)
    Op0 = Ref(0.0); g0 = Ref(0.0)
    check(precomp.handle, ccall((:kls_scan, LIBKLS), Cint,
          (Ptr{Cvoid}, Ref{KlsScanCfg}, Ptr{ComplexF64}, Ptr{Float64}, Ref{Float64}, Ref{Float64}),
          precomp.handle, sc, det_grid, C_NULL, Op0, g0))
    return det_grid, Op0[], g0[]
end

"newton_search (NewtonSolver.jl:36) -> NewtonResult."
function newton_search(config, precomp::PrecomputedData, devprecomp, gpu_type, Tcpu::Type,
                       Omega_p_init::Real, gamma_init::Real; verbose::Bool=false)
    n = config.newton
    nc = Ref(KlsNewtonCfg(n.max_iter, n.tol, n.delta, n.use_line_search, n.max_line_search,
                          modeof(devprecomp)))
    res = Ref(KlsNewtonResult())
    hist = zeros(Float64, 3, n.max_iter)          # row-major (iter, 3) on the C side
    check(precomp.handle, ccall((:kls_newton, LIBKLS), Cint,
          (Ptr{Cvoid}, Cdouble, Cdouble, Ref{KlsNewtonCfg}, Ref{KlsNewtonResult}, Ptr{Float64}),
          precomp.handle, Omega_p_init, gamma_init, nc, res, hist))
    r = res[]
    h = permutedims(hist[:, 1:r.iterations])
    return NewtonResult{Float64}(r.Omega_p, r.gamma, complex(r.omega_re, r.omega_im),
                                 complex(r.det_re, r.det_im), r.iterations, r.converged != 0, h)
end

# ---- beyond the reference's API --------------------------------------------

struct KlsHybridCfg
    mixed_delta::Float64; mixed_step_tol::Float64; mixed_max_iter::Int32; fp64_max_iter::Int32
    anchor_radius::Float64; final_fp64::Int32; far_step::Float64
end

struct KlsTuneResult
    mode::Int32; splits::Int32; default_splits::Int32; candidates::Int32
    ms_per_omega::Float64; default_ms_per_omega::Float64; form::Int32
end

"""
newton_search_hybrid: split-BF16 secant steps, then an FP64 anchor and
anchored steps to the reference's stopping rule |det| < tol on an
FP64-accurate determinant (kls_newton_hybrid).  Keyword defaults are the
library's recommended ones.
"""
function newton_search_hybrid(config, precomp::PrecomputedData, Omega_p_init::Real,
                              gamma_init::Real; mixed_delta::Real=1e-3,
                              mixed_step_tol::Real=1e-5, mixed_max_iter::Integer=30,
                              fp64_max_iter::Integer=50, anchor_radius::Real=1e-5,
                              final_fp64::Bool=false, far_step::Real=2e-2)
    n = config.newton
    check(precomp.handle, ccall((:kls_prepare_mixed, LIBKLS), Cint, (Ptr{Cvoid},), precomp.handle))
    nc = Ref(KlsNewtonCfg(n.max_iter, n.tol, n.delta, n.use_line_search, n.max_line_search,
                          KLS_MODE_FP64))
    hc = Ref(KlsHybridCfg(mixed_delta, mixed_step_tol, mixed_max_iter, fp64_max_iter,
                          anchor_radius, Int32(final_fp64), far_step))
    res = Ref(KlsNewtonResult())
    evals = zeros(Int32, 3)
    hist = zeros(Float64, 3, n.max_iter)
    check(precomp.handle, ccall((:kls_newton_hybrid, LIBKLS), Cint,
          (Ptr{Cvoid}, Cdouble, Cdouble, Ref{KlsNewtonCfg}, Ref{KlsHybridCfg},
           Ref{KlsNewtonResult}, Ptr{Int32}, Ptr{Float64}),
          precomp.handle, Omega_p_init, gamma_init, nc, hc, res, evals, hist))
    r = res[]
    h = permutedims(hist[:, 1:min(r.iterations, n.max_iter)])
    return NewtonResult{Float64}(r.Omega_p, r.gamma, complex(r.omega_re, r.omega_im),
                                 complex(r.det_re, r.det_im), r.iterations, r.converged != 0, h)
end

"autotune: K split count (and the split-BF16 tile form) chosen by timing (kls_autotune)."
function autotune(precomp::PrecomputedData, Tgpu::Type; batch::Integer=2)
    mode = Tgpu === Float64 ? KLS_MODE_FP64 : KLS_MODE_MIXED
    r = Ref{KlsTuneResult}()
    check(precomp.handle, ccall((:kls_autotune, LIBKLS), Cint,
          (Ptr{Cvoid}, Cint, Cint, Ref{KlsTuneResult}), precomp.handle, mode, batch, r))
    return r[]
end

"release_fp64: keep only the split-BF16 table of a precompute (kls_release_fp64)."
release_fp64(precomp::PrecomputedData) =
    check(precomp.handle, ccall((:kls_release_fp64, LIBKLS), Cint, (Ptr{Cvoid},), precomp.handle))

function multi_error(h)
    unsafe_string(ccall((:kls_multi_last_error, LIBKLS), Cstring, (Ptr{Cvoid},), h))
end

"""
grid_scan_multi: grid_scan (GridScan.jl:25) of many precomputes (any sizes) in
shared launches (kls_multi, kls_scan_multi).  Returns (det_grids
[n_gamma, n_Op, n_models], Omega_p_init [n_models], gamma_init [n_models]).
"""
function grid_scan_multi(config, precomps::Vector{PrecomputedData}, Tgpu::Type;
                         batch::Integer=16)
    mode = Tgpu === Float64 ? KLS_MODE_FP64 : KLS_MODE_MIXED
    if mode == KLS_MODE_MIXED
        for p in precomps
            check(p.handle, ccall((:kls_prepare_mixed, LIBKLS), Cint, (Ptr{Cvoid},), p.handle))
        end
    end
    handles = Ptr{Cvoid}[p.handle for p in precomps]
    mm = Ref{Ptr{Cvoid}}(C_NULL)
    code = ccall((:kls_multi_create, LIBKLS), Cint,
                 (Ptr{Ptr{Cvoid}}, Cint, Cint, Cint, Ref{Ptr{Cvoid}}),
                 handles, length(handles), mode, batch, mm)
    code == 0 || error("libkls status $code: " * multi_error(C_NULL))
    s = config.scan
    nm = length(precomps)
    sc = Ref(KlsScanCfg(s.n_Op, s.n_gamma, s.Omega_p_min, s.Omega_p_max, s.gamma_min,
                        s.gamma_max, mode, batch))
    dets = Array{ComplexF64}(undef, s.n_gamma, s.n_Op, nm)   # column-major block per model
    Op0 = zeros(Float64, nm)
    g0 = zeros(Float64, nm)
    try
        code = ccall((:kls_scan_multi, LIBKLS), Cint,
                     (Ptr{Cvoid}, Ref{KlsScanCfg}, Ptr{ComplexF64}, Ptr{Float64}, Ptr{Float64},
                      Ptr{Float64}), mm[], sc, dets, C_NULL, Op0, g0)
        code == 0 || error("libkls status $code: " * multi_error(mm[]))
    finally
        ccall((:kls_multi_destroy, LIBKLS), Cint, (Ptr{Cvoid},), mm[])
    end
    return dets, Op0, g0
end

end # module
