# ==============================================================================
# FivoGPU.jl — Julia binding of libfivo2d.so (include/fivo2d.h) for the 2+1D
# driver of FiVoHydro.jl. Include it from main2D.jl after the src2d files:
#
#     include(joinpath(@__DIR__, "..", "fivohydro.jl_b200", "julia", "FivoGPU.jl"))
#
# and pass `work = GPUWork2D(g, model)` to run_sim_2d! (the one-line hook is the
# integrator selection of run_sim_2d!). The stage then runs on the GPU with the reference's own driver
# semantics: the same keywords, the same (ok, Δ) step convention, the same
# NamedTuple result, dumps through on_dump.
# ==============================================================================

const LIBFIVO2D = get(ENV, "FIVO2D_LIB",
                      joinpath(@__DIR__, "..", "csrc", "libfivo2d.so"))

const FIVO_OK = Cint(0)
const FIVO_EOS_CONFORMAL_HQ = Cint(0)
const FIVO_EOS_LATTICE_HRG = Cint(1)
const FIVO_BULK_ZERO, FIVO_BULK_LORENTZ, FIVO_BULK_GAUSS = Cint(0), Cint(1), Cint(2)
const FIVO_SSPRK2, FIVO_SSPRK3 = Cint(2), Cint(3)

# fivo_params, field for field (doubles first, then Int32, then UInt32)
mutable struct FivoParams
    g_eff::Float64; m_hq::Float64; g_hq::Float64
    lhrg_a::NTuple{4,Float64}; lhrg_b::NTuple{4,Float64}
    lhrg_c::Float64; lhrg_d::Float64; canon_factor::Float64
    kappa_coeff::Float64; tauN_coeff::Float64; deltaN_factor::Float64
    nu_clip_factor::Float64; vacuum_n_lo::Float64; vacuum_n_hi::Float64
    eta_over_s::Float64; tauShear_coeff::Float64; deltaShear_factor::Float64
    taupi_pi_factor::Float64; lambda_pi_Pi_factor::Float64; pi_clip_factor::Float64
    zeta_over_s::Float64; tauPi_coeff::Float64; bulk_T0::Float64; bulk_width::Float64
    deltaPi_factor::Float64; lambda_Pi_pi_factor::Float64; Pi_clip_factor::Float64
    r_domain::Float64; T_vac_cut::Float64; E_vac_cut::Float64; primrec_tol::Float64
    transport_mass::Float64
    eos_kind::Int32; hq_times_fmGeV3::Int32; with_charge::Int32
    enable_diff::Int32; enable_shear::Int32; enable_bulk::Int32
    shear_kind::Int32; bulk_kind::Int32
    advect_nu::Int32; relax_advect_nu::Int32; advect_pi::Int32; relax_advect_pi::Int32
    advect_Pi::Int32; relax_advect_Pi::Int32; vacuum_ramp_relax::Int32
    shear_projected_deriv::Int32; diff_projected_deriv::Int32; shear_constraint_project::Int32
    consistent_fm::Int32; consistent_m2::Int32; primrec_maxit::Int32; terms::UInt32
    relax_advect_m2::Int32; reserved0::Int32
    FivoParams() = new()
end

struct FivoRunResult
    ok::Int32; pad0::Int32; tau::Float64; nsteps::Int64; nprimfail::Int64; nvacuum::Int64
    max_shear_res::Float64; maxu::Float64; dQ::Float64; Q0::Float64; Q1::Float64; minPtot::Float64
end

# fivo_lockstep_info: the lockstep batch's candidate schedules and the one kept
struct FivoLockstepInfo
    enabled::Int32; flags::Int32; ncand::Int32; chosen::Int32
    cand_order::NTuple{16,Int32}; cand_slow::NTuple{16,Int32}; cand_fused::NTuple{16,Int32}
    cand_ms::NTuple{16,Float64}
    steps::Int64; fallbacks::Int64; ms_step::Float64; ms_post::Float64; kernels::Int64
end

fivo_error() = unsafe_string(ccall((:fivo_last_error, LIBFIVO2D), Cstring, ()))
fivocheck(st, what) = st == FIVO_OK || error("$what: status $st: $(fivo_error())")

_b(x::Bool) = Int32(x)

"""Flatten an IdealDiffVisc2DModel into fivo_params (src2d/primitives2d.jl:41-210)."""
function fivo_params(model)
    p = FivoParams()
    ccall((:fivo_params_default, LIBFIVO2D), Cvoid, (Ref{FivoParams},), p)
    eos = model.eos
    if eos isa LatticeHRGEOS
        p.eos_kind = FIVO_EOS_LATTICE_HRG
        p.lhrg_a = (eos.a1, eos.a2, eos.a3, eos.a4); p.lhrg_b = (eos.b1, eos.b2, eos.b3, eos.b4)
        p.lhrg_c = eos.c; p.lhrg_d = eos.d; p.canon_factor = eos.canon_factor
    elseif eos isa ConformalHQEOS
        p.eos_kind = FIVO_EOS_CONFORMAL_HQ; p.g_eff = eos.g_eff
    else
        error("FivoGPU: EOS $(typeof(eos)) is not built")
    end
    p.m_hq = eos.m_hq; p.g_hq = eos.g_hq; p.hq_times_fmGeV3 = _b(eos.hq_times_fmGeV3)
    L = model.layout
    p.with_charge = _b(L.hasNu)
    p.enable_diff = _b(model.enable_diff); p.enable_shear = _b(model.enable_shear)
    p.enable_bulk = _b(model.enable_bulk)
    sh = model.shear
    if sh isa QGPViscosity
        p.shear_kind = 1; p.eta_over_s = sh.ηs; p.tauShear_coeff = sh.Cs
    end
    bu = model.bulk
    if bu isa SimpleBulkViscosity
        p.bulk_kind = FIVO_BULK_LORENTZ; p.zeta_over_s = bu.ζs; p.tauPi_coeff = bu.Cζ
    elseif nameof(typeof(bu)) === :GaussianBulkViscosity
        p.bulk_kind = FIVO_BULK_GAUSS; p.zeta_over_s = bu.ζs; p.tauPi_coeff = bu.Cζ
        p.bulk_T0 = bu.T0; p.bulk_width = bu.width
    else
        p.bulk_kind = FIVO_BULK_ZERO
    end
    for f in (:kappa_coeff, :tauN_coeff, :deltaN_factor, :nu_clip_factor, :vacuum_n_lo, :vacuum_n_hi,
              :deltaShear_factor, :taupi_pi_factor, :lambda_pi_Pi_factor, :pi_clip_factor,
              :deltaPi_factor, :lambda_Pi_pi_factor, :Pi_clip_factor, :r_domain, :T_vac_cut, :E_vac_cut,
              :transport_mass)
        setfield!(p, f, Float64(getfield(model, f)))
    end
    for f in (:advect_nu, :relax_advect_nu, :advect_pi, :relax_advect_pi, :advect_Pi, :relax_advect_Pi,
              :vacuum_ramp_relax, :shear_projected_deriv, :diff_projected_deriv, :consistent_fm, :consistent_m2,
              :relax_advect_m2)
        setfield!(p, f, _b(getfield(model, f)))
    end
    p.shear_constraint_project = _b(model.shear_constraint === :project)
    t = model.terms
    p.terms = UInt32(sum(UInt32(getfield(t, n)) << (k - 1) for (k, n) in enumerate(fieldnames(typeof(t)))))
    return p
end

"""A device-resident Work2D: the library context for one (grid, model) pair."""
mutable struct GPUWork2D
    h::Ptr{Cvoid}
    nv::Int
    ntot::Int
    function GPUWork2D(g::Grid2D, model)
        p = fivo_params(model)
        h = Ref{Ptr{Cvoid}}(C_NULL)
        fivocheck(ccall((:fivo_ctx_create, LIBFIVO2D), Cint,
                        (Ref{FivoParams}, Cint, Cint, Cint, Cdouble, Cdouble, Ref{Ptr{Cvoid}}),
                        p, g.Nx, g.Ny, g.nghost, g.xmax, g.ymax, h), "fivo_ctx_create")
        w = new(h[], nvars(model.layout), g.Ntot)
        finalizer(w -> ccall((:fivo_ctx_destroy, LIBFIVO2D), Cint, (Ptr{Cvoid},), w.h), w)
        return w
    end
end

upload!(w::GPUWork2D, U::Matrix{Float64}) =
    fivocheck(ccall((:fivo_upload_state, LIBFIVO2D), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cint, Int64),
                    w.h, U, size(U, 1), size(U, 2)), "fivo_upload_state")
download!(U::Matrix{Float64}, w::GPUWork2D) =
    fivocheck(ccall((:fivo_download_state, LIBFIVO2D), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cint, Int64),
                    w.h, U, size(U, 1), size(U, 2)), "fivo_download_state")

_bc(bc::Symbol) = bc === :periodic ? Cint(1) : Cint(0)

"""step_ssprk2_2d! on the GPU (src2d/timestepper2d.jl:74-103); U is updated in place."""
function step_ssprk2_2d!(U::AbstractMatrix, g::Grid2D, τ::Float64, Δτ::Float64, model, work::GPUWork2D;
                         bc::Symbol = :outflow, max_halve::Int = 12, max_mood::Int = 2)
    upload!(work, U)
    used = Ref{Float64}(0.0); ok = Ref{Cint}(0)
    fivocheck(ccall((:fivo_step, LIBFIVO2D), Cint,
                    (Ptr{Cvoid}, Cint, Cdouble, Cdouble, Cint, Cint, Cint, Ref{Float64}, Ref{Cint}),
                    work.h, FIVO_SSPRK2, τ, Δτ, max_halve, max_mood, _bc(bc), used, ok), "fivo_step")
    download!(U, work)
    return ok[] != 0, used[]
end

"""step_ssprk3_2d! on the GPU (src2d/timestepper2d.jl:148-188)."""
function step_ssprk3_2d!(U::AbstractMatrix, g::Grid2D, τ::Float64, Δτ::Float64, model, work::GPUWork2D;
                         bc::Symbol = :outflow, max_halve::Int = 12)
    upload!(work, U)
    used = Ref{Float64}(0.0); ok = Ref{Cint}(0)
    fivocheck(ccall((:fivo_step, LIBFIVO2D), Cint,
                    (Ptr{Cvoid}, Cint, Cdouble, Cdouble, Cint, Cint, Cint, Ref{Float64}, Ref{Cint}),
                    work.h, FIVO_SSPRK3, τ, Δτ, max_halve, 0, _bc(bc), used, ok), "fivo_step")
    download!(U, work)
    return ok[] != 0, used[]
end

"""rhs_2d! on the GPU (src2d/rhs2d.jl:169-249)."""
function rhs_2d!(dU::AbstractMatrix, U::AbstractMatrix, g::Grid2D, τ::Float64, model, work::GPUWork2D;
                 bc::Symbol = :outflow, Emin::Float64 = E_FLOOR,
                 force_first_order::Union{Nothing,BitVector} = nothing)
    upload!(work, U)
    mask = force_first_order === nothing ? C_NULL : UInt8.(force_first_order)
    fivocheck(ccall((:fivo_rhs, LIBFIVO2D), Cint, (Ptr{Cvoid}, Cdouble, Cint, Ptr{UInt8}, Ptr{Float64}),
                    work.h, τ, _bc(bc), mask, dU), "fivo_rhs")
    download!(U, work)          # rhs_2d! refills the ghost frame of U
    return true
end

"""compute_dt_2d (src2d/timestepper2d.jl:37-47) from the device's last amax."""
function compute_dt_2d(work::GPUWork2D, g::Grid2D, τ::Float64; CFL::Float64 = 0.2, CFLτ::Float64 = 0.05)
    dt = Ref{Float64}(0.0)
    fivocheck(ccall((:fivo_compute_dt, LIBFIVO2D), Cint, (Ptr{Cvoid}, Cdouble, Cdouble, Cdouble, Ref{Float64}),
                    work.h, τ, CFL, CFLτ, dt), "fivo_compute_dt")
    return dt[]
end

"""run_sim_2d! on the GPU (main2D.jl:371-561): same keywords and result fields.
`on_dump(τ, U, work)` gets the host U, refreshed at each dump time."""
function run_sim_2d_gpu!(U::AbstractMatrix, g::Grid2D, model, work::GPUWork2D;
                         τ0::Float64 = 0.4, τfinal::Float64 = 13.0, CFL::Float64 = 0.2, CFLτ::Float64 = 0.05,
                         integrator::Symbol = :ssprk2, bc::Symbol = :outflow, reset_history::Bool = true,
                         on_dump = nothing, dump_dt::Float64 = 0.5, max_steps::Int = 2_000_000)
    integ = integrator === :ssprk3 ? FIVO_SSPRK3 : FIVO_SSPRK2
    upload!(work, U)
    res = Ref{FivoRunResult}()
    if on_dump === nothing
        fivocheck(ccall((:fivo_run, LIBFIVO2D), Cint,
                        (Ptr{Cvoid}, Cdouble, Cdouble, Cdouble, Cdouble, Cint, Cint, Int64, Cint, Ref{FivoRunResult}),
                        work.h, τ0, τfinal, CFL, CFLτ, integ, _bc(bc), max_steps, Cint(reset_history), res),
                  "fivo_run")
        download!(U, work)
        r = res[]
    else
        # prime with a zero-step run, then advance in chunks between dumps
        fivocheck(ccall((:fivo_run, LIBFIVO2D), Cint,
                        (Ptr{Cvoid}, Cdouble, Cdouble, Cdouble, Cdouble, Cint, Cint, Int64, Cint, Ref{FivoRunResult}),
                        work.h, τ0, τ0, CFL, CFLτ, integ, _bc(bc), 0, Cint(reset_history), res), "fivo_run")
        download!(U, work); on_dump(τ0, U, work)
        Q0 = res[].Q0
        τ = τ0; next = τ0 + dump_dt; nsteps = 0; ok = true
        nprimfail = 0; nvacuum = 0; max_shear_res = 0.0
        while τ < τfinal && nsteps < max_steps
            fivocheck(ccall((:fivo_advance, LIBFIVO2D), Cint,
                            (Ptr{Cvoid}, Cdouble, Cdouble, Cdouble, Cdouble, Cint, Cint, Int64, Ref{FivoRunResult}),
                            work.h, τ, min(τfinal, next), CFL, CFLτ, integ, _bc(bc), max_steps - nsteps, res),
                      "fivo_advance")
            τ = res[].tau; nsteps += res[].nsteps
            nprimfail += res[].nprimfail; nvacuum += res[].nvacuum
            max_shear_res = max(max_shear_res, res[].max_shear_res)
            res[].ok == 0 && (ok = false; break)
            if τ >= next - 1e-12
                download!(U, work); on_dump(τ, U, work); next += dump_dt
            end
        end
        download!(U, work); on_dump(τ, U, work)
        # the end-of-run diagnostics of run_sim_2d! (main2D.jl:532-556); NaN after a failed step
        Q1 = Ref{Float64}(NaN); maxu = Ref{Float64}(NaN); minPtot = Ref{Float64}(NaN)
        if ok
            fivocheck(ccall((:fivo_run_diagnostics, LIBFIVO2D), Cint,
                            (Ptr{Cvoid}, Ref{Float64}, Ref{Float64}, Ref{Float64}), work.h, Q1, maxu, minPtot),
                      "fivo_run_diagnostics")
        end
        dQ = ok ? (abs(Q0) > 0 ? abs(Q1[] - Q0)/abs(Q0) : 0.0) : NaN
        return (ok = ok, τ = τ, nsteps = nsteps, nprimfail = nprimfail, nvacuum = nvacuum,
                max_shear_res = max_shear_res, work = work, maxu = maxu[], dQ = dQ, Q0 = Q0, Q1 = Q1[],
                minPtot = minPtot[])
    end
    return (ok = r.ok != 0, τ = r.tau, nsteps = r.nsteps, nprimfail = r.nprimfail, nvacuum = r.nvacuum,
            max_shear_res = r.max_shear_res, work = work, maxu = r.maxu, dQ = r.dQ, Q0 = r.Q0, Q1 = r.Q1,
            minPtot = r.minPtot)
end

"""
    fields_2d(g, U, work::GPUWork2D, model) -> NamedTuple

The reference's readout (main2D.jl:588-600) from the device's primitives: the same
NamedTuple (x, y, T, mu, alpha, n, e, P, ux, uy and every stored dissipative row by
its layout name, in physical units), so the reference's own
`save_fields(path, fields_2d(g, U, res.work, m); model = m)` writes it unchanged.
"""
function fields_2d(g::Grid2D, U::AbstractMatrix, work::GPUWork2D, model)
    N = work.ntot
    yT, φ, μ, α, ux, uy, P, n, e = (Vector{Float64}(undef, N) for _ in 1:9)
    ok = Vector{UInt8}(undef, N)
    fivocheck(ccall((:fivo_get_primitives, LIBFIVO2D), Cint,
                    (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                     Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{UInt8}),
                    work.h, N, yT, φ, μ, α, ux, uy, P, n, e, ok), "fivo_get_primitives")
    L = model.layout; ng = g.nghost
    ixs = (ng+1):(ng+g.Nx); iys = (ng+1):(ng+g.Ny)
    grab(f) = [f(lin(g, ix, iy)) for ix in ixs, iy in iys]
    prim = (x = g.xC[ixs], y = g.yC[iys],
            T = grab(i -> exp(yT[i])), mu = grab(i -> μ[i]), alpha = grab(i -> α[i]), n = grab(i -> n[i]),
            e = grab(i -> e[i]), P = grab(i -> P[i]), ux = grab(i -> ux[i]), uy = grab(i -> uy[i]))
    diss = [s => grab(i -> phys_from_stored(U[L.idx[s], i])) for s in L.names[5:end]]
    return merge(prim, NamedTuple(diss))
end

"""Device checkpoint: `dst` continues bit for bit as `src` would (same grid and model)."""
clone_state!(dst::GPUWork2D, src::GPUWork2D) =
    fivocheck(ccall((:fivo_ctx_clone_state, LIBFIVO2D), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), dst.h, src.h),
              "fivo_ctx_clone_state")

"""Per-kernel-class CUDA-event times (fivo_kernel_times): classes prim_fast, prim_slow,
faces, update, adm_slow, relax, other."""
struct FivoKernelTimes
    launches::NTuple{8,Int64}; ms::NTuple{8,Float64}; units::NTuple{8,Int64}; total_launches::Int64
end

profile!(w::GPUWork2D, on::Bool) =
    fivocheck(ccall((:fivo_profile, LIBFIVO2D), Cint, (Ptr{Cvoid}, Cint), w.h, Cint(on)), "fivo_profile")

function kernel_times(w::GPUWork2D; reset::Bool = false)
    kt = Ref{FivoKernelTimes}()
    fivocheck(ccall((:fivo_profile_read, LIBFIVO2D), Cint, (Ptr{Cvoid}, Ref{FivoKernelTimes}, Cint),
                    w.h, kt, Cint(reset)), "fivo_profile_read")
    return kt[]
end

# ----------------------------------------------------------------------------- freeze-out

"""Cooper-Frye grid and constants of pion_yield (freezeout2d.jl:144-190)."""
mutable struct FivoCFParams
    T_fo::Float64; m::Float64; pt_lo::Float64; pt_hi::Float64; eta_max::Float64; f_yield::Float64
    n_eta::Int32; n_pt::Int32; n_phi::Int32; pad::Int32
end
function FivoCFParams(; kw...)
    p = FivoCFParams(0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    ccall((:fivo_cf_params_default, LIBFIVO2D), Cvoid, (Ref{FivoCFParams},), p)
    for (k, v) in kw; setfield!(p, k, convert(fieldtype(FivoCFParams, k), v)); end
    return p
end

"""The device freeze-out surface tau_fo(x, y) of a GPUWork2D (freeze_surface's record!)."""
mutable struct GPUFreezeOut
    h::Ptr{Cvoid}
    nx::Int
    ny::Int
    function GPUFreezeOut(w::GPUWork2D, g::Grid2D; T_fo::Float64 = 0.156)
        h = Ref{Ptr{Cvoid}}(C_NULL)
        fivocheck(ccall((:fivo_fo_create, LIBFIVO2D), Cint, (Ptr{Cvoid}, Cdouble, Ref{Ptr{Cvoid}}), w.h, T_fo, h),
                  "fivo_fo_create")
        f = new(h[], g.Nx, g.Ny)
        finalizer(f -> ccall((:fivo_fo_destroy, LIBFIVO2D), Cint, (Ptr{Cvoid},), f.h), f)
        return f
    end
end

"""record!(τ) after update_primitives_2d! (freezeout2d.jl:94-115)."""
record!(f::GPUFreezeOut, w::GPUWork2D, τ::Float64) =
    fivocheck(ccall((:fivo_fo_record, LIBFIVO2D), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cdouble), f.h, w.h, τ),
              "fivo_fo_record")

"""(; τfo, uxf, uyf, nhot, nfroze, refroze) as freeze_surface returns them (row-major a*ny + b
on the device, returned as nx x ny Julia matrices)."""
function surface(f::GPUFreezeOut)
    n = f.nx * f.ny
    t = Vector{Float64}(undef, n); ux = similar(t); uy = similar(t); c = zeros(Int64, 3)
    fivocheck(ccall((:fivo_fo_surface, LIBFIVO2D), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Int64}), f.h, t, ux, uy, c),
              "fivo_fo_surface")
    m(v) = permutedims(reshape(v, f.ny, f.nx))
    return (; τfo = m(t), uxf = m(ux), uyf = m(uy), nhot = c[1], nfroze = c[2], refroze = c[3])
end

"""pion_yield on the device: (N_boltzmann, N_bose, negative-dSigma fraction)."""
function pion_yield(f::GPUFreezeOut; kw...)
    p = FivoCFParams(; kw...)
    out = zeros(3)
    fivocheck(ccall((:fivo_cooper_frye, LIBFIVO2D), Cint, (Ptr{Cvoid}, Ref{FivoCFParams}, Ptr{Float64}),
                    f.h, p, out), "fivo_cooper_frye")
    return (out[1], out[2], out[3])
end

# ----------------------------------------------------------------------------- learned recovery guess

"""The learned Newton starting guess (fivo_guess_*): harvest pairs from plain runs,
train on the GPU, attach to a GPUWork2D."""
mutable struct GPURecoveryGuess
    h::Ptr{Cvoid}
    function GPURecoveryGuess(w::GPUWork2D; seed::Integer = 1)
        h = Ref{Ptr{Cvoid}}(C_NULL)
        fivocheck(ccall((:fivo_guess_create, LIBFIVO2D), Cint, (Ptr{Cvoid}, UInt64, Ref{Ptr{Cvoid}}),
                        w.h, UInt64(seed), h), "fivo_guess_create")
        gg = new(h[])
        finalizer(gg -> ccall((:fivo_guess_destroy, LIBFIVO2D), Cint, (Ptr{Cvoid},), gg.h), gg)
        return gg
    end
end

reserve!(gg::GPURecoveryGuess, n::Integer) =
    fivocheck(ccall((:fivo_guess_reserve, LIBFIVO2D), Cint, (Ptr{Cvoid}, Int64), gg.h, n), "fivo_guess_reserve")
harvest!(gg::GPURecoveryGuess, w::GPUWork2D, τ::Float64; stride::Integer = 1, phase::Integer = 0) =
    fivocheck(ccall((:fivo_guess_harvest, LIBFIVO2D), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Cint, Cint),
                    w.h, gg.h, τ, stride, phase), "fivo_guess_harvest")
function train!(gg::GPURecoveryGuess; steps::Integer = 3000, ctas::Integer = 148, lr::Float32 = 2f-3,
                seed::Integer = 5)
    fivocheck(ccall((:fivo_guess_fit_norm, LIBFIVO2D), Cint, (Ptr{Cvoid},), gg.h), "fivo_guess_fit_norm")
    loss = zeros(2)
    fivocheck(ccall((:fivo_guess_train, LIBFIVO2D), Cint, (Ptr{Cvoid}, Cint, Cint, Cfloat, UInt64, Ptr{Float64}),
                    gg.h, steps, ctas, lr, UInt64(seed), loss), "fivo_guess_train")
    return (first = loss[1], last = loss[2])
end
attach!(w::GPUWork2D, gg::Union{GPURecoveryGuess,Nothing}) =
    fivocheck(ccall((:fivo_ctx_set_guess, LIBFIVO2D), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), w.h,
                    gg === nothing ? C_NULL : gg.h), "fivo_ctx_set_guess")

# ----------------------------------------------------------------------------- mixed precision

"""The face pass of rhs_2d! in FP32 (`:fp32_faces`) or the reference's FP64 (`:fp64`);
recovery, SSPRK combination, floors and relaxation stay FP64 either way."""
function set_precision!(w::GPUWork2D, mode::Symbol)
    m = mode === :fp32_faces ? Cint(1) : mode === :fp64 ? Cint(0) : mode === :fp32 ? Cint(2) :
        throw(ArgumentError("precision must be :fp64, :fp32_faces or :fp32"))
    fivocheck(ccall((:fivo_ctx_set_precision, LIBFIVO2D), Cint, (Ptr{Cvoid}, Cint), w.h, m),
              "fivo_ctx_set_precision")
end
