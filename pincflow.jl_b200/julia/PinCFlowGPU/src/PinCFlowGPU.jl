# PinCFlowGPU.jl -- the C ABI of libpincflow_poisson.so (include/pincflow_poisson.h),
# the sm_100a pressure Poisson solver for PinCFlow.jl, bound through ccall.
#
# This module knows nothing of PinCFlow's types: it mirrors the library's
# structs and wraps its entry points on plain arrays.  The package extension
# PinCFlowGPUExt (ext/PinCFlowGPUExt.jl), which Julia loads as soon as both
# PinCFlowGPU and PinCFlow are loaded, adds the methods of
#     PinCFlow.PoissonSolver.solve_poisson!    (src/PoissonSolver/solve_poisson!.jl:39-75)
#     PinCFlow.PoissonSolver.apply_corrector!  (src/PoissonSolver/apply_corrector!.jl:38-61)
#     PinCFlow.Integration.implicit_integration! (src/Integration/implicit_integration!.jl:37-80)
# that route a State to the library once `enable!` has been called.
#
#     using PinCFlow, PinCFlowGPU
#     PinCFlowGPU.enable!(precision = :mixed, multigrid = true)
#     integrate(namelists)       # solve_poisson! now runs on the GPU
#
# Single MPI rank only (npx = npy = npz = 1).
module PinCFlowGPU

using Libdl

const LIB = get(ENV, "PINCFLOW_POISSON_LIB",
                joinpath(@__DIR__, "..", "..", "..", "lib", "libpincflow_poisson.so"))

struct PcfDims
    nx::Cint; ny::Cint; nz::Cint
    nbx::Cint; nby::Cint; nbz::Cint
    model::Cint; device::Cint
end

mutable struct PcfParams
    tolerance::Cdouble
    poisson_iterations::Cint
    preconditioner::Cint
    dtau::Cdouble
    preconditioner_iterations::Cint
    tolerance_is_relative::Cint
    damp_horizontal_wind_on_rhs::Cint
    precision::Cint
    residual::Cint
    inner_tolerance::Cdouble
    max_refinements::Cint
    learned::Cint
    check_interval::Cint
    restart_interval::Cint
    multigrid::Cint
    mg_dtau::Cdouble
    mg_coarse_iterations::Cint
    mg_min_columns::Cint
    autotune::Cint
    mg_operator_bf16::Cint
    mg_fused_coarse::Cint
    mg_smoother_fp8::Cint
end

mutable struct PcfResult
    errflag::Cint; niter::Cint; nrefine::Cint; status::Cint
    residual::Cdouble; true_residual::Cdouble; b_norm::Cdouble
    ms_upload::Cdouble; ms_assemble::Cdouble; ms_solve::Cdouble
    ms_download::Cdouble; ms_total::Cdouble
end
PcfResult() = PcfResult(0, 0, 0, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0)

const MODEL = Dict(:Boussinesq => 0, :PseudoIncompressible => 1, :Compressible => 2)
const PRECISION = Dict(:fp64 => 0, :mixed => 1)

"""Settings of the GPU path; `enabled` false leaves every call to the reference."""
const SETTINGS = Ref((enabled = false, precision = :fp64, multigrid = false, corrector = false,
                      implicit_step = false, device = 0))

check(rc, what) = rc == 0 || error("$what: " *
    unsafe_string(ccall((:pcf_strerror, LIB), Cstring, (Cint,), rc)))

"""
    create(nx, ny, nz, nbx, nby, nbz, model; device = 0) -> Ptr{Cvoid}

A library handle (pcf_create) for one grid; it owns the grid's device memory
until `destroy`.
"""
function create(nx, ny, nz, nbx, nby, nbz, model::Symbol; device::Integer = 0)
    dims = Ref(PcfDims(nx, ny, nz, nbx, nby, nbz, MODEL[model], device))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:pcf_create, LIB), Cint, (Ptr{Ptr{Cvoid}}, Ptr{PcfDims}), h, dims), "pcf_create")
    return h[]
end

destroy(h::Ptr{Cvoid}) = h == C_NULL ? 0 : ccall((:pcf_destroy, LIB), Cint, (Ptr{Cvoid},), h)

"""The grid metric (pcf_set_grid): jac and the (1,3), (2,3), (3,3) planes of met."""
function set_grid!(h, dx, dy, dz, jac::Array{Float64}, met::Array{Float64, 5})
    # met[:, :, :, r, c] is a contiguous block of the 5-D column-major array
    m13 = @view met[:, :, :, 1, 3]
    m23 = @view met[:, :, :, 2, 3]
    m33 = @view met[:, :, :, 3, 3]
    GC.@preserve jac met begin
        check(ccall((:pcf_set_grid, LIB), Cint,
                    (Ptr{Cvoid}, Cdouble, Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
                    h, dx, dy, dz, jac, pointer(m13), pointer(m23), pointer(m33)), "pcf_set_grid")
    end
    return nothing
end

"""The background atmosphere (pcf_set_background)."""
function set_background!(h, pbar, rhobar, thetabar, n2)
    GC.@preserve pbar rhobar thetabar n2 begin
        check(ccall((:pcf_set_background, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
                    h, pbar, rhobar, thetabar, n2), "pcf_set_background")
    end
    return nothing
end

"""
    params(namelist_fields...) -> PcfParams

The library's settings from PoissonNamelist's fields (PoissonNamelist.jl:38-66)
and the GPU path's SETTINGS.
"""
function params(; tolerance, poisson_iterations, preconditioner, dtau, preconditioner_iterations,
                tolerance_is_relative, damp_horizontal_wind_on_rhs)
    p = PcfParams(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    ccall((:pcf_params_default, LIB), Cint, (Ref{PcfParams},), p)
    p.tolerance = tolerance
    p.poisson_iterations = poisson_iterations
    p.preconditioner = preconditioner
    p.dtau = dtau
    p.preconditioner_iterations = preconditioner_iterations
    p.tolerance_is_relative = tolerance_is_relative
    p.damp_horizontal_wind_on_rhs = damp_horizontal_wind_on_rhs
    p.precision = PRECISION[SETTINGS[].precision]
    p.multigrid = SETTINGS[].multigrid
    p.autotune = 1
    return p
end

"""
    solve!(h, rhs, rho, betar, p, dt, rayleigh_factor, tolref, prm, dpip) -> (errflag, niter)

solve_poisson! on host arrays (pcf_solve): rhs interior, the others haloed;
`p` is `nothing` unless the model is Compressible.  dt == 0 raises like
solve_poisson!.jl:52-54.
"""
function solve!(h, rhs, rho, betar, p, dt, rayleigh_factor, tolref, prm::PcfParams, dpip)
    dt == 0.0 && error("Error in solve_poisson!: dt = 0.0!")
    pp = p === nothing ? C_NULL : p
    res = PcfResult()
    GC.@preserve rhs rho p betar dpip begin
        rc = ccall((:pcf_solve, LIB), Cint,
                   (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Cdouble, Cdouble,
                    Cdouble, Ref{PcfParams}, Ptr{Cdouble}, Ref{PcfResult}),
                   h, rhs, rho, betar, pp, dt, rayleigh_factor, tolref, prm, dpip, res)
    end
    check(rc, "pcf_solve")
    return (res.errflag != 0, Int(res.niter))
end

"""compute_lhs! on host arrays (pcf_compute_lhs): writes rhs, returns tolref."""
function compute_lhs!(h, u, v, w, heating, rhs)
    tolref = Ref{Cdouble}(0.0)
    hh = heating === nothing ? C_NULL : heating
    GC.@preserve u v w heating rhs begin
        check(ccall((:pcf_compute_lhs, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{Cdouble}),
                    h, u, v, w, hh, rhs, tolref), "pcf_compute_lhs")
    end
    return tolref[]
end

"""The dpip halo fill and correct! on host arrays (pcf_correct)."""
function correct!(h, dt, rayleigh_factor, damp, dpip, u, v, w, rhop, pip)
    GC.@preserve dpip u v w rhop pip begin
        check(ccall((:pcf_correct, LIB), Cint,
                    (Ptr{Cvoid}, Cdouble, Cdouble, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                     Ptr{Cdouble}, Ptr{Cdouble}),
                    h, dt, rayleigh_factor, damp, dpip, u, v, w, rhop, pip), "pcf_correct")
    end
    return nothing
end

"""
    implicit_step!(h, dtstage, rayleigh_factor, prm, u, v, w, rho, rhop, pip, p, betar,
                   dudt, dvdt, heating, wold, dpip) -> PcfResult

The implicit half step (pcf_implicit_step): predictor with its boundary fills,
compute_lhs!, the solve, the dpip fill and correct! in one call.  `p`,
`dudt`, `dvdt` and `heating` may be `nothing`.
"""
function implicit_step!(h, dtstage, rayleigh_factor, prm::PcfParams, u, v, w, rho, rhop, pip, p, betar,
                        dudt, dvdt, heating, wold, dpip)
    nul(a) = a === nothing ? C_NULL : a
    res = PcfResult()
    GC.@preserve u v w rho rhop pip p betar dudt dvdt heating wold dpip begin
        rc = ccall((:pcf_implicit_step, LIB), Cint,
                   (Ptr{Cvoid}, Cdouble, Cdouble, Ref{PcfParams}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                    Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                    Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{PcfResult}),
                   h, dtstage, rayleigh_factor, prm, u, v, w, rho, rhop, pip, nul(p), betar, nul(dudt), nul(dvdt),
                   nul(heating), wold, dpip, res)
    end
    check(rc, "pcf_implicit_step")
    return res
end

"""
    enable!(; precision = :fp64, multigrid = false, corrector = false, implicit_step = false, device = 0)

Route PinCFlow's `solve_poisson!` to the GPU (the methods of the package
extension PinCFlowGPUExt).  `precision = :mixed` selects the FP32-inner /
FP64-refined solve (same FP64 tolerance), and `multigrid = true` (with
`:mixed`) its multigrid preconditioner.  `corrector = true` also routes
`apply_corrector!` (compute_lhs!, the solve and correct! on the GPU);
`implicit_step = true` routes the whole `implicit_integration!` (predictor,
corrector and the boundary fills of the predictands in one library call).
"""
function enable!(; precision::Symbol = :fp64, multigrid::Bool = false, corrector::Bool = false,
                 implicit_step::Bool = false, device::Integer = 0)
    haskey(PRECISION, precision) || error("precision must be :fp64 or :mixed")
    SETTINGS[] = (enabled = true, precision = precision, multigrid = multigrid, corrector = corrector,
                  implicit_step = implicit_step, device = device)
    return nothing
end

"""
    release!(state)

Frees the device memory of the library handle made for a PinCFlow State
(State is immutable, so this is explicit; the extension frees every handle
at exit).  Its method lives in the package extension.
"""
function release! end

"""Back to the reference's own methods (the handles stay until `release!`)."""
function disable!()
    SETTINGS[] = merge(SETTINGS[], (enabled = false,))
    return nothing
end

end # module
