# PinCFlowGPU.jl -- routes PinCFlow.jl's pressure Poisson solve to the sm_100a
# library libpincflow_poisson.so (include/pincflow_poisson.h) through ccall.
#
# Usage (after `using PinCFlow`):
#     include("PinCFlowGPU.jl"); using .PinCFlowGPU
#     PinCFlowGPU.enable!()          # later solve_poisson! calls run on the GPU
#
# The methods below replace
#     PinCFlow.PoissonSolver.solve_poisson!(state, dt, rayleigh_factor, tolref)
# (src/PoissonSolver/solve_poisson!.jl:39-75) and, with enable!(corrector = true),
#     PinCFlow.PoissonSolver.apply_corrector!(state, dt, rayleigh_factor)
# (src/PoissonSolver/apply_corrector!.jl:44-61: compute_lhs!, the solve, the
# dpip halo fill and correct!) with the same signatures and return convention
# (errflag, niter); dt == 0 raises as in the reference, a non-converged solve
# returns (true, niter) and leaves dpip and the fields untouched.  With
# enable!(implicit_step = true) the whole
#     PinCFlow.Integration.implicit_integration!(state, dtstage, time, ntotalbicg,
#                                                side, rayleigh_factor, iout,
#                                                machine_start_time)
# (src/Integration/implicit_integration!.jl:40-80) is one library call.
# Single MPI rank only (npx = npy = npz = 1).
module PinCFlowGPU

using PinCFlow
const PS = PinCFlow.PoissonSolver

const LIB = get(ENV, "PINCFLOW_POISSON_LIB",
                joinpath(@__DIR__, "..", "lib", "libpincflow_poisson.so"))

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

# one handle per State, created on first use (grid and background uploaded once)
const HANDLES = IdDict{Any, Ptr{Cvoid}}()
const SETTINGS = Ref((precision = :fp64, multigrid = false, device = 0))

check(rc, what) = rc == 0 || error("$what: " *
    unsafe_string(ccall((:pcf_strerror, LIB), Cstring, (Cint,), rc)))

function handle(state)
    haskey(HANDLES, state) && return HANDLES[state]
    (; nx, ny, nz) = state.domain
    (; nbx, nby, nbz) = state.namelists.domain
    model = MODEL[state.namelists.atmosphere.model]
    dims = Ref(PcfDims(nx, ny, nz, nbx, nby, nbz, model, SETTINGS[].device))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:pcf_create, LIB), Cint, (Ptr{Ptr{Cvoid}}, Ptr{PcfDims}), h, dims), "pcf_create")
    (; dx, dy, dz, jac, met) = state.grid
    (; pbar, rhobar, thetabar, n2) = state.atmosphere
    # met[:, :, :, r, c] is a contiguous block of the 5-D column-major array
    m13 = @view met[:, :, :, 1, 3]
    m23 = @view met[:, :, :, 2, 3]
    m33 = @view met[:, :, :, 3, 3]
    GC.@preserve jac met begin
        check(ccall((:pcf_set_grid, LIB), Cint,
                    (Ptr{Cvoid}, Cdouble, Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
                    h[], dx, dy, dz, jac, pointer(m13), pointer(m23), pointer(m33)), "pcf_set_grid")
    end
    GC.@preserve pbar rhobar thetabar n2 begin
        check(ccall((:pcf_set_background, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
                    h[], pbar, rhobar, thetabar, n2), "pcf_set_background")
    end
    HANDLES[state] = h[]
    return h[]
end

"""
    release!(state)

Frees the device memory of the handle created for `state` (State is immutable,
so this is explicit rather than a finalizer).
"""
function release!(state)
    h = pop!(HANDLES, state, C_NULL)
    h == C_NULL || ccall((:pcf_destroy, LIB), Cint, (Ptr{Cvoid},), h)
    return nothing
end

function params(state)
    (; tolerance, poisson_iterations, preconditioner, dtau, preconditioner_iterations,
       tolerance_is_relative) = state.namelists.poisson
    p = PcfParams(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    ccall((:pcf_params_default, LIB), Cint, (Ref{PcfParams},), p)
    p.tolerance = tolerance
    p.poisson_iterations = poisson_iterations
    p.preconditioner = preconditioner
    p.dtau = dtau
    p.preconditioner_iterations = preconditioner_iterations
    p.tolerance_is_relative = tolerance_is_relative
    p.damp_horizontal_wind_on_rhs = state.namelists.sponge.damp_horizontal_wind_on_rhs
    p.precision = PRECISION[SETTINGS[].precision]
    p.multigrid = SETTINGS[].multigrid
    p.autotune = 1
    return p
end

function solve_poisson_gpu!(state, dt::AbstractFloat, rayleigh_factor::AbstractFloat,
                            tolref::AbstractFloat)
    dt == 0.0 && error("Error in solve_poisson!: dt = 0.0!")
    h = handle(state)
    (; rhs) = state.poisson
    (; rho, p) = state.variables.predictands
    (; betar) = state.sponge
    (; dpip) = state.variables.increments
    pp = state.namelists.atmosphere.model == :Compressible ? p : C_NULL
    prm = params(state)
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

# apply_corrector!.jl:44-61 through the library: compute_lhs! (with the
# Compressible model's heating from the reference's own compute_volume_force),
# the solve, then the dpip halo fill and correct!.
function apply_corrector_gpu!(state, dt::AbstractFloat, rayleigh_factor::AbstractFloat)
    h = handle(state)
    (; u, v, w, rhop, pip) = state.variables.predictands
    (; dpip) = state.variables.increments
    (; rhs) = state.poisson
    heating = C_NULL
    if state.namelists.atmosphere.model == :Compressible
        (; i0, i1, j0, j1, k0, k1) = state.domain
        heating = [PinCFlow.Update.compute_volume_force(state, i, j, k, PinCFlow.P())
                   for i in i0:i1, j in j0:j1, k in k0:k1]
    end
    tolref = Ref{Cdouble}(0.0)
    GC.@preserve u v w heating rhs begin
        check(ccall((:pcf_compute_lhs, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{Cdouble}),
                    h, u, v, w, heating, rhs, tolref), "pcf_compute_lhs")
    end
    (errflag, niter) = solve_poisson_gpu!(state, dt, rayleigh_factor, tolref[])
    errflag && return (errflag, niter)
    damp = state.namelists.sponge.damp_horizontal_wind_on_rhs
    GC.@preserve dpip u v w rhop pip begin
        check(ccall((:pcf_correct, LIB), Cint,
                    (Ptr{Cvoid}, Cdouble, Cdouble, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                     Ptr{Cdouble}, Ptr{Cdouble}),
                    h, dt, rayleigh_factor, damp, dpip, u, v, w, rhop, pip), "pcf_correct")
    end
    return (errflag, niter)
end

# implicit_integration!.jl:40-80 through the library: modify_compressible_wind!,
# the predictor update!(U, V, W, RhoP; Implicit()) with set_boundaries!,
# apply_corrector!, the inverse wind factors and set_boundaries! in one call
# (pcf_implicit_step).  Tracer boundaries are not the library's: the Julia
# fills run once afterwards (the step leaves tracers unchanged).
function implicit_integration_gpu!(state, dtstage::AbstractFloat, time::AbstractFloat, ntotalbicg::Integer,
                                   side, rayleigh_factor::AbstractFloat, iout::Integer, machine_start_time)
    h = handle(state)
    (; rho, rhop, u, v, w, pip, p) = state.variables.predictands
    (; wold) = state.variables.backups
    (; dpip) = state.variables.increments
    (; betar) = state.sponge
    compressible = state.namelists.atmosphere.model == :Compressible
    pp = compressible ? p : C_NULL
    dudt = dvdt = C_NULL
    if state.namelists.wkb.wkb_mode != :NoWKB
        (; dudt, dvdt) = state.wkb.tendencies
    end
    heating = C_NULL
    if compressible  # compute_volume_force(P) reads rho and fluxes, which the predictor leaves alone
        (; i0, i1, j0, j1, k0, k1) = state.domain
        heating = [PinCFlow.Update.compute_volume_force(state, i, j, k, PinCFlow.P())
                   for i in i0:i1, j in j0:j1, k in k0:k1]
    end
    prm = params(state)
    res = PcfResult()
    GC.@preserve u v w rho rhop pip p betar dudt dvdt heating wold dpip begin
        rc = ccall((:pcf_implicit_step, LIB), Cint,
                   (Ptr{Cvoid}, Cdouble, Cdouble, Ref{PcfParams}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                    Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                    Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{PcfResult}),
                   h, dtstage, rayleigh_factor, prm, u, v, w, rho, rhop, pip, pp, betar, dudt, dvdt, heating,
                   wold, dpip, res)
    end
    check(rc, "pcf_implicit_step")
    if res.errflag != 0
        iout = PinCFlow.Output.write_output(state, time, iout, machine_start_time)
        error("BiCGSTAB errored! Output last state into record ", iout, ".")
    end
    B = PinCFlow.Boundaries
    B.set_tracer_zonal_boundaries!(state, B.BoundaryPredictands())
    B.set_tracer_meridional_boundaries!(state, B.BoundaryPredictands())
    B.set_tracer_vertical_boundaries!(state, B.BoundaryPredictands())
    return ntotalbicg + Int(res.niter)
end

"""
    enable!(; precision = :fp64, multigrid = false, corrector = false, implicit_step = false, device = 0)

Make `PinCFlow.PoissonSolver.solve_poisson!` run on the GPU.  `precision = :mixed`
selects the FP32-inner / FP64-refined solve (same FP64 tolerance), and
`multigrid = true` (with `:mixed`) its multigrid preconditioner.
`corrector = true` also replaces `apply_corrector!` (compute_lhs!, the solve and
correct! all on the GPU); `implicit_step = true` replaces the whole
`implicit_integration!` (the implicit predictor, the corrector and the
boundary fills of the predictands in one library call per half step).
"""
function enable!(; precision::Symbol = :fp64, multigrid::Bool = false, corrector::Bool = false,
                 implicit_step::Bool = false, device::Integer = 0)
    SETTINGS[] = (precision = precision, multigrid = multigrid, device = device)
    @eval PS function solve_poisson!(state::PinCFlow.State, dt::AbstractFloat,
                                     rayleigh_factor::AbstractFloat, tolref::AbstractFloat)
        return $(solve_poisson_gpu!)(state, dt, rayleigh_factor, tolref)
    end
    if corrector
        @eval PS function apply_corrector!(state::PinCFlow.State, dt::AbstractFloat,
                                           rayleigh_factor::AbstractFloat)
            return $(apply_corrector_gpu!)(state, dt, rayleigh_factor)
        end
    end
    if implicit_step
        @eval PinCFlow.Integration function implicit_integration!(state::PinCFlow.State, dtstage::AbstractFloat,
                                                                  time::AbstractFloat, ntotalbicg::Integer,
                                                                  side::RHS, rayleigh_factor::AbstractFloat,
                                                                  iout::Integer, machine_start_time::DateTime)
            return $(implicit_integration_gpu!)(state, dtstage, time, ntotalbicg, side, rayleigh_factor, iout,
                                                machine_start_time)
        end
    end
    return nothing
end

end # module
