# PinCFlowGPUExt -- the package extension that connects PinCFlow.jl's State to
# the sm_100a Poisson library (loaded by Julia once PinCFlow and PinCFlowGPU
# are both loaded; PinCFlow is a weak dependency of PinCFlowGPU).
#
# It adds Float64 methods of
#     PinCFlow.PoissonSolver.solve_poisson!(state, dt, rayleigh_factor, tolref)
#         src/PoissonSolver/solve_poisson!.jl:39-75
#     PinCFlow.PoissonSolver.apply_corrector!(state, dt, rayleigh_factor)
#         src/PoissonSolver/apply_corrector!.jl:38-61
#     PinCFlow.Integration.implicit_integration!(state, dtstage, time, ntotalbicg,
#                                                side, rayleigh_factor, iout,
#                                                machine_start_time)
#         src/Integration/implicit_integration!.jl:37-80
# The reference declares its arguments AbstractFloat, so these methods are
# more specific and take the calls without overwriting the reference's
# methods (which precompilation forbids).  Until PinCFlowGPU.enable! is
# called, and for the parts not enabled, each one `invoke`s the reference's
# own method.  The return conventions are the reference's: (errflag, niter),
# dt == 0 raises, a non-converged solve returns (true, niter) and leaves dpip
# and the fields untouched.
#
# One library handle is kept per State for the whole run (grid and background
# uploaded once), so the initial cleaning (integrate.jl:141) and the two
# solves of every time step (integrate.jl:291, :329) share it.
module PinCFlowGPUExt

using PinCFlow
using PinCFlowGPU
using Dates: DateTime

const G = PinCFlowGPU
const PS = PinCFlow.PoissonSolver
const IN = PinCFlow.Integration

const HANDLES = IdDict{Any, Ptr{Cvoid}}()

function handle(state)
    haskey(HANDLES, state) && return HANDLES[state]
    (; nx, ny, nz) = state.domain
    (; nbx, nby, nbz) = state.namelists.domain
    h = G.create(nx, ny, nz, nbx, nby, nbz, state.namelists.atmosphere.model; device = G.SETTINGS[].device)
    (; dx, dy, dz, jac, met) = state.grid
    (; pbar, rhobar, thetabar, n2) = state.atmosphere
    G.set_grid!(h, dx, dy, dz, jac, met)
    G.set_background!(h, pbar, rhobar, thetabar, n2)
    HANDLES[state] = h
    return h
end

function G.release!(state)
    G.destroy(pop!(HANDLES, state, C_NULL))
    return nothing
end

function params(state)
    pn = state.namelists.poisson
    return G.params(; tolerance = pn.tolerance, poisson_iterations = pn.poisson_iterations,
                    preconditioner = pn.preconditioner, dtau = pn.dtau,
                    preconditioner_iterations = pn.preconditioner_iterations,
                    tolerance_is_relative = pn.tolerance_is_relative,
                    damp_horizontal_wind_on_rhs = state.namelists.sponge.damp_horizontal_wind_on_rhs)
end

compressible(state) = state.namelists.atmosphere.model == :Compressible

# the Compressible model's heating, from the reference's own compute_volume_force
function heating(state)
    compressible(state) || return nothing
    (; i0, i1, j0, j1, k0, k1) = state.domain
    return [PinCFlow.Update.compute_volume_force(state, i, j, k, PinCFlow.P())
            for i in i0:i1, j in j0:j1, k in k0:k1]
end

function solve_gpu!(state, dt, rayleigh_factor, tolref)
    (; rhs) = state.poisson
    (; rho, p) = state.variables.predictands
    (; betar) = state.sponge
    (; dpip) = state.variables.increments
    return G.solve!(handle(state), rhs, rho, betar, compressible(state) ? p : nothing, dt, rayleigh_factor,
                    tolref, params(state), dpip)
end

function PS.solve_poisson!(state::PinCFlow.State, dt::Float64, rayleigh_factor::Float64, tolref::Float64)
    G.SETTINGS[].enabled ||
        return invoke(PS.solve_poisson!, Tuple{PinCFlow.State, AbstractFloat, AbstractFloat, AbstractFloat},
                      state, dt, rayleigh_factor, tolref)
    return solve_gpu!(state, dt, rayleigh_factor, tolref)
end

# apply_corrector!.jl:44-61: compute_lhs!, the solve, the dpip halo fill and correct!
function PS.apply_corrector!(state::PinCFlow.State, dt::Float64, rayleigh_factor::Float64)
    (G.SETTINGS[].enabled && G.SETTINGS[].corrector) ||
        return invoke(PS.apply_corrector!, Tuple{PinCFlow.State, AbstractFloat, AbstractFloat},
                      state, dt, rayleigh_factor)
    h = handle(state)
    (; u, v, w, rhop, pip) = state.variables.predictands
    (; dpip) = state.variables.increments
    tolref = G.compute_lhs!(h, u, v, w, heating(state), state.poisson.rhs)
    (errflag, niter) = solve_gpu!(state, dt, rayleigh_factor, tolref)
    errflag && return (errflag, niter)
    G.correct!(h, dt, rayleigh_factor, state.namelists.sponge.damp_horizontal_wind_on_rhs, dpip, u, v, w, rhop,
               pip)
    return (errflag, niter)
end

# implicit_integration!.jl:40-80 in one library call; tracer boundaries are
# not the library's, so the Julia fills run once afterwards (the step leaves
# tracers unchanged)
function IN.implicit_integration!(state::PinCFlow.State, dtstage::Float64, time::Float64, ntotalbicg::Integer,
                                  side::PinCFlow.Update.RHS, rayleigh_factor::Float64, iout::Integer,
                                  machine_start_time::DateTime)
    (G.SETTINGS[].enabled && G.SETTINGS[].implicit_step) ||
        return invoke(IN.implicit_integration!,
                      Tuple{PinCFlow.State, AbstractFloat, AbstractFloat, Integer, PinCFlow.Update.RHS, AbstractFloat,
                            Integer, DateTime},
                      state, dtstage, time, ntotalbicg, side, rayleigh_factor, iout, machine_start_time)
    (; rho, rhop, u, v, w, pip, p) = state.variables.predictands
    (; wold) = state.variables.backups
    (; dpip) = state.variables.increments
    (; betar) = state.sponge
    dudt = dvdt = nothing
    if state.namelists.wkb.wkb_mode != :NoWKB
        (; dudt, dvdt) = state.wkb.tendencies
    end
    res = G.implicit_step!(handle(state), dtstage, rayleigh_factor, params(state), u, v, w, rho, rhop, pip,
                           compressible(state) ? p : nothing, betar, dudt, dvdt, heating(state), wold, dpip)
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

function __init__()
    atexit() do
        for h in values(HANDLES)
            G.destroy(h)
        end
        empty!(HANDLES)
    end
end

end # module
