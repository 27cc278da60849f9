# IBPMGPU.jl — drop-in GPU backend for IBPM.jl's static-body time step.
#
# Binds libibpm_gpu.so (include/ibpm_gpu.h) with ccall and adds
#     advance!(state::ibpm.IBState, prob::IBProblemGPU, t::Float64)
# so callers of the reference's advance! (src/timestepping/timestepping.jl:35-67),
# run_sim! (src/ibpm.jl:90-106) included, run unchanged.  The GPU owns the
# state between calls; `prob.sync_fields = true` copies Γ, ψ, q and the
# nonlinear terms back after every step (parity runs), otherwise only CD, CL
# and F̃b come back and `sync!(state, prob)` pulls the fields on demand.
module IBPMGPU

using ..ibpm: ibpm, IBState, AbstractIBProblem, MultiGrid, RigidBody, Static, get_body_info

export IBProblemGPU, sync!, push!

const LIB = get(ENV, "IBPM_GPU_LIB", joinpath(@__DIR__, "..", "lib", "libibpm_gpu.so"))

# Mirror of ibpm_problem_desc (include/ibpm_gpu.h); field order and types must match.
struct ProblemDesc
    nx::Int32; ny::Int32; mg::Int32
    h::Float64; offx::Float64; offy::Float64
    Re::Float64; dt::Float64
    Ux::Float64; Uy::Float64; inclination::Float64
    beta::NTuple{2,Float64}
    nbodies::Int32; nb::Int32
    body_npts::Ptr{Int32}; xb::Ptr{Float64}; ds::Ptr{Float64}
    precision::Int32; device::Int32
end

mutable struct IBProblemGPU <: AbstractIBProblem
    handle::Ptr{Cvoid}
    model_grid::MultiGrid
    nbodies::Int
    dt::Float64
    sync_fields::Bool
end

lasterr(h) = unsafe_string(ccall((:ibpm_last_error, LIB), Cstring, (Ptr{Cvoid},), h))
check(rc, h) = rc == 0 || error("libibpm_gpu error $rc: $(lasterr(h))")

"""
    IBProblemGPU(grid, bodies, dt, Re; freestream, device=0, sync_fields=false)

GPU counterpart of `IBProblem(grid, bodies, dt, Re; freestream)`
(src/pre-processing/problem-types.jl:188-199) for `RigidBody{Static}` bodies.
The freestream functions are evaluated at t = 0, as IBState's base_flux! does
for static bodies.
"""
function IBProblemGPU(grid::MultiGrid, bodies::Vector{<:RigidBody{Static}}, dt::Float64, Re::Float64;
                      freestream=(Ux=t->1.0, Uy=t->0.0, inclination=t->0.0), device::Integer=0,
                      sync_fields::Bool=false)
    nb, _ = get_body_info(bodies)
    xb = vcat([b.xb for b in bodies]...)           # (nb, 2) column-major
    ds = vcat([b.ds for b in bodies]...)
    npts = Int32.(nb)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve xb ds npts begin
        d = ProblemDesc(grid.nx, grid.ny, grid.mg, grid.h, grid.offx, grid.offy, Re, dt,
                        freestream.Ux(0.0), freestream.Uy(0.0), freestream.inclination(0.0),
                        (1.5, -0.5), length(bodies), sum(nb),
                        pointer(npts), pointer(xb), pointer(ds), 0, device)
        rc = ccall((:ibpm_create, LIB), Cint, (Ref{ProblemDesc}, Ref{Ptr{Cvoid}}), d, h)
        check(rc, C_NULL)
    end
    p = IBProblemGPU(h[], grid, length(bodies), dt, sync_fields)
    finalizer(p) do x
        x.handle == C_NULL || ccall((:ibpm_destroy, LIB), Cint, (Ptr{Cvoid},), x.handle)
        x.handle = C_NULL
    end
    return p
end

"Copy every IBState field to the device (the reference's column-major layouts)."
function push!(state::IBState, prob::IBProblemGPU)
    rc = ccall((:ibpm_set_state, LIB), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                Ptr{Float64}, Ptr{Float64}),
               prob.handle, state.Γ, state.q, state.q0, state.ψ, state.nonlin[1], state.nonlin[2],
               state.F̃b)
    check(rc, prob.handle)
end

"Copy the device state into `state`."
function sync!(state::IBState, prob::IBProblemGPU)
    rc = ccall((:ibpm_get_state, LIB), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                Ptr{Float64}, Ptr{Float64}),
               prob.handle, state.Γ, state.q, state.q0, state.ψ, state.nonlin[1], state.nonlin[2],
               state.F̃b)
    check(rc, prob.handle)
end

"""
    advance!(state, prob::IBProblemGPU, t)

One step of advance!(state, prob, t) on the GPU.  A non-finite CD/CL leaves
NaN in state.CL (as the reference would), so run_sim!'s isfinite check stops
the loop.
"""
function ibpm.advance!(state::IBState, prob::IBProblemGPU, t::Float64)
    cd = zeros(prob.nbodies); cl = zeros(prob.nbodies)
    rc = ccall((:ibpm_advance, LIB), Cint, (Ptr{Cvoid}, Float64, Int32, Ptr{Float64}, Ptr{Float64}),
               prob.handle, t, 1, cd, cl)
    state.CD .= cd
    state.CL .= cl
    prob.sync_fields && sync!(state, prob)
    rc == -3 && return nothing          # IBPM_ERR_NONFINITE: CL carries the NaN
    check(rc, prob.handle)
    return nothing
end

end # module
