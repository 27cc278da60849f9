# IBPMGPU.jl — drop-in GPU backend for IBPM.jl's static-body time step.
#
# Binds libibpm_gpu.so (include/ibpm_gpu.h) with ccall and adds
#     advance!(state::ibpm.IBState, prob::IBProblemGPU, t::Float64)
# for static bodies, one body on a MovingGrid, and MotionFunction bodies
# so callers of the reference's advance! (src/timestepping/timestepping.jl:35-67),
# run_sim! (src/ibpm.jl:90-106) included, run unchanged.  The GPU owns the
# state between calls; `prob.sync_fields = true` copies Γ, ψ, q and the
# nonlinear terms back after every step (parity runs), otherwise only CD, CL
# and F̃b come back and `sync!(state, prob)` pulls the fields on demand.
# What run_sim! reads besides advance! is served from the device too:
# compute_cfl (src/ibpm.jl:83-88) pulls the fine-level flux first, and
# save_data! (src/timestepping/save_info.jl:93-106) pulls the whole state
# before any step whose time it saves, so neither sees stale fields.
# `prob.scheme` is the reference's AB2(dt) (models.jl:70-72) and `prob.model`
# carries the grid, bodies, Re, freestream and the q5 work array that
# compute_cfl's generic method uses, so `ibpm.IBState(prob)` builds a state
# for a GPU problem as it does for a reference one (state-types.jl:25-47; its
# base_flux! call takes the device's base flux).
module IBPMGPU

using ..ibpm: ibpm, IBState, AbstractIBProblem, MultiGrid, RigidBody, Static, MovingGrid, MotionFunction,
              MotionType, get_body_info, AB2, AdamsBashforth

export IBProblemGPU, sync!, push_state!, adjoint_run, set_vorticity!, set_transform_plan!, set_level_chain!

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
    refine_sweeps::Int32
end

# Mirror of ibpm_objective.
struct Objective
    window::Int32
    w_cd::Float64
    w_cl::Float64
end

const PRECISIONS = Dict(:fp64 => Int32(0), :fp32_refined => Int32(1))

mutable struct IBProblemGPU <: AbstractIBProblem
    handle::Ptr{Cvoid}
    model_grid::MultiGrid
    nbodies::Int
    dt::Float64
    sync_fields::Bool
    motion::Union{Nothing, MovingGrid}
    body_motions::Union{Nothing, Vector{MotionFunction}}
    # the IBProblem fields that run_sim!'s helpers read (problem-types.jl:23-28):
    # model.grid, model.bodies, model.Re, model.freestream, model.work.q5; scheme.dt
    model::NamedTuple
    scheme::AdamsBashforth
end

lasterr(h) = unsafe_string(ccall((:ibpm_last_error, LIB), Cstring, (Ptr{Cvoid},), h))
check(rc, h) = rc == 0 || error("libibpm_gpu error $rc: $(lasterr(h))")

"""
    IBProblemGPU(grid, bodies, dt, Re; freestream, device=0, sync_fields=false,
                 precision=:fp64, refine_sweeps=1)

GPU counterpart of `IBProblem(grid, bodies, dt, Re; freestream)`
(src/pre-processing/problem-types.jl:23-41) for `RigidBody{Static}` bodies,
or one `RigidBody{MovingGrid}` (its base flux is recomputed from the motion at
every step's t, timestepping.jl:41-43, 273-318).  For static bodies the
freestream functions are evaluated at t = 0 only, as the reference does: its
base flux is set once when the IBState is built (state-types.jl:45) and
advance! updates it only for a MovingGrid (timestepping.jl:41-43).
`precision = :fp32_refined` runs the sine transforms of the projection solve
and of the final `vort2flux!` in FP32 with FP64-residual refinement (the trial
solve and the trial `vort2flux!` stay FP64).
"""
function IBProblemGPU(grid::MultiGrid, bodies::Vector{<:RigidBody}, dt::Float64, Re::Float64;
                      freestream=(Ux=t->1.0, Uy=t->0.0, inclination=t->0.0), device::Integer=0,
                      sync_fields::Bool=false, precision::Symbol=:fp64, refine_sweeps::Integer=1)
    nb, _ = get_body_info(bodies)
    xb = vcat([b.xb for b in bodies]...)           # (nb, 2) column-major
    ds = vcat([b.ds for b in bodies]...)
    npts = Int32.(nb)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve xb ds npts begin
        d = ProblemDesc(grid.nx, grid.ny, grid.mg, grid.h, grid.offx, grid.offy, Re, dt,
                        freestream.Ux(0.0), freestream.Uy(0.0), freestream.inclination(0.0),
                        (1.5, -0.5), length(bodies), sum(nb),
                        pointer(npts), pointer(xb), pointer(ds), PRECISIONS[precision], device,
                        refine_sweeps)
        rc = ccall((:ibpm_create, LIB), Cint, (Ref{ProblemDesc}, Ref{Ptr{Cvoid}}), d, h)
        check(rc, C_NULL)
    end
    mt = MotionType(bodies)
    motion = mt == MovingGrid ? bodies[1].motion : nothing
    body_motions = mt == MotionFunction ? MotionFunction[b.motion for b in bodies] : nothing
    mt in (Static, MovingGrid, MotionFunction) ||
        error("IBProblemGPU: bodies must be Static, one MovingGrid, or all MotionFunction")
    model = (grid=grid, bodies=bodies, Re=Re, freestream=freestream, work=(q5=zeros(grid.nq),))
    p = IBProblemGPU(h[], grid, length(bodies), dt, sync_fields, motion, body_motions, model, AB2(dt))
    finalizer(p) do x
        x.handle == C_NULL || ccall((:ibpm_destroy, LIB), Cint, (Ptr{Cvoid},), x.handle)
        x.handle = C_NULL
    end
    if body_motions !== nothing
        # the points as created are x0; E and B⁻¹ are rebuilt on the device every step
        check(ccall((:ibpm_set_motion_function, LIB), Cint, (Ptr{Cvoid},), p.handle), p.handle)
    end
    if motion !== nothing
        # rotation about the IBModel's (0, 0), as IBProblem builds it (models.jl:127-153)
        rc = ccall((:ibpm_set_moving_grid, LIB), Cint, (Ptr{Cvoid}, Float64, Float64, Ptr{Float64}),
                   p.handle, 0.0, 0.0, motion_row(motion, 0.0))
        check(rc, p.handle)
    end
    return p
end

"U, V, θ, θ̇ of a MovingGrid at t (motion-types.jl:40-48)."
motion_row(m::MovingGrid, t::Float64) = Float64[m.U(t), m.V(t), m.θ(t), m.θ̇(t)]

"x, y, θ, ẋ, ẏ, θ̇ of a MotionFunction at t (get_transformation, move-body-utils.jl:70-84)."
motion_row(m::MotionFunction, t::Float64) =
    Float64[m.xc[1](t), m.xc[2](t), m.xc[3](t), m.uc[1](t), m.uc[2](t), m.uc[3](t)]

"""
    base_flux!(state, prob::IBProblemGPU, t)

The base flux q0 that the device uses (base_flux!, timestepping.jl:228-233,
252-270): uniform per level for static bodies, that of the last step's motion
for a MovingGrid.  `ibpm.IBState(prob)` calls it at construction.
"""
function ibpm.base_flux!(state::IBState, prob::IBProblemGPU, t::Float64)
    rc = ccall((:ibpm_get_state, LIB), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                Ptr{Float64}, Ptr{Float64}),
               prob.handle, C_NULL, C_NULL, state.q0, C_NULL, C_NULL, C_NULL, C_NULL)
    check(rc, prob.handle)
end

"Copy every IBState field to the device (the reference's column-major layouts)."
function push_state!(state::IBState, prob::IBProblemGPU)
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
    compute_cfl(state, prob::IBProblemGPU)

The reference's CFL number max|q₁|·Δt/Δx (src/ibpm.jl:83-88) from the device's
fine-level flux, which is copied into `state.q[:, 1]` first.
"""
function ibpm.compute_cfl(state::IBState, prob::IBProblemGPU)
    g = prob.model_grid
    qall = zeros(g.nq, g.mg)
    rc = ccall((:ibpm_get_state, LIB), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                Ptr{Float64}, Ptr{Float64}),
               prob.handle, C_NULL, qall, C_NULL, C_NULL, C_NULL, C_NULL, C_NULL)
    check(rc, prob.handle)
    state.q .= qall
    return maximum(abs, @view state.q[:, 1]) * prob.scheme.dt / g.h
end

"""
    save_data!(tnow, t, prob::IBProblemGPU, state, data)

The reference's save_data! (src/timestepping/save_info.jl:93-106), after
copying the device state into `state` whenever one of `data`'s save times
is `tnow` (the same test the reference applies), so a saved state — the
restart state by default — is never stale.
"""
function ibpm.save_data!(tnow, t, prob::IBProblemGPU, state, data)
    saves = any(j -> sum(@. (abs(data[j].t - tnow) + 1.0) ≈ 1.0) > 0, 1:length(data))
    saves && !prob.sync_fields && sync!(state, prob)
    return invoke(ibpm.save_data!, Tuple{Any, Any, Any, Any, Any}, tnow, t, prob, state, data)
end

"""
    advance!(state, prob::IBProblemGPU, t)

One step of advance!(state, prob, t) on the GPU.  A non-finite CD/CL leaves
NaN in state.CL (as the reference would), so run_sim!'s isfinite check stops
the loop.
"""
function ibpm.advance!(state::IBState, prob::IBProblemGPU, t::Float64)
    cd = zeros(prob.nbodies); cl = zeros(prob.nbodies)
    rc = if prob.body_motions !== nothing
        rows = reduce(vcat, [motion_row(m, t) for m in prob.body_motions])
        ccall((:ibpm_advance_bodies, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
              prob.handle, 1, rows, cd, cl)
    elseif prob.motion === nothing
        ccall((:ibpm_advance, LIB), Cint, (Ptr{Cvoid}, Float64, Int32, Ptr{Float64}, Ptr{Float64}),
              prob.handle, t, 1, cd, cl)
    else
        ccall((:ibpm_advance_moving, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
              prob.handle, 1, motion_row(prob.motion, t), cd, cl)
    end
    state.CD .= cd
    state.CL .= cl
    prob.sync_fields && sync!(state, prob)
    rc == -3 && return nothing          # IBPM_ERR_NONFINITE: CL carries the NaN
    check(rc, prob.handle)
    return nothing
end

"""
    set_vorticity!(prob, ω)

Start state from a finest-level vorticity field ω ((nx-1)×(ny-1)): Γ = h²ω on
level 1, zero elsewhere and zero history, then vort2flux! (curl.jl:133-165)
makes ψ and q consistent.  This is the start state whose gradient
`adjoint_run` returns as `grad_omega0`.
"""
function set_vorticity!(prob::IBProblemGPU, ω::AbstractMatrix{Float64})
    g = prob.model_grid
    nΓ = (g.nx - 1) * (g.ny - 1)
    Γ = zeros(nΓ, g.mg); Γ[:, 1] .= vec(ω) .* g.h^2
    z = zeros(nΓ, g.mg)
    rc = ccall((:ibpm_set_state, LIB), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                Ptr{Float64}, Ptr{Float64}),
               prob.handle, Γ, zeros(g.nq, g.mg), C_NULL, z, z, z, C_NULL)
    check(rc, prob.handle)
    check(ccall((:ibpm_vort2flux, LIB), Cint, (Ptr{Cvoid},), prob.handle), prob.handle)
end

"""
    set_transform_plan!(prob; single=:latency, multi=:auto)

Plans of the device sine transforms for launches over one level (`single`)
and over several (`multi`): `:latency` (radix 4, N/4 threads per line pair,
the shortest chain per launch) or `:throughput` (radix 8, N/8 threads, fewer
instructions); `multi` may also be `:auto` (the throughput plan for launches
of 4 or more slabs, else `single`).  No counterpart in the reference, whose FFTW plans are fixed
(src/fluid-operators/dst-inversion.jl:10-20).
"""
function set_transform_plan!(prob::IBProblemGPU; single::Symbol=:latency, multi::Symbol=:auto)
    code(s) = s === :latency ? Int32(0) : s === :throughput ? Int32(1) : s === :auto ? Int32(2) :
              throw(ArgumentError("plan must be :latency, :throughput or :auto"))
    check(ccall((:ibpm_set_transform_plan, LIB), Cint, (Ptr{Cvoid}, Int32, Int32), prob.handle,
                code(single), code(multi)), prob.handle)
end

"""
    set_level_chain!(prob, chain::Symbol)

How `vort2flux!` runs its levels on the device: `:sequential` (the
reference's order, src/fluid-operators/curl.jl:133-165, one level after
another) or `:boundary_transfer` (the default: every level per launch, the
edge values from a low-rank factorisation of the level-to-level transfer).
The results agree to rounding.
"""
function set_level_chain!(prob::IBProblemGPU, chain::Symbol)
    c = chain === :sequential ? Int32(0) : chain === :boundary_transfer ? Int32(1) :
        throw(ArgumentError("chain must be :sequential or :boundary_transfer"))
    check(ccall((:ibpm_set_level_chain, LIB), Cint, (Ptr{Cvoid}, Int32), prob.handle, c), prob.handle)
end

"""
    adjoint_run(prob, nsteps; k=50, window=nsteps, w_cd=1.0, w_cl=0.0, want_xb=false)

Discrete adjoint of `nsteps` steps from the device state: J = the mean over
the last `window` steps of Σ_bodies (w_cd·CD + w_cl·CL), and its gradients
with respect to the start state (Γ, q as independent inputs), to the
vorticity the start state was built from (`set_vorticity!`), to the
freestream angle and (`want_xb`) to the body-point positions, an (nb, 2)
matrix like `body.xb`.  A checkpoint every `k` steps bounds the device memory.
"""
function adjoint_run(prob::IBProblemGPU, nsteps::Integer; k::Integer=50, window::Integer=nsteps,
                     w_cd::Real=1.0, w_cl::Real=0.0, want_xb::Bool=false)
    g = prob.model_grid
    nΓ = (g.nx - 1) * (g.ny - 1)
    J = Ref(0.0); α = Ref(0.0)
    gΓ = zeros(nΓ, g.mg); gq = zeros(g.nq, g.mg); gω = zeros(g.nx - 1, g.ny - 1)
    nf = Ref{Int32}(0)
    check(ccall((:ibpm_sizes, LIB), Cint, (Ptr{Cvoid}, Ptr{Int64}, Ptr{Int64}, Ptr{Int32}, Ref{Int32}, Ptr{Int32}),
                prob.handle, C_NULL, C_NULL, C_NULL, nf, C_NULL), prob.handle)
    gx = want_xb ? zeros(nf[] ÷ 2, 2) : nothing
    obj = Objective(window, w_cd, w_cl)
    rc = ccall((:ibpm_adjoint_run, LIB), Cint,
               (Ptr{Cvoid}, Int32, Int32, Ref{Objective}, Ref{Float64}, Ptr{Float64}, Ptr{Float64},
                Ptr{Float64}, Ref{Float64}, Ptr{Float64}),
               prob.handle, nsteps, k, obj, J, gΓ, gq, gω, α, gx === nothing ? C_NULL : gx)
    check(rc, prob.handle)
    return (J=J[], grad_Gamma0=gΓ, grad_q0=gq, grad_omega0=gω, grad_alpha=α[], grad_xb=gx)
end

end # module
