# IBPMGPUChainRules.jl — reverse-mode rule for objectives of IBPMGPU runs.
#
# Load after IBPMGPU.jl when ChainRulesCore is available (a weak dependency
# of the shim):
#     include("IBPMGPU.jl"); include("IBPMGPUChainRules.jl")
# The function below maps a start vorticity to the time-averaged force
# objective of a GPU run; its rrule returns the gradient from the discrete
# adjoint (ibpm_adjoint_run), so Zygote / ChainRules-based optimisers can
# differentiate through the solver without tracing it.
module IBPMGPUChainRules

using ChainRulesCore
using ..IBPMGPU: IBProblemGPU, adjoint_run, set_vorticity!

export mean_force

"""
    mean_force(ω, prob; nsteps, window=nsteps, k=50, w_cd=1.0, w_cl=0.0)

Run `nsteps` steps from the start state built from ω (`set_vorticity!`) and
return J = mean over the last `window` steps of Σ_bodies (w_cd·CD + w_cl·CL).
"""
function mean_force(ω::AbstractMatrix{Float64}, prob::IBProblemGPU; nsteps::Integer,
                    window::Integer=nsteps, k::Integer=50, w_cd::Real=1.0, w_cl::Real=0.0)
    set_vorticity!(prob, ω)
    return adjoint_run(prob, nsteps; k=k, window=window, w_cd=w_cd, w_cl=w_cl).J
end

function ChainRulesCore.rrule(::typeof(mean_force), ω::AbstractMatrix{Float64}, prob::IBProblemGPU;
                              nsteps::Integer, window::Integer=nsteps, k::Integer=50,
                              w_cd::Real=1.0, w_cl::Real=0.0)
    set_vorticity!(prob, ω)
    r = adjoint_run(prob, nsteps; k=k, window=window, w_cd=w_cd, w_cl=w_cl)
    pullback(ΔJ) = (NoTangent(), unthunk(ΔJ) .* r.grad_omega0, NoTangent())
    return r.J, pullback
end

end # module
