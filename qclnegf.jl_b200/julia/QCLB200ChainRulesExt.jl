# Package extension of QCLB200 (QCLB200.jl beside this file) that makes the
# converged SCBA current differentiable for ChainRulesCore-based AD
# (Zygote, Diffractor, ...).  A maintainer adds to QCLB200's Project.toml
#
#     [weakdeps]
#     ChainRulesCore = "d360d2e6-b24c-11e9-a2a3-2a2ae2dbcce4"
#     [extensions]
#     QCLB200ChainRulesExt = "ChainRulesCore"
#
# and copies this file to ext/.  The rule: J = converged_current(build, p)
# with the pullback ΔJ -> ΔJ * dJ/dp from QCLB200.implicit_gradient
# (implicit-function theorem at the FP64 fixed point, qcl_scba_tangent_*);
# `build` is not differentiated (NoTangent).  `steps` are the difference
# steps of the explicit part Phi_p, J_p (per parameter).
#
# This image has no Julia: the extension is written against the C ABI that the
# Python tests exercise (qclb200.gradient), and has not been run.
module QCLB200ChainRulesExt

using QCLB200
import ChainRulesCore: rrule, NoTangent, unthunk

function rrule(::typeof(QCLB200.converged_current), build, p::AbstractVector{<:Real};
               steps = fill(1e-3, length(p)), tol = 1e-11, max_iter = 20000)
    J, dJdp = QCLB200.implicit_gradient(build, p, steps; tol = tol, max_iter = max_iter)
    converged_current_pullback(ΔJ) = (NoTangent(), NoTangent(), unthunk(ΔJ) .* dJdp)
    return J, converged_current_pullback
end

end # module
