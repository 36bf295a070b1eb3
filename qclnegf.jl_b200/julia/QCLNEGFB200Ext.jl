# Package extension of QCLNEGF.jl that routes its production operators
# through libqclb200 (module QCLB200, QCLB200.jl beside this file).
#
# A maintainer adds to QCLNEGF.jl's Project.toml
#
#     [weakdeps]
#     QCLB200 = "<uuid of the QCLB200 package>"
#     [extensions]
#     QCLNEGFB200Ext = "QCLB200"
#
# and copies this file to ext/.  Loading `using QCLNEGF, QCLB200` then makes
# the routing below available.  No reference source changes: routing is by
# Julia dispatch on the reference's own extension points.
#
#   * Operator level.  `_production_static_contraction!` dispatches on the
#     AbstractProductionKernel subtype of each cached operator
#     (numerics/optimized/production_contracts.jl:262-323; methods at
#     numerics/optimized/production_operators.jl:402-670).  `b200_cache(cache)`
#     returns the ProductionCache (production_contracts.jl:332-344) with every
#     kernel wrapped in `B200Kernel`, whose method calls qcl_static_contraction
#     with the wrapped operator's arrays.  `B200SeparableKernel` is the
#     Kronecker-sum form K(m, m') = sum_i radial_i(m, m') block_i that keeps the
#     momentum-dependent kernels of large grids out of the dense (N_k N_b^2)^2
#     matrix (QCL_KERNEL_SEPARABLE_SUM).
#   * Fixed-point level.  `B200Problem(problem)` wraps an NEGFProblem; the
#     method solve_scba_production(::B200Problem, Uᴴ; ...) runs the device
#     SCBA (QCLB200.create / seed! / step!) under the reference's stopping
#     tolerance on r_Sigma.  solver_backend in AlgorithmOptions
#     (domain/algorithm_options.jl:19-39) is left as is: its validation
#     (:42-93) admits :educational and :production only, so the device path is
#     selected by the wrapper type instead of a new symbol.
#
# This image has no Julia: the extension is written against the reference's
# sources and the C ABI that the Python tests exercise, and has not been run.
module QCLNEGFB200Ext

using QCLNEGF
using QCLB200

import QCLNEGF: _production_static_contraction!, solve_scba_production

const _OPT = QCLNEGF  # the optimised-operator names live in the package namespace

"""A cached production operator routed to the GPU."""
struct B200Kernel{K<:_OPT.AbstractProductionKernel} <: _OPT.AbstractProductionKernel
    inner::K
    precision::Symbol
end

"""K(m, m') = sum_i radial[:, :, i] * block[:, :, i] (rows (a, b), columns
(c, d)) -- QCL_KERNEL_SEPARABLE_SUM."""
struct B200SeparableKernel <: _OPT.AbstractProductionKernel
    radial::Array{ComplexF64,3}
    block::Array{ComplexF64,3}
    N_k::Int
    N_b::Int
end

_arrays(op::_OPT.DenseProductionKernel) = (:dense, (; matrix = op.matrix))
_arrays(op::_OPT.MomentumIndependentProductionKernel) = (:momentum_independent, (; block = op.block))
_arrays(op::_OPT._SeparableIFRProductionKernel) = (:ifr, (; left = op.left, right = op.right, radial = op.radial))
_arrays(op::_OPT.LowRankProductionKernel) = (:low_rank, (; left = op.left, right = op.right_adjoint))
_arrays(op::B200SeparableKernel) = (:separable_sum, (; radial = op.radial, block = op.block))

function _production_static_contraction!(
    Σ::AbstractArray{ComplexF64,4},
    op::B200Kernel,
    G::AbstractArray{<:Number,4},
    wᵏ::AbstractVector{<:Real},
    qᴷ::Real,
    energy_chunk::Integer;
    α::Number = 1,
    β::Number = 0,
    parallel_backend::Symbol = :blas,
    worker_count::Integer = 0,
)
    kind, arrays = _arrays(op.inner)
    QCLB200.production_static_contraction(kind, arrays, Array{ComplexF64,4}(G), Vector{Float64}(wᵏ), qᴷ;
                                          α = real(α), β = real(β), Σ = Σ)
    return Σ
end

function _production_static_contraction!(Σ::AbstractArray{ComplexF64,4}, op::B200SeparableKernel,
                                         G::AbstractArray{<:Number,4}, wᵏ::AbstractVector{<:Real}, qᴷ::Real,
                                         energy_chunk::Integer; α::Number = 1, β::Number = 0, kwargs...)
    QCLB200.production_static_contraction(:separable_sum, (; radial = op.radial, block = op.block),
                                          Array{ComplexF64,4}(G), Vector{Float64}(wᵏ), qᴷ;
                                          α = real(α), β = real(β), Σ = Σ)
    return Σ
end

"""The cache with every kernel operator routed to the GPU (the shift plans,
FFT plan and estimate are kept; the Hilbert transforms and shifts can be
routed the same way through QCLB200.fft_hilbert_transform and
QCLB200.apply_energy_shift!)."""
function b200_cache(cache::_OPT.ProductionCache; precision::Symbol = :c128)
    kernels = Dict{Symbol,_OPT.AbstractProductionKernel}(
        name => (op isa _OPT.LiteralProductionKernel ? op : B200Kernel(op, precision)) for
        (name, op) in cache.kernels
    )
    return _OPT.ProductionCache(cache.W̃₊ᴱᵖ, cache.W̃₋ᴱᵖ, cache.W̃₊ᴸᴼ, cache.W̃₋ᴸᴼ, kernels,
                                cache.fft_hilbert_plan, cache.product_hilbert_operator, cache.estimate,
                                cache.source_grids, cache.source_kernel_arrays, cache.algorithms)
end

"""An NEGFProblem whose fixed-point solve runs on the GPU."""
struct B200Problem{P}
    inner::P
    precision::Symbol
    mechanisms::Vector{QCLB200.Mechanism}
    keep::Vector{Any}
end

B200Problem(problem; precision::Symbol = :c128) = B200Problem(problem, precision, QCLB200.Mechanism[], Any[])

"""solve_scba_production on the device: the problem's grids, projected
Hamiltonians, neighbour couplings and kernel operators are uploaded once
(QCLB200.create), the seed and the iterations run on the GPU, and the loop
stops at the reference's tolerance on r_Sigma or at max_iter; each step's
SCBAIteration row (domain/types.jl:908) is returned in the history."""
function solve_scba_production(p::B200Problem, Uᴴ::AbstractVector{<:Real};
                               options::_OPT.SolverOptions = _OPT.baseline_options(),
                               production_options::_OPT.ProductionOptions = _OPT.ProductionOptions(),
                               kwargs...)
    problem = p.inner
    h = _OPT.project_hamiltonians(problem, Uᴴ)
    sp = _OPT._scaled_physics(problem.physical, problem.scales)
    NLO = _OPT._thermal_lo_occupation(problem.physical)
    kBT = _OPT.scaled_value(_OPT.CODATA.kᴮ * problem.physical.Tᴸ, problem.scales, :energy)
    ηseed = _OPT.scaled_value(problem.numerical.η_seed, problem.scales, :energy)
    cache = _OPT.build_production_cache(problem; options = production_options)
    # the cached operators in the reference's mechanism order (_SCATTERING_MECHANISM_ORDER)
    names = [n for n in _OPT._SCATTERING_MECHANISM_ORDER if haskey(cache.kernels, n)]
    ops = [(n, cache.kernels[n], problem.kernels.qᴷ[n]) for n in names]
    problem_struct, mechanisms = QCLB200.problem_and_mechanisms(
        problem.grids.ε, problem.grids.wᴱ, problem.grids.wᵏ, h, problem.basis.T₊, problem.basis.T₋, sp.Eᵖ,
        sp.ħωᴸᴼ, NLO, 2, sp.Nᴰ²ᴰ, ηseed, kBT, options.α_Σ, problem.scales.J₀, ops, p.keep;
        precision = p.precision)
    solver = QCLB200.create(problem_struct, mechanisms, p.keep)
    QCLB200.seed!(solver)
    history = QCLB200.Row[]
    for ν = 1:options.max_scba
        row = QCLB200.step!(solver)
        push!(history, row)
        (row.status != 0 || row.r_Sigma <= options.tolerances.r_Σ) && break
    end
    return history, solver
end

end # module
