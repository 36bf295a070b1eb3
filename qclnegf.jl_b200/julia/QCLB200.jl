"""
    QCLB200

Julia binding of libqclb200.so, the B200 (sm_100a) implementation of the SCBA
hot path of QCLNEGF.jl.  Every function keeps the argument meaning and the
array layout of the QCLNEGF.jl function it replaces (fields are
`Array{ComplexF64,4}` of size `(N_E, N_k, N_b, N_b)`, energy fastest), calls
the library through `ccall` in the same way QCLNEGF.jl already calls LAPACK
(`numerics/optimized/production_operators.jl:20-61`), and maps the library
status to the same exceptions.

Set `ENV["QCLB200_LIB"]` to the path of `libqclb200.so` before loading.
"""
module QCLB200

using LinearAlgebra

const libqcl = get(ENV, "QCLB200_LIB", joinpath(@__DIR__, "..", "lib", "libqclb200.so"))

const QCL_C128 = Cint(0)
const QCL_C64 = Cint(1)
const QCL_MIXED = Cint(2)

function check(status::Cint)
    status == 0 && return nothing
    msg = unsafe_string(ccall((:qcl_last_error, libqcl), Cstring, ()))
    # the index of the failing pivot, as _production_inverse! reports LAPACK's info
    status == 1 && throw(SingularException(Int(ccall((:qcl_last_singular_pivot, libqcl), Cint, ()))))
    status == 2 && throw(DomainError(msg))
    status == 3 && throw(DimensionMismatch(msg))
    status == 4 && throw(ArgumentError(msg))
    # the memory preflight refuses as build_production_cache does (production_cache.jl:764-770)
    status == 8 && throw(ArgumentError(msg))
    error("qclb200 status $status: $msg")
end

"""Fused `_retarded_green_production` + the raw sandwiches of
`_current_green_production`: returns `(Gᴿ, Gˡ, Gᵍ, scale)`."""
function dyson_keldysh(ε::Vector{Float64}, h::Array{ComplexF64,3}, Σᴿ::Array{ComplexF64,4},
                       Σˡ::Array{ComplexF64,4}, Σᵍ::Array{ComplexF64,4}; η::Real = 0.0)
    NE, Nk, Nb, _ = size(Σᴿ)
    size(h) == (Nk, Nb, Nb) || throw(DimensionMismatch("h has wrong shape"))
    Gᴿ = similar(Σᴿ); Gˡ = similar(Σᴿ); Gᵍ = similar(Σᴿ)
    scale = zeros(Float64, NE, Nk)
    check(ccall((:qcl_dyson_keldysh, libqcl), Cint,
                (Cint, Cint, Cint, Cint, Ptr{Float64}, Float64, Ptr{ComplexF64}, Ptr{ComplexF64},
                 Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{ComplexF64},
                 Ptr{Float64}, Ptr{ComplexF64}, Ptr{ComplexF64}),
                QCL_C128, NE, Nk, Nb, ε, Float64(η), h, Σᴿ, Σˡ, Σᵍ, Gᴿ, Gˡ, Gᵍ, scale, C_NULL, C_NULL))
    return Gᴿ, Gˡ, Gᵍ, scale
end

"""`production_fft_hilbert_transform(Γ, ε, wᴱ, plan; return_roundoff)`."""
function fft_hilbert_transform(Γ::Array{ComplexF64,4}, ε::Vector{Float64}, wᴱ::Vector{Float64};
                               return_roundoff::Bool = false)
    NE = size(Γ, 1)
    Λ = similar(Γ)
    r = Ref{Float64}(0.0)
    check(ccall((:qcl_fft_hilbert_transform, libqcl), Cint,
                (Cint, Cint, Csize_t, Ptr{Float64}, Ptr{Float64}, Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{Float64}),
                QCL_C128, NE, length(Γ) ÷ NE, ε, wᴱ, Γ, Λ, return_roundoff ? r : C_NULL))
    return return_roundoff ? (Λ, r[]) : Λ
end

"""`apply_energy_shift!(destination, build_shift_plan(ε, δ), X)`."""
function apply_energy_shift!(dst::Array{ComplexF64,4}, ε::Vector{Float64}, δ::Real, X::Array{ComplexF64,4})
    Base.mightalias(dst, X) && throw(ArgumentError("in-place aliasing is not supported"))
    NE = size(X, 1)
    check(ccall((:qcl_apply_energy_shift, libqcl), Cint,
                (Cint, Cint, Csize_t, Ptr{Float64}, Float64, Ptr{ComplexF64}, Ptr{ComplexF64}),
                QCL_C128, NE, length(X) ÷ NE, ε, Float64(δ), X, dst))
    return dst
end

struct Mechanism
    kind::Cint
    is_LO::Cint
    J::Cint
    q::Float64
    block::Ptr{ComplexF64}
    matrix::Ptr{ComplexF64}
    left::Ptr{ComplexF64}
    right::Ptr{ComplexF64}
    radial::Ptr{ComplexF64}
end

"""`production_static_contraction(op, G, wᵏ, qᴷ)` for the factorised
operators: `:momentum_independent` (block), `:dense` (matrix), `:ifr`
(left, right, radial), `:low_rank` (left, right = right_adjoint of a
`LowRankProductionKernel`).  Arrays must stay rooted during the call."""
function production_static_contraction(kind::Symbol, arrays::NamedTuple, G::Array{ComplexF64,4},
                                       wᵏ::Vector{Float64}, qᴷ::Real; α::Real = 1, β::Real = 0,
                                       Σ::Array{ComplexF64,4} = zeros(ComplexF64, size(G)))
    NE, Nk, Nb, _ = size(G)
    k = kind === :momentum_independent ? 0 : kind === :dense ? 1 : kind === :ifr ? 2 :
        kind === :low_rank ? 3 : kind === :separable_sum ? 4 : throw(ArgumentError("unknown kernel kind $kind"))
    GC.@preserve arrays begin
        p(name) = haskey(arrays, name) ? pointer(getfield(arrays, name)) : Ptr{ComplexF64}(C_NULL)
        J = k == 4 ? size(arrays.radial, 3) : haskey(arrays, :left) ? size(arrays.left, 2) : 0
        op = Ref(Mechanism(k, 0, J, Float64(qᴷ), p(:block), p(:matrix), p(:left), p(:right), p(:radial)))
        check(ccall((:qcl_static_contraction, libqcl), Cint,
                    (Cint, Ref{Mechanism}, Cint, Cint, Cint, Ptr{Float64}, Float64, Float64,
                     Ptr{ComplexF64}, Ptr{ComplexF64}),
                    QCL_C128, op, NE, Nk, Nb, wᵏ, Float64(α), Float64(β), G, Σ))
    end
    return Σ
end

"""`condition_number(ε, h, Gᴿ, Σᴿ; η)` → `(κD, scaleD)`: the condition_number
and dyson_scale outputs of `_retarded_green_production` for the Dyson solve
that produced `Gᴿ`."""
function condition_number(ε::Vector{Float64}, h::Array{ComplexF64,3}, Gᴿ::Array{ComplexF64,4},
                          Σᴿ::Union{Nothing,Array{ComplexF64,4}} = nothing; η::Real = 0.0)
    NE, Nk, Nb, _ = size(Gᴿ)
    κ = zeros(Float64, NE, Nk); s = zeros(Float64, NE, Nk)
    check(ccall((:qcl_condition_number, libqcl), Cint,
                (Cint, Cint, Cint, Cint, Ptr{Float64}, Float64, Ptr{ComplexF64}, Ptr{ComplexF64},
                 Ptr{ComplexF64}, Ptr{Float64}, Ptr{Float64}),
                QCL_C128, NE, Nk, Nb, ε, Float64(η), h,
                Σᴿ === nothing ? Ptr{ComplexF64}(C_NULL) : Σᴿ, Gᴿ, κ, s))
    return κ, s
end

"""`spectral_function(Gᴿ)` = i(Gᴿ − Gᴿ†) per block."""
function spectral_function(Gᴿ::Array{ComplexF64,4})
    NE, Nk, Nb, _ = size(Gᴿ)
    A = similar(Gᴿ)
    check(ccall((:qcl_spectral_function, libqcl), Cint,
                (Cint, Cint, Cint, Cint, Ptr{ComplexF64}, Ptr{ComplexF64}), QCL_C128, NE, Nk, Nb, Gᴿ, A))
    return A
end

"""`production_residual_suite(ε, h, green, total, candidate)` →
`(r_D, r_A, r_K, r_PSD, r_caus)`."""
function production_residual_suite(ε, h, Gᴿ, Gˡ, Gᵍ, Σᴿ, Σˡ, Σᵍ, candidate_Σˡ)
    NE, Nk, Nb, _ = size(Gᴿ)
    out = zeros(Float64, 5)
    check(ccall((:qcl_residual_suite, libqcl), Cint,
                (Cint, Cint, Cint, Cint, Ptr{Float64}, Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{ComplexF64},
                 Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{ComplexF64},
                 Ptr{Float64}),
                QCL_C128, NE, Nk, Nb, ε, h, Gᴿ, Gˡ, Gᵍ, Σᴿ, Σˡ, Σᵍ, candidate_Σˡ, out))
    return (r_D = out[1], r_A = out[2], r_K = out[3], r_PSD = out[4], r_caus = out[5])
end

# ---------------------------------------------------------------------------
# SCBA level (solve_scba_production inner loop on the device)
# ---------------------------------------------------------------------------
struct Problem
    NE::Cint; Nk::Cint; Nb::Cint
    eps::Ptr{Float64}; wE::Ptr{Float64}; wk::Ptr{Float64}
    h::Ptr{ComplexF64}; Tplus::Ptr{ComplexF64}; Tminus::Ptr{ComplexF64}
    Ep::Float64; hw_LO::Float64; N_LO::Float64
    gs::Cint; target::Float64; eta_seed::Float64; kBT::Float64; alpha::Float64; J0::Float64
    precision::Cint; verify_roundoff::Cint; nmech::Cint
    # AlgorithmOptions model switches, 0 = default:
    # self_energy_structure (:full/:diagonal), transverse_momentum (:resolved/:averaged),
    # retarded_real_part (:kramers_kronig/:drop), elastic_retarded (:hilbert/:direct_green)
    self_energy_structure::Cint; transverse_momentum::Cint; retarded_real_part::Cint; elastic_retarded::Cint
    occupation_normalization::Cint  # :paired_convex / :scalar_lesser
    mixing::Cint                    # :linear / :anderson
    anderson_history_depth::Cint; anderson_damping::Float64; anderson_regularization::Float64
    memory_budget_bytes::Csize_t    # preflight budget (ProductionOptions.memory_budget_bytes); 0 = free memory
    refinement::Cint                # 1: a mixed context that can finish in FP64 (promote!)
end

struct MemoryEstimate
    fields::Csize_t; operators::Csize_t; workspace::Csize_t; anderson::Csize_t; resident::Csize_t; peak::Csize_t
end

struct Row
    nu::Cint; status::Cint
    r_D::Float64; r_A::Float64; r_K::Float64; r_Sigma::Float64; r_lambda::Float64; lambda::Float64
    r_PSD::Float64; r_caus::Float64; r_roundoff::Float64; r_J::Float64; r_pop::Float64
    J::Float64; Jbar::Float64; number::Float64; holes::Float64
    occupied_fraction::Float64; empty_fraction::Float64
    target_charge::Float64; normalized_charge::Float64; lambda_change::Float64
end

mutable struct Solver
    handle::Ptr{Cvoid}
    keep::Vector{Any}
end

"""The `Problem` struct and the mechanism operators of one fixed-point
solve, from the reference's grids (ModelGrids ε, wᴱ, wᵏ), projected
Hamiltonians h (N_k, N_b, N_b), neighbour couplings (BasisData.T₊, T₋) and
scaled physics (Eᵖ, ħωᴸᴼ, N_LO, g_s, Nᴰ²ᴰ, η_seed, k_B T, α_Σ, J₀);
`ops` = [(name, cached AbstractProductionKernel, qᴷ)] in the reference's
mechanism order.  Every array is pushed to `keep` (rooted for the life of the
solver).  Kernel types map to QCL_KERNEL_*: MomentumIndependent -> 0 (block),
Dense -> 1 (matrix), _SeparableIFR -> 2 (left, right, radial), LowRank -> 3
(left, right_adjoint); a wrapper with fields `radial`, `block` -> 4."""
function problem_and_mechanisms(ε, wᴱ, wᵏ, h, T₊, T₋, Eᵖ, ħω, NLO, gs, target, ηseed, kBT, α, J₀, ops,
                                keep::Vector{Any}; precision::Symbol = :c128)
    prec = precision === :c128 ? QCL_C128 : precision === :c64 ? Cint(1) : Cint(2)
    arrays = Any[Vector{Float64}(ε), Vector{Float64}(wᴱ), Vector{Float64}(wᵏ), Array{ComplexF64,3}(h),
                 Matrix{ComplexF64}(T₊), Matrix{ComplexF64}(T₋)]
    append!(keep, arrays)
    mechs = Mechanism[]
    nullp = Ptr{ComplexF64}(C_NULL)
    for (name, op, q) in ops
        isLO = Cint(name === :LO)
        if hasfield(typeof(op), :radial) && hasfield(typeof(op), :block)       # separable sum
            push!(keep, op.radial, op.block)
            push!(mechs, Mechanism(4, isLO, size(op.radial, 3), q, pointer(op.block), nullp, nullp, nullp,
                                   pointer(op.radial)))
        elseif hasfield(typeof(op), :right_adjoint)                          # LowRankProductionKernel
            push!(keep, op.left, op.right_adjoint)
            push!(mechs, Mechanism(3, isLO, size(op.left, 2), q, nullp, nullp, pointer(op.left),
                                   pointer(op.right_adjoint), nullp))
        elseif hasfield(typeof(op), :radial)                                 # _SeparableIFRProductionKernel
            push!(keep, op.left, op.right, op.radial)
            push!(mechs, Mechanism(2, isLO, size(op.left, 2), q, nullp, nullp, pointer(op.left),
                                   pointer(op.right), pointer(op.radial)))
        elseif hasfield(typeof(op), :block)                                  # MomentumIndependent
            push!(keep, op.block)
            push!(mechs, Mechanism(0, isLO, 0, q, pointer(op.block), nullp, nullp, nullp, nullp))
        else                                                                 # DenseProductionKernel
            push!(keep, op.matrix)
            push!(mechs, Mechanism(1, isLO, 0, q, nullp, pointer(op.matrix), nullp, nullp, nullp))
        end
    end
    p = Problem(length(ε), size(h, 1), size(h, 2), pointer(arrays[1]), pointer(arrays[2]), pointer(arrays[3]),
                pointer(arrays[4]), pointer(arrays[5]), pointer(arrays[6]), Eᵖ, ħω, NLO, Cint(gs), target,
                ηseed, kBT, α, J₀, prec, Cint(1), Cint(length(mechs)), 0, 0, 0, 0, 0, 0, 5, 1.0, 1e-12,
                Csize_t(0), Cint(0))
    return p, mechs
end

function create(problem::Problem, mechanisms::Vector{Mechanism}, keep::Vector{Any})
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:qcl_scba_create, libqcl), Cint, (Ref{Problem}, Ptr{Mechanism}, Ref{Ptr{Cvoid}}),
                problem, mechanisms, h))
    s = Solver(h[], keep)
    finalizer(x -> ccall((:qcl_scba_destroy, libqcl), Cvoid, (Ptr{Cvoid},), x.handle), s)
    return s
end

# _estimate_production_memory / build_production_cache's refusal (production_cache.jl:475-668, 764-770)
function estimate_memory(problem::Problem, mechanisms::Vector{Mechanism})
    out = Ref{MemoryEstimate}()
    check(ccall((:qcl_scba_estimate_memory, libqcl), Cint, (Ref{Problem}, Ptr{Mechanism}, Ref{MemoryEstimate}),
                problem, mechanisms, out))
    return out[]
end

# FP64 refinement of a mixed-precision state (a context created with refinement = 1)
promote!(s::Solver) = check(ccall((:qcl_scba_promote, libqcl), Cint, (Ptr{Cvoid},), s.handle))

seed!(s::Solver) = (μ = Ref(0.0); check(ccall((:qcl_scba_seed, libqcl), Cint, (Ptr{Cvoid}, Ref{Float64}), s.handle, μ)); μ[])

function step!(s::Solver)
    r = Ref{Row}()
    check(ccall((:qcl_scba_step, libqcl), Cint, (Ptr{Cvoid}, Ref{Row}), s.handle, r))
    return r[]
end

function download(s::Solver, which::Integer, shape::NTuple{4,Int})
    out = Array{ComplexF64,4}(undef, shape)
    check(ccall((:qcl_scba_download, libqcl), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), s.handle, which, out))
    return out
end

upload!(s::Solver, which::Integer, X::Array{ComplexF64,4}) =
    check(ccall((:qcl_scba_upload, libqcl), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), s.handle, which, X))

function download_candidate(s::Solver, which::Integer, shape::NTuple{4,Int})
    out = Array{ComplexF64,4}(undef, shape)
    check(ccall((:qcl_scba_download_candidate, libqcl), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), s.handle,
                which, out))
    return out
end

# ---------------------------------------------------------------------------
# Implicit differentiation of the converged fixed point (qcl_scba_tangent_*)
# ---------------------------------------------------------------------------
tangent_init!(s::Solver) = check(ccall((:qcl_scba_tangent_init, libqcl), Cint, (Ptr{Cvoid},), s.handle))
tangent_set!(s::Solver, which::Integer, X::Array{ComplexF64,4}) =
    check(ccall((:qcl_scba_tangent_set, libqcl), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), s.handle, which, X))
tangent_reset!(s::Solver) =
    check(ccall((:qcl_scba_tangent_set, libqcl), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), s.handle, -1, C_NULL))
function tangent_step!(s::Solver)
    out = zeros(2)
    check(ccall((:qcl_scba_tangent_step, libqcl), Cint, (Ptr{Cvoid}, Ptr{Float64}), s.handle, out))
    return out[1], out[2]  # J_Sigma v (solver units), largest relative change of v
end

"""A problem family for differentiation: `build(p)` returns
`(problem, mechanisms, keep, shape)` for the parameter vector p (the bias, layer
thicknesses, ...), `shape` = (N_E, N_k, N_b, N_b)."""
const ProblemFamily = Function

_families(nmech) = 3 .+ 3 .* (0:nmech+1)  # first component index of each self-energy family

function _converged(build, p, tol, max_iter)
    problem, mechs, keep, shape = build(p)
    s = create(problem, mechs, keep)
    seed!(s)
    row = step!(s)
    while row.r_Sigma > tol && row.nu < max_iter
        row = step!(s)
    end
    row.r_Sigma <= tol || error("SCBA did not reach r_Sigma <= $tol in $max_iter iterations")
    return s, row, problem, mechs, shape
end

normalization_branch(s::Solver) = (b = Ref{Cint}(0); check(ccall((:qcl_scba_normalization_branch, libqcl), Cint,
                                   (Ptr{Cvoid}, Ref{Cint}), s.handle, b)); Int(b[]))
set_normalization_branch!(s::Solver, b::Integer) =
    check(ccall((:qcl_scba_set_normalization_branch, libqcl), Cint, (Ptr{Cvoid}, Cint), s.handle, b))

# One application of the map Phi at the fixed-point state `fams` for the
# problem at p: Phi per family component and J (the explicit dependence), with
# the paired normalisation held in the fixed point's form `branch`.
function _map_at(build, p, fams, α, branch)
    problem, mechs, keep, shape = build(p)
    s = create(problem, mechs, keep)
    set_normalization_branch!(s, branch)
    for (which, X) in fams
        upload!(s, which, X)
    end
    row = step!(s)
    phi = Dict(which => X .+ (download_candidate(s, which, shape) .- X) ./ α for (which, X) in fams)
    return phi, row.J
end

"""dJ/dp at p0 by implicit differentiation of the FP64 fixed point
(qcl_scba_tangent_*), with the explicit part Phi_p, J_p by central
differences of ONE map application at the fixed point (steps[k] for p_k).
Returns (J, dJ/dp)."""
function implicit_gradient(build::ProblemFamily, p0::AbstractVector{<:Real}, steps::AbstractVector{<:Real};
                           tol = 1e-11, max_iter = 20000, tangent_tol = 1e-11, max_tangent = 20000)
    s, row, problem, mechs, shape = _converged(build, p0, tol, max_iter)
    fams = [(which + c, download(s, which + c, shape)) for which in _families(length(mechs)) for c in 0:2]
    branch = normalization_branch(s)
    tangent_init!(s)
    grad = zeros(length(p0))
    for k in eachindex(p0)
        e = zeros(length(p0)); e[k] = steps[k]
        φp, Jp = _map_at(build, p0 .+ e, fams, problem.alpha, branch)
        φm, Jm = _map_at(build, p0 .- e, fams, problem.alpha, branch)
        for (which, _) in fams
            tangent_set!(s, which, (φp[which] .- φm[which]) ./ (2steps[k]))
        end
        tangent_reset!(s)
        n, change = 0, Inf
        while change > tangent_tol && n < max_tangent
            _, change = tangent_step!(s)
            n += 1
        end
        jv, _ = tangent_step!(s)
        grad[k] = jv * problem.J0 + (Jp - Jm) / (2steps[k])
    end
    return row.J, grad
end

"""The converged current density J(p) of a problem family (the primal of
the ChainRulesCore rrule in QCLB200ChainRulesExt)."""
converged_current(build::ProblemFamily, p::AbstractVector{<:Real}; tol = 1e-11, max_iter = 20000) =
    _converged(build, p, tol, max_iter)[2].J

end # module
