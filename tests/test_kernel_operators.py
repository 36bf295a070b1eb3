"""Factorised kernel operators: the host builder (_production_kernel /
_low_rank_production_kernel, numerics/optimized/production_cache.jl:339-409)
and the low-rank contraction (production_operators.jl:597-658).

CPU tests restate test/numerics/literal_blas_and_low_rank_kernel_operators.jl
with this project's RNG (the reference's Xoshiro streams are Julia-only): the
dense and full-rank operators reproduce the literal six-index map
(3e-14 / 2e-13), and a truncated operator meets its tolerance with the
reported residual.  GPU tests run the low-rank contraction through the C ABI
against the oracle, alone and inside the SCBA loop.
"""
import numpy as np
import pytest

from helpers import approx_err


def _random_kernel(seed=0xA190, NE=5, Nk=3, Nb=2):
    rng = np.random.default_rng(seed)
    K = rng.standard_normal((Nk, Nk, Nb, Nb, Nb, Nb)) + 1j * rng.standard_normal((Nk, Nk, Nb, Nb, Nb, Nb))
    G = rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb))
    w = rng.uniform(0.0, 1.0, Nk)
    return np.asfortranarray(K), np.asfortranarray(G), w


# ---------------------------------------------------------------------------
# host builder + oracle (CPU)
# ---------------------------------------------------------------------------

def test_literal_dense_and_low_rank_operators(orc):
    from qclb200.problem import production_kernel

    NE, Nk, Nb = 5, 3, 2
    K, G, w = _random_kernel(NE=NE, Nk=Nk, Nb=Nb)
    scale = 0.13
    ref = orc.contraction_literal(K, G, w, scale)

    dense = production_kernel("x", scale, K, contraction="dense_blas")
    assert dense.kind == "dense"
    assert approx_err(orc.contraction(dense, G, w), ref) < 3e-14

    literal = production_kernel("x", scale, K, contraction="literal")
    assert approx_err(orc.contraction(literal, G, w), ref) < 3e-14

    full = production_kernel("x", scale, K, contraction="low_rank", low_rank_relative_tolerance=0.0)
    assert full.kind == "low_rank"
    assert full.left.shape[1] == Nk * Nb ** 2
    assert full.residual == 0.0
    assert approx_err(orc.contraction(full, G, w), ref) < 2e-13

    ctl = production_kernel("x", scale, K, contraction="low_rank", low_rank_relative_tolerance=0.45)
    assert ctl.left.shape[1] < Nk * Nb ** 2
    approx = ctl.left @ ctl.right
    measured = np.linalg.norm(approx - dense.matrix) / np.linalg.norm(dense.matrix)
    assert measured <= 0.45 + 128 * np.finfo(float).eps
    assert measured == pytest.approx(ctl.residual, rel=2e-13)
    # the truncated operator is the literal map of its own reconstruction
    assert approx_err(orc.contraction(ctl, G, w), orc.contraction_literal(ctl.literal_kernel(Nk, Nb), G, w,
                                                                          scale)) < 2e-13


def test_low_rank_rank_is_minimal_for_the_tolerance():
    from qclb200.problem import low_rank_production_kernel

    rng = np.random.default_rng(5)
    n = 24
    U, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    V, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    s = 2.0 ** -np.arange(n)
    M = (U * s) @ V.conj().T
    for tol in (1e-1, 1e-3, 1e-6):
        op = low_rank_production_kernel("x", 1.0, M, tol)
        r = op.left.shape[1]
        tail = lambda k: np.linalg.norm(s[k:]) / np.linalg.norm(s)
        assert tail(r) <= tol + 64 * np.finfo(float).eps
        assert tail(r - 1) > tol
        assert op.residual == pytest.approx(tail(r), rel=1e-12)


def test_low_rank_cap_that_misses_the_tolerance_raises():
    from qclb200.problem import low_rank_production_kernel

    rng = np.random.default_rng(6)
    M = rng.standard_normal((12, 12)) + 1j * rng.standard_normal((12, 12))
    with pytest.raises(ValueError, match="cannot satisfy"):
        low_rank_production_kernel("x", 1.0, M, relative_tolerance=1e-3, maximum_rank=2)
    with pytest.raises(ValueError):
        low_rank_production_kernel("x", 1.0, M, relative_tolerance=1.0)
    # a cap that still meets the tolerance is accepted
    op = low_rank_production_kernel("x", 1.0, M, relative_tolerance=0.0, maximum_rank=12)
    assert op.left.shape[1] == 12


def test_momentum_independent_kernel_is_detected(orc):
    from qclb200.problem import production_kernel

    K, G, w = _random_kernel(seed=11, NE=7, Nk=4, Nb=3)
    K[...] = K[0, 0][None, None]
    op = production_kernel("x", 0.7, K)
    assert op.kind == "momentum_independent"
    assert approx_err(orc.contraction(op, G, w), orc.contraction_literal(K, G, w, 0.7)) < 3e-14
    with pytest.raises(ValueError):
        production_kernel("x", 1.0, K[:, :, :, :, :, :1])


# ---------------------------------------------------------------------------
# CUDA path (GPU)
# ---------------------------------------------------------------------------

def _dense_problem_kernel(seed, NE, Nk, Nb):
    """A smooth (numerically low-rank) covariance kernel like the LO /
    impurity forms, plus a random field."""
    rng = np.random.default_rng(seed)
    kappa = np.linspace(0.0, 2.0, Nk)
    Nq = 4
    F = rng.standard_normal((Nq, Nb, Nb)) + 1j * rng.standard_normal((Nq, Nb, Nb))
    R = np.array([1.0 / (1.0 + (kappa[:, None] - kappa[None, :]) ** 2 + h) for h in range(Nq)])
    K = np.einsum("hmn,hac,hbd->mnacdb", R, F, np.conj(F))
    G = rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb))
    w = rng.uniform(0.1, 1.0, Nk)
    return np.asfortranarray(K), np.asfortranarray(G), w


@pytest.mark.gpu
@pytest.mark.parametrize("NE,Nk,Nb,tol,beta", [(5, 3, 2, 0.0, 0.0), (5, 3, 2, 0.45, 0.5), (300, 4, 4, 1e-3, 0.0),
                                                (129, 6, 3, 0.0, 1.0)])
def test_low_rank_contraction_c128_matches_oracle(gpu_ops, orc, NE, Nk, Nb, tol, beta):
    from qclb200.problem import production_kernel

    K, G, w = _dense_problem_kernel(NE + Nk, NE, Nk, Nb)
    op = production_kernel("x", 0.37, K, contraction="low_rank", low_rank_relative_tolerance=tol)
    S0 = np.asfortranarray(np.random.default_rng(2).standard_normal(G.shape) + 0j)
    want = orc.contraction(op, G, w, alpha=1.3, beta=beta, S=S0.copy(order="F"))
    got = gpu_ops.production_static_contraction(op, G, w, alpha=1.3, beta=beta, S=S0)
    assert approx_err(got, want) < 1e-13
    if tol == 0.0:
        assert approx_err(got, orc.contraction_literal(K, G, w, 0.37 * 1.3) + beta * S0) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["c64", "mixed"])
def test_low_rank_contraction_c64_matches_oracle(gpu_ops, orc, precision):
    from qclb200.problem import production_kernel

    K, G, w = _dense_problem_kernel(9, 257, 5, 4)
    op = production_kernel("x", 0.37, K, contraction="low_rank", low_rank_relative_tolerance=1e-4)
    want = orc.contraction(op, G, w)
    got = gpu_ops.production_static_contraction(op, G, w, precision=precision)
    assert got.dtype == np.complex64
    assert approx_err(got, want) < 2e-6


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["momentum_independent", "dense_blas", "low_rank"])
def test_built_operators_match_literal_map_on_gpu(gpu_ops, orc, form):
    """Random (index-asymmetric) six-index kernels through the host builder and
    the C ABI: each factorised form reproduces the literal map."""
    from qclb200.problem import production_kernel

    K, G, w = _random_kernel(seed=21, NE=67, Nk=3, Nb=3)
    if form == "momentum_independent":
        K[...] = K[0, 0][None, None]
    op = production_kernel("x", 0.21, K, contraction="low_rank" if form == "low_rank" else "dense_blas")
    assert op.kind == {"momentum_independent": "momentum_independent", "dense_blas": "dense",
                       "low_rank": "low_rank"}[form]
    got = gpu_ops.production_static_contraction(op, G, w)
    assert approx_err(got, orc.contraction_literal(K, G, w, 0.21)) < 1e-13


@pytest.mark.gpu
def test_low_rank_operator_rejects_zero_rank(gpu_ops):
    from qclb200.problem import Mechanism

    Nk, Nb = 2, 2
    op = Mechanism("x", "low_rank", 1.0, left=np.zeros((Nk * Nb * Nb, 0), complex),
                   right=np.zeros((0, Nk * Nb * Nb), complex))
    G = np.zeros((4, Nk, Nb, Nb), dtype=complex, order="F")
    with pytest.raises(Exception, match="rank"):
        gpu_ops.production_static_contraction(op, G, np.ones(Nk))


@pytest.mark.gpu
def test_scba_with_low_rank_impurity_matches_oracle(gpu_ops, orc):
    from qclb200.problem import low_rank_production_kernel, small_problem
    from qclb200.scba import solve_scba_production

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "impurity"))
    for i, m in enumerate(pr.mechanisms):
        if m.kind == "dense":
            pr.mechanisms[i] = low_rank_production_kernel(m.name, m.q, m.matrix, relative_tolerance=1e-3)
    assert sum(m.kind == "low_rank" for m in pr.mechanisms) == 2
    hist_o, _ = orc.scba(pr, 3)
    hist_g, solver = solve_scba_production(pr, 3)
    solver.close()
    for ro, rg in zip(hist_o, hist_g):
        for ko, kg in (("J", "J"), ("rSigma", "r_Sigma"), ("lam", "lam"), ("rK", "r_K")):
            a, b = ro[ko], rg[kg]
            assert abs(a - b) <= 1e-9 * max(abs(a), abs(b)) + 1e-15, (ro["nu"], ko, a, b)
