"""The Kronecker-sum (separable-sum) kernel operator.

K(m, m') = q sum_i radial_i(m, m') block_i holds the momentum-dependent
kernels without their (N_k N_b^2)^2 dense matrix: the exact LO kernel
(lo_phonon_kernel, numerics/reference/kernels.jl:321-356) and the tabulated
impurity kernel (_assemble_lookup_kernel + _production_impurity_evaluator,
numerics/optimized/kernels.jl:122-158, 303-320).

CPU: the host compression reproduces the oracle's literal six-index kernels
to 1e-13 (relative, max norm), and its contraction in the oracle equals the
literal contraction.  GPU: the contraction against the oracle's literal
six-index map (complex128 1e-13, complex64 on the tensor cores 2e-6), with
several term chunks and beta != 0, and an SCBA whose LO and impurity kernels
are separable sums against the oracle's dense-operator SCBA.
"""
import dataclasses

import numpy as np
import pytest

from helpers import approx_err


def _structure(seed=5, Nb=3, Nz=40, Nk=4):
    rng = np.random.default_rng(seed)
    x = np.linspace(0.025, 1.975, Nz)
    wx = np.full(Nz, 2.0 / Nz)
    chi = np.zeros((Nz, Nb))
    for a in range(Nb):
        chi[:, a] = np.exp(-((x - 0.4 - 0.5 * a) / 0.3) ** 2) * (1 + 0.2 * rng.standard_normal())
    chi /= np.sqrt((chi ** 2 * wx[:, None]).sum(axis=0))
    kappa = np.linspace(0.0, 1.5, Nk)
    return x, wx, chi.astype(complex), kappa


def _maxrel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b)))


def _lo(Nb=3, Nk=4, Nphi=8, Nq=21, qscreen=0.4, prefactor=2.3):
    from qclb200.kernel_build import lo_form_factors, lo_weights, separable_sum_operator

    x, wx, chi, kappa = _structure(Nb=Nb, Nk=Nk)
    qz = np.linspace(-6.0, 6.0, Nq)
    wqz = np.full(Nq, qz[1] - qz[0])
    F = lo_form_factors(chi, x, wx, qz)
    W = lo_weights(kappa, Nphi, qz, wqz, qscreen, prefactor)
    mech = separable_sum_operator("LO", W, F.reshape((Nq, Nb * Nb), order="F"))
    return mech, (F, qz, wqz, kappa, Nphi, qscreen, prefactor)


def _impurity(Nb=4, Nk=5, Nphi=10, T=17):
    from qclb200.kernel_build import impurity_pair_factors, lookup_weights, separable_sum_operator, transfer_momenta

    x, wx, chi, kappa = _structure(Nb=Nb, Nk=Nk)
    donors = np.where(x < 0.5, 0.8, 0.0) * wx
    qmax = float(transfer_momenta(kappa, Nphi).max())
    nodes = qmax * (np.arange(T) / (T - 1)) ** 2
    V, d = zip(*(impurity_pair_factors(q, chi, x, wx, donors, 0.3, 1.7) for q in nodes))
    mech = separable_sum_operator("impurity", lookup_weights(nodes, kappa, Nphi), np.array(V), d[0])
    return mech, (nodes, chi, x, wx, donors, kappa, Nphi)


@pytest.mark.parametrize("Nb,Nk,Nq", [(3, 4, 21), (5, 6, 41)])
def test_separable_lo_kernel_matches_literal(orc, Nb, Nk, Nq):
    mech, (F, qz, wqz, kappa, Nphi, qs, pre) = _lo(Nb=Nb, Nk=Nk, Nq=Nq)
    K = orc.lo_kernel_literal(F, qz, wqz, kappa, Nphi, qs, pre)
    assert mech.radial.shape[2] < Nq  # fewer terms than q_z nodes
    assert _maxrel(mech.q * mech.literal_kernel(Nk, Nb), K) < 1e-13
    assert mech.q >= float(np.max(np.abs(K))) * (1 - 1e-12)  # an upper bound of max|K|


def test_separable_tabulated_impurity_kernel_matches_literal(orc):
    mech, (nodes, chi, x, wx, donors, kappa, Nphi) = _impurity()
    blocks = [orc.impurity_block_literal(q, chi, x, wx, donors, 0.3, 1.7) for q in nodes]
    K = orc.assemble_lookup_kernel(nodes, blocks, kappa, Nphi)
    Nb, Nk = chi.shape[1], len(kappa)
    assert _maxrel(mech.q * mech.literal_kernel(Nk, Nb), K) < 1e-13


def test_separable_sum_rejects_zero_kernel_and_tight_cap():
    from qclb200.kernel_build import lo_form_factors, lo_weights, separable_sum_operator

    x, wx, chi, kappa = _structure()
    qz = np.linspace(-6.0, 6.0, 21)
    W = lo_weights(kappa, 8, qz, np.full(21, 0.6), 0.4, 1.0)
    F = lo_form_factors(chi, x, wx, qz).reshape((21, 9), order="F")
    with pytest.raises(ValueError):
        separable_sum_operator("LO", W, np.zeros_like(F))
    with pytest.raises(ValueError):
        separable_sum_operator("LO", W, F, max_terms=1)
    loose = separable_sum_operator("LO", W, F, rtol=1e-6)
    tight = separable_sum_operator("LO", W, F, rtol=1e-15)
    assert loose.radial.shape[2] < tight.radial.shape[2]
    assert 0 < loose.residual <= 1e-6


def test_oracle_contraction_of_separable_sum_is_the_literal_map(orc):
    mech, _ = _lo()
    rng = np.random.default_rng(2)
    Nk, Nb = mech.radial.shape[0], 3
    G = np.asfortranarray(rng.standard_normal((11, Nk, Nb, Nb)) + 1j * rng.standard_normal((11, Nk, Nb, Nb)))
    wk = rng.uniform(0.5, 1.5, Nk)
    got = orc.contraction(mech, G, wk, alpha=0.7)
    lit = orc.contraction_literal(mech.literal_kernel(Nk, Nb), G, wk, 0.7 * mech.q)
    assert approx_err(got, lit) < 1e-14


def _random_separable(rng, Nk, Nb, J):
    from qclb200.problem import Mechanism

    radial = rng.standard_normal((Nk, Nk, J)) + 1j * rng.standard_normal((Nk, Nk, J))
    block = rng.standard_normal((Nb * Nb, Nb * Nb, J)) + 1j * rng.standard_normal((Nb * Nb, Nb * Nb, J))
    return Mechanism("impurity", "separable_sum", 0.37, radial=np.asfortranarray(radial),
                     block=np.asfortranarray(block))


@pytest.mark.gpu
@pytest.mark.parametrize("J", [1, 8, 11])  # one chunk, a full chunk, two chunks
@pytest.mark.parametrize("beta", [0.0, 1.0])
def test_separable_contraction_matches_literal_oracle(gpu_ops, orc, J, beta):
    rng = np.random.default_rng(J)
    NE, Nk, Nb = 37, 4, 4
    mech = _random_separable(rng, Nk, Nb, J)
    G = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    S0 = np.asfortranarray(rng.standard_normal(G.shape) + 1j * rng.standard_normal(G.shape))
    wk = rng.uniform(0.2, 1.0, Nk)
    lit = orc.contraction_literal(mech.literal_kernel(Nk, Nb), G, wk, 1.7 * mech.q) + beta * S0
    got = gpu_ops.production_static_contraction(mech, G, wk, alpha=1.7, beta=beta, S=S0)
    assert approx_err(got, lit) < 1e-13
    got32 = gpu_ops.production_static_contraction(mech, G, wk, alpha=1.7, beta=beta, S=S0, precision="c64")
    assert approx_err(got32, lit) < 2e-6


@pytest.mark.gpu
def test_separable_contraction_physical_kernels_on_gpu(gpu_ops, orc):
    """The compressed LO and impurity operators against the literal
    contraction of the oracle's literal kernels (not of the compressed
    factors): compression and contraction together."""
    lo, (F, qz, wqz, kappa, Nphi, qs, pre) = _lo(Nb=5, Nk=6, Nq=41)
    K_lo = orc.lo_kernel_literal(F, qz, wqz, kappa, Nphi, qs, pre)
    imp, (nodes, chi, x, wx, donors, kappa2, Nphi2) = _impurity(Nb=5, Nk=6)
    blocks = [orc.impurity_block_literal(q, chi, x, wx, donors, 0.3, 1.7) for q in nodes]
    K_imp = orc.assemble_lookup_kernel(nodes, blocks, kappa2, Nphi2)
    rng = np.random.default_rng(9)
    NE, Nk, Nb = 29, 6, 5
    G = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    wk = rng.uniform(0.2, 1.0, Nk)
    for mech, K in ((lo, K_lo), (imp, K_imp)):
        lit = orc.contraction_literal(K, G, wk, 1.0)
        assert approx_err(gpu_ops.production_static_contraction(mech, G, wk), lit) < 1e-13
        assert approx_err(gpu_ops.production_static_contraction(mech, G, wk, precision="c64"), lit) < 2e-6


def _separable_problem():
    """small_problem with its dense LO and impurity operators replaced by
    separable sums of the same kernels (rtol 1e-15)."""
    from qclb200.kernel_build import separable_sum_operator
    from qclb200.problem import small_problem

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "impurity", "IFR"))
    mechs = []
    for m in pr.mechanisms:
        if m.kind == "dense":
            K = m.literal_kernel(pr.Nk, pr.Nb)  # [m, m', a, c, d, b]
            Nk, Nb = pr.Nk, pr.Nb
            W = np.eye(Nk * Nk)  # one node per (m, m'): X_(m,m') = K[m, m'] in pair layout
            X = np.transpose(K, (0, 1, 2, 3, 5, 4)).reshape((Nk * Nk, Nb * Nb, Nb * Nb), order="F")
            # factor each Hermitian node tensor X = V diag(d) V^H (it is PSD for these kernels)
            Vs, ds = [], []
            for t in range(Nk * Nk):
                w, U = np.linalg.eigh(0.5 * (X[t] + X[t].conj().T))
                Vs.append(U * np.sqrt(np.maximum(w, 0.0))[None, :])
            sep = separable_sum_operator(m.name, W, np.array(Vs))
            sep.q *= m.q
            mechs.append(sep)
        else:
            mechs.append(m)
    return dataclasses.replace(pr, mechanisms=mechs), pr


def test_separable_problem_reproduces_dense_kernels():
    sep, dense = _separable_problem()
    for a, b in zip(sep.mechanisms, dense.mechanisms):
        if b.kind == "dense":
            Ka = a.q * a.literal_kernel(dense.Nk, dense.Nb)
            Kb = b.q * b.literal_kernel(dense.Nk, dense.Nb)
            assert _maxrel(Ka, Kb) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("c128", 1e-9), ("mixed", 2e-5)])
def test_scba_with_separable_operators_matches_dense_oracle(gpu_ops, orc, precision, tol):
    from qclb200.scba import solve_scba_production

    sep, dense = _separable_problem()
    hist_o, _ = orc.scba(dense, 3)
    hist_g, solver = solve_scba_production(sep, 3, precision=precision)
    solver.close()
    for ro, rg in zip(hist_o, hist_g):
        assert abs(rg["J"] - ro["J"]) <= tol * abs(ro["J"])
        assert abs(rg["r_Sigma"] - ro["rSigma"]) <= max(tol, 1e-6) * abs(ro["rSigma"]) + 1e-12


@pytest.mark.gpu
def test_separable_contraction_large_operands(gpu_ops):
    """Operands larger than L2 (stage 1: 524 288 rows x 64, 134 MB of FP16
    pairs; stage 2: 65 536 rows x 4096, 1.07 GB as FP16 pairs and 2.1 GB as
    complex128), where the tensor-core and DMMA kernels run their tiles
    column-fastest so that the large A is read once: both precisions against
    the two stages of the Kronecker sum evaluated in numpy (complex128 1e-12,
    complex64 2e-6)."""
    rng = np.random.default_rng(21)
    NE, Nk, Nb, J = 2048, 32, 16, 8
    mech = _random_separable(rng, Nk, Nb, J)
    G = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    wk = rng.uniform(0.2, 1.0, Nk)
    alpha = 0.9
    Gf = G.reshape((NE, Nk, Nb * Nb), order="F") * wk[None, :, None]
    want = np.zeros((NE, Nk, Nb * Nb), dtype=np.complex128)
    for i in range(J):
        Z = np.einsum("mn,enc->emc", mech.radial[:, :, i], Gf)  # stage 1
        want += Z @ mech.block[:, :, i].T  # stage 2: S[e, m, ab] += sum_cd block[ab, cd] Z[e, m, cd]
    want = (alpha * mech.q * want).reshape(G.shape, order="F")
    got = gpu_ops.production_static_contraction(mech, G, wk, alpha=alpha)
    assert approx_err(got, want) < 1e-12
    got32 = gpu_ops.production_static_contraction(mech, G, wk, alpha=alpha, precision="c64")
    assert approx_err(got32, want) < 2e-6
