"""Anderson mixing of the SCBA families with its causality guard
(numerics/optimized/production_mixing.jl:1-317; mixing = :anderson in
production_solver.jl:798-818).

CPU: the oracle's coefficient solve on known Gram matrices, its guard on
planted defects (each failure code at its block, first failure in the
reference's (family, e, m) order), history eviction and the
residual-increase restart, and faster early contraction than linear mixing
on the all-mechanism test structure.  GPU: the guard kernel on the same
planted cases, and the device SCBA loop with Anderson mixing against the
oracle's (rows within 1e-7: the coefficients come from a regularised Gram
solve, which amplifies the last-bit differences of the inner products; the
mixer's decisions must agree exactly), eager and graph-replayed.
"""
import dataclasses
import math

import numpy as np
import pytest

from helpers import psd_blocks


def test_coefficients_known_gram(orc):
    assert np.array_equal(orc.anderson_coefficients(np.array([[3.0]]), 1e-12), [1.0])
    # orthogonal residuals: c_i proportional to 1 / |R_i|^2
    c = orc.anderson_coefficients(np.diag([4.0, 1.0]), 0.0)
    np.testing.assert_allclose(c, [0.2, 0.8], rtol=1e-14)
    # identical residuals: the null direction is cut off, the rest is split evenly
    c = orc.anderson_coefficients(np.array([[2.0, 2.0], [2.0, 2.0]]), 1e-12)
    np.testing.assert_allclose(c, [0.5, 0.5], rtol=1e-12)
    with pytest.raises(ValueError):
        orc.anderson_coefficients(np.zeros((2, 2)), 0.0)


def _families(seed=4, NE=9, Nk=3, Nb=4, nfam=3):
    """Causal, Keldysh-consistent families: S< = i P<, S> = -i P>, S^R =
    -i (P< + P>)/2 + Hermitian."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nfam):
        PL, PG = psd_blocks(rng, NE, Nk, Nb, 0.02), psd_blocks(rng, NE, Nk, Nb, 0.03)
        herm = 0.01 * (rng.standard_normal(PL.shape) + 1j * rng.standard_normal(PL.shape))
        herm = herm + np.conj(np.transpose(herm, (0, 1, 3, 2)))
        out.append(tuple(np.asfortranarray(x) for x in (-0.5j * (PL + PG) + herm, 1j * PL, -1j * PG)))
    return out


def _planted():
    """(name, families, expected (first 1-based index, code)); NE = 9, Nk = 3."""
    NE, Nk = 9, 3
    idx = lambda f, e, m: f * NE * Nk + e * Nk + m + 1
    cases = [("clean", _families(), (0, 0))]
    F = [list(f) for f in _families()]
    R = F[1][0].copy(order="F")
    R[4, 2] += 0.2j * np.eye(4)                      # Im Sigma^R > 0: acausal
    F[1][0] = R
    F2 = [list(f) for f in _families()]
    L = F2[2][1].copy(order="F")
    L[2, 0, 0, 1] += 0.05                             # -i Sigma< loses Hermiticity
    F2[2][1] = L
    F3 = [list(f) for f in _families()]
    L = F3[0][1].copy(order="F")
    L[6, 1] += -0.5j * np.eye(4)                      # -i Sigma< gains a negative eigenvalue
    F3[0][1] = L
    F3[0][0] = F3[0][0].copy(order="F")
    F3[0][0][6, 1] += -0.25j * np.eye(4)              # ... with Sigma^R kept Keldysh-consistent
    F4 = [list(f) for f in _families()]
    G = F4[1][2].copy(order="F")
    G[3, 0] += -0.1j * np.eye(4)                      # Sigma> moved alone: Keldysh identity broken
    F4[1][2] = G
    F5 = [list(f) for f in _families()]
    L = F5[2][1].copy(order="F")
    L[8, 2, 1, 1] = np.nan
    F5[2][1] = L
    F6 = [list(f) for f in F]                         # two failures: the earlier family wins
    F6[0] = list(F4[1])
    F6[0][2] = F4[1][2]
    cases += [("acausal", F, (idx(1, 4, 2), 2)), ("non_hermitian", F2, (idx(2, 2, 0), 3)),
              ("negative", F3, (idx(0, 6, 1), 4)), ("keldysh", F4, (idx(1, 3, 0), 5)),
              ("nonfinite", F5, (idx(2, 8, 2), 1)), ("first_of_two", F6, (idx(0, 3, 0), 5))]
    return cases


@pytest.mark.parametrize("case", [c[0] for c in _planted()])
def test_oracle_guard_planted(orc, case):
    name, fams, (first, code) = next(c for c in _planted() if c[0] == case)
    passed, f, k = orc.anderson_guard([tuple(x) for x in fams])
    assert (f, k) == (first, code)
    assert passed == (first == 0)


def test_oracle_history_eviction_and_restart(orc):
    fams = _families(nfam=2)
    mixer = orc.AndersonMixer(depth=3)
    zero = [tuple(np.zeros_like(c) for c in f) for f in fams]
    for k in range(5):  # shrinking residuals: no restart, the history stays at depth 3
        cand = [tuple(z + (0.5 ** k) * c for z, c in zip(zf, f)) for zf, f in zip(zero, fams)]
        mixer.mix(zero, cand, 0.3)
        assert mixer.info["reset_reason"] == "none" and mixer.info["history_depth"] == min(k + 1, 3)
    cand = [tuple(z + 10.0 * c for z, c in zip(zf, f)) for zf, f in zip(zero, fams)]
    mixer.mix(zero, cand, 0.3)  # a larger residual restarts the history
    assert mixer.info["reset_reason"] == "residual_increase" and mixer.info["history_depth"] == 1


def _anderson_problem(**kw):
    from qclb200.problem import small_problem

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "impurity", "IFR", "alloy"))
    return dataclasses.replace(pr, mixing="anderson", **kw)


def test_oracle_anderson_contracts_faster_than_linear(orc):
    pa = _anderson_problem()
    ha, _ = orc.scba(pa, 6)
    hl, _ = orc.scba(dataclasses.replace(pa, mixing="linear"), 6)
    assert ha[-1]["rSigma"] < 0.5 * hl[-1]["rSigma"]
    assert [r["mixer"]["history_depth"] for r in ha] == [1, 2, 3, 4, 5, 5]


def test_guard_budgets_of_a_state_stored_in_complex64(orc, monkeypatch):
    """A state made in complex64 (a mixed-precision run promoted to
    complex128 for its FP64 refinement) carries FP32 rounding in every entry.
    The guard's budgets at FP64 roundoff (64 n eps ||X||) reject nearly every
    block of it -- Sigma^R - Sigma^A = Sigma^> - Sigma^< and the
    definiteness tests hold only to FP32 -- so a convex fallback towards
    that state is refused and the refinement stops with a DomainError.  At
    the FP32 roundoff the same blocks pass: the budgets a promoted context's
    guard keeps (the roundoff argument of launch_anderson_guard, set by
    qcl_scba_promote)."""
    from qclb200.problem import small_problem

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "IFR"))
    _, st = orc.scba(pr, 8, keep_state=True)
    fams = [st["scattering"][m.name] for m in pr.mechanisms] + [st["plus"], st["minus"]]

    def stored(a):
        return np.asarray(a, np.complex64).astype(np.complex128)

    def antiherm(a):  # the promotion keeps the anti-Hermitian part of Sigma^<, Sigma^>
        return 0.5 * (a - np.conj(np.swapaxes(a, -1, -2)))

    blocks = [(stored(R)[e, m], antiherm(stored(L))[e, m], antiherm(stored(G))[e, m])
              for R, L, G in fams for e in range(pr.NE) for m in range(pr.Nk)]
    # the FP64 state itself passes at FP64 budgets
    assert all(orc.anderson_block_failure(R[e, m], L[e, m], G[e, m]) == 0
               for R, L, G in fams for e in range(pr.NE) for m in range(pr.Nk))
    failing = sum(orc.anderson_block_failure(*b) != 0 for b in blocks)
    assert failing > len(blocks) // 2
    monkeypatch.setattr(orc, "_EPS", 2.0 ** -23)
    assert all(orc.anderson_block_failure(*b) == 0 for b in blocks)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("case", [c[0] for c in _planted()])
def test_gpu_guard_planted(gpu_ops, orc, case):
    name, fams, (first, code) = next(c for c in _planted() if c[0] == case)
    passed, f, k = gpu_ops.anderson_guard([tuple(x) for x in fams])
    assert (f, k) == (first, code)
    assert passed == (first == 0)


def _compare_rows(ho, hg, rtol):
    assert len(ho) == len(hg)
    for ro, rg in zip(ho, hg):
        for ko, kg in (("J", "J"), ("rSigma", "r_Sigma"), ("lam", "lam"), ("rK", "r_K"), ("rA", "r_A")):
            a, b = ro[ko], rg[kg]
            assert abs(a - b) <= rtol * max(abs(a), abs(b)) + 1e-14, (ro["nu"], ko, a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [False, True])
def test_scba_anderson_matches_oracle(gpu_ops, orc, use_graph):
    from qclb200.scba import ProductionSCBA

    pr = _anderson_problem()
    hist_o, _ = orc.scba(pr, 8)
    s = ProductionSCBA(pr, use_graph=use_graph)
    s.seed()
    hist_g, infos = [], []
    for _ in range(8):
        hist_g.append(s.step())
        infos.append(s.mixer_info())
    s.close()
    _compare_rows(hist_o, hist_g, 1e-7)
    for ro, info in zip(hist_o, infos):
        mo = ro["mixer"]
        assert info["history_depth"] == mo["history_depth"]
        assert info["reset_reason"] == mo["reset_reason"]
        assert bool(info["fallback"]) == mo["fallback"]
        assert bool(info["acceleration_accepted"]) == mo["acceleration_accepted"]
        assert info["coefficients_l1"] == pytest.approx(mo["coefficients_l1"], rel=1e-6)


@pytest.mark.gpu
def test_scba_anderson_depth_and_damping(gpu_ops, orc):
    from qclb200.scba import solve_scba_production

    pr = _anderson_problem(anderson_history_depth=2, anderson_damping=0.7)
    hist_o, _ = orc.scba(pr, 5)
    hist_g, s = solve_scba_production(pr, 5)
    s.close()
    _compare_rows(hist_o, hist_g, 1e-7)


@pytest.mark.gpu
def test_scba_anderson_rejects_bad_options(gpu_ops):
    from qclb200.scba import ProductionSCBA

    for kw in (dict(anderson_history_depth=0), dict(anderson_damping=0.0), dict(anderson_damping=1.5),
               dict(anderson_regularization=-1.0), dict(anderson_history_depth=9)):
        with pytest.raises(Exception):
            ProductionSCBA(_anderson_problem(**kw))
