"""Scattering-model switches of the SCBA candidate (AlgorithmOptions
self_energy_structure / transverse_momentum / retarded_real_part /
elastic_retarded; numerics/optimized/production_operators.jl:1165-1335).

CPU: the oracle is pinned to the reference's direct-static-closure anchor
(test/physics/direct_static_retarded.jl:80-114, restated: analytic G^R of
H = [0 1+i; 1-i 2], a two-vertex covariance kernel, the candidate against the
literal covariance sum at 5e-13 and no Hilbert roundoff), and the switches'
defining properties.  GPU: the device SCBA loop with each switch against the
oracle's SCBA, every history metric within 1e-9.
"""
import dataclasses
import math

import numpy as np
import pytest

from helpers import approx_err


def _approx(x, y, rtol=5e-13, atol=2e-12):
    x, y = np.asarray(x).ravel(), np.asarray(y).ravel()
    return np.linalg.norm(x - y) <= max(atol, rtol * max(np.linalg.norm(x), np.linalg.norm(y)))


def _closure_fixture():
    """The anchor's fixture: NE = 9, Nk = 2, Nb = 2 (its grids are the
    reference's tutorial grids; the identities hold on any grid, so a
    uniform one stands in)."""
    from qclb200.problem import SCBAProblem, energy_grid, production_kernel

    NE, Nk, Nb = 9, 2, 2
    eps, wE = energy_grid(-0.5, 1.5, NE)
    wk = np.array([0.31, 0.77])
    GR = np.zeros((NE, Nk, Nb, Nb), dtype=complex, order="F")
    for e in range(NE):
        for m in range(1, Nk + 1):
            z = eps[e] - 0.17 * m + (0.2 + 0.1 * m) * 1j
            GR[e, m - 1] = np.array([[z - 2, 1 + 1j], [1 - 1j, z]]) / (z * z - 2 * z - 2)
    A = 1j * (GR - np.conj(np.transpose(GR, (0, 1, 3, 2))))
    green = dict(GR=GR, GL=np.asfortranarray(0.37j * A), GG=np.asfortranarray(-0.63j * A))
    vertices = [np.array([[1, 0.2 + 0.3j], [0.2 - 0.3j, 0.7]]), np.array([[0.5, 0.4j], [-0.4j, 1.2]])]
    assert np.linalg.norm(vertices[0] @ vertices[1] - vertices[1] @ vertices[0]) > 0.1
    K = np.zeros((Nk, Nk, Nb, Nb, Nb, Nb), dtype=complex)
    for m in range(Nk):
        for mp in range(Nk):
            coef = (m + 1 + mp + 1) / (Nk + 1)
            K[m, mp] = coef * sum(np.einsum("ac,bd->acdb", V, np.conj(V)) for V in vertices)
    qscale = 7.25
    mechs = [production_kernel(n, qscale, K / qscale) for n in ("acoustic", "impurity", "IFR", "alloy")]
    assert all(m.kind == "dense" for m in mechs)
    pr = SCBAProblem(NE=NE, Nk=Nk, Nb=Nb, eps=eps, wE=wE, wk=wk, h=np.zeros((Nk, Nb, Nb), complex, order="F"),
                     Tplus=np.zeros((Nb, Nb), complex), Tminus=np.zeros((Nb, Nb), complex), Ep=0.3, hw_LO=0.36,
                     N_LO=0.2, gs=2, target=0.1, kBT=0.1, eta_seed=0.02, alpha=0.3, mechanisms=mechs,
                     elastic_retarded="direct_green")

    def covariance(X):
        out = np.zeros_like(X)
        for m in range(Nk):
            for mp in range(Nk):
                coef = (m + 1 + mp + 1) / (Nk + 1)
                for V in vertices:
                    out[:, m] += coef * wk[mp] * np.einsum("ac,ecd,bd->eab", V, X[:, mp], np.conj(V))
        return out

    return pr, green, covariance, A


def _broadening(R):
    return 1j * (R - np.conj(np.transpose(R, (0, 1, 3, 2))))


def test_direct_static_closure_anchor(orc):
    pr, green, covariance, A = _closure_fixture()
    cand, rround = orc.scattering_candidate(pr, green, orc.make_plans(pr), verify=True)
    truthR, truthL, truthG, truthA = (covariance(green["GR"]), covariance(green["GL"]), covariance(green["GG"]),
                                      covariance(A))
    for name in ("acoustic", "impurity", "IFR", "alloy"):
        SR, SL, SG = cand[name]
        assert _approx(SR, truthR) and _approx(SL, truthL) and _approx(SG, truthG), name
        assert _approx(_broadening(SR), truthA)
        assert _approx(1j * (SG - SL), truthA)
    for e in range(pr.NE):
        for m in range(pr.Nk):
            assert np.linalg.eigvalsh(0.5 * (truthA[e, m] + truthA[e, m].conj().T)).min() >= -2e-12
    assert rround == 0.0


def _small(**switches):
    from qclb200.problem import small_problem

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "impurity", "IFR", "alloy"))
    return dataclasses.replace(pr, **switches)


def test_switch_properties_on_oracle_candidates(orc):
    base = _small()
    green, _ = orc.seed_green(base)
    plans = orc.make_plans(base)
    ref, r0 = orc.scattering_candidate(base, green, plans, verify=True)
    assert r0 > 0

    diag, _ = orc.scattering_candidate(_small(self_energy_structure="diagonal"), green, plans)
    for name, fam in diag.items():
        for X, Y in zip(fam, ref[name]):
            off = np.ones((4, 4), bool) & ~np.eye(4, dtype=bool)
            assert np.all(X[:, :, off] == 0)
            assert np.array_equal(X[:, :, ~off], Y[:, :, ~off])

    avg, _ = orc.scattering_candidate(_small(transverse_momentum="averaged"), green, plans)
    w = base.wk / base.wk.sum()
    for name, fam in avg.items():
        for X, Y in zip(fam, ref[name]):
            assert np.array_equal(X[:, 0], X[:, 1]) and np.array_equal(X[:, 0], X[:, 2])
            assert approx_err(X[:, 0], np.einsum("m,emab->eab", w, Y)) < 1e-14

    drop, rd = orc.scattering_candidate(_small(retarded_real_part="drop"), green, plans, verify=True)
    assert rd == 0.0
    for name, (SR, SL, SG) in drop.items():
        assert np.array_equal(SL, ref[name][1]) and np.array_equal(SG, ref[name][2])
        assert np.array_equal(SR, 0.5 * (SG - SL))

    direct, _ = orc.scattering_candidate(_small(elastic_retarded="direct_green"), green, plans)
    for m in base.mechanisms:
        SR = direct[m.name][0]
        if m.name == "LO":
            assert np.array_equal(SR, ref["LO"][0])
        else:
            assert approx_err(SR, orc.contraction(m, green["GR"], base.wk)) == 0.0


def test_scalar_lesser_normalisation_on_oracle(orc):
    """occupation_normalization = :scalar_lesser (production_state.jl:54-61):
    N(G<) equals the target and G> = G^R - G^A + G<."""
    pr = _small(occupation_normalization="scalar_lesser")
    plans = orc.make_plans(pr)
    green, _ = orc.seed_green(pr)
    scattering, _ = orc.scattering_candidate(pr, green, plans, verify=False)
    plus, minus = orc.embedding_candidate(pr, green, plans)
    g, lam = orc.current_green(pr, orc.total_family(pr, scattering, plus, minus))
    assert g["normalized"] == pytest.approx(pr.target, rel=1e-12)
    GR = g["GR"]
    assert approx_err(g["GG"], GR - np.conj(np.transpose(GR, (0, 1, 3, 2))) + g["GL"]) < 1e-15
    paired = _small()
    gp, lp = orc.current_green(paired, orc.total_family(paired, scattering, plus, minus))
    assert lp == lam and gp["normalized"] == pytest.approx(pr.target, rel=1e-12)


def test_switch_codes_validate_symbols():
    from qclb200.scba import _switch_codes

    assert _switch_codes(_small()) == [0, 0, 0, 0, 0, 0]
    assert _switch_codes(_small(self_energy_structure="diagonal", elastic_retarded="direct_green")) == [1, 0, 0, 1, 0,
                                                                                                         0]
    with pytest.raises(ValueError, match="transverse_momentum"):
        _switch_codes(_small(transverse_momentum="mean"))


# ---------------------------------------------------------------------------
# device SCBA loop with the switches (GPU)
# ---------------------------------------------------------------------------

SWITCH_CASES = [
    dict(self_energy_structure="diagonal"),
    dict(transverse_momentum="averaged"),
    dict(retarded_real_part="drop"),
    dict(elastic_retarded="direct_green"),
    dict(self_energy_structure="diagonal", transverse_momentum="averaged", elastic_retarded="direct_green"),
    dict(occupation_normalization="scalar_lesser"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("switches", SWITCH_CASES, ids=lambda d: "+".join(f"{k}={v}" for k, v in d.items()))
def test_scba_with_model_switches_matches_oracle(gpu_ops, orc, switches):
    from qclb200.scba import solve_scba_production

    pr = _small(**switches)
    hist_o, _ = orc.scba(pr, 3)
    hist_g, solver = solve_scba_production(pr, 3)
    solver.close()
    for ro, rg in zip(hist_o, hist_g):
        for ko, kg in (("J", "J"), ("rSigma", "r_Sigma"), ("lam", "lam"), ("rK", "r_K"), ("rA", "r_A")):
            a, b = ro[ko], rg[kg]
            floor = 1e-14 if ko == "rA" else 1e-15  # r_A sits at roundoff
            assert abs(a - b) <= 1e-9 * max(abs(a), abs(b)) + floor, (ro["nu"], ko, a, b)
        np.testing.assert_allclose(rg["populations"], ro["populations"], rtol=1e-9, atol=1e-13)
        if switches.get("retarded_real_part") == "drop":
            assert rg["r_roundoff"] == 0.0
        assert rg["target_charge"] == pr.target
        assert rg["normalized_charge"] == pytest.approx(ro["normalized"], rel=1e-9)
        assert rg["normalized_charge"] == pytest.approx(pr.target, rel=1e-9)
        if ro["nu"] == 1:
            assert math.isnan(rg["lambda_change"])
        else:
            assert rg["lambda_change"] == pytest.approx(ro["lambda_change"], rel=1e-6, abs=1e-12)


@pytest.mark.gpu
def test_direct_green_rejects_truncated_low_rank(gpu_ops):
    from qclb200.problem import low_rank_production_kernel
    from qclb200.scba import ProductionSCBA

    pr = _small(elastic_retarded="direct_green")
    for i, m in enumerate(pr.mechanisms):
        if m.name == "impurity":
            pr.mechanisms[i] = low_rank_production_kernel(m.name, m.q, m.matrix, relative_tolerance=1e-2)
            assert pr.mechanisms[i].left.shape[1] < m.matrix.shape[0]
    with pytest.raises(Exception, match="untruncated"):
        ProductionSCBA(pr)
    # with the real part dropped the pair is allowed (algorithm_options.jl:66-75)
    ProductionSCBA(dataclasses.replace(pr, retarded_real_part="drop")).close()
