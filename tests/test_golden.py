"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py
from the FP64 oracle on seeded inputs).

CPU tests: the oracle still reproduces every fixture (a regression pin of the
oracle itself).  GPU tests: the CUDA path reproduces the same stored values,
at the tolerances of the operator tests.
"""
import os

import numpy as np
import pytest

from helpers import approx_err

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(HERE, name + ".npz"))


# ---------------------------------------------------------------------------
# oracle pinned to the fixtures (CPU)
# ---------------------------------------------------------------------------

def test_oracle_reproduces_dyson_keldysh_fixture(orc):
    d = load("dyson_keldysh_N7")
    GR, _, scale, _ = orc.retarded_green(d["eps"], d["h"], d["SR"])
    assert approx_err(GR, d["GR"]) < 1e-14
    assert approx_err(orc.keldysh_green(GR, d["SL"]), d["GL"]) < 1e-14
    assert approx_err(orc.keldysh_green(GR, d["SG"]), d["GG"]) < 1e-14
    np.testing.assert_allclose(scale, d["scale"], rtol=1e-15)


def test_oracle_reproduces_hilbert_fixture(orc):
    d = load("hilbert_NE300")
    Lam, r = orc.fft_hilbert(d["Gam"], d["eps"], d["wE"], return_roundoff=True)
    assert approx_err(Lam, d["Lam"]) < 1e-14
    assert r == pytest.approx(float(d["roundoff"]), rel=1e-6, abs=1e-18)
    SR, Gam = orc.retarded_self_energy(d["SL"], d["SG"], d["eps"], d["wE"], method="direct")
    assert approx_err(SR, d["SR"]) < 1e-14
    assert np.array_equal(Gam, d["GamSE"])


def test_oracle_reproduces_shift_and_embedding_fixture(orc):
    d = load("shift_embedding")
    for i, delta in enumerate(d["deltas"]):
        plan = orc.ShiftPlan(d["eps"], float(delta))
        assert approx_err(plan.apply(d["X"]), d[f"shift{i}"]) < 1e-15
        assert approx_err(orc.embedding_component(d["T"], d["X"], plan), d[f"embed{i}"]) < 1e-14


def test_oracle_reproduces_contraction_fixture(orc):
    from qclb200.problem import small_problem

    d = load("contraction_NE19")
    pr = small_problem(NE=19, Nk=3, Nb=3, mechanisms=("acoustic", "impurity", "IFR"))
    for m in pr.mechanisms:
        got = orc.contraction_literal(m.literal_kernel(pr.Nk, pr.Nb), d["G"], pr.wk, 1.3 * m.q)
        assert approx_err(got, d["sigma_" + m.name]) < 1e-14, m.name


def test_oracle_reproduces_residual_fixture(orc):
    d = load("residual_suite_N6")
    res = orc.residual_suite(d["eps"], d["h"], d["GR"], d["GL"], d["GG"], (d["SR"], d["SL"], d["SG"]), d["cand"])
    for k in ("rD", "rA", "rK", "rPSD", "rcaus"):
        assert res[k] == pytest.approx(float(d[k]), rel=1e-12, abs=1e-16), k


def test_oracle_reproduces_scba_fixture(orc):
    from qclb200.problem import small_problem

    d = load("scba_small_LO_acoustic")
    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic"))
    hist, _ = orc.scba(pr, 3)
    for k in ("J", "Jbar", "rSigma", "rK", "lam", "number"):
        np.testing.assert_allclose([row[k] for row in hist], d[k], rtol=1e-11, err_msg=k)
    np.testing.assert_allclose([row["populations"] for row in hist], d["populations"], rtol=1e-11, atol=1e-16)


# ---------------------------------------------------------------------------
# CUDA path against the fixtures (GPU)
# ---------------------------------------------------------------------------

@pytest.mark.gpu
def test_gpu_dyson_keldysh_fixture(gpu_ops):
    d = load("dyson_keldysh_N7")
    GR, GL, GG, scale = gpu_ops.dyson_keldysh(d["eps"], d["h"], d["SR"], d["SL"], d["SG"])
    assert approx_err(GR, d["GR"]) < 1e-12
    assert approx_err(GL, d["GL"]) < 1e-12
    assert approx_err(GG, d["GG"]) < 1e-12
    np.testing.assert_allclose(scale, d["scale"], rtol=1e-14)


@pytest.mark.gpu
def test_gpu_hilbert_fixture(gpu_ops):
    d = load("hilbert_NE300")
    Lam, r = gpu_ops.fft_hilbert_transform(d["Gam"], d["eps"], d["wE"], return_roundoff=True)
    assert approx_err(Lam, d["Lam"]) < 2e-13
    assert r < 100 * float(d["roundoff"]) + 1e-15
    SR, Gam = gpu_ops.retarded_self_energy_fft(d["SL"], d["SG"], d["eps"], d["wE"])
    assert approx_err(SR, d["SR"]) < 2e-13
    assert np.array_equal(Gam, d["GamSE"])


@pytest.mark.gpu
def test_gpu_shift_and_embedding_fixture(gpu_ops):
    d = load("shift_embedding")
    for i, delta in enumerate(d["deltas"]):
        assert approx_err(gpu_ops.apply_energy_shift(d["X"], d["eps"], float(delta)), d[f"shift{i}"]) < 5e-15
        assert approx_err(gpu_ops.embedding_component(d["T"], d["X"], d["eps"], float(delta)), d[f"embed{i}"]) < 1e-13


@pytest.mark.gpu
def test_gpu_contraction_fixture(gpu_ops):
    from qclb200.problem import small_problem

    d = load("contraction_NE19")
    pr = small_problem(NE=19, Nk=3, Nb=3, mechanisms=("acoustic", "impurity", "IFR"))
    for m in pr.mechanisms:
        got = gpu_ops.production_static_contraction(m, d["G"], pr.wk, alpha=1.3)
        assert approx_err(got, d["sigma_" + m.name]) < 1e-13, m.name


@pytest.mark.gpu
def test_gpu_residual_fixture(gpu_ops):
    d = load("residual_suite_N6")
    got = gpu_ops.production_residual_suite(d["eps"], d["h"], d["GR"], d["GL"], d["GG"], (d["SR"], d["SL"], d["SG"]),
                                            d["cand"])
    for k in ("rA", "rK"):
        assert abs(got[k] - float(d[k])) <= 1e-10 * max(float(d[k]), 1e-14) + 1e-15, k
    assert abs(got["rD"] - float(d["rD"])) <= 1e-14
    assert got["rPSD"] == pytest.approx(float(d["rPSD"]), abs=1e-13)
    assert got["rcaus"] == pytest.approx(float(d["rcaus"]), abs=1e-13)


@pytest.mark.gpu
def test_gpu_scba_fixture(gpu_ops):
    from qclb200.problem import small_problem
    from qclb200.scba import solve_scba_production

    d = load("scba_small_LO_acoustic")
    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic"))
    hist, solver = solve_scba_production(pr, 3)
    solver.close()
    np.testing.assert_allclose([r["J"] for r in hist], d["J"], rtol=1e-9)
    np.testing.assert_allclose([r["r_Sigma"] for r in hist], d["rSigma"], rtol=1e-9)
    np.testing.assert_allclose([r["lam"] for r in hist], d["lam"], rtol=1e-11)
    np.testing.assert_allclose([r["populations"] for r in hist], d["populations"], rtol=1e-9, atol=1e-14)
