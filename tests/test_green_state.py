"""The derived GreenState fields (domain/types.jl:733-740): the spectral
function A = i(G^R - G^R^H), condition_number = cond_2(D) and dyson_scale,
as retarded_green / _retarded_green_production / _green_state_production
write them (numerics/reference/greens.jl:18-57,
numerics/optimized/production_operators.jl:1337-1415).

CPU: the oracle's cond_2(D) against numpy's SVD-based cond (the reference
uses LAPACK's SVD), including the scalar anchor kappa = 1
(test/physics/scalar_dyson_and_spectral_identity.jl:4-21).  GPU: the C ABI
against the oracle, at the operator level and from a running SCBA context.
"""
import numpy as np
import pytest

from helpers import approx_err, dyson_inputs


def test_oracle_condition_number_matches_svd(orc):
    NE, Nk, N = 11, 2, 6
    eps, h, SR, _, _ = dyson_inputs(5, NE, Nk, N)
    _, k2, scale, _ = orc.retarded_green(eps, h, SR)
    for e in range(NE):
        for m in range(Nk):
            D = eps[e] * np.eye(N) - h[m] - SR[e, m]
            assert k2[e, m] == pytest.approx(np.linalg.cond(D, 2), rel=1e-11)
            assert scale[e, m] == pytest.approx(np.abs(D).sum(axis=1).max(), rel=1e-15)


def test_oracle_scalar_condition_number_is_one(orc):
    eps = np.linspace(-1.0, 1.0, 9)
    h = np.full((1, 1, 1), 0.2 + 0j, order="F")
    SR = np.asfortranarray(np.full((9, 1, 1, 1), -0.05j))
    GR, k2, _, _ = orc.retarded_green(eps, h, SR)
    np.testing.assert_allclose(k2, 1.0, rtol=0, atol=4e-16)
    A = orc.spectral_function(GR)
    lorentz = 2 * 0.05 / ((eps - 0.2) ** 2 + 0.05 ** 2)
    np.testing.assert_allclose(A[:, 0, 0, 0].real, lorentz, rtol=1e-13)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("N", [1, 3, 8, 13, 24, 32, 40, 48])
@pytest.mark.parametrize("eta", [0.0, 0.02])
def test_condition_number_matches_oracle(gpu_ops, orc, N, eta):
    NE, Nk = 37, 3
    eps, h, SR, _, _ = dyson_inputs(300 + N, NE, Nk, N)
    GR = gpu_ops.dyson_keldysh(eps, h, SR, eta=eta, precision="c128")[0]
    kappa, scale = gpu_ops.condition_number(eps, h, GR, SR, eta=eta)
    _, ok2, oscale, _ = orc.retarded_green(eps, h, SR, eta=eta)
    np.testing.assert_allclose(kappa, ok2, rtol=1e-10)
    np.testing.assert_allclose(scale, oscale, rtol=1e-14)
    assert np.all(kappa >= 1.0 - 1e-14)  # cond_2 >= 1 up to rounding


@pytest.mark.gpu
def test_condition_number_scalar_anchor_and_null_sigma(gpu_ops):
    eps = np.linspace(-1.0, 1.0, 9)
    h = np.full((1, 1, 1), 0.2 + 0j, order="F")
    GR = gpu_ops.dyson_keldysh(eps, h, np.zeros((9, 1, 1, 1), complex, order="F"), eta=0.05)[0]
    kappa, scale = gpu_ops.condition_number(eps, h, GR, None, eta=0.05)
    np.testing.assert_allclose(kappa, 1.0, rtol=0, atol=4e-16)
    np.testing.assert_allclose(scale[:, 0], np.hypot(eps - 0.2, 0.05), rtol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_spectral_function_matches_oracle(gpu_ops, orc, precision):
    eps, h, SR, _, _ = dyson_inputs(7, 41, 3, 12)
    GR = orc.retarded_green(eps, h, SR)[0]
    want = orc.spectral_function(GR)
    if precision == "c128":
        assert np.array_equal(gpu_ops.spectral_function(GR), want)
    else:
        got = gpu_ops.spectral_function(GR.astype(np.complex64), precision="c64")
        assert approx_err(got, want) < 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["c128", "mixed"])
def test_scba_green_state_matches_oracle(gpu_ops, orc, precision):
    from qclb200.problem import small_problem
    from qclb200.scba import ProductionSCBA

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "impurity"))
    s = ProductionSCBA(pr, precision=precision)
    with pytest.raises(Exception, match="seed or step"):
        s.green_state()
    s.seed()
    rtol = 1e-10 if precision == "c128" else 1e-4
    # after the seed: eta_seed, Sigma = 0
    gs = s.green_state()
    GR, k2, scale, _ = orc.retarded_green(pr.eps, pr.h, None, eta=pr.eta_seed)
    np.testing.assert_allclose(gs["condition_number"], k2, rtol=rtol)
    np.testing.assert_allclose(gs["dyson_scale"], scale, rtol=1e-14 if precision == "c128" else 1e-6)
    assert approx_err(gs["A"], orc.spectral_function(GR)) < (1e-12 if precision == "c128" else 1e-5)
    # after two steps: the total Sigma^R of the (unmixed) state that produced G^R
    s.step()
    s.step()
    gs = s.green_state()
    total = sum(s.family(f)[0].astype(np.complex128) for f in range(len(pr.mechanisms) + 2))
    GR, k2, scale, _ = orc.retarded_green(pr.eps, pr.h, total)
    np.testing.assert_allclose(gs["condition_number"], k2, rtol=rtol)
    np.testing.assert_allclose(gs["dyson_scale"], scale, rtol=1e-14 if precision == "c128" else 1e-6)
    assert approx_err(gs["A"], orc.spectral_function(GR)) < (1e-12 if precision == "c128" else 1e-5)
    s.close()
