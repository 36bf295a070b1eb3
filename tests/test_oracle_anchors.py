"""Pins the CPU oracle against the reference test suite's known answers.

Each test restates one analytic anchor or operator-equivalence check of the
reference (file:line of the Julia test cited) at the reference's own
tolerance.  The Julia random streams cannot be reproduced here, so random
inputs use numpy generators with the same shapes; the anchors themselves are
closed-form.
"""
import math

import numpy as np
import pytest


def approx(x, y, rtol=0.0, atol=0.0):
    """Julia's isapprox for arrays: norm(x - y) <= max(atol, rtol*max(norm(x), norm(y)))."""
    x, y = np.asarray(x), np.asarray(y)
    d = np.linalg.norm((x - y).ravel())
    return d <= max(atol, rtol * max(np.linalg.norm(x.ravel()), np.linalg.norm(y.ravel())))


def _uniform(lo, hi, n):
    eps = np.linspace(lo, hi, n)
    de = eps[1] - eps[0]
    w = np.full(n, de)
    w[[0, -1]] /= 2
    return eps, w


def test_scalar_lorentzian_and_identity(orc):
    # test/physics/scalar_dyson_and_spectral_identity.jl:4-21
    eps = np.linspace(-1.0, 1.0, 2001)
    Estar, Gam = 0.17, 0.08
    h = np.full((1, 1, 1), Estar, dtype=complex)
    SR = np.full((len(eps), 1, 1, 1), -0.5j * Gam, order="F")
    GR, k2, sc, k1 = orc.retarded_green(eps, h, SR)
    A = orc.spectral_function(GR)
    exact = Gam / ((eps - Estar) ** 2 + (Gam / 2) ** 2)
    assert approx(A[:, 0, 0, 0].real, exact, rtol=2e-13)
    assert approx(k2, 1.0, rtol=1e-14)
    f = 1 / (np.exp(eps / 0.1) + 1)
    GL = np.zeros_like(GR)
    GL[:, 0, 0, 0] = 1j * f * A[:, 0, 0, 0]
    GG = orc.greater_green(GR, GL)
    assert np.max(np.abs(GG - GL - (GR - np.conj(GR)))) < 1e-12


def test_kms_fdt_and_sum_rule(orc):
    # analytic_equilibrium_sum_rule_lo_balance_and_zero_current_anchors.jl:5-52
    eps = np.linspace(-0.40, 0.40, 4001)
    level, broad, mu, kBT = 0.03, 0.07, -0.02, 0.025
    h = np.full((1, 1, 1), level, dtype=complex)
    SR = np.full((len(eps), 1, 1, 1), -0.5j * broad, order="F")
    GR = orc.retarded_green(eps, h, SR)[0]
    A = orc.spectral_function(GR)
    occ = 1 / (np.exp((eps - mu) / kBT) + 1)
    GL = np.zeros_like(GR)
    GL[:, 0, 0, 0] = 1j * occ * A[:, 0, 0, 0]
    GG = orc.greater_green(GR, GL)
    assert approx(GG[:, 0, 0, 0], -1j * (1 - occ) * A[:, 0, 0, 0], rtol=3e-13)
    inner = (occ > 1e-7) & (occ < 1 - 1e-7)
    ratio = GG[inner, 0, 0, 0].imag / GL[inner, 0, 0, 0].imag
    assert approx(ratio, -np.exp((eps[inner] - mu) / kBT), rtol=2e-12)

    eps, w = _uniform(-10.0, 10.0, 40001)
    level, broad = 0.17, 0.08
    h = np.full((1, 1, 1), level, dtype=complex)
    SR = np.full((len(eps), 1, 1, 1), -0.5j * broad, order="F")
    A = orc.spectral_function(orc.retarded_green(eps, h, SR)[0])[:, 0, 0, 0].real
    numerical = np.dot(w, A) / (2 * math.pi)
    exact = (math.atan(2 * (eps[-1] - level) / broad) - math.atan(2 * (eps[0] - level) / broad)) / math.pi
    assert abs(numerical - exact) < 1e-5 and 0 < numerical < 1


def test_detailed_balance():
    # analytic_...anchors.jl:54-69 (pure scalar identity used by the LO closure)
    kBT = 8.617333262e-5 * 200.0
    hw = 0.0367
    bose = 1 / math.expm1(hw / kBT)
    assert abs((bose + 1) / bose - math.exp(hw / kBT)) <= 2e-15 * math.exp(hw / kBT)
    mu = 0.01
    fermi = lambda x: 1 / (math.exp((x - mu) / kBT) + 1)
    for lo in (-0.05, 0.0, 0.05):
        up = lo + hw
        down = (bose + 1) * fermi(up) * (1 - fermi(lo))
        upw = bose * fermi(lo) * (1 - fermi(up))
        assert abs(down - upw) <= 3e-14 * abs(down)


def test_inverse_matches_numpy_and_backward_error(orc):
    # production_exact_operations.jl:7-28 and production_hotpaths.jl:7-50
    for nb in (1, 2, 5, 8, 16):
        a, b = np.meshgrid(np.arange(1, nb + 1), np.arange(1, nb + 1), indexing="ij")
        M = np.sin(a + 2 * b) + 1j * np.cos(2 * a - b) + 4 * np.eye(nb)
        out = orc.inverse(M)
        assert approx(out, np.linalg.inv(M), rtol=5e-13, atol=5e-14)
    rng = np.random.default_rng(1082)
    for n in range(1, 10):
        rnd = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        q, _ = np.linalg.qr(rnd)
        spec = np.array([1e-10]) if n == 1 else np.linspace(1e-10, 1, n)
        cases = [rnd + 0.1 * np.eye(n), q @ np.diag(spec) @ q.conj().T + 1e-12j * np.eye(n)]
        if n > 1:
            P = np.eye(n, dtype=complex)
            P[[0, n - 1]] = P[[n - 1, 0]]
            cases.append(P)
        for M in cases:
            for scale in (1e-150, 1.0, 1e150):
                a = M * scale
                out = orc.inverse(a)
                den = np.linalg.norm(a) * np.linalg.norm(out) + math.sqrt(n)
                assert np.linalg.norm(a @ out - np.eye(n)) / den < 32 * n * np.finfo(float).eps
        with pytest.raises(orc.OracleError):
            orc.inverse(np.zeros((n, n), dtype=complex))


def test_hermitian_eigvals_match_numpy(orc):
    rng = np.random.default_rng(5)
    for n in (1, 2, 5, 12, 24):
        X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        H = X + X.conj().T
        assert approx(orc.eigvalsh(H), np.linalg.eigvalsh(H), rtol=1e-12, atol=1e-12 * np.abs(H).max())


def test_direct_principal_value_antisymmetry(orc):
    # test/numerics/direct_principal_value_transform.jl:4-13
    eps = np.arange(-40, 41) / 20.0  # the Julia range -2.0:0.05:2.0 (correctly rounded nodes)
    w = np.full(len(eps), 0.05)
    w[[0, -1]] /= 2
    G = np.zeros((len(eps), 1, 1, 1), dtype=complex, order="F")
    G[:, 0, 0, 0] = np.exp(-eps ** 2)
    L = orc.direct_hilbert(G, eps, w)
    c = int(np.argmin(np.abs(eps)))
    assert abs(L[c, 0, 0, 0]) < 1e-14
    assert abs(L[c + 5, 0, 0, 0].real + L[c - 5, 0, 0, 0].real) <= 1e-12 * abs(L[c + 5, 0, 0, 0].real)


def test_fft_hilbert_equals_direct(orc):
    # fft_linear_hilbert_map_equals_direct_principal_value.jl:5-58
    rng = np.random.default_rng(0xFF71)
    NE, Nk, Nb = 37, 2, 2
    eps, w = _uniform(-1.3, 0.9, NE)
    G = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    direct = orc.direct_hilbert(G, eps, w)
    fft, rround = orc.fft_hilbert(G, eps, w, return_roundoff=True)
    assert approx(fft, direct, rtol=2e-13, atol=2e-13)
    assert math.isfinite(rround) and rround < 1e-12
    SL = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    SG = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    SRd, Gd = orc.retarded_self_energy(SL, SG, eps, w, method="direct")
    SRf, Gf = orc.retarded_self_energy(SL, SG, eps, w, method="fft")
    assert np.array_equal(Gd, Gf)
    assert approx(SRf, SRd, rtol=2e-13, atol=2e-13)


def test_contractions_equal_literal_six_index_map(orc):
    # production_contractions_equal_literal_six_index_map.jl:5-26
    from qclb200.problem import Mechanism

    rng = np.random.default_rng(0xB05C0)
    NE, Nk, Nb = 7, 4, 2
    G = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    K = np.asfortranarray(rng.standard_normal((Nk, Nk, Nb, Nb, Nb, Nb)) + 1j * rng.standard_normal((Nk, Nk, Nb, Nb, Nb, Nb)))
    wk = rng.random(Nk)
    q = 0.037
    direct = orc.contraction_literal(K, G, wk, q)
    M = np.transpose(K, (0, 2, 5, 1, 3, 4)).reshape((Nk * Nb * Nb, Nk * Nb * Nb), order="F")
    dense = orc.contraction(Mechanism("x", "dense", q, matrix=np.asfortranarray(M)), G, wk)
    assert approx(dense, direct, rtol=2e-14, atol=2e-14)
    block = rng.standard_normal((Nb * Nb,) * 2) + 1j * rng.standard_normal((Nb * Nb,) * 2)
    mech = Mechanism("y", "momentum_independent", q, block=np.asfortranarray(block))
    Kind = mech.literal_kernel(Nk, Nb)
    np.testing.assert_allclose(orc.contraction(mech, G, wk), orc.contraction_literal(Kind, G, wk, q),
                               rtol=2e-14, atol=2e-14)
    # separable IFR (exact_ifr_structured_contraction.jl:36-177)
    J = 3
    left = rng.standard_normal((Nb * Nb, J)) + 1j * rng.standard_normal((Nb * Nb, J))
    right = rng.standard_normal((J, Nb * Nb)) + 1j * rng.standard_normal((J, Nb * Nb))
    radial = rng.standard_normal((Nk, Nk)) + 0j
    ifr = Mechanism("IFR", "ifr", q, left=np.asfortranarray(left), right=np.asfortranarray(right),
                    radial=np.asfortranarray(radial))
    np.testing.assert_allclose(orc.contraction(ifr, G, wk), orc.contraction_literal(ifr.literal_kernel(Nk, Nb), G, wk, q),
                               rtol=5e-13, atol=5e-13)


def test_shift_plan_equals_dense_matrix(orc):
    # production_exact_operations.jl:56-109 (sparse plan == dense matrix)
    eps, _ = _uniform(-1.0, 2.0, 41)
    rng = np.random.default_rng(9)
    X = np.asfortranarray(rng.standard_normal((41, 3, 2, 2)) + 1j * rng.standard_normal((41, 3, 2, 2)))
    for delta in (0.367, -0.367, 0.3, -0.3, 0.0, 3.0, 0.075):
        W = orc.shift_matrix(eps, delta)
        dense = np.einsum("ef,fmab->emab", W, X)
        assert approx(orc.ShiftPlan(eps, delta).apply(X), dense, rtol=5e-14, atol=5e-14)


def test_zero_bias_equilibrium_current(orc):
    # analytic_...anchors.jl:71-138: a reservoir in equilibrium carries no flux
    from qclb200.problem import small_problem

    pr = small_problem(NE=61, Nk=3, Nb=4)
    shape = pr.shape
    gamma = 0.02
    f = 1 / (np.exp(pr.eps / pr.kBT) + 1)
    SR = np.zeros(shape, dtype=complex, order="F")
    SL = np.zeros(shape, dtype=complex, order="F")
    SG = np.zeros(shape, dtype=complex, order="F")
    for a in range(pr.Nb):
        SR[:, :, a, a] = -0.5j * gamma
        SL[:, :, a, a] = (1j * f * gamma)[:, None]
        SG[:, :, a, a] = (-1j * (1 - f) * gamma)[:, None]
    GR = orc.retarded_green(pr.eps, pr.h, SR)[0]
    GL = orc.keldysh_green(GR, SL)
    GG = orc.greater_green(GR, GL)
    assert abs(orc.current(pr, SG, SL, GL, GG)) < 2e-13


def test_nonlinear_scalar_scba_root(orc):
    # independent_nonlinear_and_continuum_anchors.jl:21-98 (linear mixing)
    z = 0.2 + 0.3j
    lam = 0.04
    roots = [(z - np.sqrt(z * z - 4 * lam)) / (2 * lam), (z + np.sqrt(z * z - 4 * lam)) / (2 * lam)]
    truth = [r for r in roots if r.imag < 0][0]
    h = np.zeros((1, 1, 1), dtype=complex)
    for seed in (0.01, 0.1, 0.5):
        sig = -1j * seed
        green = None
        for it in range(1000):
            SR = np.full((1, 1, 1, 1), sig, dtype=complex, order="F")
            green = orc.retarded_green(np.array([z.real]), h, SR, eta=z.imag)[0][0, 0, 0, 0]
            cand = lam * green
            if abs(cand - sig) / (abs(cand) + 1e-14) < 1e-10:
                break
            sig = 0.4 * sig + 0.6 * cand
        assert abs(green - truth) <= 2e-9 * abs(truth)
        assert green.imag < 0


def test_paired_normalisation_preserves_sum_and_target(orc):
    # greens.jl:155-199: Gn + Gp preserved, number -> target
    rng = np.random.default_rng(4)
    n = 50
    GL = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    GG = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for number, holes, target in ((2.0, 3.0, 1.5), (1.0, 3.0, 1.5)):
        a, c, lam = orc.paired_coefficients(number, holes, target)
        L2, G2 = GL.copy(), GG.copy()
        orc.normalize_pair(L2, G2, a, c)
        assert approx(G2 - L2, GG - GL, rtol=1e-15, atol=1e-15)  # Gn + Gp = i(G> - G<) is kept
        assert lam == number / target
        # number after transfer: a*N + c*H (G< = i Gn, G> = -i Gp)
        assert abs(a * number + c * holes - target) < 1e-14
    with pytest.raises(orc.OracleError):
        orc.paired_coefficients(1.0, 0.1, 2.0)  # beyond the Pauli capacity
