"""The outer Hartree-Poisson loop (production_solver.jl:993-1151) around the
device SCBA.

CPU: the bordered periodic Poisson solve of the host mirror and of the
oracle against the discrete analytic answer for a cosine charge (r_P at
rounding, zero mean, zeta = 0), the projected Hamiltonians' linearity in U,
charge neutrality of the density built from a normalised state, and the
oracle's outer loop itself.  GPU: the device coherence matrix against the
oracle, and the whole outer loop (device SCBA warm-started across outer
iterations via retarget) against the oracle's, every OuterIteration field
within 1e-8.
"""
import math

import numpy as np
import pytest


def _cosine_case():
    from qclb200.outer import outer_small

    st, pr = outer_small()
    N = len(st.x)
    Lp = st.Lp
    k = 2 * math.pi / Lp
    A = 0.3 * st.ND2D / Lp
    st.eps_r = np.full(N, 12.9)
    nbar = st.ND - A * np.cos(k * st.x)
    dx = st.wx[0]
    lam_k = (2 - 2 * math.cos(k * dx)) / dx ** 2
    U_exact = -st.lambda_P * A * np.cos(k * st.x) / (12.9 * lam_k)
    return st, nbar, U_exact


def test_poisson_cosine_charge_host_and_oracle(orc):
    from qclb200.outer import solve_periodic_poisson

    st, nbar, U_exact = _cosine_case()
    for solve in (solve_periodic_poisson, orc.poisson_solve):
        U, zeta, rP, neutral = solve(st, nbar)
        np.testing.assert_allclose(U, U_exact, rtol=0, atol=1e-11 * np.max(np.abs(U_exact)))
        assert abs(zeta) < 1e-12 and rP < 1e-12 and neutral < 1e-14
        assert abs(np.sum(U)) < 1e-10 * np.max(np.abs(U))


def test_projection_is_linear_and_hermitian():
    from qclb200.outer import outer_small, project_hamiltonians

    st, pr = outer_small()
    rng = np.random.default_rng(1)
    U1, U2 = rng.standard_normal(len(st.x)), rng.standard_normal(len(st.x))
    h0, h1, h2 = (project_hamiltonians(st, U) for U in (0 * U1, U1, U2))
    h12 = project_hamiltonians(st, U1 + 2 * U2)
    np.testing.assert_allclose(h12 - h0, (h1 - h0) + 2 * (h2 - h0), atol=1e-13)
    assert np.allclose(h1, np.conj(np.transpose(h1, (0, 2, 1))), atol=1e-14)
    np.testing.assert_allclose(st.Phi.T @ st.Phi, np.eye(pr.Nb), atol=1e-13)
    c = 0.37
    np.testing.assert_allclose(project_hamiltonians(st, np.full(len(st.x), c)) - h0,
                               c * np.broadcast_to(np.eye(pr.Nb), h0.shape), atol=1e-13)


def test_oracle_outer_loop_is_neutral(orc):
    from qclb200.outer import outer_small

    st, pr = outer_small()
    rows = orc.outer_loop(pr, st, max_poisson=2, inner_iterations=2)
    for r in rows:
        assert r["r_P"] < 1e-12 and r["r_neutral"] < 1e-12
        assert math.isfinite(r["J"]) and math.isfinite(r["r_U"])
    assert math.isinf(rows[0]["r_n"]) and math.isfinite(rows[1]["r_n"])


@pytest.mark.gpu
def test_density_matrix_matches_oracle(gpu_ops, orc):
    from qclb200 import _lib
    import ctypes

    rng = np.random.default_rng(3)
    NE, Nk, Nb = 57, 4, 5
    GL = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    wE, wk = rng.uniform(0.1, 1, NE), rng.uniform(0.1, 1, Nk)
    rho = np.zeros((Nb, Nb), dtype=np.complex128, order="F")
    _lib.check(_lib.lib().qcl_density_matrix(0, NE, Nk, Nb, ctypes.c_void_p(wE.ctypes.data),
                                             ctypes.c_void_p(wk.ctypes.data), ctypes.c_void_p(GL.ctypes.data),
                                             ctypes.c_void_p(rho.ctypes.data)))
    want = orc.density_matrix(GL, wE, wk)
    np.testing.assert_allclose(rho, want, rtol=1e-13, atol=1e-13 * np.abs(want).max())


@pytest.mark.gpu
def test_outer_loop_matches_oracle(gpu_ops, orc):
    from qclb200.outer import outer_small, solve_production_outer

    st, pr = outer_small()
    want = orc.outer_loop(pr, st, max_poisson=3, inner_iterations=3)
    got, solver = solve_production_outer(pr, st, max_poisson=3, inner_iterations=3)
    solver.close()
    for ro, rg in zip(want, got):
        for k in ("r_U", "r_J", "J", "zeta", "r_Jchange", "r_population", "r_n"):
            a, b = ro[k], rg[k]
            if math.isinf(a):
                assert math.isinf(b), k
            else:
                assert abs(a - b) <= 1e-8 * max(abs(a), abs(b)) + 1e-14, (ro["mu"], k, a, b)
        for k in ("r_P", "r_neutral"):
            assert rg[k] < 1e-12 and ro[k] < 1e-12
        np.testing.assert_allclose(rg["n"], ro["n"], rtol=1e-8, atol=1e-12)
        np.testing.assert_allclose(rg["populations"], ro["populations"], rtol=1e-8, atol=1e-13)
