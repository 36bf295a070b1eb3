"""Kernel builders on the device (numerics/reference/kernels.jl:5-19,
104-160, 321-407; numerics/optimized/kernels.jl:122-158, 205-217, 303-320).

CPU: the host-side node weights (angular means of the LO factors and of the
lookup interpolation weights) and the vectorised impurity covariance against
the oracle's literal loops.  GPU: the exact LO phonon kernel and a tabulated
impurity kernel assembled on the device into the production dense layout,
against the oracle's literal six-index kernels (1e-12) and their q^K scale.
"""
import math

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


def test_lookup_weights_match_oracle_lookup(orc):
    from qclb200.kernel_build import lookup_weights

    x, wx, chi, kappa = _structure()
    nodes = np.linspace(0.0, 3.0, 9)
    Nphi = 7
    W = lookup_weights(nodes, kappa, Nphi)
    np.testing.assert_allclose(W.sum(axis=1), 1.0, rtol=1e-14)
    # scalar node values v_t = t: the weighted sum equals the oracle's lookup average
    vals = [np.full((1, 1, 1, 1), float(t)) for t in range(len(nodes))]
    K = orc.assemble_lookup_kernel(nodes, vals, kappa, Nphi)[:, :, 0, 0, 0, 0]
    Nk = len(kappa)
    np.testing.assert_allclose((W @ np.arange(len(nodes))).reshape((Nk, Nk), order="F"), K.real, rtol=1e-13)
    with pytest.raises(ValueError):
        lookup_weights(nodes[:4], kappa, Nphi)


def test_impurity_covariance_matches_literal(orc):
    from qclb200.kernel_build import impurity_pair_covariance

    x, wx, chi, kappa = _structure()
    Nb = chi.shape[1]
    donors = np.where(x < 0.5, 0.8, 0.0) * wx
    for q in (0.0, 0.7, 2.5):
        C = impurity_pair_covariance(q, chi, x, wx, donors, 0.3, 1.7)
        blk = orc.impurity_block_literal(q, chi, x, wx, donors, 0.3, 1.7)  # (a,c,d,b)
        want = np.transpose(blk, (0, 1, 3, 2)).reshape((Nb * Nb, Nb * Nb), order="F")
        assert approx_err(C, want) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("Nb,Nk,Nphi,Nq", [(3, 4, 8, 5), (5, 6, 12, 9)])
def test_lo_kernel_assembled_on_gpu_matches_literal(gpu_ops, orc, Nb, Nk, Nphi, Nq):
    from qclb200.kernel_build import lo_form_factors, lo_kernel_operator

    x, wx, chi, kappa = _structure(Nb=Nb, Nk=Nk)
    qz = np.linspace(-6.0, 6.0, Nq)
    wqz = np.full(Nq, qz[1] - qz[0])
    mech = lo_kernel_operator(chi, x, wx, qz, wqz, kappa, Nphi, qscreen=0.4, prefactor=2.3)
    F = lo_form_factors(chi, x, wx, qz)
    K, q = orc.normalize_kernel(orc.lo_kernel_literal(F, qz, wqz, kappa, Nphi, 0.4, 2.3))
    assert mech.q == pytest.approx(q, rel=1e-12)
    assert approx_err(mech.literal_kernel(Nk, Nb), K) < 1e-12


@pytest.mark.gpu
def test_tabulated_impurity_kernel_assembled_on_gpu_matches_literal(gpu_ops, orc):
    from qclb200.kernel_build import impurity_pair_covariance, table_kernel_operator, transfer_momenta

    Nb, Nk, Nphi = 4, 5, 10
    x, wx, chi, kappa = _structure(Nb=Nb, Nk=Nk)
    donors = np.where(x < 0.5, 0.8, 0.0) * wx
    qmax = float(transfer_momenta(kappa, Nphi).max())
    nodes = np.linspace(0.0, qmax, 17)
    covs = np.array([impurity_pair_covariance(q, chi, x, wx, donors, 0.3, 1.7) for q in nodes])
    mech = table_kernel_operator("impurity", nodes, covs, kappa, Nphi)
    blocks = [np.transpose(c.reshape((Nb, Nb, Nb, Nb), order="F"), (0, 1, 3, 2)) for c in covs]  # (a,c,d,b)
    K, q = orc.normalize_kernel(orc.assemble_lookup_kernel(nodes, blocks, kappa, Nphi))
    assert mech.q == pytest.approx(q, rel=1e-12)
    assert approx_err(mech.literal_kernel(Nk, Nb), K) < 1e-12


@pytest.mark.gpu
def test_assembly_rejects_bad_arguments(gpu_ops):
    from qclb200.kernel_build import TABLE, assemble_operator

    with pytest.raises(Exception):
        assemble_operator("x", 7, 2, 2, np.ones((4, 1)), np.ones((1, 16)))
    with pytest.raises(ValueError, match="zero"):
        assemble_operator("x", TABLE, 2, 2, np.ones((4, 1)), np.zeros((16, 1)))


@pytest.mark.gpu
def test_device_built_operator_feeds_scba_without_host_copy(gpu_ops):
    """The LO operator assembled into device memory and handed to the SCBA
    context directly gives the same rows as the host copy of it."""
    import dataclasses

    from qclb200.kernel_build import RANK1, assemble_operator, assemble_operator_device, lo_form_factors, lo_weights
    from qclb200.problem import small_problem
    from qclb200.scba import solve_scba_production

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic"))
    x, wx, chi, _ = _structure(Nb=4, Nk=3)
    qz = np.linspace(-6.0, 6.0, 7)
    F = lo_form_factors(chi, x, wx, qz)
    W = lo_weights(np.linspace(0.0, 1.2, 3), 8, qz, np.full(7, 2.0), 0.4, 1.0)
    Fm = F.reshape((7, 16), order="F")
    host = assemble_operator("LO", RANK1, 3, 4, W, Fm)
    dev = assemble_operator_device("LO", RANK1, 3, 4, W, Fm)
    assert dev.q == host.q
    np.testing.assert_array_equal(dev.matrix.cpu().numpy().T, host.matrix)
    rows = []
    for lo in (host, dev):
        lo = dataclasses.replace(lo, q=0.05 * lo.q / lo.q)
        p2 = dataclasses.replace(pr, mechanisms=[lo] + [m for m in pr.mechanisms if m.name != "LO"])
        hist, s = solve_scba_production(p2, 3)
        s.close()
        rows.append([r["J"] for r in hist])
    assert rows[0] == rows[1]
