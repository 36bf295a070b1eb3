"""Pins against outputs of the reference itself.

The reference's physics atlas (examples/10_physics_atlas.jl, run by the
reference's authors; its CSVs ship in docs/src/assets/physics/data) holds
two results this library recomputes with its own code, extracted into
tests/golden/atlas_pins.npz by tests/golden/make_atlas_pins.py:

* form_factors.csv: |<a| exp(i q z) |b>|^2 of two PzP-tail basis states
  (atlas lines 284-310) -- the longitudinal LO form factors F_h[a, c] that
  kernel_build.lo_form_factors computes for the LO kernel builder
  (lo_phonon_kernel, numerics/reference/kernels.jl:329-338);
* hartree.csv: the Hartree energy of one bordered periodic Poisson solve for
  a trial electron profile (atlas lines 256-282, solve_periodic_poisson,
  numerics/reference/poisson.jl:41-65) -- the host Poisson step of the outer
  loop (outer.solve_periodic_poisson);
* basis_operators.csv / basis_metrics.csv / spectral_population.csv: the
  projected 25 x 25 PzP-tail Hamiltonian, its eigen-energies, the
  central-period weight of each eigenstate and the local density of states
  on the central rows at eta = 2 meV (atlas lines 128-131, 224-247) -- the
  retarded Dyson solve G^R = ((E + i eta) I - H)^-1 (_retarded_green_production,
  numerics/optimized/production_operators.jl:1337-1385, with Sigma^R = 0):
  tr G^R against sum_n 1 / (E + i eta - e_n), and the central density of
  states sum_n w_n (-Im G_nn / pi) in the eigenbasis against the LDOS summed
  over z.  CPU: the oracle's retarded_green; GPU: the Dyson kernel;
* spectral_population.csv's occupied column with optical_parameters.csv
  (mu = 60 meV, T = 200 K): the Fermi function times that density of states
  -- the equilibrium Keldysh function G^< = -f (G^R - G^A) of the SCBA seed
  (_seed_green_production, numerics/optimized/seed.jl:151-197), with the
  oracle's fermi() and the CODATA Boltzmann constant.

The CSVs carry 12 significant digits; the form factors and the Hartree
energy agree to about 1e-12, the spectral pins to about 1e-10.
"""
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _pins():
    return np.load(os.path.join(HERE, "golden", "atlas_pins.npz"))


def test_lo_form_factors_reproduce_reference_atlas():
    from qclb200.kernel_build import lo_form_factors

    d = _pins()
    z = d["z_nm"]
    dx = float(d["period_nm"]) / float(d["points_per_period"])
    assert np.allclose(np.diff(z), dx, rtol=1e-9)
    chi = np.stack([d["psi_a"], d["psi_b"]], axis=1)
    F = lo_form_factors(chi, z, np.full(len(z), dx), d["q_per_nm"])
    assert np.max(np.abs(np.abs(F[:, 0, 0]) ** 2 - d["diagonal_F2"])) < 1e-10
    assert np.max(np.abs(np.abs(F[:, 0, 1]) ** 2 - d["transition_F2"])) < 1e-10
    assert abs(np.abs(F[0, 0, 0]) ** 2 - 1.0) < 1e-10  # normalised envelope


def test_periodic_poisson_reproduces_reference_hartree_energy():
    from qclb200.outer import OuterStructure, solve_periodic_poisson

    d = _pins()
    e, eps0 = 1.602176634e-19, 8.8541878128e-12  # CODATA 2018 (domain/constants.jl)
    E0, L0 = 0.1 * e, 1e-8  # ScaleSystem: E0 = 0.1 eV, L0 = 10 nm (domain/scaling.jl:10-24)
    lam = e ** 2 / (eps0 * E0 * L0)  # lambda_P (scaling.jl:20-21)
    x = d["hartree_z_nm"] / 10.0
    N = len(x)
    wx = np.full(N, float(d["period_nm"]) / float(d["points_per_period"]) / 10.0)
    st = OuterStructure(x=x, wx=wx, chi=None, Phi=None, H0=None, Z=None, Minv=None, F=0.0, z0=0.0, Cbar=0.0,
                        kappa=np.zeros(1), ND=d["donors_m3"] * L0 ** 3, eps_r=np.full(N, 12.9), lambda_P=lam)
    U, zeta, rP, neutrality = solve_periodic_poisson(st, d["electrons_m3"] * L0 ** 3)
    ref = d["hartree_meV"]
    assert np.max(np.abs(U * 100.0 - ref)) <= 1e-10 * np.max(np.abs(ref))
    assert rP < 1e-10 and neutrality < 1e-12  # the atlas's own checks (checks.csv)
    assert abs(np.sum(U)) / N < 1e-10


def _spectral_checks(GR):
    """Relative errors of tr G^R and of the central density of states against
    the reference's spectral data; GR is (N_E, 1, 25, 25)."""
    d = _pins()
    E, eta = d["spectral_E_meV"], float(d["eta_meV"])
    H = d["H_pzp_meV"]
    _, V = np.linalg.eigh(0.5 * (H + H.conj().T))
    tr = np.trace(GR[:, 0], axis1=1, axis2=2)
    want_tr = np.array([np.sum(1.0 / (e + 1j * eta - d["levels_meV"])) for e in E])
    Gn = np.einsum("an,eab,bn->en", V.conj(), GR[:, 0], V)
    dos = -(Gn.imag / math.pi) @ d["central_weight"]
    ref = d["central_dos_per_meV"]
    return (float(np.max(np.abs(tr - want_tr)) / np.max(np.abs(want_tr))),
            float(np.max(np.abs(dos - ref)) / np.max(ref)))


def _spectral_inputs():
    d = _pins()
    E = np.asarray(d["spectral_E_meV"], dtype=np.float64)
    h = np.asfortranarray(d["H_pzp_meV"][None, :, :])
    sig = np.zeros((len(E), 1) + h.shape[1:], dtype=np.complex128, order="F")
    return E, h, sig, float(d["eta_meV"])


def test_oracle_dyson_reproduces_reference_spectrum(orc):
    E, h, sig, eta = _spectral_inputs()
    GR = orc.retarded_green(E, h, sig, eta=eta)[0]
    err_tr, err_dos = _spectral_checks(GR)
    assert err_tr < 1e-10 and err_dos < 1e-9, (err_tr, err_dos)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("c128", 1e-9), ("c64", 2e-5)])
def test_gpu_dyson_reproduces_reference_spectrum(gpu_ops, precision, tol):
    E, h, sig, eta = _spectral_inputs()
    GR = gpu_ops.retarded_green(E, h, sig.astype(np.complex64) if precision == "c64" else sig, eta=eta,
                                precision=precision)
    err_tr, err_dos = _spectral_checks(np.asarray(GR, dtype=np.complex128))
    assert err_tr < tol and err_dos < tol, (err_tr, err_dos)


def test_seed_keldysh_function_reproduces_reference_occupation(orc):
    """-i G^< / 2 pi of G^< = -f (G^R - G^A) on the central states against
    the reference's occupied density of states (Fermi function at 60 meV and
    200 K times the density of states, summed over z)."""
    d = _pins()
    E, h, sig, eta = _spectral_inputs()
    GR = orc.retarded_green(E, h, sig, eta=eta)[0]
    kBT = 8.617333262e-5 * 1e3 * float(d["temperature_K"])  # meV; CODATA 2018 k_B (domain/constants.jl)
    f = orc.fermi(E, float(d["mu_meV"]), kBT)
    GL = -f[:, None, None, None] * (GR - np.conj(np.transpose(GR, (0, 1, 3, 2))))
    H = d["H_pzp_meV"]
    _, V = np.linalg.eigh(0.5 * (H + H.conj().T))
    Ln = np.einsum("an,eab,bn->en", V.conj(), GL[:, 0], V)
    occ = (np.real(-1j * Ln) / (2 * math.pi)) @ d["central_weight"]
    ref = d["central_occupied_per_meV"]
    assert float(np.max(np.abs(occ - ref)) / np.max(ref)) < 1e-9
