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
  loop (outer.solve_periodic_poisson).

The CSVs carry 12 significant digits; both agree to about 1e-12.
"""
import math
import os

import numpy as np

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
