"""The FP64 reference gradient on the CPU oracle.

oracle.implicit_gradient differentiates the oracle's converged SCBA by the
implicit-function theorem, with directional differences of the oracle's own
map for Phi_Sigma v and J_Sigma v and GMRES for (I - Phi_Sigma) v = Phi_p.
It shares no code with the device tangent (qcl_scba_tangent_*, which
linearises the Dyson, Keldysh and normalisation steps analytically), so it is
an independent FP64 reference for the same derivative.  Checked here against
central differences of the oracle's converged solves, for the structure and
parameters of the device test (the bias drop per period E^p and the
scattering strength of an LO + acoustic + IFR structure).
"""
import dataclasses

import numpy as np


def _build(p):
    from qclb200.problem import small_problem

    Ep, strength = p
    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "IFR"), strength=strength)
    return dataclasses.replace(pr, Ep=Ep, alpha=0.7)


def test_oracle_implicit_gradient_matches_converged_differences(orc):
    p0 = np.array([0.31, 0.05])  # E^p off the energy nodes: the shift interpolation is smooth there
    steps = [1e-4, 1e-5]
    grad, J, rS, _ = orc.implicit_gradient(_build, p0, steps, iterations=900)
    assert rS < 1e-14
    for k, h in enumerate(steps):
        e = np.zeros(2)
        e[k] = h
        Jp = orc.scba(_build(p0 + e), 900, verify=False)[0][-1]["J"]
        Jm = orc.scba(_build(p0 - e), 900, verify=False)[0][-1]["J"]
        fd = (Jp - Jm) / (2 * h)
        # measured 1.1e-6 (E^p) and 6e-9 (strength) against these differences;
        # against their Richardson extrapolation (steps h and h/2) 9e-8 and
        # 1.6e-8: the rest is the differences' own truncation error
        assert abs(grad[k] - fd) <= 1e-5 * abs(fd), (k, grad[k], fd)
