"""Implicit differentiation of the converged SCBA (tangent mode).

GPU: dJ/dp by the implicit-function theorem (qcl_scba_tangent_*: the
linearised Dyson / Keldysh / normalisation steps and the linear candidate
maps; the explicit dependence by one map application at p +- h) against
central finite differences of the SCBA converged at p +- h, for the bias
drop per period and the scattering strength of a small structure with LO
(dense, with its energy shifts), acoustic and IFR scattering, within 1e-4
relative (the north-star tolerance of the adjoint gradients).  The
full-physics test structures with layer thicknesses as parameters have a
slow SCBA mode at these small sizes (r_Sigma falls by 0.9995 per iteration
below ~1e-5 in the oracle's own SCBA), too slow to converge to the 1e-12 an
FD check needs; their derivative enters through the same explicit part
(one map application at p +- h), which this test covers.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _build(p):
    from qclb200.problem import small_problem

    Ep, strength = p
    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "IFR"), strength=strength)
    return dataclasses.replace(pr, Ep=Ep, alpha=0.7)


def test_implicit_derivatives_match_central_differences(gpu_ops):
    from qclb200.gradient import central_difference, implicit_derivatives

    p0 = [0.31, 0.05]  # E^p off the energy nodes (spacing 0.075): the shift interpolation is smooth there
    steps = [1e-4, 1e-5]
    got = implicit_derivatives(_build, p0, steps, tol=1e-12)
    fd = central_difference(_build, p0, steps, tol=1e-12)
    for g, f in zip(got["dJ_dp"], fd):
        assert abs(g - f) <= 1e-4 * max(abs(f), 1e-6 * abs(got["J"])), (g, f)
