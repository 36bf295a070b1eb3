"""Implicit differentiation of the converged SCBA (tangent mode).

GPU: dJ/dp by the implicit-function theorem (qcl_scba_tangent_*: the
linearised Dyson / Keldysh / normalisation steps and the linear candidate
maps; the explicit dependence by one map application at p +- h) against
central finite differences of the SCBA converged at p +- h, for the bias and
the four layer thicknesses of a small full-physics-shaped structure
(acoustic + IFR: with LO as well, this 2-period, 3-state structure has no
stable fixed point under linear mixing -- the oracle's SCBA cycles at
r_Sigma ~ 0.5 for alpha = 0.3 and decays only as 0.996 per iteration at
alpha = 0.2), within 1e-4 relative (the north-star tolerance of the adjoint
gradients).
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _build(p):
    from qclb200.problem import full_physics_problem

    bias, d0, d1, d2, d3 = p
    return full_physics_problem(seed=2, NE=96, Nk=6, periods=2, states=3, Nqz=41, Nphi=16, lookup_nodes=9,
                                alpha=0.5, bias_mV=bias, mechanisms=("acoustic", "IFR"),
                                layers=(d0, d1, d2, d3))


def test_implicit_derivatives_match_central_differences(gpu_ops):
    from qclb200.gradient import central_difference, implicit_derivatives

    p0 = [50.0, 4.0, 8.5, 2.0, 16.0]
    steps = [0.1, 1e-3, 1e-3, 1e-3, 1e-3]  # mV, nm (the steps of the adjoint check)
    got = implicit_derivatives(_build, p0, steps, tol=1e-12)
    fd = central_difference(_build, p0, steps, tol=1e-12)
    for g, f in zip(got["dJ_dp"], fd):
        assert abs(g - f) <= 1e-4 * max(abs(f), 1e-6 * abs(got["J"])), (g, f)
