"""Implicit differentiation of the converged SCBA (tangent mode).

GPU: dJ/dp by the implicit-function theorem (qcl_scba_tangent_*: the
linearised Dyson / Keldysh / normalisation steps and the linear candidate
maps; the explicit dependence by one map application at p +- h) against
central finite differences of the SCBA converged at p +- h, for the bias
drop per period and the scattering strength of a small structure with LO
(dense, with its energy shifts), acoustic and IFR scattering, within 1e-4
relative (the tolerance asked of the gradients); and the four layer
thicknesses of a full-physics-shaped stack with 20 meV couplings at 300 K.  (With the builder's default 4 meV couplings at 100 K
these small stacks have a slow SCBA mode -- r_Sigma falls by 0.9995 per
iteration below ~1e-5 in the oracle's own SCBA -- too slow for the 1e-12 an
FD check needs.)
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


def test_implicit_derivatives_match_the_oracle_reference_gradient(gpu_ops, orc):
    """The same derivatives against the FP64 reference gradient of the CPU
    oracle (oracle.implicit_gradient: directional differences of the
    oracle's own SCBA map and GMRES, no code shared with the device tangent),
    which lies within 1e-7 of the converged-solve differences' Richardson
    limit here.  Bounded at 2e-4: the device derivative's agreement with the
    differences (1e-4, the test above) plus their truncation (1e-6)."""
    from qclb200.gradient import implicit_derivatives

    p0 = [0.31, 0.05]
    steps = [1e-4, 1e-5]
    got = implicit_derivatives(_build, p0, steps, tol=1e-12)
    ref, J, rS, _ = orc.implicit_gradient(_build, p0, steps, iterations=900)
    assert rS < 1e-14
    for g, r in zip(got["dJ_dp"], ref):
        assert abs(g - r) <= 2e-4 * abs(r), (g, r)


def _build_stack(p):
    from qclb200.problem import full_physics_problem

    d0, d1, d2, d3 = p
    return full_physics_problem(seed=2, NE=96, Nk=6, periods=2, states=3, Nqz=41, Nphi=16, lookup_nodes=9,
                                alpha=0.8, bias_mV=50.0, mechanisms=("LO", "acoustic", "IFR"),
                                layers=(d0, d1, d2, d3), coupling_ev=0.02, temperature_K=300.0)


def test_thickness_derivatives_match_central_differences(gpu_ops):
    """dJ/d(four layer thicknesses) of a 2-period, 3-state stack (LO +
    acoustic + IFR, 20 meV couplings at 300 K: its SCBA falls by about 0.95
    per iteration and reaches 1e-12).  The thicknesses enter the builder
    through the period length (basis functions on a grid of fixed cell count,
    round(30.5 nm / 0.5 nm) = 61 cells, so 1e-3 nm steps cross no cell) and
    the IFR interface positions.  (The stack's bias is left out: it moves the
    raw carrier number of the map across the switch of the paired
    normalisation (number above or below the target), a kink of the map that
    a particle-conserving fixed point sits on (lambda -> 1); the central
    difference of the explicit part then mixes the two one-sided branches,
    measured 9x off the converged-solve difference, while the thicknesses
    agree to 1e-7.)"""
    from qclb200.gradient import central_difference, implicit_derivatives

    p0 = [4.0, 8.5, 2.0, 16.0]
    steps = [1e-3, 1e-3, 1e-3, 1e-3]  # nm
    got = implicit_derivatives(_build_stack, p0, steps, tol=1e-12, tangent_tol=1e-9, max_tangent=5000)
    fd = central_difference(_build_stack, p0, steps, tol=1e-12)
    for g, f in zip(got["dJ_dp"], fd):
        assert abs(g - f) <= 1e-4 * max(abs(f), 1e-6 * abs(got["J"])), (g, f)


def _build_stack_bias(p):
    from qclb200.problem import full_physics_problem

    (bias,) = p
    return full_physics_problem(seed=2, NE=96, Nk=6, periods=2, states=3, Nqz=41, Nphi=16, lookup_nodes=9,
                                alpha=0.8, bias_mV=bias, mechanisms=("LO", "acoustic", "IFR"),
                                layers=(4.0, 8.5, 2.0, 16.0), coupling_ev=0.02, temperature_K=300.0)


def test_stack_bias_derivative_holds_the_normalisation_form(gpu_ops):
    """dJ/dbias of the same stack.  The explicit part is evaluated with the
    paired normalisation held in the fixed point's form on both sides
    (qcl_scba_set_normalization_branch): one map application at p +- h can
    move the raw carrier number across the switch of the paired
    normalisation (number above or below the target), and with the
    reference's choice on each side the central difference mixed the two
    one-sided branches and came out 9x off.

    The converged current curves on a 1 mV scale here (J'' ~ -1.2e6 A/m^2
    per mV^2; the oracle's converged solves, r_Sigma <= 1e-15, at 50 +- h mV
    for h = 0.1 ... 0.00625), so a central difference at h = 0.1 mV is
    1.4e-3 off the derivative, which Richardson extrapolation of those
    differences puts at -1.0712050e6 per mV.  With the explicit part's own
    step at 0.1 mV the implicit derivative was -1.0715e6 (2.8e-4 off, the
    error of that step; the oracle's FP64 implicit gradient with the branch
    held gives -1.0715221e6 at that step and -1.0712342e6, 2.7e-5 off, at
    0.01 mV).  The test takes the explicit step at 0.01 mV and checks
    against the Richardson combination of the converged-solve differences at
    0.1 and 0.05 mV; expected agreement about 3e-5, asserted at 1e-3."""
    from qclb200.gradient import central_difference, implicit_derivatives

    got = implicit_derivatives(_build_stack_bias, [50.0], [0.01], tol=1e-12, tangent_tol=1e-9, max_tangent=5000)
    d1 = central_difference(_build_stack_bias, [50.0], [0.1], tol=1e-12)[0]
    d2 = central_difference(_build_stack_bias, [50.0], [0.05], tol=1e-12)[0]
    fd = (4.0 * d2 - d1) / 3.0
    assert abs(got["dJ_dp"][0] - fd) <= 1e-3 * abs(fd), (got["dJ_dp"][0], fd, d1, d2)
