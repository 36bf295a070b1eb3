"""Derivatives of the converged current density by implicit differentiation.

The reference has no derivatives.  At a converged fixed point
Sigma_fp = Phi(Sigma_fp, p) of the SCBA map the implicit-function theorem
gives dSigma_fp/dp = v with

    v = Phi_Sigma v + Phi_p,        dJ/dp = J_Sigma v + J_p.

Phi_Sigma v and J_Sigma v are formed on the GPU by the linearised SCBA
iteration (qcl_scba_tangent_*: the Dyson, Keldysh and normalisation steps
linearised analytically, the candidate maps reused as the linear maps they
are), and the linear fixed point is solved by the same damped iteration as
the SCBA itself.  The explicit dependence Phi_p, J_p -- everything a
parameter changes in the problem's inputs (the Hamiltonian, the bias drop,
the kernels, ...) -- is the central difference of ONE application of the map
at the fixed point (not of a converged solve), so it carries no convergence
error: the problem is rebuilt at p +- h, the fixed-point state is uploaded and
one step is taken.  The paired number normalisation is held in the form the
fixed point used (qcl_scba_set_normalization_branch): a particle-conserving
fixed point sits on the switch between its two forms, and a difference
across the switch would mix the two one-sided derivatives.

`central_difference` converges the SCBA at p +- h instead: the check.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Sequence

import numpy as np

from ._lib import check, lib
from .scba import ProductionSCBA


def _families(solver, nfam):
    return [[solver.download(3 + 3 * f + c) for c in range(3)] for f in range(nfam)]


def _converge(problem, tol, max_iter):
    s = ProductionSCBA(problem, precision="c128", use_graph=True)
    s.seed()
    rows = s.run(max_iter, tol)
    if rows[-1]["r_Sigma"] > tol:
        s.close()
        raise RuntimeError(f"SCBA did not reach r_Sigma <= {tol} in {max_iter} iterations "
                           f"(last {rows[-1]['r_Sigma']:.3e})")
    return s, rows


def _branch(solver):
    b = ctypes.c_int(0)
    check(lib().qcl_scba_normalization_branch(solver._h, ctypes.byref(b)))
    return b.value


def _map_at(problem, fams, branch):
    """One application of the map at the uploaded state: (Phi(Sigma) per
    family component, J(Sigma)), with the paired normalisation held in the
    form `branch` of the fixed point (a particle-conserving fixed point sits
    on the switch between its two forms, and p +- h must not straddle it)."""
    s = ProductionSCBA(problem, precision="c128", use_graph=False)
    check(lib().qcl_scba_set_normalization_branch(s._h, int(branch)))
    for f, comps in enumerate(fams):
        for c, a in enumerate(comps):
            s.upload(3 + 3 * f + c, a)
    row = s.step()
    alpha = problem.alpha
    phi = []
    for f, comps in enumerate(fams):
        out = []
        for c, a in enumerate(comps):
            mixed = s.download_candidate(3 + 3 * f + c)
            out.append(a + (mixed - a) / alpha)
        phi.append(out)
    s.close()
    return phi, row["J"]


def implicit_derivatives(build: Callable[[np.ndarray], object], p0: Sequence[float], steps: Sequence[float], *,
                         tol: float = 1e-11, max_iter: int = 20000, tangent_tol: float = 1e-11,
                         max_tangent: int = 20000):
    """dJ/dp_k at p0 for every parameter of the problem family `build(p)`,
    by implicit differentiation of the FP64 fixed point.  `steps[k]` is the
    difference step of the explicit part Phi_p, J_p.  Returns a dict with the
    derivatives (A/m^2 per unit of p), J, and iteration counts."""
    p0 = np.asarray(p0, dtype=np.float64)
    pr0 = build(p0)
    nfam = len(pr0.mechanisms) + 2
    s, rows = _converge(pr0, tol, max_iter)
    fams = _families(s, nfam)
    branch = _branch(s)
    J0 = pr0.J0
    lib_s = s
    check(lib().qcl_scba_tangent_init(lib_s._h))
    grads, tangent_iters = [], []
    for k, h in enumerate(steps):
        e = np.zeros_like(p0)
        e[k] = h
        phi_p, Jp = _map_at(build(p0 + e), fams, branch)
        phi_m, Jm = _map_at(build(p0 - e), fams, branch)
        for f in range(nfam):
            for c in range(3):
                src = np.asfortranarray((phi_p[f][c] - phi_m[f][c]) / (2 * h))
                check(lib().qcl_scba_tangent_set(lib_s._h, 3 + 3 * f + c, ctypes.c_void_p(src.ctypes.data)))
        check(lib().qcl_scba_tangent_set(lib_s._h, -1, None))
        out = np.zeros(2)
        n = 0
        while n < max_tangent:
            check(lib().qcl_scba_tangent_step(lib_s._h, ctypes.c_void_p(out.ctypes.data)))
            n += 1
            if out[1] <= tangent_tol:
                break
        # one more step: out[0] is J_Sigma v of the converged v
        check(lib().qcl_scba_tangent_step(lib_s._h, ctypes.c_void_p(out.ctypes.data)))
        grads.append(out[0] * J0 + (Jp - Jm) / (2 * h))
        tangent_iters.append(n)
    s.close()
    return {"dJ_dp": np.array(grads), "J": rows[-1]["J"], "scba_iterations": len(rows),
            "tangent_iterations": tangent_iters}


def central_difference(build: Callable[[np.ndarray], object], p0: Sequence[float], steps: Sequence[float], *,
                       tol: float = 1e-11, max_iter: int = 20000):
    """(J(p0 + h e_k) - J(p0 - h e_k)) / 2h with the SCBA converged at each
    point (the check of implicit_derivatives)."""
    p0 = np.asarray(p0, dtype=np.float64)
    out = []
    for k, h in enumerate(steps):
        e = np.zeros_like(p0)
        e[k] = h
        Js = []
        for sign in (1, -1):
            s, rows = _converge(build(p0 + sign * e), tol, max_iter)
            s.close()
            Js.append(rows[-1]["J"])
        out.append((Js[0] - Js[1]) / (2 * h))
    return np.array(out)
