"""The outer Hartree-Poisson loop around the device SCBA.

Mirror of the outer loop of ``solve_production`` (numerics/optimized/
production_solver.jl:993-1151): for a Hartree energy U(x) on the position
grid, project the Hamiltonians h_m(U) (``project_hamiltonians``,
numerics/reference/basis.jl:288-307), solve the inner SCBA on the device
(warm-started from the previous outer iteration's state), integrate the
electron density n(x) from the device's coherence matrix
(``_electron_density_bar``, physics/observables.jl:1-22), solve the bordered
periodic Poisson system for the candidate U (``solve_periodic_poisson``,
numerics/reference/poisson.jl:41-65) and mix U <- (1 - alpha_P) U + alpha_P U*.
Each outer iteration returns the reference's ``OuterIteration`` fields.

The Poisson system is an (N_z + 1)-square dense solve and the projection an
N_z x N_b^2 product: both stay FP64 on the host, as in the reference's design;
the N_E N_k N_b^2 work (the SCBA and the density integral) is on the GPU.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

from .problem import (E0_EV, E_CHARGE, L0_NM, SCBAProblem, _localized_states, small_problem)


@dataclasses.dataclass
class OuterStructure:
    """The pieces of an NEGFProblem the outer loop reads (solver units).

    ``chi`` (N_z, N_b) basis functions for the density; ``Phi`` the same
    functions weighted by sqrt(wx) for the Hartree projection (basis.Phi);
    ``H0``, ``Z`` (position matrix), ``Minv`` (inverse in-plane mass) the
    basis matrices; ``F`` the field, ``z0`` its reference position; ``Cbar``
    and ``kappa`` the in-plane kinetic coefficient and momenta; ``ND`` the
    donor density L0^3 N_D(x); ``eps_r`` the relative permittivity;
    ``lambda_P`` the Poisson scale (scaling.jl)."""

    x: np.ndarray
    wx: np.ndarray
    chi: np.ndarray
    Phi: np.ndarray
    H0: np.ndarray
    Z: np.ndarray
    Minv: np.ndarray
    F: float
    z0: float
    Cbar: float
    kappa: np.ndarray
    ND: np.ndarray
    eps_r: np.ndarray
    lambda_P: float

    @property
    def ND2D(self):
        return float(np.dot(self.wx, self.ND))

    @property
    def Lp(self):
        return float(np.sum(self.wx))


def project_hamiltonians(st: OuterStructure, U) -> np.ndarray:
    """h_m = H0 - F (Z - z0 I) + Phi^H diag(U) Phi + Cbar kappa_m^2 Minv
    (project_hamiltonians, numerics/reference/basis.jl:288-307)."""
    U = np.asarray(U, dtype=np.float64)
    if U.shape != st.x.shape or not np.all(np.isfinite(U)):
        raise ValueError("Hartree field must be finite and match the spatial grid")
    Nb = st.H0.shape[0]
    Uproj = st.Phi.conj().T @ (U[:, None] * st.Phi)
    static = st.H0 - st.F * (st.Z - st.z0 * np.eye(Nb)) + Uproj
    h = np.zeros((len(st.kappa), Nb, Nb), dtype=np.complex128, order="F")
    for m, k in enumerate(st.kappa):
        h[m] = static + st.Cbar * k * k * st.Minv
    return h


def electron_density_bar(st: OuterStructure, rho: np.ndarray, gs: int) -> np.ndarray:
    """n(x_g) = g_s/(2 pi) Re(-i sum_ab chi_ga rho_ab conj(chi_gb)) from the
    integrated coherences (_electron_density_bar, physics/observables.jl:1-22)."""
    v = np.einsum("ga,ab,gb->g", st.chi, rho, np.conj(st.chi))
    return gs / (2 * math.pi) * np.real(-1j * v)


def build_poisson_matrix(st: OuterStructure) -> np.ndarray:
    """Cyclic tridiagonal -d/dx(eps_r d/dx) with harmonic-mean face
    permittivities (build_poisson_matrix, numerics/reference/poisson.jl:12-28)."""
    N = len(st.x)
    dx = st.wx[0]
    e = st.eps_r
    face = np.array([2 * e[g] * e[(g + 1) % N] / (e[g] + e[(g + 1) % N]) for g in range(N)])
    L = np.zeros((N, N))
    for g in range(N):
        gm, gp = (g - 1) % N, (g + 1) % N
        L[g, g] = (face[gm] + face[g]) / dx ** 2
        L[g, gm] = -face[gm] / dx ** 2
        L[g, gp] = -face[g] / dx ** 2
    return L


def solve_periodic_poisson(st: OuterStructure, nbar) -> tuple:
    """Bordered periodic Poisson solve for U, the border multiplier zeta, the
    relative residual r_P and the neutrality defect (solve_periodic_poisson,
    numerics/reference/poisson.jl:41-65)."""
    N = len(st.x)
    nbar = np.asarray(nbar, dtype=np.float64)
    ND2D = st.ND2D
    neutrality = abs(float(np.dot(st.wx, st.ND - nbar))) / ND2D
    L = build_poisson_matrix(st)
    b = -st.lambda_P * (st.ND - nbar)
    sP = float(np.max(np.sum(np.abs(L), axis=1)))
    v = np.full(N, 1.0 / math.sqrt(N))
    B = np.zeros((N + 1, N + 1))
    B[:N, :N] = L / sP
    B[:N, N] = v
    B[N, :N] = v
    ans = np.linalg.solve(B, np.r_[b / sP, 0.0])
    U, zeta = ans[:N], float(ans[N])
    rP = float(np.linalg.norm(L @ U - b) / (np.linalg.norm(b) + st.lambda_P * 1e-14))
    return U, zeta, rP, neutrality


def outer_structure(problem: SCBAProblem, seed: int = 11, Nz: int = 48, length: float = 2.0,
                    field: float = 0.05) -> tuple:
    """A synthetic outer structure for `problem` (same N_b, N_k, target):
    an orthonormalised localised basis on an N_z grid of `length` (L0), donors in the first
    quarter of the cell carrying the problem's sheet density, GaAs-like
    permittivity with a lower-permittivity barrier, lambda_P = e^2 /
    (E0 eps0 L0).  The static Hamiltonian is the problem's h at kappa = 0
    with the field term moved into F (Z - z0), so project_hamiltonians(U = 0)
    reproduces problem.h up to the in-plane term.  Returns (structure,
    problem with h = project_hamiltonians(st, 0))."""
    rng = np.random.default_rng(seed)
    Nb, Nk = problem.Nb, problem.Nk
    x, wx, chi = _localized_states(rng, Nb, Nz=Nz, length=length)
    # Loewdin orthonormalisation under the quadrature weights, so that the
    # basis is orthonormal (Phi^T Phi = I) as the reference's localised basis is
    S = chi.T @ (wx[:, None] * chi)
    vals, vecs = np.linalg.eigh(S)
    chi = chi @ (vecs @ np.diag(vals ** -0.5) @ vecs.T)
    Phi = np.sqrt(wx)[:, None] * chi
    Z = Phi.T @ (x[:, None] * Phi)
    z0 = float(np.mean(x))
    H0 = np.array(problem.h[0], dtype=np.complex128) + field * (Z - z0 * np.eye(Nb))
    kappa = np.sqrt(np.maximum(np.real(np.diagonal(problem.h[:, 0:1, 0:1], axis1=1, axis2=2)[:, 0]
                                       - problem.h[0, 0, 0]), 0.0))
    ND = np.zeros(Nz)
    ND[: Nz // 4] = 1.0
    ND *= problem.target / float(np.dot(wx, ND))
    eps_r = np.full(Nz, 12.9)
    eps_r[Nz // 2: Nz // 2 + Nz // 8] = 12.2
    eps0 = 8.8541878128e-12
    lam = E_CHARGE ** 2 / (E0_EV * E_CHARGE * eps0 * L0_NM * 1e-9)
    st = OuterStructure(x=x, wx=wx, chi=chi, Phi=Phi, H0=H0, Z=Z, Minv=np.eye(Nb), F=field, z0=z0, Cbar=1.0,
                        kappa=kappa, ND=ND, eps_r=eps_r, lambda_P=lam)
    pr = dataclasses.replace(problem, h=project_hamiltonians(st, np.zeros(Nz)))
    return st, pr


def solve_production_outer(problem: SCBAProblem, st: OuterStructure, *, U0=None, max_poisson: int = 5,
                           alpha_P: float = 0.3, inner_iterations: int = 10, tol_sigma: float = -1.0,
                           precision: str = "c128", use_graph: bool = False):
    """The outer loop with the SCBA on the device.  Returns (rows, solver):
    one dict per outer iteration with the OuterIteration fields
    (production_solver.jl:1042-1088): mu, r_P, r_U, r_n, r_neutral, r_J,
    r_Jchange, r_population, zeta, J, populations, n."""
    from . import operators
    from .scba import ProductionSCBA

    Nz = len(st.x)
    U = np.zeros(Nz) if U0 is None else np.array(U0, dtype=np.float64)
    rows: List[dict] = []
    solver: Optional[ProductionSCBA] = None
    nprev = Jprev = pprev = None
    for mu in range(1, max_poisson + 1):
        h = project_hamiltonians(st, U)
        if solver is None:
            solver = ProductionSCBA(dataclasses.replace(problem, h=h), precision=precision, use_graph=use_graph)
            solver.seed()
        else:  # warm start from the previous outer iteration's state
            solver.retarget(h=h)
        hist = solver.run(inner_iterations, tol_sigma)
        last = hist[-1]
        rho = solver.density_matrix()
        nbar = electron_density_bar(st, rho, problem.gs)
        cand, zeta, rP, rneutral = solve_periodic_poisson(st, nbar)
        Unew = (1 - alpha_P) * U + alpha_P * cand
        rU = float(np.max(np.abs(cand - U)))
        rn = math.inf if nprev is None else float(
            math.sqrt(np.sum(st.wx * (nbar - nprev) ** 2)) / (st.ND2D / math.sqrt(st.Lp)))
        # _outer_current_residual (numerics/reference/solver.jl:66-72)
        M = len(solver.problem.mechanisms)
        g = solver.green()
        plus, minus = solver.family(M), solver.family(M + 1)
        pr = solver.problem
        jp = operators.current_and_populations(pr, plus[2], plus[1], g["GL"], g["GG"], precision=precision)[0]
        jm = operators.current_and_populations(pr, minus[2], minus[1], g["GL"], g["GG"], precision=precision)[0]
        rJ = abs(jp + jm) / max(abs(jp), abs(jm), 1e-12)
        J = jp * pr.J0
        pops = np.array(last["populations"])
        rJc = math.inf if Jprev is None else abs(J - Jprev) / max(abs(J), abs(Jprev), 1e-12)
        rpop = math.inf if pprev is None else float(np.linalg.norm(pops - pprev) / (np.linalg.norm(pops) + 1e-14))
        rows.append(dict(mu=mu, r_P=rP, r_U=rU, r_n=rn, r_neutral=rneutral, r_J=rJ, r_Jchange=rJc,
                         r_population=rpop, zeta=zeta, J=J, populations=pops, n=nbar, inner=hist))
        U, nprev, Jprev, pprev = Unew, nbar, J, pops
    return rows, solver


def outer_small(seed: int = 3) -> tuple:
    """The outer structure of the small all-mechanism test problem."""
    pr = small_problem(seed=seed, NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "impurity", "IFR", "alloy"))
    return outer_structure(pr)
