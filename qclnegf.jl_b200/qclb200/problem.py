"""Host-side SCBA problem description and seeded synthetic structures.

The reference assembles an ``NEGFProblem`` from a layer stack (grids, basis,
projected Hamiltonian, kernels; ``numerics/reference/{grids,basis,kernels}.jl``
and ``numerics/optimized/kernels.jl:790-836``).  Those builders are one-time
host set-up and stay outside the accelerated path; here a problem is the
finished set of inputs the SCBA fixed-point map consumes:

* grids ``eps, wE`` (``grids.jl:20-27``: uniform energies, trapezoid weights)
  and ``wk`` (``grids.jl:29-37``: annulus weights ``(b_{m+1}^2-b_m^2)/(4 pi)``);
* the projected Hamiltonians ``h[m, a, b]`` (``basis.jl:288-331``);
* the neighbour couplings ``T+`` and ``T- = T+^H`` (``basis.jl:56-57``);
* the kernel operators per mechanism (the factorised forms built by
  ``production_cache.jl:387-448``);
* the scalars ``g_s``, the target sheet density ``N_D`` (solver units),
  ``E^p = F L_p`` and ``hbar omega_LO`` (``scaling.jl:95-110``).

All arrays use the reference's Julia layout: numpy arrays in Fortran order
with shape ``(N_E, N_k, N_b, N_b)`` for fields, ``(N_k, N_b, N_b)`` for ``h``.

The structures below are synthetic and seeded: they have the shapes, sizes
and value ranges of the workloads they stand for, not the reference's
converged physics of a particular device.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

# Solver units (scaling.jl:10-24): E0 = 0.1 eV, L0 = 10 nm, m_ref = 0.067 m0.
E0_EV = 0.1
L0_NM = 10.0
HBAR2_OVER_2M0_EV_NM2 = 0.0380998212  # hbar^2 / (2 m0) in eV nm^2
KB_EV = 8.617333262e-5
E_CHARGE = 1.602176634e-19
HBAR_EV_S = 6.582119569e-16
# J0 = e E0 / (hbar L0^2) in A/m^2 (scaling.jl:22)
J0_A_M2 = E_CHARGE * E0_EV / (HBAR_EV_S * (L0_NM * 1e-9) ** 2)

MECHANISM_ORDER = ("LO", "acoustic", "impurity", "IFR", "alloy")


def fortran_zeros(shape, dtype=np.complex128):
    return np.zeros(shape, dtype=dtype, order="F")


@dataclasses.dataclass
class Mechanism:
    """One enabled scattering mechanism in its factorised operator form.

    kind:
      * ``"momentum_independent"`` -- ``block`` is the ``(Nb^2, Nb^2)``
        matrix of ``K[1,1,a,c,d,b]`` with rows ``(a,b)`` and columns ``(c,d)``
        (``production_cache.jl:396-399``);
      * ``"dense"`` -- ``matrix`` has rows ``(m,a,b)`` and columns
        ``(m',c,d)`` (``production_cache.jl:400-405``);
      * ``"ifr"`` -- ``left (Nb^2,J)``, ``right (J,Nb^2)``, ``radial (Nk,Nk)``
        (``production_cache.jl:414-448``);
      * ``"low_rank"`` -- ``left (Nk Nb^2, r)`` (U S), ``right (r, Nk Nb^2)``
        (V^H) of the dense matrix (``production_cache.jl:348-385``);
      * ``"separable_sum"`` -- ``radial (Nk, Nk, J)`` and ``block (Nb^2, Nb^2,
        J)`` (rows ``(a,b)``, columns ``(c,d)``): ``K(m,m') = sum_i
        radial_i(m,m') block_i``, the Kronecker-sum form of the momentum
        dependent kernels (``kernel_build.separable_sum_operator``).
    ``q`` is the kernel scale ``q^K`` (``kernels.jl:388-405``).
    """

    name: str
    kind: str
    q: float
    block: Optional[np.ndarray] = None
    matrix: Optional[np.ndarray] = None
    left: Optional[np.ndarray] = None
    right: Optional[np.ndarray] = None
    radial: Optional[np.ndarray] = None
    residual: float = 0.0  # low rank: attained relative discarded singular-value norm

    def literal_kernel(self, Nk: int, Nb: int) -> np.ndarray:
        """The six-index tensor K[m,m',a,c,d,b] this operator represents."""
        K = np.zeros((Nk, Nk, Nb, Nb, Nb, Nb), dtype=np.complex128, order="F")
        if self.kind == "momentum_independent":
            # block[(a,b),(c,d)] -> K[a,c,d,b]
            blk = np.transpose(np.asarray(self.block).reshape((Nb, Nb, Nb, Nb), order="F"), (0, 2, 3, 1))
            for m in range(Nk):
                for mp in range(Nk):
                    K[m, mp] = blk
        elif self.kind == "dense":
            # rows (m,a,b), cols (m',c,d), first index fastest
            M = self.matrix.reshape((Nk, Nb, Nb, Nk, Nb, Nb), order="F")
            # M[m,a,b,m',c,d] -> K[m,m',a,c,d,b]
            K[...] = np.transpose(M, (0, 3, 1, 4, 5, 2))
        elif self.kind == "low_rank":
            M = (self.left @ self.right).reshape((Nk, Nb, Nb, Nk, Nb, Nb), order="F")
            K[...] = np.transpose(M, (0, 3, 1, 4, 5, 2))
        elif self.kind == "separable_sum":
            J = self.radial.shape[2]
            blk = np.asarray(self.block).reshape((Nb, Nb, Nb, Nb, J), order="F")  # [a,b,c,d,i]
            K[...] = np.einsum("mni,abcdi->mnacdb", np.asarray(self.radial), blk)
        elif self.kind == "ifr":
            J = self.left.shape[1]
            L = self.left.reshape((Nb, Nb, J), order="F")  # [a,b,j]
            R = self.right.reshape((J, Nb, Nb), order="F")  # [j,c,d]
            blk = np.einsum("abj,jcd->acdb", L, R)
            for m in range(Nk):
                for mp in range(Nk):
                    K[m, mp] = self.radial[m, mp] * blk
        else:
            raise ValueError(self.kind)
        return K


def _is_momentum_independent(K: np.ndarray) -> bool:
    """_is_momentum_independent (production_cache.jl:338-346): every (m, m')
    slice of K equals K[1,1]."""
    ref = K[0, 0]
    return all(np.array_equal(K[m, mp], ref) for m in range(K.shape[0]) for mp in range(K.shape[1]))


def low_rank_production_kernel(name: str, q: float, matrix: np.ndarray, relative_tolerance: float = 0.0,
                               maximum_rank: int = 0) -> Mechanism:
    """_low_rank_production_kernel (production_cache.jl:348-385): thin SVD of
    the dense (m,a,b) x (m',c,d) matrix, truncated at the smallest rank whose
    discarded singular values have norm <= tol * ||s||, capped at
    ``maximum_rank`` (0 = no cap).  ``left = U_r diag(s_r)``, ``right =
    V_r^H``.  Raises ValueError (the reference's ArgumentError) when the cap
    cannot meet the tolerance.  ``.residual`` holds the attained relative
    discarded norm."""
    if not 0.0 <= relative_tolerance < 1.0:
        raise ValueError("low_rank_relative_tolerance must lie in [0,1)")
    if maximum_rank < 0:
        raise ValueError("low_rank_maximum_rank cannot be negative")
    U, sv, Vh = np.linalg.svd(np.asarray(matrix, dtype=np.complex128), full_matrices=False)
    total = float(np.linalg.norm(sv))
    cap = len(sv) if maximum_rank == 0 else min(maximum_rank, len(sv))
    rank = len(sv)
    if total > 0 and relative_tolerance > 0:
        tail = float(np.sum(np.abs(sv) ** 2))
        for cand in range(len(sv)):
            tail -= float(abs(sv[cand]) ** 2)
            rank = cand + 1
            if math.sqrt(max(tail, 0.0)) <= relative_tolerance * total:
                break
    rank = min(rank, cap)
    discarded = 0.0 if rank == len(sv) else float(np.linalg.norm(sv[rank:]))
    residual = 0.0 if total == 0 else discarded / total
    if not residual <= relative_tolerance + 64 * np.finfo(np.float64).eps:
        raise ValueError(f"low_rank_maximum_rank={cap} cannot satisfy the requested relative tolerance "
                         f"{relative_tolerance} (attained {residual})")
    left = np.asfortranarray(U[:, :rank] * sv[:rank][None, :])
    right = np.asfortranarray(Vh[:rank, :])
    return Mechanism(name, "low_rank", q, left=left, right=right, residual=residual)


def production_kernel(name: str, q: float, K: np.ndarray, contraction: str = "dense_blas",
                      low_rank_relative_tolerance: float = 0.0, low_rank_maximum_rank: int = 0) -> Mechanism:
    """_production_kernel (production_cache.jl:387-409): the factorised
    operator of a six-index kernel K[m,m',a,c,d,b].  A momentum-independent K
    becomes its (a,b) x (c,d) block; otherwise K is permuted to the (m,a,b) x
    (m',c,d) matrix, dense or truncated (``contraction="low_rank"``).
    ``contraction="literal"`` keeps the literal six-index map, which as a
    linear map is that same dense matrix, so it is returned in dense form."""
    if contraction not in ("literal", "dense_blas", "low_rank"):
        raise ValueError("contraction must be :literal, :dense_blas, or :low_rank")
    K = np.asarray(K, dtype=np.complex128)
    Nk, Nk2, Nb, Nb2, Nb3, Nb4 = K.shape
    if not (Nk == Nk2 and Nb == Nb2 == Nb3 == Nb4):
        raise ValueError("kernel order must be (m,m',a,c,d,b)")
    if contraction != "literal" and _is_momentum_independent(K):
        return Mechanism(name, "momentum_independent", q, block=block_matrix(K[0, 0]))
    # rows (m,a,b), cols (m',c,d): permute (m,m',a,c,d,b) -> (m,a,b,m',c,d)
    matrix = np.transpose(K, (0, 2, 5, 1, 3, 4)).reshape((Nk * Nb * Nb, Nk * Nb * Nb), order="F")
    if contraction == "low_rank":
        return low_rank_production_kernel(name, q, matrix, low_rank_relative_tolerance, low_rank_maximum_rank)
    return Mechanism(name, "dense", q, matrix=np.asfortranarray(matrix))


@dataclasses.dataclass
class SCBAProblem:
    NE: int
    Nk: int
    Nb: int
    eps: np.ndarray
    wE: np.ndarray
    wk: np.ndarray
    h: np.ndarray  # (Nk, Nb, Nb) F-order complex
    Tplus: np.ndarray  # (Nb, Nb)
    Tminus: np.ndarray
    Ep: float
    hw_LO: float
    N_LO: float
    gs: int
    target: float
    kBT: float
    eta_seed: float
    alpha: float
    mechanisms: List[Mechanism]
    J0: float = J0_A_M2
    name: str = "problem"
    # scattering-model switches of AlgorithmOptions (algorithm_options.jl:19-39)
    self_energy_structure: str = "full"           # or "diagonal"
    transverse_momentum: str = "resolved"         # or "averaged"
    retarded_real_part: str = "kramers_kronig"    # or "drop"
    elastic_retarded: str = "hilbert"             # or "direct_green"
    occupation_normalization: str = "paired_convex"  # or "scalar_lesser"
    mixing: str = "linear"                        # or "anderson"
    anderson_history_depth: int = 5
    anderson_damping: float = 1.0
    anderson_regularization: float = 1e-12

    @property
    def shape(self):
        return (self.NE, self.Nk, self.Nb, self.Nb)

    def field_bytes(self, itemsize=16):
        return self.NE * self.Nk * self.Nb * self.Nb * itemsize


def energy_grid(emin: float, emax: float, NE: int):
    """Uniform grid and trapezoid weights (grids.jl:20-27)."""
    eps = np.linspace(emin, emax, NE)
    de = (emax - emin) / (NE - 1)
    wE = np.full(NE, de)
    wE[[0, -1]] /= 2
    return eps, wE


def momentum_grid(kmax: float, Nk: int):
    """Uniform radial grid and annulus weights (grids.jl:29-37)."""
    kappa = np.linspace(0.0, kmax, Nk)
    bnd = np.zeros(Nk + 1)
    for m in range(1, Nk):
        bnd[m] = 0.5 * (kappa[m - 1] + kappa[m])
    bnd[-1] = kmax
    wk = (bnd[1:] ** 2 - bnd[:-1] ** 2) / (4 * math.pi)
    return kappa, wk


def _kinetic_coefficient(mass_ratio=0.067):
    """hbar^2/(2 m*) in solver units (E0 L0^2)."""
    return HBAR2_OVER_2M0_EV_NM2 / mass_ratio / (E0_EV * L0_NM ** 2)


def _supercell(rng, periods, states, level_ev, Ep, coupling_ev, mass_spread=0.03):
    """Onsite block h0 (solver units) of a `periods` x `states` supercell,
    the neighbour coupling T+ and a weak mass-mixing matrix."""
    Nb = periods * states
    h0 = np.zeros((Nb, Nb), dtype=np.complex128)
    for p in range(periods):
        for s in range(states):
            h0[p * states + s, p * states + s] = level_ev[s] / E0_EV - p * Ep
    c = coupling_ev / E0_EV
    for p in range(periods - 1):
        blk = c * (rng.standard_normal((states, states)) + 1j * rng.standard_normal((states, states))) / math.sqrt(2)
        h0[p * states:(p + 1) * states, (p + 1) * states:(p + 2) * states] = blk
        h0[(p + 1) * states:(p + 2) * states, p * states:(p + 1) * states] = blk.conj().T
    intra = 0.2 * c * (rng.standard_normal((Nb, Nb)) + 1j * rng.standard_normal((Nb, Nb)))
    intra = np.triu(intra, 1)
    h0 += intra + intra.conj().T
    Tplus = np.zeros((Nb, Nb), dtype=np.complex128)
    blk = c * (rng.standard_normal((states, states)) + 1j * rng.standard_normal((states, states))) / math.sqrt(2)
    Tplus[(periods - 1) * states:, :states] = blk
    mix = mass_spread * rng.standard_normal((Nb, Nb))
    mix = 0.5 * (mix + mix.T)
    return h0, Tplus, mix


def _localized_states(rng, Nb, Nz=96, length=3.0):
    """Real, normalised, localised synthetic basis functions chi[g, a] on a
    cell-centred grid (the role of basis.chi, basis.jl:15-110)."""
    dx = length / Nz
    x = (np.arange(Nz) + 0.5) * dx
    centres = np.linspace(0.1 * length, 0.9 * length, Nb) + 0.02 * rng.standard_normal(Nb)
    widths = 0.12 * length / max(Nb / 4, 1) * (1 + 0.2 * rng.random(Nb))
    chi = np.exp(-0.5 * ((x[:, None] - centres[None, :]) / widths[None, :]) ** 2)
    chi *= 1 + 0.3 * np.sin(3 * x[:, None] / length * math.pi * (1 + np.arange(Nb)[None, :] % 3))
    chi /= np.sqrt((chi ** 2).sum(axis=0) * dx)[None, :]
    return x, np.full(Nz, dx), chi


def block_matrix(K4: np.ndarray) -> np.ndarray:
    """The (Nb^2, Nb^2) operator of a momentum-independent kernel slice
    K[a,c,d,b]: rows (a,b), columns (c,d), first index fastest
    (production_cache.jl:396-399)."""
    Nb = K4.shape[0]
    return np.asfortranarray(np.transpose(K4, (0, 3, 1, 2)).reshape((Nb * Nb, Nb * Nb), order="F"))


def acoustic_block(chi, wx, prefactor):
    """Deformation-potential kernel slice K[a,c,d,b] = P sum_g w chi_a chi_c
    chi_d chi_b (acoustic_kernel, numerics/reference/kernels.jl:246-283, real
    basis functions) in (a,c,d,b) order."""
    K = prefactor * np.einsum("g,ga,gc,gd,gb->acdb", wx, chi, chi, chi, chi)
    return np.asfortranarray(K.astype(np.complex128))


def tutorial_problem(seed: int = 1, NE: int = 400, Nk: int = 16, alpha: float = 0.3) -> SCBAProblem:
    """Plain-FP64 tutorial-scale SCBA structure: 3 periods x 4 states
    (N_b = 12), N_E = 400 energies over 0.3 eV, N_k = 16 in-plane momenta on
    0-60 meV kinetic energy, acoustic phonons only, T = 50 K, 50 mV/period,
    linear mixing 0.3."""
    rng = np.random.default_rng(seed)
    periods, states = 3, 4
    Nb = periods * states
    Ep = 0.050 / E0_EV
    eps, wE = energy_grid(-0.13 / E0_EV, 0.17 / E0_EV, NE)
    Cbar = _kinetic_coefficient()
    kmax = math.sqrt(0.060 / E0_EV / Cbar)
    kappa, wk = momentum_grid(kmax, Nk)
    h0, Tplus, mix = _supercell(rng, periods, states, [0.010, 0.045, 0.085, 0.120], Ep, 0.004)
    h = np.zeros((Nk, Nb, Nb), dtype=np.complex128, order="F")
    for m in range(Nk):
        h[m] = h0 + Cbar * kappa[m] ** 2 * (np.eye(Nb) + mix)
    x, wx, chi = _localized_states(rng, Nb)
    # Xi^2 kB T / (rho v_s^2) / (L0 K0) with Xi = 7 eV, T = 50 K, GaAs rho, v_s
    # (acoustic_kernel prefactor, kernels.jl:262-266; presets.jl:76-78).
    Xi = 7.0 * E_CHARGE
    kBT_J = 1.380649e-23 * 50.0
    pref = Xi ** 2 * kBT_J / (5317.0 * 5220.0 ** 2) / (L0_NM * 1e-9)
    K0 = (E0_EV * E_CHARGE) ** 2 * (L0_NM * 1e-9) ** 2
    K = acoustic_block(chi, wx, pref / K0)
    q = float(np.max(np.abs(K)))
    mech = Mechanism("acoustic", "momentum_independent", q, block=block_matrix(K / q))
    # 4.5e14 m^-2 sheet doping (presets.jl:62) in solver units (x L0^2)
    target = 4.5e14 * (L0_NM * 1e-9) ** 2
    kBT = KB_EV * 50.0 / E0_EV
    hw_LO = 0.0367 / E0_EV
    return SCBAProblem(
        NE=NE, Nk=Nk, Nb=Nb, eps=eps, wE=wE, wk=wk, h=h, Tplus=np.asfortranarray(Tplus),
        Tminus=np.asfortranarray(Tplus.conj().T), Ep=Ep, hw_LO=hw_LO,
        N_LO=1.0 / math.expm1(0.0367 / (KB_EV * 50.0)), gs=2, target=target, kBT=kBT,
        eta_seed=0.0005 / E0_EV, alpha=alpha, mechanisms=[mech], name="tutorial_N12",
    )


def small_problem(seed=3, NE=33, Nk=3, Nb=4, mechanisms=("acoustic",), alpha=0.3,
                  strength=0.05) -> SCBAProblem:
    """A tiny structure for exhaustive oracle/GPU comparisons of every
    mechanism kind (LO with its shifts, dense impurity, separable IFR,
    momentum-independent acoustic and alloy)."""
    rng = np.random.default_rng(seed)
    states = Nb if Nb < 4 else Nb // 2
    periods = max(Nb // states, 1)
    Ep = 0.3
    eps, wE = energy_grid(-1.0, 2.0, NE)
    kappa, wk = momentum_grid(2.0, Nk)
    Cbar = 0.06
    h0 = np.diag(np.linspace(-0.3, 1.2, Nb)).astype(np.complex128)
    cpl = 0.05 * (rng.standard_normal((Nb, Nb)) + 1j * rng.standard_normal((Nb, Nb)))
    cpl = np.triu(cpl, 1)
    h0 += cpl + cpl.conj().T
    h = np.zeros((Nk, Nb, Nb), dtype=np.complex128, order="F")
    for m in range(Nk):
        h[m] = h0 + Cbar * kappa[m] ** 2 * np.eye(Nb)
    Tplus = 0.05 * (rng.standard_normal((Nb, Nb)) + 1j * rng.standard_normal((Nb, Nb)))
    x, wx, chi = _localized_states(rng, Nb, Nz=48, length=2.0)
    mechs = []
    for name in MECHANISM_ORDER:
        if name not in mechanisms:
            continue
        if name in ("acoustic", "alloy"):
            K = acoustic_block(chi, wx, 1.0)
            q = float(np.max(np.abs(K)))
            mechs.append(Mechanism(name, "momentum_independent", strength * (1.3 if name == "alloy" else 1.0),
                                   block=block_matrix(K / q)))
        elif name in ("LO", "impurity"):
            # sum_h R_h(m,m') F_h (x) F_h^* -- the LO/impurity covariance form
            # (kernels.jl:321-356) with synthetic form factors.
            Nq = 5
            F = rng.standard_normal((Nq, Nb, Nb)) + 1j * rng.standard_normal((Nq, Nb, Nb))
            F = 0.5 * (F + np.conj(np.transpose(F, (0, 2, 1))))
            R = np.empty((Nq, Nk, Nk))
            for hq in range(Nq):
                R[hq] = 1.0 / (1.0 + (kappa[:, None] - kappa[None, :]) ** 2 + hq)
            K = np.einsum("hmn,hac,hbd->mnacdb", R, F, np.conj(F))
            q = float(np.max(np.abs(K)))
            K = K / q
            # rows (m,a,b), cols (m',c,d)
            M = np.transpose(K, (0, 2, 5, 1, 3, 4)).reshape((Nk * Nb * Nb, Nk * Nb * Nb), order="F")
            mechs.append(Mechanism(name, "dense", strength * (0.8 if name == "LO" else 0.5),
                                   matrix=np.asfortranarray(M.astype(np.complex128))))
        elif name == "IFR":
            J = 3
            v = rng.standard_normal((Nb, J)) + 0.3j * rng.standard_normal((Nb, J))
            left = np.zeros((Nb * Nb, J), dtype=np.complex128)
            right = np.zeros((J, Nb * Nb), dtype=np.complex128)
            for j in range(J):
                for b in range(Nb):
                    for a in range(Nb):
                        val = v[a, j] * np.conj(v[b, j])
                        left[a + Nb * b, j] = val
                        right[j, a + Nb * b] = np.conj(val)
            radial = np.exp(-0.5 * (kappa[:, None] - kappa[None, :]) ** 2).astype(np.complex128)
            mech = Mechanism(name, "ifr", 1.0, left=np.asfortranarray(left), right=np.asfortranarray(right),
                             radial=np.asfortranarray(radial))
            K = mech.literal_kernel(Nk, Nb)
            q = float(np.max(np.abs(K)))
            mech.left = np.asfortranarray(left / q)
            mech.q = strength * 0.6
            mechs.append(mech)
    return SCBAProblem(
        NE=NE, Nk=Nk, Nb=Nb, eps=eps, wE=wE, wk=wk, h=h, Tplus=np.asfortranarray(Tplus),
        Tminus=np.asfortranarray(Tplus.conj().T), Ep=Ep, hw_LO=0.367, N_LO=0.25, gs=2,
        target=0.05, kBT=0.2, eta_seed=0.02, alpha=alpha, mechanisms=mechs, name="small",
    )


def operator_batch_hamiltonian(N: int, Nk: int, seed: int = 7):
    """Hermitian block-tridiagonal h per k (blocks of 8 states, diagonal
    subband energies U(0, 250 meV), inter-period couplings N(0, 2 meV)) plus
    a parabolic in-plane dispersion; solver units."""
    rng = np.random.default_rng(seed)
    blocks = N // 8
    h0 = np.zeros((N, N), dtype=np.complex128)
    h0[np.arange(N), np.arange(N)] = rng.uniform(0.0, 0.250, N) / E0_EV
    for p in range(blocks - 1):
        blk = (rng.standard_normal((8, 8)) + 1j * rng.standard_normal((8, 8))) * (0.002 / E0_EV) / math.sqrt(2)
        h0[p * 8:(p + 1) * 8, (p + 1) * 8:(p + 2) * 8] = blk
        h0[(p + 1) * 8:(p + 2) * 8, p * 8:(p + 1) * 8] = blk.conj().T
    Cbar = _kinetic_coefficient()
    kappa, wk = momentum_grid(math.sqrt(0.060 / E0_EV / Cbar), Nk)
    h = np.zeros((Nk, N, N), dtype=np.complex128, order="F")
    for m in range(Nk):
        h[m] = h0 + Cbar * kappa[m] ** 2 * np.eye(N)
    eps, wE = energy_grid(-0.05 / E0_EV, 0.35 / E0_EV, 4096)
    return h, wk, kappa


# GaAs / Al0.15Ga0.85As constants used by the full-physics synthetic structure
# (presets.jl:45-47, 76-78; SI).
_EPS0 = 8.8541878128e-12
_KB_J = 1.380649e-23
_GAAS_EPS_INF, _GAAS_EPS_S = 10.89, 12.9
_GAAS_RHO, _GAAS_VS, _GAAS_XI_EV = 5317.0, 5220.0, 7.0


def _period_basis(rng, periods, states, layers_nm, dz_nm=0.5):
    """Real, normalised, localised basis functions chi[g, a] (a = period *
    states + s) on a cell-centred grid over `periods` periods of the layer
    stack, in solver units (x / L0, sum_g wx chi^2 = 1); also the interface
    coordinates (layer edges, the period seam included once per period)."""
    Lp = sum(layers_nm) / L0_NM
    nz = int(round(sum(layers_nm) / dz_nm))
    dx = Lp / nz
    x = (np.arange(periods * nz) + 0.5) * dx
    chi = np.zeros((len(x), periods * states))
    for p in range(periods):
        centres = p * Lp + Lp * (np.arange(states) + 0.5) / states + 0.03 * Lp * rng.standard_normal(states)
        widths = Lp * (0.10 + 0.12 * rng.random(states))
        for s in range(states):
            a = p * states + s
            u = (x - centres[s]) / widths[s]
            chi[:, a] = np.exp(-0.5 * u ** 2) * (1 + 0.4 * np.sin((1 + s % 3) * math.pi * u))
    chi /= np.sqrt((chi ** 2).sum(axis=0) * dx)[None, :]
    edges = np.cumsum(layers_nm) / L0_NM
    interfaces = np.array([p * Lp + e for p in range(periods) for e in np.concatenate(([0.0], edges[:-1]))])
    return x, np.full(len(x), dx), chi, interfaces


def full_physics_problem(seed: int = 11, NE: int = 2048, Nk: int = 64, periods: int = 4, states: int = 8,
                         Nqz: int = 401, Nphi: int = 64, lookup_nodes: int = 129, rtol: float = 1e-15,
                         alpha: float = 0.5, bias_mV: float = 50.0,
                         mechanisms=("LO", "acoustic", "impurity", "IFR", "alloy"),
                         kernels=None, layers=(4.0, 8.5, 2.0, 16.0), coupling_ev: float = 0.004,
                         temperature_K: float = 100.0) -> SCBAProblem:
    """Full-physics-shaped SCBA structure: a supercell of `periods` periods x
    `states` localised states (N_b = 32 by default) of the GaAs /
    Al0.15Ga0.85As stack 4.0 / 8.5 / 2.0 / 16.0 nm, N_E = 2048 energies over
    [-0.25, 0.40] eV, N_k = 64 momenta on 0-80 meV kinetic energy, T = 100 K,
    with all five mechanisms built from the basis functions:

    * LO phonon (36.7 meV): the exact screened Froehlich kernel
      (lo_phonon_kernel, numerics/reference/kernels.jl:321-356) on N_qz = 401
      longitudinal nodes (|q_z| <= 10 nm^-1) and N_phi = 64 angles, as a
      separable sum;
    * acoustic deformation potential (Xi = 7 eV, kernels.jl:246-283) and
      alloy disorder (kernels.jl:285-319), momentum independent;
    * ionised impurities, 2D sheet doping 3e10 cm^-2 per period in the 4 nm
      layer: the tabulated screened covariance (numerics/optimized/
      kernels.jl:122-158, 303-320) on `lookup_nodes` nodes, as a separable sum;
    * interface roughness (Delta = 0.1 nm, Lambda = 8 nm) at every layer edge
      (interface_roughness_kernel, kernels.jl:176-244), separable.

    The basis functions, level scheme and couplings are synthetic and seeded;
    the kernels follow the reference formulas with these basis functions.
    `rtol` is the compression tolerance of the separable sums.  `mechanisms`
    selects the mechanisms (in the reference order); `kernels` (the
    mechanism list of an earlier call with the same seed, structure and N_k)
    is reused as is -- the kernels do not depend on the bias or the energy
    grid, as retarget_problem keeps them (composition/operating_point.jl:
    25-150).  `coupling_ev` is the scale of the random inter-period and
    (x 0.2) intra-period couplings of the supercell Hamiltonian;
    `temperature_K` the lattice temperature (phonon occupation, acoustic
    kernel, k_B T of the seed)."""
    from .kernel_build import (impurity_pair_factors, lo_form_factors, lo_weights, lookup_weights,
                               separable_sum_operator, transfer_momenta)

    rng = np.random.default_rng(seed)
    Nb = periods * states
    layers = [float(d) for d in layers]
    Ep = bias_mV * 1e-3 / E0_EV
    eps, wE = energy_grid(-0.25 / E0_EV, 0.40 / E0_EV, NE)
    Cbar = _kinetic_coefficient()
    kmax = math.sqrt(0.080 / E0_EV / Cbar)
    kappa, wk = momentum_grid(kmax, Nk)
    levels = list(np.linspace(0.0, 0.24, states) + 0.004 * rng.standard_normal(states))
    h0, Tplus, mix = _supercell(rng, periods, states, levels, Ep, coupling_ev)
    h = np.zeros((Nk, Nb, Nb), dtype=np.complex128, order="F")
    for m in range(Nk):
        h[m] = h0 + Cbar * kappa[m] ** 2 * (np.eye(Nb) + mix)
    x, wx, chi, interfaces = _period_basis(rng, periods, states, layers)
    L0 = L0_NM * 1e-9
    K0 = (E0_EV * E_CHARGE) ** 2 * L0 ** 2
    T_K = float(temperature_K)
    hw = 0.0367
    mechs = []
    want = set(mechanisms)
    # LO: prefactor e^2 hbar w / (2 eps0) (1/eps_inf - 1/eps_s) L0 / K0 (kernels.jl:340-355)
    pre_lo = E_CHARGE ** 2 * hw * E_CHARGE / (2 * _EPS0) * (1 / _GAAS_EPS_INF - 1 / _GAAS_EPS_S) * L0 / K0
    qz = np.linspace(-10.0 * L0_NM, 10.0 * L0_NM, Nqz)
    wqz = np.full(Nqz, qz[1] - qz[0])
    if kernels is None and "LO" in want:
        F = lo_form_factors(chi, x, wx, qz).reshape((Nqz, Nb * Nb), order="F")
        W = lo_weights(kappa, Nphi, qz, wqz, qscreen=0.05 * L0_NM, prefactor=pre_lo)
        mechs.append(separable_sum_operator("LO", W, F, rtol=rtol))
    # acoustic: Xi^2 kB T / (rho v_s^2) / (L0 K0) sum_g w chi^4 (kernels.jl:262-283)
    pre_ac = (_GAAS_XI_EV * E_CHARGE) ** 2 * _KB_J * T_K / (_GAAS_RHO * _GAAS_VS ** 2) / L0 / K0
    if kernels is None and "acoustic" in want:
        Kac = acoustic_block(chi, wx, pre_ac)
        q = float(np.max(np.abs(Kac)))
        mechs.append(Mechanism("acoustic", "momentum_independent", q, block=block_matrix(Kac / q)))
    # impurity: 3e10 cm^-2 per period over the cells of each period's first (4 nm) layer
    Lp = sum(layers) / L0_NM
    doped = ((x % Lp) < layers[0] / L0_NM)
    sheet = 3e14 * L0 ** 2  # N_D L0^2 per period
    donor_w = np.where(doped, wx, 0.0)
    donor_w *= sheet * periods / donor_w.sum()
    pre_imp = math.sqrt(E_CHARGE ** 4 / (2 * _EPS0 * _GAAS_EPS_S) ** 2 / K0)  # V in sqrt(K0) units
    qmax = float(transfer_momenta(kappa, Nphi).max())
    nodes = qmax * (np.arange(lookup_nodes) / (lookup_nodes - 1)) ** 2
    qs_imp = 0.1 * L0_NM
    if kernels is None and "impurity" in want:
        VD = [impurity_pair_factors(qn, chi, x, wx, donor_w, qs_imp, pre_imp) for qn in nodes]
        mechs.append(separable_sum_operator("impurity", lookup_weights(nodes, kappa, Nphi),
                                            np.array([v for v, _ in VD]), VD[0][1], rtol=rtol))
    # IFR: D_j[a,c] = dEc chi_a(z_j) chi_c(z_j); block = sum_j D_j (x) conj D_j; radial = angular
    # mean of pi Delta^2 Lambda^2 exp(-q^2 Lambda^2 / 4) (interface_roughness_kernel, kernels.jl:176-244)
    dEc = 0.831 * 0.15 / E0_EV
    u = np.array([[np.interp(z, x, chi[:, a]) for a in range(Nb)] for z in interfaces])  # (J, Nb)
    Jn = len(interfaces)
    left = np.zeros((Nb * Nb, Jn), dtype=np.complex128)
    for j in range(Jn):
        left[:, j] = (dEc * np.outer(u[j], u[j])).reshape(Nb * Nb, order="F")
    right = np.asfortranarray(left.conj().T)
    Delta, Lam = 0.1 / L0_NM, 8.0 / L0_NM
    qt = transfer_momenta(kappa, Nphi)
    radial = (math.pi * Delta ** 2 * Lam ** 2 * np.exp(-qt ** 2 * Lam ** 2 / 4).mean(axis=2)).astype(np.complex128)
    qifr = float(np.max(np.abs(radial))) * float(np.max(np.abs(left @ right)))
    if kernels is None and "IFR" in want:
        mechs.append(Mechanism("IFR", "ifr", qifr, left=np.asfortranarray(left), right=right,
                               radial=np.asfortranarray(radial / qifr)))
    # alloy: Omega dV^2 x(1 - x) in the barriers (kernels.jl:285-319), Omega = a^3 / 4, dV = 0.6 eV
    # barriers: the even layers of the stack (Al0.15Ga0.85As), wells the odd ones
    edges = np.concatenate(([0.0], np.cumsum(layers) / L0_NM))
    layer_of = np.clip(np.searchsorted(edges, x % Lp, side="right") - 1, 0, len(layers) - 1)
    xal = np.where(layer_of % 2 == 0, 0.15, 0.0)
    pre_al = (0.565e-9) ** 3 / 4 * (0.6 * E_CHARGE) ** 2 / L0 / K0
    if kernels is None and "alloy" in want:
        Kal = acoustic_block(chi, wx * xal * (1 - xal), pre_al)
        q = float(np.max(np.abs(Kal)))
        mechs.append(Mechanism("alloy", "momentum_independent", q, block=block_matrix(Kal / q)))
    if kernels is not None:
        mechs = list(kernels)
    kBT = KB_EV * T_K / E0_EV
    target = 3e14 * L0 ** 2 * periods
    return SCBAProblem(
        NE=NE, Nk=Nk, Nb=Nb, eps=eps, wE=wE, wk=wk, h=h, Tplus=np.asfortranarray(Tplus),
        Tminus=np.asfortranarray(Tplus.conj().T), Ep=Ep * periods, hw_LO=hw / E0_EV,
        N_LO=1.0 / math.expm1(hw / (KB_EV * T_K)), gs=2, target=target, kBT=kBT,
        eta_seed=0.0005 / E0_EV, alpha=alpha, mechanisms=mechs, name=f"full_physics_N{Nb}",
    )


def bias_sweep_problems(npoints: int = 64, seed: int = 5, Nk: int = 32, classes=((2, 8), (3, 8), (4, 8), (6, 8)),
                        NE_choices=(1024, 1536, 2048, 2560, 3072, 3584, 4096), bias_mV=(20.0, 70.0),
                        alpha: float = 0.5, Nqz: int = 401, Nphi: int = 64) -> List[SCBAProblem]:
    """A batched bias sweep: `npoints` operating points from bias_mV[0] to
    bias_mV[1] mV per period, each on one of the structure classes (periods x
    states: N_b = 16, 24, 32, 48) and an energy grid of N_E drawn from
    NE_choices, with N_k momenta and LO + acoustic + IFR scattering
    (full_physics_problem).  The kernels of a class are built once and shared
    by its points, since they do not depend on the bias or the energy grid."""
    rng = np.random.default_rng(seed)
    cls = rng.integers(0, len(classes), npoints)
    nes = rng.choice(np.asarray(NE_choices), npoints)
    biases = np.linspace(bias_mV[0], bias_mV[1], npoints)
    kernels = {}
    out = []
    for i in range(npoints):
        periods, states = classes[int(cls[i])]
        key = (periods, states)
        kw = dict(seed=seed + 100 * int(cls[i]), NE=int(nes[i]), Nk=Nk, periods=periods, states=states, Nqz=Nqz,
                  Nphi=Nphi, alpha=alpha, bias_mV=float(biases[i]), mechanisms=("LO", "acoustic", "IFR"))
        pr = full_physics_problem(kernels=kernels.get(key), **kw)
        kernels.setdefault(key, pr.mechanisms)
        out.append(dataclasses.replace(pr, name=f"sweep_{i}_N{pr.Nb}_NE{pr.NE}_{biases[i]:.1f}mV"))
    return out
