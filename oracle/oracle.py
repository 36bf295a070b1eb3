"""Python driver of the CPU FP64 oracle (test infrastructure only).

Binds ``oracle/_build/liborc.so`` (built from ``qcl_oracle.c`` by
``oracle/Makefile``) with ctypes and composes the reference's SCBA inner
loop from its operators, following ``numerics/reference/scba.jl:142-354``
(educational loop) with the production operator choices of
``numerics/optimized/production_solver.jl:435-844`` (sparse shift plans,
FFT Hilbert with roundoff verification, factorised kernel operators, paired
number normalisation, linear mixing).

Only tests, the smoke check and the benchmark's CPU-baseline leg import this
module.  Arrays follow the Julia layout: numpy Fortran order, fields of
shape (N_E, N_k, N_b, N_b).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

REALNESS_LIMIT = 1.0e-10  # _NUMBER_FUNCTIONAL_REALNESS_LIMIT (domain/numerical_invariants.jl:5)
FERMI_SATURATION = 40.0  # _FERMI_EXPONENT_SATURATION (domain/numerical_invariants.jl:10)


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (status {code})")
        self.code = code


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    """The loaded library.  Each wrapper calls lib() before building its
    argument list; that is where the previous call's temporaries are dropped."""
    del _ALIVE[:]
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liborc.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
        _declare(_LIB)
    return _LIB


P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double
Z = ctypes.c_size_t
L = ctypes.c_long


def _declare(l):
    sig = {
        "orc_inverse": (I, [I, P, P, P]),
        "orc_hermitian_eigvals": (None, [I, P, P]),
        "orc_retarded_green": (I, [I, I, I, P, D, P, P, P, P, P, P, P]),
        "orc_keldysh_green": (None, [I, I, I, P, P, P]),
        "orc_greater_green": (None, [I, I, I, P, P, P]),
        "orc_spectral_function": (None, [I, I, I, P, P]),
        "orc_number_functional": (I, [I, I, I, P, P, P, I, D, P]),
        "orc_paired_coefficients": (I, [D, D, D, P, P, P]),
        "orc_normalize_pair": (None, [Z, P, P, D, D]),
        "orc_shift_plan": (I, [I, P, D, P, P, P, P]),
        "orc_apply_shift": (None, [I, Z, P, P, P, P, P, P]),
        "orc_shift_matrix": (None, [I, P, D, P]),
        "orc_contraction_literal": (None, [I, I, I, P, P, P, D, P]),
        "orc_contraction_momentum_independent": (None, [I, I, I, P, P, P, D, D, P]),
        "orc_contraction_dense": (None, [I, I, I, P, P, P, D, D, P]),
        "orc_contraction_ifr": (None, [I, I, I, I, P, P, P, P, P, D, D, P]),
        "orc_contraction_low_rank": (None, [I, I, I, I, P, P, P, P, D, D, P]),
        "orc_direct_hilbert": (None, [I, Z, P, P, P, P, I]),
        "orc_fft_hilbert": (I, [I, Z, P, P, P, P, I]),
        "orc_fft_hilbert_roundoff": (I, [I, Z, P, P, P, P, P]),
        "orc_retarded_self_energy": (I, [I, Z, P, P, P, P, P, P, I, P]),
        "orc_embedding_component": (None, [I, I, I, P, P, P, P, P, P, P]),
        "orc_current": (D, [I, I, I, P, P, P, I, P, P, P, P]),
        "orc_populations": (None, [I, I, I, P, P, I, D, P, P]),
        "orc_mix": (None, [Z, P, P, D]),
        "orc_relative_change": (D, [Z, P, P]),
        "orc_residual_suite": (None, [I, I, I, P, P, P, P, P, P, P, P, P, P]),
        "orc_residual_witness": (None, [I, I, I, P, P, P, P, P, P, P]),
        "orc_dyson_keldysh": (I, [I, I, I, P, P, P, P, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(l, name)
        fn.restype = res
        fn.argtypes = args


_ALIVE = []


def _p(a):
    """Pointer to a numpy array's data.  The array is kept referenced until the
    next call that starts (`_begin`), so temporaries made by layout
    conversions inside an argument list outlive the C call they feed."""
    if a is None:
        return None
    _ALIVE.append(a)
    return ctypes.c_void_p(a.ctypes.data)


def _field(x, shape=None):
    a = np.asarray(x, dtype=np.complex128)
    a = np.asfortranarray(a)
    if shape is not None and a.shape != tuple(shape):
        raise ValueError(f"shape {a.shape} != {shape}")
    return a


def _real(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


# --------------------------------------------------------------------------
# Operators
# --------------------------------------------------------------------------

def inverse(A):
    A = _field(A).copy(order="F")
    n = A.shape[0]
    work = np.zeros((n, n), dtype=np.complex128, order="F")
    piv = np.zeros(n, dtype=np.int32)
    st = lib().orc_inverse(n, _p(A), _p(work), _p(piv))
    if st:
        raise OracleError(st, f"singular pivot {st}")
    return A


def eigvalsh(H):
    H = _field(H).copy(order="F")
    n = H.shape[0]
    vals = np.zeros(n)
    lib().orc_hermitian_eigvals(n, _p(H), _p(vals))
    return vals


def retarded_green(eps, h, sigR=None, eta=0.0):
    """retarded_green (numerics/reference/greens.jl:18-42).  Returns
    (GR, kappa2, scale, kappa1)."""
    eps = _real(eps)
    h = _field(h)
    Nk, Nb = h.shape[0], h.shape[1]
    NE = eps.shape[0]
    sigR = None if sigR is None else _field(sigR, (NE, Nk, Nb, Nb))
    GR = np.zeros((NE, Nk, Nb, Nb), dtype=np.complex128, order="F")
    k1 = np.zeros((NE, Nk), order="F")
    k2 = np.zeros((NE, Nk), order="F")
    sc = np.zeros((NE, Nk), order="F")
    bad = ctypes.c_long(-1)
    st = lib().orc_retarded_green(NE, Nk, Nb, _p(eps), eta, _p(h), _p(sigR), _p(GR), _p(k1), _p(k2),
                                  _p(sc), ctypes.byref(bad))
    if st:
        raise OracleError(st, f"singular Dyson block {bad.value}")
    return GR, k2, sc, k1


def keldysh_green(GR, sig):
    GR = _field(GR)
    sig = _field(sig, GR.shape)
    out = np.zeros_like(GR, order="F")
    NE, Nk, Nb, _ = GR.shape
    lib().orc_keldysh_green(NE, Nk, Nb, _p(GR), _p(sig), _p(out))
    return out


def greater_green(GR, GL):
    GR, GL = _field(GR), _field(GL)
    out = np.zeros_like(GR, order="F")
    NE, Nk, Nb, _ = GR.shape
    lib().orc_greater_green(NE, Nk, Nb, _p(GR), _p(GL), _p(out))
    return out


def spectral_function(GR):
    GR = _field(GR)
    out = np.zeros_like(GR, order="F")
    NE, Nk, Nb, _ = GR.shape
    lib().orc_spectral_function(NE, Nk, Nb, _p(GR), _p(out))
    return out


def number_functional(GL, wE, wk, gs):
    GL = _field(GL)
    NE, Nk, Nb, _ = GL.shape
    out = ctypes.c_double()
    st = lib().orc_number_functional(NE, Nk, Nb, _p(GL), _p(_real(wE)), _p(_real(wk)), gs, REALNESS_LIMIT,
                                     ctypes.byref(out))
    if st:
        raise OracleError(st, "number functional is not real")
    return out.value


def paired_coefficients(number, holes, target):
    a, c, lam = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    st = lib().orc_paired_coefficients(number, holes, target, ctypes.byref(a), ctypes.byref(c),
                                       ctypes.byref(lam))
    if st:
        raise OracleError(st, "paired number coefficients rejected")
    return a.value, c.value, lam.value


def normalize_pair(GL, GG, a, c):
    lib().orc_normalize_pair(GL.size, _p(GL), _p(GG), a, c)


class ShiftPlan:
    """EnergyShiftPlan (numerics/optimized/production_contracts.jl:13-19),
    0-based."""

    def __init__(self, eps, delta):
        eps = _real(eps)
        NE = eps.shape[0]
        self.NE = NE
        self.delta = float(delta)
        self.left = np.zeros(NE, dtype=np.int32)
        self.right = np.zeros(NE, dtype=np.int32)
        self.theta = np.zeros(NE)
        self.valid = np.zeros(NE, dtype=np.uint8)
        st = lib().orc_shift_plan(NE, _p(eps), float(delta), _p(self.left), _p(self.right), _p(self.theta),
                                  _p(self.valid))
        if st:
            raise OracleError(st, "invalid shift plan")

    def apply(self, X):
        X = _field(X)
        Y = np.zeros_like(X, order="F")
        lib().orc_apply_shift(self.NE, X.size // self.NE, _p(self.left), _p(self.right), _p(self.theta),
                              _p(self.valid), _p(X), _p(Y))
        return Y


def shift_matrix(eps, delta):
    eps = _real(eps)
    W = np.zeros((eps.shape[0], eps.shape[0]), order="F")
    lib().orc_shift_matrix(eps.shape[0], _p(eps), float(delta), _p(W))
    return W


def contraction_literal(K, G, wk, q=1.0):
    G = _field(G)
    K = _field(K)
    NE, Nk, Nb, _ = G.shape
    S = np.zeros_like(G, order="F")
    lib().orc_contraction_literal(NE, Nk, Nb, _p(K), _p(G), _p(_real(wk)), float(q), _p(S))
    return S


def contraction(mech, G, wk, alpha=1.0, beta=0.0, S=None):
    """production_static_contraction for one factorised operator
    (production_operators.jl:402-658, the LowRank method at :597-658):
    S = beta S + alpha q K[wk G]."""
    G = _field(G)
    NE, Nk, Nb, _ = G.shape
    if S is None:
        S = np.zeros_like(G, order="F")
    wk = _real(wk)
    aq = float(alpha * mech.q)
    if mech.kind == "momentum_independent":
        lib().orc_contraction_momentum_independent(NE, Nk, Nb, _p(_field(mech.block)), _p(G), _p(wk), aq,
                                                   float(beta), _p(S))
    elif mech.kind == "dense":
        lib().orc_contraction_dense(NE, Nk, Nb, _p(_field(mech.matrix)), _p(G), _p(wk), aq, float(beta), _p(S))
    elif mech.kind == "ifr":
        J = mech.left.shape[1]
        lib().orc_contraction_ifr(NE, Nk, Nb, J, _p(_field(mech.left)), _p(_field(mech.right)),
                                  _p(_field(mech.radial)), _p(G), _p(wk), aq, float(beta), _p(S))
    elif mech.kind == "separable_sum":
        # The reference has no Kronecker-sum operator: its contraction of the
        # same kernel is the dense BLAS map (production_operators.jl:402-465)
        # of the permuted six-index tensor (_production_kernel,
        # production_cache.jl:400-405), which is what is evaluated here.
        K = mech.literal_kernel(Nk, Nb)
        M = np.transpose(K, (0, 2, 5, 1, 3, 4)).reshape((Nk * Nb * Nb, Nk * Nb * Nb), order="F")
        lib().orc_contraction_dense(NE, Nk, Nb, _p(_field(M)), _p(G), _p(wk), aq, float(beta), _p(S))
    elif mech.kind == "low_rank":
        r = mech.left.shape[1]
        lib().orc_contraction_low_rank(NE, Nk, Nb, r, _p(_field(mech.left)), _p(_field(mech.right)), _p(G),
                                       _p(wk), aq, float(beta), _p(S))
    else:
        raise ValueError(mech.kind)
    return S


def direct_hilbert(Gam, eps, wE, reverse=False):
    Gam = _field(Gam)
    NE = Gam.shape[0]
    out = np.zeros_like(Gam, order="F")
    lib().orc_direct_hilbert(NE, Gam.size // NE, _p(_real(eps)), _p(_real(wE)), _p(Gam), _p(out), int(reverse))
    return out


def fft_hilbert(Gam, eps, wE, L=0, return_roundoff=False):
    Gam = _field(Gam)
    NE = Gam.shape[0]
    out = np.zeros_like(Gam, order="F")
    if return_roundoff:
        r = ctypes.c_double()
        st = lib().orc_fft_hilbert_roundoff(NE, Gam.size // NE, _p(_real(eps)), _p(_real(wE)), _p(Gam), _p(out),
                                            ctypes.byref(r))
        if st:
            raise OracleError(st, "fft hilbert")
        return out, r.value
    st = lib().orc_fft_hilbert(NE, Gam.size // NE, _p(_real(eps)), _p(_real(wE)), _p(Gam), _p(out), int(L))
    if st:
        raise OracleError(st, "fft hilbert")
    return out


def retarded_self_energy(SL, SG, eps, wE, method="fft", return_roundoff=False):
    SL, SG = _field(SL), _field(SG)
    NE = SL.shape[0]
    SR = np.zeros_like(SL, order="F")
    Gam = np.zeros_like(SL, order="F")
    r = ctypes.c_double()
    st = lib().orc_retarded_self_energy(NE, SL.size // NE, _p(_real(eps)), _p(_real(wE)), _p(SL), _p(SG), _p(SR),
                                        _p(Gam), 0 if method == "fft" else 1,
                                        ctypes.byref(r) if return_roundoff else None)
    if st:
        raise OracleError(st, "retarded self-energy")
    return (SR, Gam, r.value) if return_roundoff else (SR, Gam)


def embedding_component(T, G, plan: ShiftPlan):
    G = _field(G)
    NE, Nk, Nb, _ = G.shape
    S = np.zeros_like(G, order="F")
    lib().orc_embedding_component(NE, Nk, Nb, _p(_field(T)), _p(G), _p(plan.left), _p(plan.right),
                                  _p(plan.theta), _p(plan.valid), _p(S))
    return S


def current(problem, SG, SL, GL, GG):
    NE, Nk, Nb = problem.NE, problem.Nk, problem.Nb
    return lib().orc_current(NE, Nk, Nb, _p(_real(problem.eps)), _p(_real(problem.wE)), _p(_real(problem.wk)),
                             problem.gs, _p(_field(SG)), _p(_field(SL)), _p(_field(GL)), _p(_field(GG)))


def populations(problem, GL):
    pop = np.zeros(problem.Nb)
    lib().orc_populations(problem.NE, problem.Nk, problem.Nb, _p(_real(problem.wE)), _p(_real(problem.wk)),
                          problem.gs, problem.target, _p(_field(GL)), _p(pop))
    return pop


def relative_change(old, new):
    return lib().orc_relative_change(old.size, _p(_field(old)), _p(_field(new)))


def residual_suite(eps, h, GR, GL, GG, total, candidate_SL):
    NE, Nk, Nb, _ = GR.shape
    out = np.zeros(5)
    SR, SL, SG = total
    lib().orc_residual_suite(NE, Nk, Nb, _p(_real(eps)), _p(_field(h)), _p(_field(GR)), _p(_field(GL)),
                             _p(_field(GG)), _p(_field(SR)), _p(_field(SL)), _p(_field(SG)),
                             _p(_field(candidate_SL)), _p(out))
    return dict(rD=out[0], rA=out[1], rK=out[2], rPSD=out[3], rcaus=out[4])


WITNESS_KINDS = ("spectral", "occupied", "unoccupied", "broadening", "raw_occupied", "raw_unoccupied")
WITNESS_FIELDS = ("minimum_eigenvalue", "block_norm", "floor", "ratio", "absolute_defect", "relative_defect",
                  "backward_error", "hermiticity_defect", "construction_scale")


def residual_witness(GR, GL, GG, total):
    """The positivity witness of production_residual_suite
    (residuals.jl:662-779, positivity_diagnostics.jl:41-91): kind (or
    "none"), 0-based e, m and the nine witness numbers."""
    NE, Nk, Nb, _ = GR.shape
    ikem = np.zeros(3, dtype=np.int32)
    w = np.zeros(9)
    _, SL, SG = total
    lib().orc_residual_witness(NE, Nk, Nb, _p(_field(GR)), _p(_field(GL)), _p(_field(GG)), _p(_field(SL)),
                               _p(_field(SG)), ikem.ctypes.data_as(ctypes.c_void_p), _p(w))
    out = dict(zip(WITNESS_FIELDS, w.tolist()))
    out.update(matrix_kind="none" if ikem[0] < 0 else WITNESS_KINDS[ikem[0]], energy_index=int(ikem[1]),
               momentum_index=int(ikem[2]))
    return out


def dyson_keldysh(eps, h, SR, SL, SG=None):
    eps = _real(eps)
    SR = _field(SR)
    NE, Nk, Nb, _ = SR.shape
    GR = np.zeros_like(SR, order="F")
    GL = np.zeros_like(SR, order="F")
    GG = np.zeros_like(SR, order="F") if SG is not None else None
    sc = np.zeros((NE, Nk), order="F")
    st = lib().orc_dyson_keldysh(NE, Nk, Nb, _p(eps), _p(_field(h)), _p(SR), _p(_field(SL)),
                                 _p(None if SG is None else _field(SG)), _p(GR), _p(GL), _p(GG), _p(sc))
    if st:
        raise OracleError(st, "singular Dyson block")
    return GR, GL, GG, sc


# --------------------------------------------------------------------------
# SCBA composition
# --------------------------------------------------------------------------

def fermi(energy, mu, kBT):
    x = (energy - mu) / kBT
    with np.errstate(over="ignore"):
        f = 1.0 / (np.exp(x) + 1.0)
    f = np.where(x > FERMI_SATURATION, 0.0, f)
    f = np.where(x < -FERMI_SATURATION, 1.0, f)
    return f


def bisection(fn, lo, hi):
    """Bisection to adjacent floating-point numbers (the role of Roots.jl
    `find_zero(f, (lo, hi), Bisection())`, seed.jl:182)."""
    flo = fn(lo)
    if flo == 0:
        return lo
    for _ in range(2000):
        mid = 0.5 * (lo + hi)
        if mid == lo or mid == hi:
            break
        fm = fn(mid)
        if fm == 0:
            return mid
        if (fm < 0) == (flo < 0):
            lo, flo = mid, fm
        else:
            hi = mid
    return lo if abs(fn(lo)) <= abs(fn(hi)) else hi


def seed_green(problem):
    """_seed_green_production (numerics/optimized/seed.jl:151-197)."""
    GR, k2, scale, _ = retarded_green(problem.eps, problem.h, None, eta=problem.eta_seed)
    NE, Nk, Nb = problem.NE, problem.Nk, problem.Nb
    # q_e = g_s/(2 pi) wE_e sum_m wk_m tr A_em  (seed.jl:28-66)
    trA = np.zeros((NE, Nk))
    for a in range(Nb):
        z = GR[:, :, a, a]
        trA += np.real(1j * (z - np.conj(z)))
    q = problem.gs / (2 * math.pi) * problem.wE * (trA @ problem.wk)

    def number_at(mu):
        return float(np.sum(q * fermi(problem.eps, mu, problem.kBT))) - problem.target

    lo = problem.eps[0] - 50 * problem.kBT
    hi = problem.eps[-1] + 50 * problem.kBT
    if number_at(lo) * number_at(hi) > 0:
        raise OracleError(4, "seed chemical-potential root is not bracketed")
    mu = bisection(number_at, lo, hi)
    f = fermi(problem.eps, mu, problem.kBT)
    diff = GR - np.conj(np.transpose(GR, (0, 1, 3, 2)))
    GL = np.asfortranarray(-f[:, None, None, None] * diff)
    GG = greater_green(GR, GL)
    return dict(GR=GR, GL=GL, GG=GG, scale=scale), mu


def apply_scattering_model(problem, family):
    """_apply_scattering_model! (production_operators.jl:1240-1256):
    _diagonalize_blocks! (:1208-1217) then _average_transverse_momentum!
    (:1219-1238), on every component of one family."""
    out = []
    for X in family:
        X = np.array(X, dtype=np.complex128, order="F")
        NE, Nk, Nb, _ = X.shape
        if getattr(problem, "self_energy_structure", "full") == "diagonal":
            for b in range(Nb):
                for a in range(Nb):
                    if a != b:
                        X[:, :, a, b] = 0
        if getattr(problem, "transverse_momentum", "resolved") == "averaged":
            w = np.asarray(problem.wk, dtype=np.float64)
            norm = float(np.sum(w))
            if not norm > 0:
                raise OracleError(4, "radial weights must have positive sum")
            for b in range(Nb):
                for a in range(Nb):
                    v = np.zeros(NE, dtype=np.complex128)
                    for m in range(Nk):
                        v = v + w[m] * X[:, m, a, b]
                    v = v / norm
                    X[:, :, a, b] = v[:, None]
        out.append(X)
    return tuple(out)


def scattering_candidate(problem, green, plans, verify=True):
    """_scattering_candidate_production (production_operators.jl:1258-1335)
    with the thermal-LO branch of _production_lo_contraction (:1045-1163),
    the retarded closure of _retarded_self_energy_selected (:1165-1206) and
    the model switches (:1240-1256)."""
    drop = getattr(problem, "retarded_real_part", "kramers_kronig") == "drop"
    direct = getattr(problem, "elastic_retarded", "hilbert") == "direct_green"
    out = {}
    roundoff = 0.0
    wk = problem.wk
    for mech in problem.mechanisms:
        if mech.name == "LO":
            N = problem.N_LO
            SL = contraction(mech, plans["+LO"].apply(green["GL"]), wk, alpha=N + 1)
            contraction(mech, plans["-LO"].apply(green["GL"]), wk, alpha=N, beta=1.0, S=SL)
            SG = contraction(mech, plans["-LO"].apply(green["GG"]), wk, alpha=N + 1)
            contraction(mech, plans["+LO"].apply(green["GG"]), wk, alpha=N, beta=1.0, S=SG)
        else:
            SL = contraction(mech, green["GL"], wk)
            SG = contraction(mech, green["GG"], wk)
        if direct and not drop and mech.name != "LO":
            SR = contraction(mech, green["GR"], wk)
        elif drop:
            SR = np.asfortranarray(-0.5j * (1j * (SG - SL)))
        elif verify:
            SR, _, r = retarded_self_energy(SL, SG, problem.eps, problem.wE, return_roundoff=True)
            roundoff = max(roundoff, r)
        else:
            SR, _ = retarded_self_energy(SL, SG, problem.eps, problem.wE)
        out[mech.name] = apply_scattering_model(problem, (SR, SL, SG))
    return out, roundoff


def embedding_candidate(problem, green, plans):
    """_embedding_self_energy_production (production_operators.jl:924-941)."""
    plus = tuple(embedding_component(problem.Tplus, green[k], plans["+Ep"]) for k in ("GR", "GL", "GG"))
    minus = tuple(embedding_component(problem.Tminus, green[k], plans["-Ep"]) for k in ("GR", "GL", "GG"))
    return plus, minus


def total_family(problem, scattering, plus, minus):
    """_total_family_production (production_operators.jl:1447-1473)."""
    tot = []
    for c in range(3):
        x = plus[c] + minus[c]
        for mech in problem.mechanisms:
            x = x + scattering[mech.name][c]
        tot.append(np.asfortranarray(x))
    return tuple(tot)


def current_green(problem, total, branch=0):
    """_current_green_production (numerics/optimized/production_state.jl).
    `branch` forces the form of the paired normalisation (1: scale G^<,
    2: move G^> weight into G^<; 0: the reference's choice by number versus
    target), as qcl_scba_set_normalization_branch does on the device."""
    GR, GL, GG, scale = dyson_keldysh(problem.eps, problem.h, total[0], total[1], total[2])
    number = number_functional(GL, problem.wE, problem.wk, problem.gs)
    lam = number / problem.target
    if not (math.isfinite(lam) and lam > 0):
        raise OracleError(2, "kinetic eigenvalue must be positive")
    if getattr(problem, "occupation_normalization", "paired_convex") == "scalar_lesser":
        # production_state.jl:54-61: G< / lambda, G> = G^R - G^A + G<
        GL = np.asfortranarray(GL / lam)
        GG = np.asfortranarray((GR - np.conj(np.transpose(GR, (0, 1, 3, 2)))) + GL)
        holes = -number_functional(GG, problem.wE, problem.wk, problem.gs)
        return dict(GR=GR, GL=GL, GG=GG, scale=scale, number=number, holes=holes, a=1.0, c=0.0,
                    normalized=number_functional(GL, problem.wE, problem.wk, problem.gs)), lam
    holes = -number_functional(GG, problem.wE, problem.wk, problem.gs)
    a, c, lam = paired_coefficients(number, holes, problem.target)
    if branch == 1:
        a, c = problem.target / number, 0.0
    elif branch == 2:
        a, c = 1.0, (problem.target - number) / holes
    normalize_pair(GL, GG, a, c)
    return dict(GR=GR, GL=GL, GG=GG, scale=scale, number=number, holes=holes, a=a, c=c,
                normalized=number_functional(GL, problem.wE, problem.wk, problem.gs)), lam


def make_plans(problem):
    return {
        "+Ep": ShiftPlan(problem.eps, +problem.Ep),
        "-Ep": ShiftPlan(problem.eps, -problem.Ep),
        "+LO": ShiftPlan(problem.eps, +problem.hw_LO),
        "-LO": ShiftPlan(problem.eps, -problem.hw_LO),
    }


# --------------------------------------------------------------------------
# Kernel builders (numerics/reference/kernels.jl, numerics/optimized/kernels.jl)
# --------------------------------------------------------------------------
def lo_kernel_literal(F, qz, wqz, kappa, Nphi, qscreen, prefactor, L0=1.0):
    """lo_phonon_kernel (kernels.jl:321-356) with _angular_average_kernel
    (:5-19): K[m,m',a,c,d,b] = prefactor/N_phi sum_phi sum_h f_h(q) F[h,a,c]
    conj(F[h,b,d]), f_h = wqz_h L0 / (2 pi (q^2 + qz_h^2 + qs^2))."""
    Nq, Nb, _ = F.shape
    Nk = len(kappa)
    K = np.zeros((Nk, Nk, Nb, Nb, Nb, Nb), dtype=np.complex128)
    outer = [np.einsum("ac,bd->acdb", F[h], np.conj(F[h])) for h in range(Nq)]
    for m in range(Nk):
        for mp in range(Nk):
            acc = np.zeros((Nb, Nb, Nb, Nb), dtype=np.complex128)
            for r in range(Nphi):
                phi = 2 * math.pi * r / Nphi
                q = math.sqrt(max(kappa[m] ** 2 + kappa[mp] ** 2 - 2 * kappa[m] * kappa[mp] * math.cos(phi), 0.0))
                Ksi = np.zeros_like(acc)
                for h in range(Nq):
                    Ksi += wqz[h] * L0 / (2 * math.pi * (q * q + qz[h] ** 2 + qscreen ** 2)) * outer[h]
                acc += prefactor * Ksi
            K[m, mp] = acc / Nphi
    return K


def lookup_block(nodes, values, q):
    """_lookup_block (numerics/optimized/kernels.jl:205-217)."""
    qlo, qhi = nodes[0], nodes[-1]
    tol = 64 * _EPS * max(abs(qlo), abs(qhi), 1.0)
    if not (qlo - tol <= q <= qhi + tol):
        raise ValueError("lookup query lies outside the tabulated interval")
    qc = min(max(q, qlo), qhi)
    if qc == qhi:
        return values[-1]
    j = min(max(int(np.searchsorted(nodes, qc, side="right")) - 1, 0), len(nodes) - 2)
    th = (qc - nodes[j]) / (nodes[j + 1] - nodes[j])
    return (1 - th) * values[j] + th * values[j + 1]


def assemble_lookup_kernel(nodes, values, kappa, Nphi):
    """_assemble_lookup_kernel (numerics/optimized/kernels.jl:303-320):
    values[t] are (a,c,d,b) blocks."""
    Nk = len(kappa)
    Nb = values[0].shape[0]
    K = np.zeros((Nk, Nk, Nb, Nb, Nb, Nb), dtype=np.complex128)
    for m in range(Nk):
        for mp in range(Nk):
            acc = np.zeros((Nb,) * 4, dtype=np.complex128)
            for r in range(Nphi):
                phi = 2 * math.pi * r / Nphi
                q = math.sqrt(max(kappa[m] ** 2 + kappa[mp] ** 2 - 2 * kappa[m] * kappa[mp] * math.cos(phi), 0.0))
                acc = acc + lookup_block(nodes, values, q)
            K[m, mp] = acc / Nphi
    return K


def impurity_block_literal(q, chi, x, wx, donor_weights, q_s, pre):
    """kernel_at_q of impurity_kernel (kernels.jl:117-141) as an (a,c,d,b)
    block: sum over donor cells of w_D V[a,c] conj(V[b,d]),
    V[a,c] = pre/(q + q_s) sum_g wx conj(chi_ga) exp(-q |x_g - x_D|) chi_gc."""
    Nb = chi.shape[1]
    Ksi = np.zeros((Nb,) * 4, dtype=np.complex128)
    for D in range(len(x)):
        if donor_weights[D] == 0:
            continue
        V = np.zeros((Nb, Nb), dtype=np.complex128)
        for a in range(Nb):
            for c in range(Nb):
                V[a, c] = pre / (q + q_s) * np.sum(wx * np.conj(chi[:, a]) * np.exp(-q * np.abs(x - x[D])) * chi[:, c])
        Ksi += donor_weights[D] * np.einsum("ac,bd->acdb", V, np.conj(V))
    return Ksi


def normalize_kernel(K):
    """build_kernels scaling (kernels.jl:393-403): (K / q, q), q = max |K|."""
    q = float(np.max(np.abs(K)))
    return K / q, q


# --------------------------------------------------------------------------
# Outer Hartree-Poisson loop (numerics/optimized/production_solver.jl:993-1151)
# --------------------------------------------------------------------------
def density_matrix(GL, wE, wk):
    """integrated[a,b] = sum_m sum_e wE_e wk_m G<[e,m,a,b] in the reference's
    loop order (_electron_density_bar, physics/observables.jl:1-22)."""
    NE, Nk, Nb, _ = GL.shape
    out = np.zeros((Nb, Nb), dtype=np.complex128)
    W = np.outer(np.asarray(wE), np.asarray(wk))
    for b in range(Nb):
        for a in range(Nb):
            out[a, b] = np.sum(W * GL[:, :, a, b])
    return out


def poisson_solve(st, nbar):
    """solve_periodic_poisson (numerics/reference/poisson.jl:41-65) with
    build_poisson_matrix (:12-28): returns (U, zeta, r_P, neutrality)."""
    N = len(st.x)
    dx = st.wx[0]
    e = np.asarray(st.eps_r, dtype=np.float64)
    L = np.zeros((N, N))
    for g in range(N):
        gp, gm = (g + 1) % N, (g - 1) % N
        fg = 2 * e[g] * e[gp] / (e[g] + e[gp])
        fm = 2 * e[gm] * e[g] / (e[gm] + e[g])
        L[g, g] = (fm + fg) / dx ** 2
        L[g, gm] = -fm / dx ** 2
        L[g, gp] = -fg / dx ** 2
    ND2D = float(np.dot(st.wx, st.ND))
    neutrality = abs(float(np.dot(st.wx, st.ND - nbar))) / ND2D
    b = -st.lambda_P * (st.ND - nbar)
    sP = float(np.max(np.sum(np.abs(L), axis=1)))
    v = np.full(N, 1 / math.sqrt(N))
    B = np.block([[L / sP, v[:, None]], [v[None, :], np.zeros((1, 1))]])
    ans = np.linalg.solve(B, np.r_[b / sP, 0.0])
    U = ans[:N]
    rP = float(np.linalg.norm(L @ U - b) / (np.linalg.norm(b) + st.lambda_P * 1e-14))
    return U, float(ans[N]), rP, neutrality


def outer_loop(problem, st, max_poisson, inner_iterations, alpha_P=0.3):
    """The outer loop of solve_production (production_solver.jl:993-1151)
    with a fixed inner iteration count, every inner solve warm-started from
    the previous terminal state."""
    import dataclasses as _dc

    Nz = len(st.x)
    U = np.zeros(Nz)
    rows = []
    state = None
    nprev = Jprev = pprev = None
    ND2D, Lp = float(np.dot(st.wx, st.ND)), float(np.sum(st.wx))
    for mu in range(1, max_poisson + 1):
        Nb = st.H0.shape[0]
        static = st.H0 - st.F * (st.Z - st.z0 * np.eye(Nb)) + st.Phi.conj().T @ np.diag(U) @ st.Phi
        h = np.zeros((len(st.kappa), Nb, Nb), dtype=np.complex128, order="F")
        for m, k in enumerate(st.kappa):
            h[m] = static + st.Cbar * k * k * st.Minv
        pr = _dc.replace(problem, h=h)
        hist, state = scba(pr, inner_iterations, state=state, keep_state=True, terminal=True)
        green = state["green"]
        rho = density_matrix(green["GL"], pr.wE, pr.wk)
        nbar = pr.gs / (2 * math.pi) * np.real(-1j * np.einsum("ga,ab,gb->g", st.chi, rho, np.conj(st.chi)))
        cand, zeta, rP, rneutral = poisson_solve(st, nbar)
        rU = float(np.max(np.abs(cand - U)))
        rn = math.inf if nprev is None else float(math.sqrt(np.sum(st.wx * (nbar - nprev) ** 2)) / (ND2D / math.sqrt(Lp)))
        jp = current(pr, state["plus"][2], state["plus"][1], green["GL"], green["GG"])
        jm = current(pr, state["minus"][2], state["minus"][1], green["GL"], green["GG"])
        rJ = abs(jp + jm) / max(abs(jp), abs(jm), 1e-12)
        J = jp * pr.J0
        pops = hist[-1]["populations"]
        rJc = math.inf if Jprev is None else abs(J - Jprev) / max(abs(J), abs(Jprev), 1e-12)
        rpop = math.inf if pprev is None else float(np.linalg.norm(pops - pprev) / (np.linalg.norm(pops) + 1e-14))
        rows.append(dict(mu=mu, r_P=rP, r_U=rU, r_n=rn, r_neutral=rneutral, r_J=rJ, r_Jchange=rJc,
                         r_population=rpop, zeta=zeta, J=J, populations=pops, n=nbar, inner=hist))
        U = (1 - alpha_P) * U + alpha_P * cand
        nprev, Jprev, pprev = nbar, J, pops
    return rows


# --------------------------------------------------------------------------
# Anderson mixing (numerics/optimized/production_mixing.jl:1-317)
# --------------------------------------------------------------------------
_EPS = float(np.finfo(np.float64).eps)
_TINY = float(np.finfo(np.float64).tiny)


def _anderson_inner(left, right):
    """_anderson_inner (production_mixing.jl:129-138): sum of Re <a, b> over
    families and components, column-major order."""
    v = 0.0
    for fa, fb in zip(left, right):
        for a, b in zip(fa, fb):
            v += float(np.real(np.vdot(np.ravel(a, order="F"), np.ravel(b, order="F"))))
    return v


def anderson_coefficients(gram, regularization):
    """_anderson_coefficients (production_mixing.jl:155-180).  Raises
    ValueError where the reference throws ArgumentError."""
    count = gram.shape[0]
    if count == 1:
        return np.ones(1)
    g = np.array(gram, dtype=np.float64)
    scale = max(float(np.max(np.abs(np.diag(g)))), _EPS)
    g[np.diag_indices(count)] += regularization * scale
    values, vectors = np.linalg.eigh(g / scale)
    cutoff = max(regularization, math.sqrt(_EPS))
    projected = vectors.T @ np.ones(count)
    weights = np.array([projected[i] / values[i] if values[i] > cutoff else 0.0 for i in range(count)])
    coef = vectors @ weights
    denom = float(np.sum(coef))
    if not (math.isfinite(denom) and abs(denom) > _EPS):
        raise ValueError("Anderson history is rank deficient")
    coef = coef / denom
    if not np.all(np.isfinite(coef)):
        raise ValueError("Anderson coefficient solve produced non-finite values")
    return coef


def anderson_block_failure(R, L, G):
    """_anderson_block_failure! (production_mixing.jl:48-96): 0 or the code."""
    n = R.shape[0]
    if not np.all(np.isfinite(R)):
        return 1
    Hm = (R - R.conj().T) / 2j
    nR = np.linalg.norm(R, 2)
    if not np.linalg.eigvalsh(0.5 * (Hm + Hm.conj().T)).max() <= 64 * _EPS * max(nR, _TINY):
        return 2
    if not (np.all(np.isfinite(L)) and np.all(np.isfinite(G))):
        return 1
    for X, f in ((L, -1j), (G, 1j)):
        F = f * X
        budget = 64 * n * _EPS * max(np.linalg.norm(F, 2), 1.0)
        if not np.linalg.norm(F - F.conj().T) / 2 <= budget:
            return 3
        if not np.linalg.eigvalsh(0.5 * (F + F.conj().T)).min() >= -budget:
            return 4
    diff = R - R.conj().T - (G - L)
    budget = 64 * n * _EPS * max(nR, np.linalg.norm(L, 2), np.linalg.norm(G, 2), 1.0)
    if not np.linalg.norm(diff) <= budget:
        return 5
    return 0


def anderson_guard(families):
    """_anderson_guard (production_mixing.jl:98-118): (passed, first failing
    1-based index over (family, e, m) with m fastest, code)."""
    for fi, (R, L, G) in enumerate(families):
        NE, Nk = R.shape[0], R.shape[1]
        for e in range(NE):
            for m in range(Nk):
                code = anderson_block_failure(R[e, m], L[e, m], G[e, m])
                if code:
                    return False, fi * NE * Nk + e * Nk + m + 1, code
    return True, 0, 0


class AndersonMixer:
    """The _AndersonWorkspace history with _anderson_append! and
    _anderson_mix! (production_mixing.jl:184-317)."""

    def __init__(self, depth=5, damping=1.0, regularization=1e-12):
        self.depth, self.damping, self.regularization = depth, damping, regularization
        self.states, self.residuals = [], []
        self.gram = np.zeros((0, 0))
        self.info = {}

    def clear(self):
        self.states, self.residuals = [], []
        self.gram = np.zeros((0, 0))

    def append(self, state, candidate):
        prior = None if not self.residuals else float(self.gram[-1, -1])
        if len(self.states) >= self.depth:
            self.states.pop(0)
            self.residuals.pop(0)
            self.gram = self.gram[1:, 1:]
        saved = [tuple(np.array(c, order="F") for c in f) for f in state]
        residual = [tuple(np.asfortranarray(cand[c] - st[c]) for c in range(3)) for st, cand in zip(state, candidate)]
        rn = _anderson_inner(residual, residual)
        reset = prior is not None and rn > (1 + 64 * _EPS) * max(prior, _TINY)
        if reset:
            self.clear()
        count = len(self.states) + 1
        gram = np.zeros((count, count))
        if count > 1:
            gram[:-1, :-1] = self.gram
        for i in range(count - 1):
            gram[i, -1] = gram[-1, i] = _anderson_inner(self.residuals[i], residual)
        gram[-1, -1] = rn
        self.gram = gram
        self.states.append(saved)
        self.residuals.append(residual)
        return reset

    def mix(self, state, candidate, alpha):
        reset = self.append(state, candidate)
        reason = "residual_increase" if reset else "none"
        try:
            coef = anderson_coefficients(self.gram, self.regularization)
        except ValueError:
            reason = "coefficient_solve"
            coef = np.r_[np.zeros(len(self.residuals) - 1), 1.0]
        if np.sum(np.abs(coef)) > 10 or not np.all(np.isfinite(coef)):
            reason = "coefficient_bound"
            coef = np.r_[np.zeros(len(self.residuals) - 1), 1.0]
        d = alpha * self.damping
        out = []
        for fi in range(len(state)):
            comps = []
            for c in range(3):
                v = np.zeros_like(self.states[0][fi][c])
                for h in range(len(coef)):
                    v = v + coef[h] * (self.states[h][fi][c] + d * self.residuals[h][fi][c])
                comps.append(np.asfortranarray(v))
            out.append(tuple(comps))
        depth = len(self.states)
        passed, first, code = anderson_guard(out)
        accepted = passed and int(np.count_nonzero(coef)) > 1
        if not passed:
            x, r = self.states[-1], self.residuals[-1]
            out = [tuple(np.asfortranarray(x[fi][c] + d * r[fi][c]) for c in range(3)) for fi in range(len(state))]
            self.clear()
            reason = "causality_guard"
            if not anderson_guard(out)[0]:
                raise OracleError(2, "convex Anderson fallback is not admissible; inspect raw self-energies")
        self.info = dict(history_depth=depth, reset_reason=reason, coefficients_l1=float(np.sum(np.abs(coef))),
                         acceleration_accepted=accepted, guard_first_failure=first, guard_failure_code=code,
                         fallback=not passed)
        return out


def scba(problem, iterations, verify=True, state=None, keep_state=False, terminal=False):
    """Run `iterations` SCBA steps (solve_scba, scba.jl:142-354, with the
    production operators).  Returns (history, state).  With `terminal` the
    last iteration is the solver's terminal row: its families stay unmixed
    (the state a warm-started solve continues from)."""
    plans = make_plans(problem)
    if state is None:
        green, mu = seed_green(problem)
        scattering, _ = scattering_candidate(problem, green, plans, verify=False)
        plus, minus = embedding_candidate(problem, green, plans)
    else:
        scattering, plus, minus = state["scattering"], state["plus"], state["minus"]
    history = []
    Jprev = None
    pprev = None
    mixer = None
    if getattr(problem, "mixing", "linear") == "anderson":
        mixer = AndersonMixer(problem.anderson_history_depth, problem.anderson_damping,
                              problem.anderson_regularization)
    for nu in range(1, iterations + 1):
        total = total_family(problem, scattering, plus, minus)
        green, lam = current_green(problem, total)
        cand_sc, rround = scattering_candidate(problem, green, plans, verify=verify)
        cplus, cminus = embedding_candidate(problem, green, plans)
        cand_total = total_family(problem, cand_sc, cplus, cminus)
        res = residual_suite(problem.eps, problem.h, green["GR"], green["GL"], green["GG"], total, cand_total[1])
        rS = 0.0
        for old, new in [(plus, cplus), (minus, cminus)] + [
                (scattering[m.name], cand_sc[m.name]) for m in problem.mechanisms]:
            for c in range(3):
                rS = max(rS, relative_change(old[c], new[c]))
        emb_old = tuple(plus[c] + minus[c] for c in range(3))
        emb_new = tuple(cplus[c] + cminus[c] for c in range(3))
        for c in range(3):
            rS = max(rS, relative_change(emb_old[c], emb_new[c]))
        Jbar = current(problem, plus[2], plus[1], green["GL"], green["GG"])
        J = Jbar * problem.J0
        pops = populations(problem, green["GL"])
        rJ = math.inf if Jprev is None else abs(J - Jprev) / max(abs(J), abs(Jprev), 1e-12)
        rp = math.inf if pprev is None else float(np.linalg.norm(pops - pprev) / (np.linalg.norm(pops) + 1e-14))
        row = dict(nu=nu, lam=lam, rlam=abs(lam - 1), rSigma=rS, rround=rround, J=J, Jbar=Jbar,
                   populations=pops, rJ=rJ, rpop=rp, number=green["number"], holes=green["holes"],
                   target=problem.target, normalized=green["normalized"],
                   lambda_change=math.nan if not history else lam - history[-1]["lam"], **res)
        history.append(row)
        a = problem.alpha
        if terminal and nu == iterations:
            break
        if mixer is not None:
            names = [m.name for m in problem.mechanisms]
            st = [scattering[n] for n in names] + [plus, minus]
            cd = [cand_sc[n] for n in names] + [cplus, cminus]
            mixed = mixer.mix(st, cd, a)
            row["mixer"] = dict(mixer.info)
            for i, n in enumerate(names):
                scattering[n] = mixed[i]
            plus, minus = mixed[-2], mixed[-1]
            Jprev, pprev = J, pops
            continue
        for m in problem.mechanisms:
            scattering[m.name] = tuple(np.asfortranarray((1 - a) * scattering[m.name][c] + a * cand_sc[m.name][c])
                                       for c in range(3))
        plus = tuple(np.asfortranarray((1 - a) * plus[c] + a * cplus[c]) for c in range(3))
        minus = tuple(np.asfortranarray((1 - a) * minus[c] + a * cminus[c]) for c in range(3))
        Jprev, pprev = J, pops
    out_state = dict(scattering=scattering, plus=plus, minus=minus, green=green) if keep_state else None
    return history, out_state


# --------------------------------------------------------------------------
# FP64 reference gradient of the converged current (the reference has no
# derivatives).  At a fixed point Sigma = Phi(Sigma, p) of the map of one
# SCBA iteration without mixing, dJ/dp = J_Sigma v + J_p with
# (I - Phi_Sigma) v = Phi_p.  Phi_Sigma v and J_Sigma v are central
# directional differences of the map (the map is smooth away from the switch
# of the paired normalisation), the linear system is solved by GMRES on the
# physical subspace (Sigma^<, Sigma^> anti-Hermitian per block), and Phi_p,
# J_p are central differences of one map application at p +- h.
# --------------------------------------------------------------------------
def scba_map(problem, families, plans=None, branch=0):
    """One SCBA iteration without the mixing step (the order of scba()):
    totals, Dyson/Keldysh with the paired normalisation (`branch` as in
    current_green), the scattering and embedding candidates, and J of the
    state.  `families` lists the mechanisms' (R, <, >) tuples in problem
    order, then plus and minus.  Returns (candidate families in the same
    order, J)."""
    plans = plans or make_plans(problem)
    M = len(problem.mechanisms)
    scattering = {m.name: families[i] for i, m in enumerate(problem.mechanisms)}
    plus, minus = families[M], families[M + 1]
    total = total_family(problem, scattering, plus, minus)
    green, _ = current_green(problem, total, branch)
    cand, _ = scattering_candidate(problem, green, plans, verify=False)
    cplus, cminus = embedding_candidate(problem, green, plans)
    J = current(problem, plus[2], plus[1], green["GL"], green["GG"]) * problem.J0
    return [tuple(cand[m.name]) for m in problem.mechanisms] + [tuple(cplus), tuple(cminus)], J


def _flatten(families):
    return np.concatenate([np.ravel(c, order="F").view(np.float64) for f in families for c in f])


def _unflatten(x, like):
    out, i = [], 0
    for f in like:
        comps = []
        for c in f:
            n = 2 * c.size
            comps.append(np.asfortranarray(x[i:i + n].view(np.complex128).reshape(c.shape, order="F")))
            i += n
        out.append(tuple(comps))
    return out


def _physical(families):
    """Sigma^< and Sigma^> of every family projected on their anti-Hermitian
    part (the subspace the map keeps)."""
    return [tuple(c if k == 0 else 0.5 * (c - np.conj(np.swapaxes(c, -1, -2))) for k, c in enumerate(f))
            for f in families]


def implicit_gradient(build, p0, steps, iterations=2000, rtol=1e-9, hold_branch=True):
    """dJ/dp_k at p0 for the problem family build(p): the SCBA converged by
    `iterations` linear-mixing steps (its last state is the fixed point to
    the map's roundoff), then the implicit-function derivative above.  With
    `hold_branch` every map application uses the paired normalisation's form
    at the fixed point (a fixed point near the switch between the two forms
    would otherwise see the kink in its differences).  Returns (gradient, J,
    r_Sigma of the last iteration, the form held: 1 or 2, 0 if none)."""
    import scipy.sparse.linalg as sla

    p0 = np.asarray(p0, dtype=np.float64)
    pr = build(p0)
    hist, st = scba(pr, iterations, verify=False, keep_state=True)
    fams = [tuple(np.array(c) for c in st["scattering"][m.name]) for m in pr.mechanisms]
    fams += [tuple(np.array(c) for c in st["plus"]), tuple(np.array(c) for c in st["minus"])]
    plans = make_plans(pr)
    branch = 0
    if hold_branch:
        M = len(pr.mechanisms)
        total = total_family(pr, {m.name: fams[i] for i, m in enumerate(pr.mechanisms)}, fams[M], fams[M + 1])
        green, _ = current_green(pr, total)
        branch = 1 if green["number"] >= pr.target else 2
    x0 = _flatten(fams)
    scale = np.linalg.norm(x0)

    def directional(v):
        e = 1e-6 * scale / max(np.linalg.norm(v), 1e-300)
        a, Ja = scba_map(pr, _unflatten(x0 + e * v, fams), plans, branch)
        b, Jb = scba_map(pr, _unflatten(x0 - e * v, fams), plans, branch)
        return (_flatten(a) - _flatten(b)) / (2 * e), (Ja - Jb) / (2 * e)

    def project(x):
        return _flatten(_physical(_unflatten(x, fams)))

    def matvec(v):  # identity off the physical subspace keeps the operator regular
        pv = project(v)
        return v - project(directional(pv)[0])

    n = x0.size
    A = sla.LinearOperator((n, n), matvec=matvec, dtype=np.float64)
    grad = []
    for k, h in enumerate(steps):
        e = np.zeros_like(p0)
        e[k] = h
        a, Ja = scba_map(build(p0 + e), fams, branch=branch)
        b, Jb = scba_map(build(p0 - e), fams, branch=branch)
        rhs = project((_flatten(a) - _flatten(b)) / (2 * h))
        v, info = sla.gmres(A, rhs, rtol=rtol, atol=0.0, restart=100, maxiter=5)
        if info < 0:
            raise OracleError(5, "implicit gradient: GMRES breakdown")
        grad.append(directional(v)[1] + (Ja - Jb) / (2 * h))
    return np.array(grad), hist[-1]["J"], hist[-1]["rSigma"], branch


# --------------------------------------------------------------------------
# The reference's production path on the host cores with library arithmetic
# (the CPU baseline of the benchmark): LAPACK through numpy (OpenBLAS) for
# the per-block inverse and products, pocketfft (scipy.fft) for the Hilbert
# transform, threads over independent slabs as the :threads backend of
# ProductionOptions (production_contracts.jl:113-121).
# --------------------------------------------------------------------------
def production_green_lapack(eps, h, SR, SL, threads=1, chunk=512):
    """_retarded_green_production (production_operators.jl:1337-1385: row-sum
    scale s, G = inv(D/s)/s with LAPACK) fused with the lesser sandwich of
    _current_green_production (production_state.jl:29-47).  The condition
    number kappa (an SVD per block) is not formed, as on the device.
    Returns (GR, GL) in the Julia layout."""
    import concurrent.futures

    eps = np.asarray(eps, dtype=np.float64)
    h = np.asarray(h)
    NE, Nk, N, _ = SR.shape
    GR = np.empty(SR.shape, dtype=np.complex128, order="F")
    GL = np.empty(SR.shape, dtype=np.complex128, order="F")
    eye = np.eye(N)

    def work(task):
        m, e0 = task
        e1 = min(NE, e0 + chunk)
        D = eps[e0:e1, None, None] * eye - h[m][None] - SR[e0:e1, m]
        s = np.max(np.sum(np.abs(D), axis=2), axis=1)[:, None, None]
        G = np.linalg.inv(D / s) / s
        GR[e0:e1, m] = G
        GL[e0:e1, m] = G @ SL[e0:e1, m] @ np.conj(np.swapaxes(G, -1, -2))

    tasks = [(m, e0) for m in range(Nk) for e0 in range(0, NE, chunk)]
    with concurrent.futures.ThreadPoolExecutor(max(1, threads)) as ex:
        list(ex.map(work, tasks))
    return GR, GL


def production_fft_hilbert_pocketfft(Gam, eps, wE, threads=1, chunk=512):
    """production_fft_hilbert_transform (fft_parallel.jl:168-291): per column
    the weighted field zero-padded to L = nextpow2(2 N_E - 1), multiplied in
    Fourier space by the spectrum of k[lag + N_E - 1] = 1 / (2 pi lag de),
    output y[e + N_E - 1]; columns in chunks, each chunk's FFTs over
    `threads` workers."""
    import scipy.fft

    Gam = np.asarray(Gam)
    NE = Gam.shape[0]
    cols = Gam.reshape((NE, -1), order="F")
    ncols = cols.shape[1]
    L = 1 << (2 * NE - 2).bit_length()
    de = float(eps[1] - eps[0])
    kern = np.zeros(L, dtype=np.complex128)
    lag = np.arange(-(NE - 1), NE)
    nz = lag != 0
    kern[lag[nz] + NE - 1] = 1.0 / (2 * math.pi * lag[nz] * de)
    khat = scipy.fft.fft(kern)
    out = np.empty((NE, ncols), dtype=np.complex128, order="F")
    w = np.asarray(wE, dtype=np.float64)
    for c0 in range(0, ncols, chunk):
        c1 = min(ncols, c0 + chunk)
        buf = np.zeros((c1 - c0, L), dtype=np.complex128)
        buf[:, :NE] = (cols[:, c0:c1] * w[:, None]).T
        y = scipy.fft.ifft(scipy.fft.fft(buf, axis=1, workers=threads) * khat[None, :], axis=1, workers=threads)
        out[:, c0:c1] = y[:, NE - 1:2 * NE - 1].T
    return out.reshape(Gam.shape, order="F")
