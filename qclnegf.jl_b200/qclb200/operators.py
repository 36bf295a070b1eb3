"""Host-array operators with the reference's names and argument meaning.

Each function takes numpy arrays in the reference's Julia layout (Fortran
order, fields ``(N_E, N_k, N_b, N_b)``), calls the C ABI of libqclb200.so
(host-buffer entry points: copy in, compute on the GPU, copy out) and returns
numpy arrays in the same layout.  Errors raise the reference's exception
types (see ``_lib``).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib

_CDT = {_lib.QCL_C128: np.complex128, _lib.QCL_C64: np.complex64, _lib.QCL_MIXED: np.complex64}


def _prec(precision):
    _begin()
    try:
        return _lib.PRECISIONS[precision]
    except KeyError:
        raise _lib.ArgumentError(_lib.QCL_ARG, f"unknown precision {precision!r}") from None


def _field(x, dtype, shape=None):
    a = np.asfortranarray(np.asarray(x, dtype=dtype))
    if shape is not None and a.shape != tuple(shape):
        raise _lib.DimensionMismatch(_lib.QCL_DIM, f"array shape {a.shape} differs from {tuple(shape)}")
    return a


_ALIVE = []


def _ptr(a):
    """Pointer to a numpy array's data; the array stays referenced until the
    next wrapper starts, so layout-converted temporaries outlive the C call."""
    if a is None:
        return None
    _ALIVE.append(a)
    return ctypes.c_void_p(a.ctypes.data)


def _begin():
    del _ALIVE[:]


def _real(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def dyson_keldysh(eps, h, sigR, sigL=None, sigG=None, *, eta=0.0, precision="c128", want_retarded=True,
                  return_traces=False):
    """Fused batched Dyson solve and Keldysh products.

    Mirrors ``_retarded_green_production`` + the raw sandwiches of
    ``_current_green_production`` (production_operators.jl:1337-1385,
    production_state.jl:23-48).  Returns ``(GR, GL, GG, scale)`` (entries
    None where not requested); with ``return_traces`` also the raw block
    traces of GL and GG."""
    p = _prec(precision)
    cdt = _CDT[p]
    eps = _real(eps)
    h = _field(h, np.complex128)
    Nk, Nb = h.shape[0], h.shape[1]
    NE = eps.shape[0]
    shape = (NE, Nk, Nb, Nb)
    if h.shape != (Nk, Nb, Nb):
        raise _lib.DimensionMismatch(_lib.QCL_DIM, "h has wrong shape")
    sigR = _field(sigR, cdt, shape)
    sigL = None if sigL is None else _field(sigL, cdt, shape)
    sigG = None if sigG is None else _field(sigG, cdt, shape)
    GR = np.zeros(shape, dtype=cdt, order="F") if want_retarded else None
    GL = np.zeros(shape, dtype=cdt, order="F") if sigL is not None else None
    GG = np.zeros(shape, dtype=cdt, order="F") if sigG is not None else None
    scale = np.zeros((NE, Nk), order="F")
    trL = np.zeros((NE, Nk), dtype=np.complex128, order="F") if (return_traces and sigL is not None) else None
    trG = np.zeros((NE, Nk), dtype=np.complex128, order="F") if (return_traces and sigG is not None) else None
    check(lib().qcl_dyson_keldysh(p, NE, Nk, Nb, _ptr(eps), float(eta), _ptr(h), _ptr(sigR), _ptr(sigL), _ptr(sigG),
                                  _ptr(GR), _ptr(GL), _ptr(GG), _ptr(scale), _ptr(trL), _ptr(trG)))
    if return_traces:
        return GR, GL, GG, scale, trL, trG
    return GR, GL, GG, scale


def retarded_green(eps, h, sigR, *, eta=0.0, precision="c128", return_scale=False):
    """retarded_green (numerics/reference/greens.jl:18-42): G^R = inv(D/s)/s.
    Returns ``(GR, scale)``; the condition number of the reference's second
    return value is not computed on the device path (only stored there)."""
    GR, _, _, scale = dyson_keldysh(eps, h, sigR, eta=eta, precision=precision)
    return (GR, scale) if return_scale else GR


def keldysh_green(eps, h, sigR, sig, *, eta=0.0, precision="c128"):
    """G^R Sigma G^A for Sigma in {<, >} with G^R from the same Dyson solve
    (keldysh_green, greens.jl:67-75)."""
    _, GL, _, _ = dyson_keldysh(eps, h, sigR, sig, eta=eta, precision=precision, want_retarded=False)
    return GL


def fft_hilbert_transform(Gam, eps, wE, *, precision="c128", return_roundoff=False):
    """fft_hilbert_transform (production_operators.jl:793-809)."""
    p = _prec(precision)
    cdt = _CDT[p]
    Gam = _field(Gam, cdt)
    NE = Gam.shape[0]
    ncols = Gam.size // NE
    eps, wE = _real(eps), _real(wE)
    if eps.shape[0] != NE or wE.shape[0] != NE:
        raise _lib.DimensionMismatch(_lib.QCL_DIM, "energy data differ")
    Lam = np.zeros_like(Gam, order="F")
    r = ctypes.c_double()
    check(lib().qcl_fft_hilbert_transform(p, NE, ncols, _ptr(eps), _ptr(wE), _ptr(Gam), _ptr(Lam),
                                          ctypes.byref(r) if return_roundoff else None))
    return (Lam, r.value) if return_roundoff else Lam


def retarded_self_energy_fft(SL, SG, eps, wE, *, precision="c128", return_roundoff=False):
    """retarded_self_energy_fft (production_operators.jl:811-840): returns
    ``(SigmaR, Gamma[, roundoff])``."""
    p = _prec(precision)
    cdt = _CDT[p]
    SL = _field(SL, cdt)
    SG = _field(SG, cdt, SL.shape)
    NE = SL.shape[0]
    ncols = SL.size // NE
    eps, wE = _real(eps), _real(wE)
    SR = np.zeros_like(SL, order="F")
    Gam = np.zeros_like(SL, order="F")
    r = ctypes.c_double()
    check(lib().qcl_retarded_self_energy(p, NE, ncols, _ptr(eps), _ptr(wE), _ptr(SL), _ptr(SG), _ptr(SR), _ptr(Gam),
                                         ctypes.byref(r) if return_roundoff else None))
    return (SR, Gam, r.value) if return_roundoff else (SR, Gam)


def condition_number(eps, h, GR, SR=None, *, eta=0.0, precision="c128"):
    """(kappa, scale): cond_2(D) and the Dyson row-sum scale per (E,k) block,
    D = (eps + i eta) I - h - SR -- the condition_number / dyson_scale outputs
    of _retarded_green_production (production_operators.jl:1337-1385).  GR is
    the Dyson solution for the same inputs."""
    p = _prec(precision)
    GR = _field(GR, _CDT[p])
    NE, Nk, Nb, _ = GR.shape
    h = _field(h, np.complex128, (Nk, Nb, Nb))
    SR = None if SR is None else _field(SR, _CDT[p], GR.shape)
    kappa = np.zeros((NE, Nk), order="F")
    scale = np.zeros((NE, Nk), order="F")
    check(lib().qcl_condition_number(p, NE, Nk, Nb, _ptr(_real(eps)), float(eta), _ptr(h),
                                     None if SR is None else _ptr(SR), _ptr(GR), _ptr(kappa), _ptr(scale)))
    return kappa, scale


def spectral_function(GR, *, precision="c128"):
    """A = i (GR - GR^H) per block (spectral_function, numerics/reference/greens.jl:50-57)."""
    p = _prec(precision)
    GR = _field(GR, _CDT[p])
    NE, Nk, Nb, _ = GR.shape
    A = np.zeros_like(GR, order="F")
    check(lib().qcl_spectral_function(p, NE, Nk, Nb, _ptr(GR), _ptr(A)))
    return A


class _Mechanism(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("is_LO", ctypes.c_int), ("J", ctypes.c_int), ("q", ctypes.c_double),
                ("block", ctypes.c_void_p), ("matrix", ctypes.c_void_p), ("left", ctypes.c_void_p),
                ("right", ctypes.c_void_p), ("radial", ctypes.c_void_p)]


_KIND = {"momentum_independent": 0, "dense": 1, "ifr": 2, "low_rank": 3, "separable_sum": 4}


def mechanism_struct(mech):
    """ctypes view of a problem.Mechanism (keeps the arrays alive on the
    returned object)."""
    keep = []

    def arr(a):
        if a is None:
            return None
        if hasattr(a, "__cuda_array_interface__"):  # device array (complex128, column-major): passed as is
            keep.append(a)
            return ctypes.c_void_p(a.__cuda_array_interface__["data"][0])
        a = np.asfortranarray(np.asarray(a, dtype=np.complex128))
        keep.append(a)
        return ctypes.c_void_p(a.ctypes.data)

    if mech.kind == "separable_sum":
        J = int(np.shape(mech.radial)[2])
    else:
        J = 0 if mech.left is None else int(np.shape(mech.left)[1])
    s = _Mechanism(_KIND[mech.kind], 1 if mech.name == "LO" else 0, J, float(mech.q),
                   arr(mech.block), arr(mech.matrix), arr(mech.left), arr(mech.right), arr(mech.radial))
    s._keep = keep
    return s


def apply_energy_shift(X, eps, delta, *, precision="c128"):
    """apply_energy_shift (production_cache.jl:300-325) with the plan of
    build_shift_plan(eps, delta)."""
    p = _prec(precision)
    X = _field(X, _CDT[p])
    NE = X.shape[0]
    Y = np.zeros_like(X, order="F")
    check(lib().qcl_apply_energy_shift(p, NE, X.size // NE, _ptr(_real(eps)), float(delta), _ptr(X), _ptr(Y)))
    return Y


def production_static_contraction(mech, G, wk, *, alpha=1.0, beta=0.0, S=None, precision="c128"):
    """production_static_contraction (production_operators.jl:682-722) for a
    factorised operator: returns beta*S + alpha*q*K[wk G]."""
    p = _prec(precision)
    G = _field(G, _CDT[p])
    NE, Nk, Nb, _ = G.shape
    out = np.zeros_like(G, order="F") if S is None else _field(S, _CDT[p], G.shape).copy(order="F")
    op = mechanism_struct(mech)
    check(lib().qcl_static_contraction(p, ctypes.byref(op), NE, Nk, Nb, _ptr(_real(wk)), float(alpha), float(beta),
                                       _ptr(G), _ptr(out)))
    return out


def embedding_component(T, G, eps, delta, *, precision="c128"):
    """_embedding_component_production (production_operators.jl:886-922)."""
    p = _prec(precision)
    G = _field(G, _CDT[p])
    NE, Nk, Nb, _ = G.shape
    T = _field(T, np.complex128, (Nb, Nb))
    S = np.zeros_like(G, order="F")
    check(lib().qcl_embedding_component(p, NE, Nk, Nb, _ptr(_real(eps)), float(delta), _ptr(T), _ptr(G), _ptr(S)))
    return S


def anderson_guard(families, *, precision="c128"):
    """_anderson_guard (production_mixing.jl:98-118) on a list of
    (SigmaR, Sigma<, Sigma>) families: (passed, first failing 1-based block
    index over (family, e, m) with m fastest, failure code)."""
    p = _prec(precision)
    cdt = _CDT[p]
    shape = np.shape(families[0][0])
    NE, Nk, Nb, _ = shape
    arrs = [_field(x, cdt, shape) for fam in families for x in fam]
    ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    first = ctypes.c_longlong()
    code = ctypes.c_int()
    check(lib().qcl_anderson_guard(p, NE, Nk, Nb, len(families), ptrs, ctypes.byref(first), ctypes.byref(code)))
    return first.value == 0, int(first.value), int(code.value)


WITNESS_KINDS = ("spectral", "occupied", "unoccupied", "broadening", "raw_occupied", "raw_unoccupied")


class PsdWitness(ctypes.Structure):
    """qcl_psd_witness: _PositivityWitness (positivity_diagnostics.jl:41-54)."""
    _fields_ = [("matrix_kind", ctypes.c_int), ("energy_index", ctypes.c_int), ("momentum_index", ctypes.c_int)] + [
        (n, ctypes.c_double) for n in ("minimum_eigenvalue", "block_norm", "floor", "ratio", "absolute_defect",
                                       "relative_defect", "backward_error", "hermiticity_defect",
                                       "construction_scale")]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_}
        d["matrix_kind"] = "none" if self.matrix_kind < 0 else WITNESS_KINDS[self.matrix_kind]
        return d


def production_residual_suite(eps, h, GR, GL, GG, total, candidate_lesser, *, precision="c128",
                              return_witness=False):
    """production_residual_suite (residuals.jl:537-770): dict r_D, r_A, r_K,
    r_PSD, r_caus (and the positivity witness as ``witness``)."""
    p = _prec(precision)
    cdt = _CDT[p]
    GR = _field(GR, cdt)
    shape = GR.shape
    NE, Nk, Nb, _ = shape
    arrs = [GR] + [_field(x, cdt, shape) for x in (GL, GG, total[0], total[1], total[2], candidate_lesser)]
    out = np.zeros(5)
    args = (p, NE, Nk, Nb, _ptr(_real(eps)), _ptr(_field(h, np.complex128)), *[_ptr(a) for a in arrs], _ptr(out))
    w = PsdWitness()
    if return_witness:
        check(lib().qcl_residual_suite_witness(*args, ctypes.byref(w)))
    else:
        check(lib().qcl_residual_suite(*args))
    res = dict(rD=out[0], rA=out[1], rK=out[2], rPSD=out[3], rcaus=out[4])
    if return_witness:
        res["witness"] = w.as_dict()
    return res


def production_selfenergy_residual(old, new, *, precision="c128"):
    p = _prec(precision)
    old = _field(old, _CDT[p])
    new = _field(new, _CDT[p], old.shape)
    out = ctypes.c_double()
    check(lib().qcl_selfenergy_residual(p, old.size, _ptr(old), _ptr(new), ctypes.byref(out)))
    return out.value


def current_and_populations(problem, SG, SL, GL, GG, *, precision="c128"):
    """(Jbar, populations): _production_boundary_flux_bar and
    _production_state_populations (production_iteration.jl:174-215)."""
    p = _prec(precision)
    cdt = _CDT[p]
    shape = problem.shape
    arrs = [_field(x, cdt, shape) for x in (SG, SL, GL, GG)]
    out = np.zeros(2 + problem.Nb)
    check(lib().qcl_current_populations(p, problem.NE, problem.Nk, problem.Nb, _ptr(_real(problem.wE)),
                                        _ptr(_real(problem.wk)), int(problem.gs), float(problem.target),
                                        *[_ptr(a) for a in arrs], _ptr(out)))
    return out[0], out[2:].copy()


def hermitian_eigvals(H):
    """Eigenvalues (ascending) of a stack of Hermitian matrices H[..., n, n]
    (the role of LAPACK zheev in residuals.jl:311-353)."""
    _begin()
    H = np.asarray(H, dtype=np.complex128)
    n = H.shape[-1]
    stack = H.reshape((-1, n, n))
    # column-major matrices back to back
    cm = np.ascontiguousarray(np.transpose(stack, (0, 2, 1)))
    vals = np.zeros((stack.shape[0], n))
    check(lib().qcl_hermitian_eigvals(n, stack.shape[0], _ptr(cm), _ptr(vals)))
    return np.sort(vals, axis=1).reshape(H.shape[:-1])


class TuneResult(ctypes.Structure):
    _fields_ = [("dyson_bpc", ctypes.c_int), ("default_bpc", ctypes.c_int), ("candidates", ctypes.c_int),
                ("bpc", ctypes.c_int * 4), ("ms", ctypes.c_float * 4)]


def autotune(Nb, *, precision="c128", NE=1024, Nk=8):
    """qcl_autotune: time every compiled CTA shape (blocks per CTA) of the
    Dyson + Keldysh kernel for the basis class of Nb on a synthetic NE x Nk
    batch; later launches of that class in this process use the fastest.
    Returns {"chosen", "default", "ms": {bpc: ms}}."""
    r = TuneResult()
    check(lib().qcl_autotune(_prec(precision), int(Nb), int(NE), int(Nk), ctypes.byref(r)))
    return {"chosen": r.dyson_bpc, "default": r.default_bpc,
            "ms": {int(r.bpc[i]): float(r.ms[i]) for i in range(r.candidates)}}


def autotune_reset():
    """Restore the built-in CTA shapes."""
    check(lib().qcl_autotune_reset())


def tuned_dyson_bpc(Nb, *, precision="c128"):
    return int(lib().qcl_tuned_dyson_bpc(_prec(precision), int(Nb)))
