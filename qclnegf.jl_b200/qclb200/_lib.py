"""Loader and ctypes signatures for libqclb200.so (the C ABI in
``include/qclb200.h``).

There is no CPU fallback: if the shared library is missing or does not load,
importing the operators raises, so nothing silently runs elsewhere.
"""
from __future__ import annotations

import ctypes
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
REPO_ROOT = os.path.dirname(PKG_ROOT)
LIB_PATH = os.environ.get("QCLB200_LIB") or os.path.join(PKG_ROOT, "lib", "libqclb200.so")
HEADER_PATH = os.path.join(REPO_ROOT, "include", "qclb200.h")

QCL_OK = 0
QCL_SINGULAR = 1
QCL_DOMAIN = 2
QCL_DIM = 3
QCL_ARG = 4
QCL_NONFINITE = 5
QCL_TIMEOUT = 6
QCL_CUDA = 7
QCL_NOMEM = 8
QCL_UNSUPPORTED = 9

QCL_C128 = 0
QCL_C64 = 1
QCL_MIXED = 2

PRECISIONS = {"c128": QCL_C128, "fp64": QCL_C128, "c64": QCL_C64, "fp32": QCL_C64, "mixed": QCL_MIXED,
              QCL_C128: QCL_C128, QCL_C64: QCL_C64, QCL_MIXED: QCL_MIXED}


class QCLError(RuntimeError):
    """Base class; `.code` is the library status."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class SingularException(QCLError):
    """Reference: LinearAlgebra.SingularException (production_operators.jl:39,94);
    ``k`` is its index: 0 for a zero row-sum scale, else the 1-based first
    zero pivot (qcl_last_singular_pivot)."""

    k = 0


class DomainError(QCLError, ValueError):
    """Reference: DomainError (e.g. production_state.jl:53)."""


class DimensionMismatch(QCLError, ValueError):
    """Reference: DimensionMismatch."""


class ArgumentError(QCLError, ValueError):
    """Reference: ArgumentError."""


class NonFiniteMetrics(QCLError):
    """Reference: the :nonfinite_metrics SCBA status (production_solver.jl:624-656)."""


class UnsupportedError(QCLError):
    pass


class CudaError(QCLError):
    pass


class MemoryBudgetError(ArgumentError):
    """QCL_NOMEM: the memory preflight refused the context (the ArgumentError
    of build_production_cache, numerics/optimized/production_cache.jl:
    764-770) or a device allocation failed."""


_EXC = {
    QCL_SINGULAR: SingularException,
    QCL_DOMAIN: DomainError,
    QCL_DIM: DimensionMismatch,
    QCL_ARG: ArgumentError,
    QCL_NONFINITE: NonFiniteMetrics,
    QCL_UNSUPPORTED: UnsupportedError,
    QCL_CUDA: CudaError,
    QCL_NOMEM: MemoryBudgetError,
    QCL_TIMEOUT: QCLError,
}

_LIB = None


def header_symbols():
    """Every function name declared in include/qclb200.h."""
    text = open(HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qcl_[a-z0-9_]+)\s*\(", text)))


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libqclb200.so is not built ({LIB_PATH}); run qclnegf.jl_b200/build.py")
        _LIB = ctypes.CDLL(LIB_PATH)
        _declare(_LIB)
    return _LIB


P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double
Z = ctypes.c_size_t


def _declare(l):
    sig = {
        "qcl_version": (I, []),
        "qcl_last_error": (ctypes.c_char_p, []),
        "qcl_max_basis": (I, []),
        "qcl_dyson_keldysh": (I, [I, I, I, I, P, D, P, P, P, P, P, P, P, P, P, P]),
        "qcl_dev_dyson_keldysh": (I, [P, I, I, I, I, P, D, P, P, P, P, P, P, P, P, P, P, P]),
        "qcl_dev_weighted_trace": (I, [P, I, I, P, P, P, P]),
        "qcl_dev_paired_coefficients": (I, [P, P, P, I, D, P, P]),
        "qcl_dev_normalize_pair": (I, [P, I, Z, P, P, P]),
        "qcl_fft_hilbert_transform": (I, [I, I, Z, P, P, P, P, P]),
        "qcl_dev_fft_hilbert_transform": (I, [P, I, I, Z, D, P, P, P, P]),
        "qcl_retarded_self_energy": (I, [I, I, Z, P, P, P, P, P, P, P]),
        "qcl_apply_energy_shift": (I, [I, I, Z, P, D, P, P]),
        "qcl_static_contraction": (I, [I, P, I, I, I, P, D, D, P, P]),
        "qcl_embedding_component": (I, [I, I, I, I, P, D, P, P, P]),
        "qcl_residual_suite": (I, [I, I, I, I, P, P, P, P, P, P, P, P, P, P]),
        "qcl_residual_suite_witness": (I, [I, I, I, I, P, P, P, P, P, P, P, P, P, P, P]),
        "qcl_selfenergy_residual": (I, [I, Z, P, P, P]),
        "qcl_hermitian_eigvals": (I, [I, Z, P, P]),
        "qcl_condition_number": (I, [I, I, I, I, P, D, P, P, P, P, P]),
        "qcl_spectral_function": (I, [I, I, I, I, P, P]),
        "qcl_dev_residual_suite_noalloc": (I, [P, I, I, I, I, P, P, P, P, P, P, P, P, P, P]),
        "qcl_current_populations": (I, [I, I, I, I, P, P, I, D, P, P, P, P, P]),
        "qcl_scba_create": (I, [P, P, P]),
        "qcl_scba_destroy": (None, [P]),
        "qcl_scba_seed": (I, [P, P]),
        "qcl_scba_step": (I, [P, P]),
        "qcl_scba_run": (I, [P, I, D, P, P]),
        "qcl_scba_populations": (I, [P, P]),
        "qcl_scba_download": (I, [P, I, P]),
        "qcl_scba_upload": (I, [P, I, P]),
        "qcl_scba_use_graph": (I, [P, I]),
        "qcl_scba_green_state": (I, [P, P, P, P]),
        "qcl_scba_witness": (I, [P, P]),
        "qcl_scba_retarget": (I, [P, D, D, D, P, P]),
        "qcl_scba_estimate_memory": (I, [P, P, P]),
        "qcl_scba_promote": (I, [P]),
        "qcl_scba_use_telemetry": (I, [P, I]),
        "qcl_scba_phase_times": (I, [P, P, P]),
        "qcl_last_singular_pivot": (I, []),
        "qcl_debug_set_wait_limit": (I, [ctypes.c_longlong]),
        "qcl_autotune": (I, [I, I, I, I, P]),
        "qcl_sweep_create": (I, [I, P, P, Z, P]),
        "qcl_scba_tangent_init": (I, [P]),
        "qcl_scba_tangent_set": (I, [P, I, P]),
        "qcl_scba_tangent_step": (I, [P, P]),
        "qcl_scba_download_candidate": (I, [P, I, P]),
        "qcl_scba_set_normalization_branch": (I, [P, I]),
        "qcl_scba_normalization_branch": (I, [P, ctypes.POINTER(ctypes.c_int)]),
        "qcl_sweep_run": (I, [P, I, D, P, P, P]),
        "qcl_sweep_destroy": (None, [P]),
        "qcl_autotune_reset": (I, []),
        "qcl_tuned_dyson_bpc": (I, [I, I]),
        "qcl_scba_mixer_info": (I, [P, P]),
        "qcl_anderson_guard": (I, [I, I, I, I, I, P, P, P]),
        "qcl_scba_density_matrix": (I, [P, P]),
        "qcl_density_matrix": (I, [I, I, I, I, P, P, P, P]),
        "qcl_assemble_kernel": (I, [I, I, I, I, P, P, P, P]),
        "qcl_dev_assemble_kernel": (I, [P, I, I, I, I, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        if hasattr(l, name):
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args


def declare(name, res, args):
    fn = getattr(lib(), name)
    fn.restype = res
    fn.argtypes = args
    return fn


def check(status):
    if status != QCL_OK:
        msg = lib().qcl_last_error().decode(errors="replace")
        exc = _EXC.get(status, QCLError)(status, msg or f"qclb200 status {status}")
        if status == QCL_SINGULAR:
            exc.k = int(lib().qcl_last_singular_pivot())
        raise exc
    return status
