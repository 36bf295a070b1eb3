"""B200-native SCBA hot path of QCLNEGF.jl: host-side mirror of the
reference's operator interface over the C ABI of libqclb200.so."""
from . import _lib, problem  # noqa: F401
from ._lib import (ArgumentError, DimensionMismatch, DomainError, NonFiniteMetrics, QCLError,  # noqa: F401
                   SingularException)

__all__ = ["problem", "operators", "QCLError", "SingularException", "DomainError", "DimensionMismatch",
           "ArgumentError", "NonFiniteMetrics"]


def __getattr__(name):
    if name in ("operators", "device", "scba"):
        import importlib

        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
