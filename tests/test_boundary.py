"""The C-ABI library loads and exports every symbol include/qclb200.h declares
(no GPU needed: nothing is launched)."""
import ctypes
import os
import subprocess

import pytest


def test_library_exports_every_declared_symbol():
    from qclb200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libqclb200.so not built")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _lib.header_symbols()
    assert len(declared) >= 8
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # and exported with C linkage (unmangled) from the dynamic symbol table
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(declared) <= exported


def test_version_and_limits_without_gpu():
    from qclb200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libqclb200.so not built")
    l = _lib.lib()
    assert l.qcl_version() >= 100
    assert l.qcl_max_basis() == 48
    assert l.qcl_last_error() == b""


def test_operator_argument_errors_map_to_reference_exceptions():
    """Argument validation happens on the host before any device work."""
    import numpy as np
    from qclb200 import _lib, operators

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libqclb200.so not built")
    with pytest.raises(_lib.DimensionMismatch):
        operators.dyson_keldysh(np.zeros(4), np.zeros((2, 3, 3), complex), np.zeros((4, 2, 2, 2), complex))
    with pytest.raises(_lib.ArgumentError):
        operators.fft_hilbert_transform(np.zeros((5, 1), complex), np.array([0, 1, 2, 3, 5.0]), np.ones(5))
    with pytest.raises(_lib.UnsupportedError):
        eps = np.linspace(0, 1, 3)
        operators.dyson_keldysh(eps, np.zeros((1, 49, 49), complex), np.zeros((3, 1, 49, 49), complex))
