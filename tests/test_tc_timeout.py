"""The bounded waits of the tensor-core contraction kernel.

Every mbarrier wait of tc_gemm_kernel gives up after a bounded number of
polling rounds and records QCL_TIMEOUT instead of hanging.  A test hook
lowers the main-loop limit to zero, so the first wait of every CTA gives up
while its TMA copies are in flight; the kernel must then wait (with the full
limit) for those copies, free its tensor memory and return, and the call must
report QCL_TIMEOUT.  With the default limit restored, the next contraction on
the same context is correct.
"""
import numpy as np
import pytest

from helpers import approx_err

pytestmark = pytest.mark.gpu


def test_tc_gemm_wait_timeout_is_reported_and_recoverable(gpu_ops, orc):
    from qclb200 import _lib
    from qclb200.problem import small_problem

    pr = small_problem(NE=37, Nk=4, Nb=4, mechanisms=("impurity",))
    mech = pr.mechanisms[0]
    rng = np.random.default_rng(7)
    G = np.asfortranarray(rng.standard_normal(pr.shape) + 1j * rng.standard_normal(pr.shape))
    lit = orc.contraction_literal(mech.literal_kernel(pr.Nk, pr.Nb), G, pr.wk, mech.q)
    lib = _lib.lib()
    _lib.check(lib.qcl_debug_set_wait_limit(0))
    try:
        with pytest.raises(_lib.QCLError) as ex:
            gpu_ops.production_static_contraction(mech, G, pr.wk, precision="c64")
        assert ex.value.code == _lib.QCL_TIMEOUT
    finally:
        _lib.check(lib.qcl_debug_set_wait_limit(-1))
    got = gpu_ops.production_static_contraction(mech, G, pr.wk, precision="c64")
    assert approx_err(got, lit) < 1e-5
