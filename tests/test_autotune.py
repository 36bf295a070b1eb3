"""The project autotuner (qcl_autotune): the Dyson + Keldysh kernel's CTA
shape (blocks per CTA) per basis class and precision, timed on the device.

GPU: every candidate is timed, the fastest is recorded and used by later
launches, the results of a launch with the tuned shape equal the oracle's
(the arithmetic per block does not depend on the shape), and a reset
restores the built-in choice.
"""
import numpy as np
import pytest

from helpers import approx_err, dyson_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,Nb", [("c128", 24), ("mixed", 16), ("c64", 32)])
def test_autotune_picks_a_timed_shape_and_keeps_results(gpu_ops, orc, precision, Nb):
    res = gpu_ops.autotune(Nb, precision=precision, NE=256, Nk=4)
    assert res["chosen"] in res["ms"] and len(res["ms"]) >= 2
    assert all(t > 0 for t in res["ms"].values())
    assert res["ms"][res["chosen"]] == min(res["ms"].values())
    assert gpu_ops.tuned_dyson_bpc(Nb, precision=precision) == res["chosen"]
    eps, h, SR, SL, SG = dyson_inputs(5, 67, 3, Nb)
    GR, GL, _, _ = gpu_ops.dyson_keldysh(eps, h, SR, SL, SG, precision=precision)
    oGR = orc.retarded_green(eps, h, SR)[0]
    tol = 1e-12 if precision == "c128" else 2e-5
    assert approx_err(GR, oGR) < tol
    assert approx_err(GL, orc.keldysh_green(oGR, SL)) < tol
    gpu_ops.autotune_reset()
    assert gpu_ops.tuned_dyson_bpc(Nb, precision=precision) == res["default"]
