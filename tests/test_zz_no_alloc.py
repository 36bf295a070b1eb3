"""The allocation-free residual suite (qcl_dev_residual_suite_noalloc).

It serves callers that cannot call cudaMalloc themselves or through the
library -- for example a Julia session whose GPU memory is owned by its own
pool allocator, or a host that reserves a fixed device budget up front.  It
keeps its scratch in a fixed device array of the library instead.  This test
calls it through the C ABI twice in a row on device arrays and checks each
result against the allocating entry point qcl_residual_suite, with the
tolerances of the other residual-suite tests.  It lives in its own file, which
pytest collects last, and passes alone in a fresh process as well as after the
other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(orc, seed, NE, Nk, Nb):
    from helpers import dyson_inputs

    eps, h, SR, SL, SG = dyson_inputs(seed, NE, Nk, Nb)
    GR = orc.retarded_green(eps, h, SR)[0]
    GL = orc.keldysh_green(GR, SL)
    GG = orc.keldysh_green(GR, SG)
    rng = np.random.default_rng(seed)
    cand = np.asfortranarray(SL * (1 + 0.01 * rng.standard_normal(SL.shape)))
    GL[1, 0, 0, 0] += 0.5j  # one indefinite block so r_PSD is non-zero
    return eps, h, GR, GL, GG, (SR, SL, SG), cand


@pytest.mark.parametrize("precision", ["c128", "c64", "mixed"])
def test_noalloc_residual_suite_matches_allocating_entry_point(gpu_ops, orc, precision):
    import torch

    from qclb200 import _lib

    lib = _lib.lib()
    dev = torch.device("cuda", 0)
    P = ctypes.c_void_p
    code = {"c128": _lib.QCL_C128, "c64": _lib.QCL_C64, "mixed": _lib.QCL_MIXED}[precision]
    cdt = np.complex128 if precision == "c128" else np.complex64
    for call, (seed, NE, Nk, Nb) in enumerate([(31, 29, 3, 12), (32, 40, 2, 5)]):
        eps, h, GR, GL, GG, tot, cand = _state(orc, seed, NE, Nk, Nb)
        # both entry points see the same rounded fields
        GR, GL, GG, cand = (np.asfortranarray(np.asarray(a, cdt)) for a in (GR, GL, GG, cand))
        tot = tuple(np.asfortranarray(np.asarray(a, cdt)) for a in tot)
        ref = gpu_ops.production_residual_suite(eps, h, GR, GL, GG, tot, cand, precision=precision)

        def dev_field(a):
            return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)

        d = [dev_field(a) for a in (GR, GL, GG, tot[0], tot[1], tot[2], cand)]
        d_eps = torch.tensor(eps, dtype=torch.float64, device=dev)
        d_h = dev_field(np.asarray(h, np.complex128))
        out = torch.full((5,), -1.0, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        st = lib.qcl_dev_residual_suite_noalloc(P(stream), code, NE, Nk, Nb, P(d_eps.data_ptr()),
                                                P(d_h.data_ptr()), *[P(x.data_ptr()) for x in d],
                                                P(out.data_ptr()))
        _lib.check(st)
        torch.cuda.synchronize()
        got = dict(zip(("rD", "rA", "rK", "rPSD", "rcaus"), out.cpu().numpy().tolist()))
        assert ref["rPSD"] > 0, call
        for k in ("rA", "rK"):
            assert abs(got[k] - ref[k]) <= 1e-10 * max(ref[k], 1e-14) + 1e-15, (call, k, got[k], ref[k])
        assert abs(got["rD"] - ref["rD"]) <= 1e-14 + 1e-10 * ref["rD"]
        assert got["rPSD"] == pytest.approx(ref["rPSD"], abs=1e-13, rel=1e-10)
        assert got["rcaus"] == pytest.approx(ref["rcaus"], abs=1e-13, rel=1e-10)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu_ops):
    from qclb200 import _lib

    lib = _lib.lib()
    z = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    st = lib.qcl_dev_residual_suite_noalloc(None, _lib.QCL_C128, 4096, 65, 4, z, z, z, z, z, z, z, z, z, z)
    assert st == _lib.QCL_UNSUPPORTED
    assert b"scratch capacity" in lib.qcl_last_error()
