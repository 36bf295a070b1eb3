"""GPU parity of the operator-level C ABI against the FP64 oracle.

Tolerances: complex128 paths must agree with the oracle within the
reference's own operator-equivalence tolerances (relative, Julia isapprox
sense: 1e-12 for Dyson/Keldysh products -- the reference pins its inverse at
5e-13 against `inv`; 2e-13 for the Hilbert transform).  complex64 / mixed
paths are checked at 2e-5 (Dyson, FP32 products) and 1e-5 (FFT in FP32).
"""
import math

import numpy as np
import pytest

from helpers import approx_err, dyson_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [1, 3, 8, 12, 16, 20, 24, 32, 40, 48])
def test_dyson_keldysh_c128_matches_oracle(gpu_ops, orc, N):
    NE, Nk = 37, 3
    eps, h, SR, SL, SG = dyson_inputs(100 + N, NE, Nk, N)
    GR, GL, GG, scale, trL, trG = gpu_ops.dyson_keldysh(eps, h, SR, SL, SG, precision="c128", return_traces=True)
    oGR, _, oscale, _ = orc.retarded_green(eps, h, SR)
    oGL = orc.keldysh_green(oGR, SL)
    oGG = orc.keldysh_green(oGR, SG)
    assert approx_err(GR, oGR) < 1e-12
    assert approx_err(GL, oGL) < 1e-12
    assert approx_err(GG, oGG) < 1e-12
    np.testing.assert_allclose(scale, oscale, rtol=1e-14)
    otr = np.trace(oGL, axis1=2, axis2=3)
    assert approx_err(trL, otr) < 1e-12
    assert approx_err(trG, np.trace(oGG, axis1=2, axis2=3)) < 1e-12


@pytest.mark.parametrize("precision", ["c64", "mixed"])
@pytest.mark.parametrize("N", [4, 12, 24, 48])
def test_dyson_keldysh_reduced_precision(gpu_ops, orc, precision, N):
    NE, Nk = 33, 2
    eps, h, SR, SL, SG = dyson_inputs(200 + N, NE, Nk, N)
    GR, GL, GG, _ = gpu_ops.dyson_keldysh(eps, h, SR, SL, SG, precision=precision)
    oGR = orc.retarded_green(eps, h, SR)[0]
    tol = 2e-5 if precision == "mixed" else 5e-5
    assert GR.dtype == np.complex64
    assert approx_err(GR, oGR) < tol
    assert approx_err(GL, orc.keldysh_green(oGR, SL)) < tol
    assert approx_err(GG, orc.keldysh_green(oGR, SG)) < tol


def test_dyson_scalar_lorentzian_on_gpu(gpu_ops):
    # test/physics/scalar_dyson_and_spectral_identity.jl:4-21 through the C ABI
    eps = np.linspace(-1.0, 1.0, 2001)
    Estar, Gam = 0.17, 0.08
    h = np.full((1, 1, 1), Estar, dtype=complex)
    SR = np.full((len(eps), 1, 1, 1), -0.5j * Gam, order="F")
    GR = gpu_ops.retarded_green(eps, h, SR)
    A = (1j * (GR - np.conj(GR)))[:, 0, 0, 0].real
    exact = Gam / ((eps - Estar) ** 2 + (Gam / 2) ** 2)
    assert np.linalg.norm(A - exact) <= 2e-13 * np.linalg.norm(exact)


def test_dyson_singular_block_raises(gpu_ops):
    from qclb200 import SingularException

    eps = np.linspace(0, 1, 5)
    h = np.zeros((1, 3, 3), dtype=complex)
    SR = np.zeros((5, 1, 3, 3), dtype=complex, order="F")
    SR[:, 0] = np.diag([0.0, 0.0, 0.0])
    # eps[0] = 0 with h = 0 and SR = 0 gives D = 0: scale 0 -> SingularException(0)
    with pytest.raises(SingularException) as ex:
        gpu_ops.retarded_green(eps, h, SR)
    assert ex.value.k == 0
    # a rank-deficient (but non-zero) block: D = ones(3, 3), whose first
    # elimination step leaves a zero column -> LAPACK getrf info = 2
    SR2 = np.zeros((5, 1, 3, 3), dtype=complex, order="F")
    for e in range(5):
        SR2[e, 0] = eps[e] * np.eye(3) - np.ones((3, 3))
    with pytest.raises(SingularException) as ex:
        gpu_ops.retarded_green(eps, h, SR2)
    assert ex.value.k == 2
    # D = diag(1, 2, 0) at every energy: the third pivot is zero -> info = 3
    SR3 = np.zeros((5, 1, 3, 3), dtype=complex, order="F")
    for e in range(5):
        SR3[e, 0] = eps[e] * np.eye(3) - np.diag([1.0, 2.0, 0.0])
    with pytest.raises(SingularException) as ex:
        gpu_ops.retarded_green(eps, h, SR3)
    assert ex.value.k == 3


@pytest.mark.parametrize("precision", ["c128", "c64", "mixed"])
@pytest.mark.parametrize("N", [20, 24])
def test_dyson_singular_block_pivot_index_at_padded_24(gpu_ops, N, precision):
    """SingularException(k) with LAPACK getrf's k for blocks padded to 24 x 24
    (the two-dimensional elimination in complex128 / complex64, one row per
    lane in mixed precision): a zero scale, a rank-one block and a diagonal
    block with one zero in the middle.  The energies are binary fractions and
    the rank-one block's row sum is a power of two, so that D = eps I -
    Sigma^R and its equilibration are exact in complex64 storage as well."""
    from qclb200 import SingularException

    NE = 6
    eps = 0.25 * np.arange(NE)
    h = np.zeros((1, N, N), dtype=complex)
    cases = [
        (lambda e: np.zeros((N, N)), 0),  # D = 0 at eps[0] = 0
        # rank one, D = 1 v^T with row sum 16 (v = 1 ... 1, 1/2 ... 1/2): the
        # equilibration is exact in complex64 too, so step 2 meets a zero column
        (lambda e: eps[e] * np.eye(N) - np.outer(np.ones(N), [1.0] * (32 - N) + [0.5] * (2 * N - 32)), 2),
        (lambda e: eps[e] * np.eye(N) - np.diag([float(j + 1) if j != 9 else 0.0 for j in range(N)]), 10),
    ]
    for make, k in cases:
        SR = np.zeros((NE, 1, N, N), dtype=complex, order="F")
        for e in range(NE):
            SR[e, 0] = make(e)
        with pytest.raises(SingularException) as ex:
            gpu_ops.retarded_green(eps, h, SR, precision=precision)
        assert ex.value.k == k, (N, precision, k, ex.value.k)


@pytest.mark.parametrize("NE", [37, 64, 400, 1000, 1025, 2048, 3001, 4096])
def test_fft_hilbert_c128_matches_direct_pv(gpu_ops, orc, NE):
    rng = np.random.default_rng(NE)
    ncols = 6
    eps = np.linspace(-1.3, 0.9, NE)
    w = np.full(NE, eps[1] - eps[0])
    w[[0, -1]] /= 2
    G = np.asfortranarray(rng.standard_normal((NE, ncols)) + 1j * rng.standard_normal((NE, ncols)))
    Lam, r = gpu_ops.fft_hilbert_transform(G, eps, w, return_roundoff=True)
    direct = orc.direct_hilbert(G, eps, w)
    assert approx_err(Lam, direct) < 2e-13
    assert approx_err(Lam, orc.fft_hilbert(G, eps, w)) < 2e-13
    assert math.isfinite(r) and r < 1e-12
    # roundoff agrees in magnitude with the oracle's 2L rerun
    _, ro = orc.fft_hilbert(G, eps, w, return_roundoff=True)
    assert r < 100 * ro + 1e-15
    # the transform without the roundoff rerun (its own kernel instance) gives
    # the same values
    Lam2 = gpu_ops.fft_hilbert_transform(G, eps, w)
    assert approx_err(Lam2, direct) < 2e-13
    assert np.max(np.abs(Lam2 - Lam)) <= 1e-13 * max(np.max(np.abs(Lam)), 1.0)


@pytest.mark.parametrize("NE", [2049, 3001, 4096])
def test_fft_hilbert_half_length_path_matches_oracle(gpu_ops, orc, NE):
    """L = 8192 complex128 with at least two columns per SM runs as two
    half-length transforms (even / odd frequencies): every column against the
    oracle's FFT convolution, some against the direct principal-value sum, and
    against the one-CTA kernel (the roundoff rerun) to rounding."""
    rng = np.random.default_rng(NE + 7)
    ncols = 300
    eps = np.linspace(-1.3, 0.9, NE)
    w = np.full(NE, eps[1] - eps[0])
    w[[0, -1]] /= 2
    G = np.asfortranarray(rng.standard_normal((NE, ncols)) + 1j * rng.standard_normal((NE, ncols)))
    Lam = gpu_ops.fft_hilbert_transform(G, eps, w)
    assert approx_err(Lam, orc.fft_hilbert(G, eps, w)) < 2e-13
    sub = [0, 1, 150, ncols - 1]
    assert approx_err(Lam[:, sub], orc.direct_hilbert(np.asfortranarray(G[:, sub]), eps, w)) < 2e-13
    Lam2, r = gpu_ops.fft_hilbert_transform(G, eps, w, return_roundoff=True)
    assert r < 1e-12
    assert np.max(np.abs(Lam2 - Lam)) <= 1e-13 * np.max(np.abs(Lam))


def test_retarded_self_energy_half_length_path(gpu_ops, orc):
    # the fused Gamma = i (S> - S<), SR = Lam - i Gamma / 2 through the
    # half-length kernel (N_E = 2500, L = 8192, 300 columns)
    rng = np.random.default_rng(0xFF72)
    NE, Nk, Nb = 2500, 3, 10
    eps = np.linspace(-1.3, 0.9, NE)
    w = np.full(NE, eps[1] - eps[0])
    w[[0, -1]] /= 2
    SL = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    SG = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    SR, Gam = gpu_ops.retarded_self_energy_fft(SL, SG, eps, w)
    oSR, oGam = orc.retarded_self_energy(SL, SG, eps, w, method="fft")
    assert np.array_equal(Gam, oGam)
    assert approx_err(SR, oSR) < 2e-13


@pytest.mark.parametrize("NE", [1500, 4096])
def test_fft_hilbert_in_place_on_device(gpu_ops, orc, NE):
    """Lam == Gam through the device entry: the transform of the original
    field (the half-length kernel, which reads the field twice, is not used
    for an overlapping output)."""
    import ctypes

    import torch
    from qclb200 import _lib

    rng = np.random.default_rng(NE + 1)
    ncols = 5
    eps = np.linspace(-1.3, 0.9, NE)
    w = np.full(NE, eps[1] - eps[0])
    G = rng.standard_normal((ncols, NE)) + 1j * rng.standard_normal((ncols, NE))
    dev = torch.device("cuda", 0)
    buf = torch.tensor(G, dtype=torch.complex128, device=dev)
    sep = torch.empty_like(buf)
    wd = torch.tensor(w, dtype=torch.float64, device=dev)
    P = ctypes.c_void_p
    st = P(torch.cuda.current_stream().cuda_stream)
    L = _lib.lib()
    de = float(eps[1] - eps[0])
    _lib.check(L.qcl_dev_fft_hilbert_transform(st, _lib.QCL_C128, NE, ncols, de, P(wd.data_ptr()),
                                               P(buf.data_ptr()), P(sep.data_ptr()), None))
    _lib.check(L.qcl_dev_fft_hilbert_transform(st, _lib.QCL_C128, NE, ncols, de, P(wd.data_ptr()),
                                               P(buf.data_ptr()), P(buf.data_ptr()), None))
    torch.cuda.synchronize()
    direct = orc.direct_hilbert(np.asfortranarray(G.T), eps, w)
    assert approx_err(sep.cpu().numpy().T, direct) < 2e-13
    assert approx_err(buf.cpu().numpy().T, direct) < 2e-13


@pytest.mark.parametrize("NE", [400, 4096])
def test_fft_hilbert_c64(gpu_ops, orc, NE):
    rng = np.random.default_rng(7)
    eps = np.linspace(-1.3, 0.9, NE)
    w = np.full(NE, eps[1] - eps[0])
    w[[0, -1]] /= 2
    G = np.asfortranarray(rng.standard_normal((NE, 4)) + 1j * rng.standard_normal((NE, 4)))
    Lam, r = gpu_ops.fft_hilbert_transform(G, eps, w, precision="c64", return_roundoff=True)
    assert Lam.dtype == np.complex64
    direct = orc.direct_hilbert(G, eps, w)
    assert approx_err(Lam, direct) < 1e-5
    assert r < 1e-5
    assert approx_err(gpu_ops.fft_hilbert_transform(G, eps, w, precision="c64"), direct) < 1e-5


@pytest.mark.parametrize("NE", [37, 2500])
def test_retarded_self_energy_fft_matches_oracle(gpu_ops, orc, NE):
    rng = np.random.default_rng(0xFF71)
    Nk, Nb = 2, 2
    eps = np.linspace(-1.3, 0.9, NE)
    w = np.full(NE, eps[1] - eps[0])
    w[[0, -1]] /= 2
    SL = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    SG = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    SR, Gam, r = gpu_ops.retarded_self_energy_fft(SL, SG, eps, w, return_roundoff=True)
    oSR, oGam = orc.retarded_self_energy(SL, SG, eps, w, method="direct")
    assert np.array_equal(Gam, oGam)
    assert approx_err(SR, oSR) < 2e-13
    assert r < 1e-12
    SR2, Gam2 = gpu_ops.retarded_self_energy_fft(SL, SG, eps, w)
    assert np.array_equal(Gam2, oGam)
    assert approx_err(SR2, oSR) < 2e-13


# ---------------------------------------------------------------------------
# shifts, contractions, embedding, residuals, observables
# ---------------------------------------------------------------------------

def _rand_field(rng, shape):
    return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


@pytest.mark.parametrize("delta", [0.367, -0.367, 0.3, 0.0, 3.5, 0.075])
def test_energy_shift_matches_oracle(gpu_ops, orc, delta):
    rng = np.random.default_rng(11)
    eps = np.linspace(-1.0, 2.0, 41)
    X = _rand_field(rng, (41, 3, 2, 2))
    Y = gpu_ops.apply_energy_shift(X, eps, delta)
    assert approx_err(Y, orc.ShiftPlan(eps, delta).apply(X)) < 5e-15


def test_energy_shift_rejects_aliasing(gpu_ops):
    import ctypes
    from qclb200 import _lib

    X = np.zeros((8, 1), dtype=complex, order="F")
    eps = np.linspace(0, 1, 8)
    p = ctypes.c_void_p(X.ctypes.data)
    st = _lib.lib().qcl_apply_energy_shift(0, 8, 1, ctypes.c_void_p(eps.ctypes.data), 0.1, p, p)
    assert st == _lib.QCL_ARG


@pytest.mark.parametrize("kind", ["momentum_independent", "dense", "ifr"])
@pytest.mark.parametrize("beta", [0.0, 1.0])
def test_static_contraction_matches_literal_oracle(gpu_ops, orc, kind, beta):
    from qclb200.problem import small_problem

    names = {"momentum_independent": ("acoustic",), "dense": ("impurity",), "ifr": ("IFR",)}[kind]
    pr = small_problem(NE=37, Nk=4, Nb=4, mechanisms=names)
    mech = pr.mechanisms[0]
    rng = np.random.default_rng(3)
    G = _rand_field(rng, pr.shape)
    S0 = _rand_field(rng, pr.shape)
    got = gpu_ops.production_static_contraction(mech, G, pr.wk, alpha=1.7, beta=beta, S=S0)
    lit = orc.contraction_literal(mech.literal_kernel(pr.Nk, pr.Nb), G, pr.wk, 1.7 * mech.q) + beta * S0
    assert approx_err(got, lit) < 1e-13
    got32 = gpu_ops.production_static_contraction(mech, G, pr.wk, alpha=1.7, beta=beta, S=S0, precision="c64")
    assert approx_err(got32, lit) < 1e-5


@pytest.mark.parametrize("Nb", [3, 12, 24])
def test_embedding_component_matches_oracle(gpu_ops, orc, Nb):
    rng = np.random.default_rng(Nb)
    NE, Nk = 45, 3
    eps = np.linspace(-1.0, 2.0, NE)
    T = rng.standard_normal((Nb, Nb)) + 1j * rng.standard_normal((Nb, Nb))
    G = _rand_field(rng, (NE, Nk, Nb, Nb))
    for delta in (0.5, -0.5, 0.0):
        got = gpu_ops.embedding_component(T, G, eps, delta)
        ref = orc.embedding_component(T, G, orc.ShiftPlan(eps, delta))
        assert approx_err(got, ref) < 1e-13


def _consistent_state(orc, seed, NE, Nk, Nb):
    from helpers import dyson_inputs

    eps, h, SR, SL, SG = dyson_inputs(seed, NE, Nk, Nb)
    GR = orc.retarded_green(eps, h, SR)[0]
    GL = orc.keldysh_green(GR, SL)
    GG = orc.keldysh_green(GR, SG)
    return eps, h, GR, GL, GG, (SR, SL, SG)


@pytest.mark.parametrize("Nb", [4, 12, 24])
def test_residual_suite_matches_oracle(gpu_ops, orc, Nb):
    NE, Nk = 29, 2
    eps, h, GR, GL, GG, tot = _consistent_state(orc, 50 + Nb, NE, Nk, Nb)
    rng = np.random.default_rng(5)
    cand = np.asfortranarray(tot[1] * (1 + 0.01 * rng.standard_normal(tot[1].shape)))
    ref = orc.residual_suite(eps, h, GR, GL, GG, tot, cand)
    got = gpu_ops.production_residual_suite(eps, h, GR, GL, GG, tot, cand)
    for k in ("rA", "rK"):
        assert abs(got[k] - ref[k]) <= 1e-10 * max(ref[k], 1e-14) + 1e-15, (k, got[k], ref[k])
    assert abs(got["rD"] - ref["rD"]) <= 1e-14
    assert got["rPSD"] == pytest.approx(ref["rPSD"], abs=1e-13)
    assert got["rcaus"] == pytest.approx(ref["rcaus"], abs=1e-13)


def test_residual_suite_detects_indefinite_and_acausal_blocks(gpu_ops, orc):
    NE, Nk, Nb = 17, 2, 5
    eps, h, GR, GL, GG, tot = _consistent_state(orc, 77, NE, Nk, Nb)
    SR, SL, SG = (np.array(t, order="F") for t in tot)
    SR[3, 1] += 0.3j * np.eye(Nb)        # Im SigmaR > 0 in one block: acausal
    GL2 = np.array(GL, order="F")
    GL2[5, 0, 0, 0] += 2.0j              # -i G< gains a negative eigenvalue
    ref = orc.residual_suite(eps, h, GR, GL2, GG, (SR, SL, SG), SL)
    got = gpu_ops.production_residual_suite(eps, h, GR, GL2, GG, (SR, SL, SG), SL)
    assert ref["rPSD"] > 1e-3 and ref["rcaus"] > 1e-3
    assert got["rPSD"] == pytest.approx(ref["rPSD"], rel=1e-10)
    assert got["rcaus"] == pytest.approx(ref["rcaus"], rel=1e-10)


def test_selfenergy_residual(gpu_ops, orc):
    rng = np.random.default_rng(8)
    a = _rand_field(rng, (33, 2, 3, 3))
    b = a + 0.01 * _rand_field(rng, a.shape)
    assert gpu_ops.production_selfenergy_residual(a, b) == pytest.approx(orc.relative_change(a, b), rel=1e-13)
    bad = np.array(b, order="F")
    bad[0, 0, 0, 0] = np.nan
    assert gpu_ops.production_selfenergy_residual(a, bad) == math.inf


def test_current_and_populations_match_oracle(gpu_ops, orc):
    from qclb200.problem import small_problem

    pr = small_problem(NE=41, Nk=3, Nb=4)
    rng = np.random.default_rng(21)
    SG, SL, GL, GG = (_rand_field(rng, pr.shape) for _ in range(4))
    Jbar, pops = gpu_ops.current_and_populations(pr, SG, SL, GL, GG)
    assert Jbar == pytest.approx(orc.current(pr, SG, SL, GL, GG), rel=1e-12, abs=1e-14)
    np.testing.assert_allclose(pops, orc.populations(pr, GL), rtol=1e-12, atol=1e-14)


def test_zero_bias_equilibrium_current_on_gpu(gpu_ops, orc):
    # analytic_equilibrium_..._anchors.jl:71-138 through the device reductions
    from qclb200.problem import small_problem

    pr = small_problem(NE=61, Nk=3, Nb=4)
    gamma = 0.02
    f = 1 / (np.exp(pr.eps / pr.kBT) + 1)
    SR = np.zeros(pr.shape, dtype=complex, order="F")
    SL = np.zeros(pr.shape, dtype=complex, order="F")
    SG = np.zeros(pr.shape, dtype=complex, order="F")
    for a in range(pr.Nb):
        SR[:, :, a, a] = -0.5j * gamma
        SL[:, :, a, a] = (1j * f * gamma)[:, None]
        SG[:, :, a, a] = (-1j * (1 - f) * gamma)[:, None]
    GR, GL, _, _ = gpu_ops.dyson_keldysh(pr.eps, pr.h, SR, SL)
    GG = GR - np.conj(np.transpose(GR, (0, 1, 3, 2))) + GL
    Jbar, _ = gpu_ops.current_and_populations(pr, SG, SL, GL, GG)
    assert abs(Jbar) < 2e-13


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 8, 12, 16, 17, 24, 32, 33, 48])
def test_batched_hermitian_eigvals_match_numpy(gpu_ops, n):
    rng = np.random.default_rng(n)
    X = rng.standard_normal((20, n, n)) + 1j * rng.standard_normal((20, n, n))
    H = X + np.conj(np.transpose(X, (0, 2, 1)))
    got = gpu_ops.hermitian_eigvals(H)
    ref = np.linalg.eigvalsh(H)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("NE,Nk,Nb,beta", [(37, 4, 4, 0.0), (200, 3, 3, 1.0), (129, 5, 4, 0.5)])
def test_dense_contraction_tensor_cores_c64(gpu_ops, orc, NE, Nk, Nb, beta):
    # complex64 dense contraction on tcgen05 (scaled FP16 hi/lo operands, FP32
    # accumulation) against the FP64 literal six-index map; ragged N_E and
    # N_k N_b^2 exercise the zero padding of the 128 x 256 x 32 tiles
    from qclb200.problem import small_problem

    pr = small_problem(NE=NE, Nk=Nk, Nb=Nb, mechanisms=("impurity",))
    mech = pr.mechanisms[0]
    rng = np.random.default_rng(NE + Nk)
    G = _rand_field(rng, pr.shape)
    S0 = _rand_field(rng, pr.shape)
    got = gpu_ops.production_static_contraction(mech, G, pr.wk, alpha=1.3, beta=beta, S=S0, precision="c64")
    lit = orc.contraction_literal(mech.literal_kernel(pr.Nk, pr.Nb), G, pr.wk, 1.3 * mech.q) + beta * S0
    assert got.dtype == np.complex64
    assert approx_err(got, lit) < 2e-6


def test_dense_contraction_tensor_cores_dynamic_range(gpu_ops, orc):
    # FP16 operand pairs need the per-row scale of the field and the operator
    # scale: rows from 1e-15 to 1e20, entries spread over 1e6 inside a row, an
    # operator scaled by 1e-9 (outputs stay normal FP32 numbers, >= ~1e-27);
    # every row keeps its FP32-level relative error
    from qclb200.problem import small_problem

    pr = small_problem(NE=150, Nk=3, Nb=4, mechanisms=("impurity",))
    mech = pr.mechanisms[0]
    mech.matrix = np.asfortranarray(mech.matrix * 1e-9)
    rng = np.random.default_rng(99)
    G = _rand_field(rng, pr.shape)
    G *= 10.0 ** rng.uniform(-6.0, 0.0, G.shape)
    G *= (10.0 ** rng.uniform(-15.0, 20.0, pr.NE))[:, None, None, None]
    G = np.asfortranarray(G)
    got = gpu_ops.production_static_contraction(mech, G, pr.wk, precision="c64").astype(np.complex128)
    lit = orc.contraction_literal(mech.literal_kernel(pr.Nk, pr.Nb), G, pr.wk, mech.q)
    d = (got - lit).reshape(pr.NE, -1)
    rel = np.linalg.norm(d, axis=1) / np.linalg.norm(lit.reshape(pr.NE, -1), axis=1)
    assert np.all(np.isfinite(got))
    assert float(np.max(rel)) < 2e-6


def test_dense_contraction_tensor_cores_wide_tile(gpu_ops):
    # N_E = 4736 (37 row tiles) x 1024 real columns: 256-wide tiles fill one
    # wave of 148 exactly, so the tile-width choice takes the 256 variant
    from qclb200.problem import Mechanism

    rng = np.random.default_rng(23)
    NE, Nk, Nb = 4736, 2, 16
    Nc = Nk * Nb * Nb
    M = rng.standard_normal((Nc, Nc)) + 1j * rng.standard_normal((Nc, Nc))
    G = rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb))
    wk = np.array([0.7, 1.3])
    mech = Mechanism("impurity", "dense", 0.9, matrix=np.asfortranarray(M))
    got = gpu_ops.production_static_contraction(mech, np.asfortranarray(G), wk, precision="c64")
    Gf = G.astype(np.complex64).astype(np.complex128).reshape(NE, Nc, order="F")
    Mf = M.astype(np.complex64).astype(np.complex128)
    wq = np.array([wk[q % Nk] for q in range(Nc)])  # column q = m' + Nk (c + Nb d)
    ref = 0.9 * (Gf * wq[None, :]) @ Mf.T
    assert approx_err(got.reshape(NE, Nc, order="F"), ref) < 2e-6


def test_dense_contraction_tensor_cores_no_accumulation_bias(gpu_ops):
    # a long positive sum (K = 2 N_k N_b^2 = 2048 real terms) exposes any
    # truncation bias of the tensor-core accumulation: the mean signed relative
    # error must stay at the FP32 rounding level, not grow with K
    from qclb200.problem import Mechanism

    rng = np.random.default_rng(17)
    NE, Nk, Nb = 256, 16, 8
    Nc = Nk * Nb * Nb
    M = rng.uniform(0.0, 1.0, (Nc, Nc)) + 0j
    G = rng.uniform(0.0, 1.0, (NE, Nk, Nb, Nb)).astype(np.complex64).astype(np.complex128)
    G = np.asfortranarray(G)
    mech = Mechanism("impurity", "dense", 1.0, matrix=np.asfortranarray(M))
    got = gpu_ops.production_static_contraction(mech, G, np.ones(Nk), precision="c64")
    got = got.reshape(NE, Nc, order="F").astype(np.complex128)
    ref = G.reshape(NE, Nc, order="F") @ M.astype(np.complex64).astype(np.complex128).T
    rel = (got.real - ref.real) / ref.real
    assert abs(float(np.mean(rel))) < 1e-6
    assert float(np.max(np.abs(rel))) < 3e-6
