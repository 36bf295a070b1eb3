"""The positivity witness of the residual suite (_PositivityWitness,
numerics/reference/positivity_diagnostics.jl:41-91; collected and reduced by
production_residual_suite / _production_positivity_witness,
numerics/optimized/residuals.jl:662-779).

CPU: the oracle's witness on a consistent state (the first block's spectral
function, ratio 0), on planted defects (the largest wins, ties go to the
first block in the reference's e-slow / m-fast order), and on a non-finite
block.  GPU: the same cases through the C ABI, the kind and block exactly,
the numbers to 1e-10, and the witness of a running SCBA context.
"""
import math

import numpy as np
import pytest

from helpers import dyson_inputs, psd_blocks


def _state(orc, seed, NE, Nk, Nb):
    """A Keldysh-consistent state whose six witness matrices are all
    positive semidefinite: S< = i P<, S> = -i P>, S^R = -i (P< + P>)/2 + a
    Hermitian part, G^{<,>} = G^R S^{<,>} G^A."""
    eps, h, _, _, _ = dyson_inputs(seed, NE, Nk, Nb)
    rng = np.random.default_rng(seed + 1)
    PL, PG = psd_blocks(rng, NE, Nk, Nb, 0.03), psd_blocks(rng, NE, Nk, Nb, 0.05)
    herm = 0.01 * (rng.standard_normal(PL.shape) + 1j * rng.standard_normal(PL.shape))
    herm = herm + np.conj(np.transpose(herm, (0, 1, 3, 2)))
    SR, SL, SG = (np.asfortranarray(x) for x in (-0.5j * (PL + PG) + herm, 1j * PL, -1j * PG))
    GR = orc.retarded_green(eps, h, SR)[0]
    GL = np.array(orc.keldysh_green(GR, SL), order="F")
    GG = np.array(orc.keldysh_green(GR, SG), order="F")
    return eps, h, GR, GL, GG, (SR, SL, SG)


def _cases(orc):
    NE, Nk, Nb = 17, 2, 5
    eps, h, GR, GL, GG, tot = _state(orc, 77, NE, Nk, Nb)
    out = {"clean": (eps, h, GR, GL, GG, tot)}
    GL2 = GL.copy(order="F")
    GL2[5, 0, 0, 0] -= 2.0j   # -i G< gains a negative eigenvalue at (e=5, m=0)
    GL2[9, 1, 1, 1] -= 0.5j   # a smaller one at (e=9, m=1)
    out["defects"] = (eps, h, GR, GL2, GG, tot)
    GL3 = GL.copy(order="F")
    GL3[6, 0] = GL3[5, 1] = GL[5, 1] - 1.5j * np.eye(Nb)  # identical defects: (5,1) comes first (lin 11 < 12)
    out["tie"] = (eps, h, GR, GL3, GG, tot)
    GG4 = GG.copy(order="F")
    GG4[3, 1, 2, 0] = np.nan   # non-finite unoccupied block
    out["nonfinite"] = (eps, h, GR, GL, GG4, tot)
    return out


EXPECT = {"clean": ("spectral", 0, 0), "defects": ("occupied", 5, 0), "tie": ("occupied", 5, 1),
          "nonfinite": ("unoccupied", 3, 1)}


@pytest.mark.parametrize("case", sorted(EXPECT))
def test_oracle_witness(orc, case):
    eps, h, GR, GL, GG, tot = _cases(orc)[case]
    w = orc.residual_witness(GR, GL, GG, tot)
    assert (w["matrix_kind"], w["energy_index"], w["momentum_index"]) == EXPECT[case]
    res = orc.residual_suite(eps, h, GR, GL, GG, tot, tot[1])
    if case == "nonfinite":
        assert math.isinf(w["ratio"]) and math.isnan(w["minimum_eigenvalue"]) and w["floor"] == 1e-14
        assert math.isinf(res["rPSD"])
    else:
        assert w["ratio"] == pytest.approx(res["rPSD"], rel=1e-12, abs=0)
        assert w["floor"] == w["backward_error"] == pytest.approx(64 * 5 * np.finfo(float).eps *
                                                                  max(w["block_norm"], 1.0), rel=1e-15)
        assert w["construction_scale"] == 1.0
    if case == "clean":
        assert w["ratio"] == 0.0
        A = 1j * (GR[0, 0] - GR[0, 0].conj().T)
        lam = np.linalg.eigvalsh(0.5 * (A + A.conj().T))
        assert w["minimum_eigenvalue"] == pytest.approx(lam.min(), rel=1e-12)
        assert w["block_norm"] == pytest.approx(np.abs(lam).max(), rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(EXPECT))
def test_gpu_witness_matches_oracle(gpu_ops, orc, case):
    eps, h, GR, GL, GG, tot = _cases(orc)[case]
    want = orc.residual_witness(GR, GL, GG, tot)
    got = gpu_ops.production_residual_suite(eps, h, GR, GL, GG, tot, tot[1], return_witness=True)
    w = got["witness"]
    assert (w["matrix_kind"], w["energy_index"], w["momentum_index"]) == EXPECT[case]
    for k in ("minimum_eigenvalue", "block_norm", "floor", "ratio", "absolute_defect", "relative_defect",
              "backward_error", "hermiticity_defect", "construction_scale"):
        a, b = w[k], want[k]
        if math.isnan(b):
            assert math.isnan(a), k
        elif math.isinf(b):
            assert a == b, k
        else:
            assert abs(a - b) <= 1e-10 * max(abs(b), 1e-3) + 1e-14, (k, a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["c128", "mixed"])
def test_scba_witness(gpu_ops, orc, precision):
    from qclb200.problem import small_problem
    from qclb200.scba import ProductionSCBA

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic"))
    s = ProductionSCBA(pr, precision=precision)
    s.seed()
    with pytest.raises(Exception, match="step first"):
        s.witness()
    row = s.step()
    w = s.witness()
    g = s.green()
    total = tuple(sum(s.family(f)[c].astype(np.complex128) for f in range(len(pr.mechanisms) + 2))
                  for c in range(3))
    want = orc.residual_witness(*(g[k].astype(np.complex128) for k in ("GR", "GL", "GG")), total)
    assert w["ratio"] == pytest.approx(row["r_PSD"], abs=1e-12)
    if precision == "c128":
        assert (w["matrix_kind"], w["energy_index"], w["momentum_index"]) == (
            want["matrix_kind"], want["energy_index"], want["momentum_index"])
        assert w["block_norm"] == pytest.approx(want["block_norm"], rel=1e-10)
    s.close()
