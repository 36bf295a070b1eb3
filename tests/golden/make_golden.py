"""Generates the golden input/output fixtures of tests/golden/ from the CPU
oracle (the reference itself is Julia, which this environment cannot run).

    python tests/golden/make_golden.py

Each fixture is a compressed .npz of seeded inputs and the oracle's outputs
for one operator of the SCBA hot path, small enough to check in.  They pin
the oracle (CPU regression test) and give the GPU path fixed reference
values (GPU parity test) that do not depend on re-running the oracle.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for sub in ("oracle", "qclnegf.jl_b200", "tests"):
    sys.path.insert(0, os.path.join(ROOT, sub))

import oracle as orc  # noqa: E402
from helpers import dyson_inputs  # noqa: E402


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


def dyson():
    eps, h, SR, SL, SG = dyson_inputs(2024, 23, 3, 7)
    GR, _, scale, _ = orc.retarded_green(eps, h, SR)
    save("dyson_keldysh_N7", eps=eps, h=h, SR=SR, SL=SL, SG=SG, GR=GR, GL=orc.keldysh_green(GR, SL),
         GG=orc.keldysh_green(GR, SG), scale=scale)


def hilbert():
    rng = np.random.default_rng(2025)
    NE = 300
    eps = np.linspace(-0.4, 0.8, NE)
    w = np.full(NE, eps[1] - eps[0])
    w[[0, -1]] /= 2
    G = np.asfortranarray(rng.standard_normal((NE, 5)) + 1j * rng.standard_normal((NE, 5)))
    Lam, r = orc.fft_hilbert(G, eps, w, return_roundoff=True)
    SL = np.asfortranarray(rng.standard_normal((NE, 2, 2, 2)) + 1j * rng.standard_normal((NE, 2, 2, 2)))
    SG = np.asfortranarray(rng.standard_normal((NE, 2, 2, 2)) + 1j * rng.standard_normal((NE, 2, 2, 2)))
    SR, Gam = orc.retarded_self_energy(SL, SG, eps, w, method="direct")
    save("hilbert_NE300", eps=eps, wE=w, Gam=G, Lam=Lam, roundoff=np.array(r), SL=SL, SG=SG, SR=SR, GamSE=Gam)


def shift_and_embedding():
    rng = np.random.default_rng(2026)
    NE, Nk, Nb = 31, 2, 3
    eps = np.linspace(-1.0, 2.0, NE)
    X = np.asfortranarray(rng.standard_normal((NE, Nk, Nb, Nb)) + 1j * rng.standard_normal((NE, Nk, Nb, Nb)))
    T = rng.standard_normal((Nb, Nb)) + 1j * rng.standard_normal((Nb, Nb))
    deltas = np.array([0.37, -0.37, 0.1])
    out = {"eps": eps, "X": X, "T": T, "deltas": deltas}
    for i, d in enumerate(deltas):
        out[f"shift{i}"] = orc.ShiftPlan(eps, d).apply(X)
        out[f"embed{i}"] = orc.embedding_component(T, X, orc.ShiftPlan(eps, d))
    save("shift_embedding", **out)


def contraction():
    from qclb200.problem import small_problem

    pr = small_problem(NE=19, Nk=3, Nb=3, mechanisms=("acoustic", "impurity", "IFR"))
    rng = np.random.default_rng(2027)
    G = np.asfortranarray(rng.standard_normal(pr.shape) + 1j * rng.standard_normal(pr.shape))
    out = {"G": G, "wk": pr.wk}
    for m in pr.mechanisms:
        out["sigma_" + m.name] = orc.contraction_literal(m.literal_kernel(pr.Nk, pr.Nb), G, pr.wk, 1.3 * m.q)
    save("contraction_NE19", **out)


def residuals():
    eps, h, SR, SL, SG = dyson_inputs(2028, 17, 2, 6)
    GR = orc.retarded_green(eps, h, SR)[0]
    GL = orc.keldysh_green(GR, SL)
    GG = orc.keldysh_green(GR, SG)
    rng = np.random.default_rng(2028)
    cand = np.asfortranarray(SL * (1 + 0.01 * rng.standard_normal(SL.shape)))
    GL2 = np.array(GL, order="F")
    GL2[4, 1, 0, 0] += 0.3j
    res = orc.residual_suite(eps, h, GR, GL2, GG, (SR, SL, SG), cand)
    save("residual_suite_N6", eps=eps, h=h, GR=GR, GL=GL2, GG=GG, SR=SR, SL=SL, SG=SG, cand=cand,
         **{k: np.array(v) for k, v in res.items() if np.isscalar(v)})


def scba():
    from qclb200.problem import small_problem

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic"))
    hist, _ = orc.scba(pr, 3)
    keys = ("J", "Jbar", "rSigma", "rD", "rA", "rK", "rPSD", "lam", "number")
    save("scba_small_LO_acoustic", **{k: np.array([row[k] for row in hist]) for k in keys},
         populations=np.array([row["populations"] for row in hist]))


if __name__ == "__main__":
    orc.lib()
    for fn in (dyson, hilbert, shift_and_embedding, contraction, residuals, scba):
        fn()
        print("wrote", fn.__name__)
