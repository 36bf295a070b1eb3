"""Batched sweep of operating points (qcl_sweep_*).

Points of different basis sizes, energy grids and biases are solved
together: the points that fit the memory budget are resident at once and
one iteration of all of them is one graph launch.  GPU: every point's rows
equal those of the same point solved alone (the same kernels run, so the
results are identical), and the oracle's SCBA (1e-9, complex128); a budget
that admits one point at a time gives the same results; with a tolerance a
point leaves the batch when it converges, after the same number of
iterations as alone.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _points():
    from qclb200.problem import small_problem

    pts = []
    for i, (Nb, NE, Ep) in enumerate([(4, 41, 0.30), (6, 57, 0.25), (4, 33, 0.40), (5, 49, 0.35)]):
        pr = small_problem(seed=3 + i, NE=NE, Nk=3, Nb=Nb, mechanisms=("LO", "acoustic", "IFR"))
        pts.append(dataclasses.replace(pr, Ep=Ep, alpha=0.6))
    return pts


def _alone(pr, iters, tol=-1.0, precision="c128"):
    from qclb200.scba import ProductionSCBA

    s = ProductionSCBA(pr, precision=precision, use_graph=True)
    s.seed()
    rows = s.run(iters, tol)
    s.close()
    return rows


@pytest.mark.parametrize("budget_points", [0, 1])
def test_sweep_rows_equal_single_point_runs_and_oracle(gpu_ops, orc, budget_points):
    from qclb200.scba import BatchedSweep, estimate_memory

    pts = _points()
    budget = 0
    if budget_points:  # room for the largest point alone: fewer points resident than in the sweep
        peaks = [estimate_memory(p, precision="c128")["peak"] for p in pts]
        budget = max(peaks)
        # the admission rule: points join in order while their peaks fit what is left
        expect, i = 0, 0
        while i < len(pts):
            used, j = 0, i
            while j < len(pts) and used + peaks[j] <= budget:
                used += peaks[j]
                j += 1
            expect = max(expect, j - i)
            i = j
    sw = BatchedSweep(pts, precision="c128", memory_budget_bytes=budget)
    rows, iters, stats = sw.run(3)
    sw.close()
    assert iters == [3] * len(pts)
    assert stats["iterations"] == 3 * len(pts)
    if budget_points:
        assert stats["max_resident"] == expect < len(pts)
    else:
        assert stats["max_resident"] == len(pts) and stats["graph_launches"] >= 1
    for pr, row in zip(pts, rows):
        alone = _alone(pr, 3)[-1]
        for key in ("J", "r_Sigma", "r_D", "r_K", "lam"):
            assert row[key] == alone[key], key
        ref = orc.scba(pr, 3)[0][-1]
        assert abs(row["J"] - ref["J"]) <= 1e-9 * abs(ref["J"])
        assert abs(row["r_Sigma"] - ref["rSigma"]) <= 1e-9 * abs(ref["rSigma"])


def test_sweep_points_leave_when_converged(gpu_ops):
    from qclb200.scba import BatchedSweep

    pts = _points()
    sw = BatchedSweep(pts, precision="mixed")
    rows, iters, stats = sw.run(300, 1e-5)
    sw.close()
    for pr, row, n in zip(pts, rows, iters):
        alone = _alone(pr, 300, 1e-5, precision="mixed")
        assert n == len(alone) and row["r_Sigma"] <= 1e-5
        assert row["J"] == alone[-1]["J"]
    assert len(set(iters)) > 1 or stats["graph_builds"] >= 1
