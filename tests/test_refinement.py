"""Memory preflight and FP64 refinement of a mixed-precision SCBA.

Preflight: the estimate and refusal of build_production_cache
(numerics/optimized/production_cache.jl:475-668, 764-770) for this
library's own allocation plan -- CPU: the estimate's field count and the
dense-vs-separable operator sizes at the full-physics size (N_E x N_k =
2048 x 64, N_b = 32); GPU: a context over budget is refused before any
allocation, and a refused create leaves the device usable.

Refinement (qcl_scba_promote): a reduced-precision context finishes in
FP64.  GPU: after promote the steps equal those of an FP64 context started
from the same (exactly converted) state, and a promoted run converges to
the FP64 fixed point of the same problem.
"""
import dataclasses

import numpy as np
import pytest


def _full_physics_shapes(kind):
    """Problem shells at the full-physics size with the LO and impurity
    kernels dense or separable (arrays are not touched by the estimate)."""
    from qclb200.problem import Mechanism, SCBAProblem, energy_grid

    NE, Nk, Nb = 2048, 64, 32
    eps, wE = energy_grid(-2.0, 4.0, NE)
    N2 = Nb * Nb
    mechs = []
    for name in ("LO", "acoustic", "impurity", "IFR", "alloy"):
        if name in ("acoustic", "alloy"):
            mechs.append(Mechanism(name, "momentum_independent", 1.0, block=np.zeros((1, 1))))
        elif name == "IFR":
            mechs.append(Mechanism(name, "ifr", 1.0, left=np.zeros((1, 4)), right=np.zeros((1, 1)),
                                   radial=np.zeros((1, 1))))
        elif kind == "dense":
            mechs.append(Mechanism(name, "dense", 1.0, matrix=np.zeros((1, 1))))
        else:
            mechs.append(Mechanism(name, "separable_sum", 1.0, radial=np.zeros((1, 1, 24)), block=np.zeros((1, 1))))
    return SCBAProblem(NE=NE, Nk=Nk, Nb=Nb, eps=eps, wE=wE, wk=np.ones(Nk), h=np.zeros((Nk, Nb, Nb)),
                       Tplus=np.zeros((Nb, Nb)), Tminus=np.zeros((Nb, Nb)), Ep=0.5, hw_LO=0.367, N_LO=0.01, gs=2,
                       target=0.03, kBT=0.086, eta_seed=0.01, alpha=0.5, mechanisms=mechs)


def test_memory_estimate_full_physics_size():
    from qclb200.scba import estimate_memory

    GB = 1e9
    field128 = 2048 * 64 * 32 * 32 * 16
    dense = estimate_memory(_full_physics_shapes("dense"), precision="c128")
    sep = estimate_memory(_full_physics_shapes("separable"), precision="c128")
    # state + candidate families (5 mechanisms + 2 embedding, 3 components), G, totals, two scratch fields
    assert sep["fields"] == (6 * 7 + 8) * field128
    # two dense (N_k N_b^2)^2 complex128 operators: 2 x 68.7 GB; separable: 24 x (N_k^2 + N_b^4) entries each
    assert dense["operators"] >= 2 * (64 * 1024) ** 2 * 16
    assert sep["operators"] < 2 * 24 * (64 * 64 + 1024 ** 2) * 16 + 8 * 1024 ** 2 * 16
    assert dense["peak"] > 180 * GB > sep["peak"]
    mixed = estimate_memory(_full_physics_shapes("separable"), precision="mixed")
    refine = estimate_memory(_full_physics_shapes("separable"), precision="mixed", refinement=True)
    assert mixed["fields"] == sep["fields"] // 2
    assert refine["fields"] == sep["fields"]  # FP64-sized state for the promote
    assert refine["operators"] > mixed["operators"]  # complex128 operator copies
    assert refine["peak"] < 180 * GB
    anderson = estimate_memory(dataclasses.replace(_full_physics_shapes("separable"), mixing="anderson"),
                               precision="c128")
    assert anderson["anderson"] == 2 * 5 * 21 * field128 + anderson["anderson"] % field128


@pytest.mark.gpu
def test_preflight_refuses_before_allocating(gpu_ops):
    import torch

    from qclb200._lib import MemoryBudgetError
    from qclb200.problem import small_problem
    from qclb200.scba import ProductionSCBA, estimate_memory

    pr = small_problem(NE=33, Nk=3, Nb=4, mechanisms=("LO", "acoustic"))
    est = estimate_memory(pr, precision="c128")
    free0 = torch.cuda.mem_get_info()[0]
    with pytest.raises(MemoryBudgetError):
        ProductionSCBA(pr, precision="c128", memory_budget_bytes=est["peak"] - 1)
    s = ProductionSCBA(pr, precision="c128", memory_budget_bytes=est["peak"])  # exactly at budget: accepted
    s.seed()
    assert np.isfinite(s.step()["J"])
    s.close()
    torch.cuda.synchronize()
    assert abs(torch.cuda.mem_get_info()[0] - free0) < 64 << 20


@pytest.mark.gpu
def test_promote_continues_as_fp64_from_the_converted_state(gpu_ops):
    from qclb200._lib import ArgumentError
    from qclb200.problem import small_problem
    from qclb200.scba import ProductionSCBA

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "impurity", "IFR"))
    m = ProductionSCBA(pr, precision="mixed", refinement=True)
    m.seed()
    m.run(3)
    m.promote()
    # the committed mixed state, exactly converted
    fams = [m.family(f) for f in range(len(pr.mechanisms) + 2)]
    assert all(a.dtype == np.complex128 for comps in fams for a in comps)
    ref = ProductionSCBA(pr, precision="c128")
    for f, comps in enumerate(fams):
        for c, a in enumerate(comps):
            ref.upload(3 + 3 * f + c, a)
    got = m.run(4)
    want = ref.run(4)
    for g, w in zip(got, want):
        for key in ("J", "r_Sigma", "r_D", "r_K", "lam"):
            assert g[key] == pytest.approx(w[key], rel=1e-12, abs=1e-300)
    m.close()
    ref.close()
    plain = ProductionSCBA(pr, precision="mixed")
    plain.seed()
    with pytest.raises(ArgumentError):
        plain.promote()
    plain.close()


@pytest.mark.gpu
def test_refined_mixed_run_reaches_the_fp64_fixed_point(gpu_ops):
    from qclb200.problem import small_problem
    from qclb200.scba import ProductionSCBA

    # linear mixing 0.7 on this problem: about one decade of r_Sigma per 70 iterations
    pr = dataclasses.replace(small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "IFR")), alpha=0.7)
    f = ProductionSCBA(pr, precision="c128", use_graph=True)
    f.seed()
    rf = f.run(3000, 1e-10)
    assert rf[-1]["r_Sigma"] <= 1e-10
    m = ProductionSCBA(pr, precision="mixed", refinement=True, use_graph=True)
    m.seed()
    rm = m.run(3000, 1e-6)
    assert rm[-1]["r_Sigma"] <= 1e-6
    m.promote()
    rr = m.run(3000, 1e-10)
    assert rr[-1]["r_Sigma"] <= 1e-10
    assert abs(rr[-1]["J"] - rf[-1]["J"]) <= 1e-8 * abs(rf[-1]["J"])
    assert len(rm) + len(rr) <= len(rf) + 10  # the FP64 phase starts from the mixed fixed point
    f.close()
    m.close()


@pytest.mark.gpu
def test_mixed_fixed_point_current_within_target_without_refinement(gpu_ops):
    """The mixed-precision fixed point itself (no FP64 phase): run to the
    r_Sigma floor of complex64 storage, its J is within 1e-6 relative of the
    converged FP64 J (the error target for J at convergence)."""
    from qclb200.problem import small_problem
    from qclb200.scba import ProductionSCBA

    pr = dataclasses.replace(small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "IFR")), alpha=0.7)
    f = ProductionSCBA(pr, precision="c128", use_graph=True)
    f.seed()
    rf = f.run(3000, 1e-10)
    f.close()
    assert rf[-1]["r_Sigma"] <= 1e-10
    m = ProductionSCBA(pr, precision="mixed", use_graph=True)
    m.seed()
    rm = m.run(3000, 1e-6)
    best = rm[-1]
    for _ in range(100):  # on to the floor: the smallest r_Sigma of 100 more iterations
        r = m.step()
        if r["r_Sigma"] < best["r_Sigma"]:
            best = r
    m.close()
    assert best["r_Sigma"] <= 1e-6
    assert abs(best["J"] - rf[-1]["J"]) <= 1e-6 * abs(rf[-1]["J"])


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [False, True])
def test_phase_telemetry_times_every_phase(gpu_ops, use_graph):
    """Per-phase device times under the reference's phase names
    (production_telemetry.jl:81-200): every phase has a non-negative time,
    their sum is within the step's wall time, and telemetry leaves the
    iteration's results unchanged."""
    import time

    from qclb200.problem import small_problem
    from qclb200.scba import PHASES, ProductionSCBA

    pr = small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "IFR"))
    a = ProductionSCBA(pr, precision="c128", use_graph=use_graph, telemetry=True)
    b = ProductionSCBA(pr, precision="c128", use_graph=use_graph)
    a.seed()
    b.seed()
    assert a.initialization_ms is not None and a.initialization_ms > 0
    for _ in range(3):
        t = time.perf_counter()
        ra = a.step()
        wall_ms = (time.perf_counter() - t) * 1e3
        rb = b.step()
        assert set(ra["phase_ms"]) == set(PHASES)
        assert all(v >= 0 for v in ra["phase_ms"].values())
        assert sum(ra["phase_ms"].values()) <= wall_ms
        assert ra["J"] == rb["J"] and ra["r_Sigma"] == rb["r_Sigma"]
    a.close()
    b.close()
