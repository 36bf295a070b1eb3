"""The SCBA inner loop at fixed Hartree potential on the GPU.

Mirror of ``solve_scba_production`` (numerics/optimized/production_solver.jl:
21-846) over the C ABI ``qcl_scba_*``: the production cache and all fields
live in device memory; each iteration returns one ``SCBAIteration``-like row
(domain/types.jl:908).  The termination policy stays on the host, as in the
reference (``scba_iteration_decision``, domain/research_policy.jl:166); the
default used here stops when r_Sigma falls below a tolerance.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import check, lib
from .operators import _CDT, _prec, mechanism_struct


class _Problem(ctypes.Structure):
    _fields_ = [("NE", ctypes.c_int), ("Nk", ctypes.c_int), ("Nb", ctypes.c_int),
                ("eps", ctypes.c_void_p), ("wE", ctypes.c_void_p), ("wk", ctypes.c_void_p),
                ("h", ctypes.c_void_p), ("Tplus", ctypes.c_void_p), ("Tminus", ctypes.c_void_p),
                ("Ep", ctypes.c_double), ("hw_LO", ctypes.c_double), ("N_LO", ctypes.c_double),
                ("gs", ctypes.c_int), ("target", ctypes.c_double), ("eta_seed", ctypes.c_double),
                ("kBT", ctypes.c_double), ("alpha", ctypes.c_double), ("J0", ctypes.c_double),
                ("precision", ctypes.c_int), ("verify_roundoff", ctypes.c_int), ("nmech", ctypes.c_int),
                ("self_energy_structure", ctypes.c_int), ("transverse_momentum", ctypes.c_int),
                ("retarded_real_part", ctypes.c_int), ("elastic_retarded", ctypes.c_int),
                ("occupation_normalization", ctypes.c_int), ("mixing", ctypes.c_int),
                ("anderson_history_depth", ctypes.c_int), ("anderson_damping", ctypes.c_double),
                ("anderson_regularization", ctypes.c_double), ("memory_budget_bytes", ctypes.c_size_t),
                ("refinement", ctypes.c_int)]


class MemoryEstimate(ctypes.Structure):
    _fields_ = [(n, ctypes.c_size_t) for n in ("fields", "operators", "workspace", "anderson", "resident", "peak")]


class AndersonInfo(ctypes.Structure):
    _fields_ = [("history_depth", ctypes.c_int), ("reset_reason", ctypes.c_int),
                ("acceleration_accepted", ctypes.c_int), ("fallback", ctypes.c_int),
                ("guard_failure_code", ctypes.c_int), ("guard_first_failure", ctypes.c_longlong),
                ("coefficients_l1", ctypes.c_double)]


RESET_REASONS = ("none", "residual_increase", "coefficient_solve", "coefficient_bound", "causality_guard")

# The per-iteration phases of solve_scba_production (production_solver.jl:438-590,
# production_iteration.jl:1-65), in the order qcl_scba_phase_times reports them.
PHASES = ("dyson", "candidate_scattering", "candidate_embedding", "candidate_assembly", "residuals", "observables",
          "mixing")


# AlgorithmOptions model switches -> the C ABI's 0/1 codes (_check_algorithm_options,
# algorithm_options.jl:42-93, rejects any other symbol with an ArgumentError)
_SWITCHES = {
    "self_energy_structure": ("full", "diagonal"),
    "transverse_momentum": ("resolved", "averaged"),
    "retarded_real_part": ("kramers_kronig", "drop"),
    "elastic_retarded": ("hilbert", "direct_green"),
    "occupation_normalization": ("paired_convex", "scalar_lesser"),
    "mixing": ("linear", "anderson"),
}


def _switch_codes(problem):
    codes = []
    for name, choices in _SWITCHES.items():
        v = getattr(problem, name, choices[0])
        if v not in choices:
            raise ValueError(f"{name} must be :{choices[0]} or :{choices[1]}")
        codes.append(choices.index(v))
    return codes


class Row(ctypes.Structure):
    _fields_ = [("nu", ctypes.c_int), ("status", ctypes.c_int)] + [
        (n, ctypes.c_double) for n in ("r_D", "r_A", "r_K", "r_Sigma", "r_lambda", "lambda_", "r_PSD", "r_caus",
                                       "r_roundoff", "r_J", "r_pop", "J", "Jbar", "number", "holes",
                                       "occupied_fraction", "empty_fraction", "target_charge",
                                       "normalized_charge", "lambda_change")]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_}
        d["lam"] = d.pop("lambda_")
        return d


def _c(a, dtype=np.complex128):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


class ProductionSCBA:
    """A device-resident SCBA solve for one problem (one context = one
    ``ProductionCache`` + state; calls on one context must be serialised,
    like the reference's plans, fft_parallel.jl:16-17)."""

    def __init__(self, problem, precision="c128", verify_roundoff=True, use_graph=False, refinement=False,
                 memory_budget_bytes=0, telemetry=False):
        """refinement: a reduced-precision context that can finish in FP64
        (``promote``); memory_budget_bytes: the preflight budget (0 = the
        device's free memory); a context above it raises MemoryBudgetError
        before any allocation; telemetry: per-phase device times in every
        row (``phase_ms``) and ``initialization_ms`` after the seed."""
        self.problem = problem
        self.precision = _prec(precision)
        self._p, self._marr = self._structs(problem, verify_roundoff, refinement, memory_budget_bytes)
        h = ctypes.c_void_p()
        check(lib().qcl_scba_create(ctypes.byref(self._p), self._marr, ctypes.byref(h)))
        self._h = h
        if use_graph:
            check(lib().qcl_scba_use_graph(self._h, 1))
        self.telemetry = bool(telemetry)
        if telemetry:
            check(lib().qcl_scba_use_telemetry(self._h, 1))
        self.mu = None
        self.initialization_ms = None

    def phase_times(self):
        """{phase: device ms} of the last step, and the seed's
        :initialization time (the phase_begin / phase_end pairs of
        production_telemetry.jl:81-200)."""
        ms = np.zeros(len(PHASES))
        init = ctypes.c_double()
        check(lib().qcl_scba_phase_times(self._h, ctypes.c_void_p(ms.ctypes.data), ctypes.byref(init)))
        return dict(zip(PHASES, ms.tolist())), init.value

    def _structs(self, problem, verify_roundoff, refinement, memory_budget_bytes):
        pr = problem
        self._keep = [np.ascontiguousarray(pr.eps, dtype=np.float64), np.ascontiguousarray(pr.wE, dtype=np.float64),
                      np.ascontiguousarray(pr.wk, dtype=np.float64), _c(pr.h), _c(pr.Tplus), _c(pr.Tminus)]
        ptr = [ctypes.c_void_p(a.ctypes.data) for a in self._keep]
        self._p = _Problem(pr.NE, pr.Nk, pr.Nb, *ptr, float(pr.Ep), float(pr.hw_LO), float(pr.N_LO), int(pr.gs),
                           float(pr.target), float(pr.eta_seed), float(pr.kBT), float(pr.alpha), float(pr.J0),
                           self.precision, 1 if verify_roundoff else 0, len(pr.mechanisms), *_switch_codes(pr),
                           int(getattr(pr, "anderson_history_depth", 5)), float(getattr(pr, "anderson_damping", 1.0)),
                           float(getattr(pr, "anderson_regularization", 1e-12)), int(memory_budget_bytes),
                           1 if refinement else 0)
        self._mechs = [mechanism_struct(m) for m in pr.mechanisms]
        arr = (type(self._mechs[0]) * max(len(self._mechs), 1))(*self._mechs) if self._mechs else None
        return self._p, arr

    def close(self):
        if getattr(self, "_h", None):
            lib().qcl_scba_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def promote(self):
        """Finish in FP64: the state converts exactly to complex128 and the
        following steps run in complex128 (a refinement context only)."""
        check(lib().qcl_scba_promote(self._h))
        self.precision = _prec("c128")

    def seed(self):
        mu = ctypes.c_double()
        check(lib().qcl_scba_seed(self._h, ctypes.byref(mu)))
        self.mu = mu.value
        if self.telemetry:
            self.initialization_ms = self.phase_times()[1]
        return self.mu

    def step(self):
        r = Row()
        check(lib().qcl_scba_step(self._h, ctypes.byref(r)))
        d = r.as_dict()
        d["populations"] = self.populations()
        if self.telemetry:
            d["phase_ms"] = self.phase_times()[0]
        return d

    def run(self, iterations, tol_sigma=-1.0):
        rows = []
        for _ in range(iterations):
            d = self.step()
            rows.append(d)
            if d["status"] != 0 or d["r_Sigma"] <= tol_sigma:
                break
        return rows

    def populations(self):
        out = np.zeros(self.problem.Nb)
        check(lib().qcl_scba_populations(self._h, ctypes.c_void_p(out.ctypes.data)))
        return out

    def download(self, which):
        out = np.zeros(self.problem.shape, dtype=_CDT[self.precision], order="F")
        check(lib().qcl_scba_download(self._h, int(which), ctypes.c_void_p(out.ctypes.data)))
        return out

    def download_candidate(self, which):
        """A family field of the last step's mixed candidate
        (1 - alpha) Sigma + alpha Phi(Sigma)."""
        out = np.zeros(self.problem.shape, dtype=_CDT[self.precision], order="F")
        check(lib().qcl_scba_download_candidate(self._h, int(which), ctypes.c_void_p(out.ctypes.data)))
        return out

    def upload(self, which, array):
        a = _c(array, _CDT[self.precision])
        check(lib().qcl_scba_upload(self._h, int(which), ctypes.c_void_p(a.ctypes.data)))

    def green(self):
        return dict(GR=self.download(0), GL=self.download(1), GG=self.download(2))

    def green_state(self):
        """The derived GreenState fields of the last Dyson solve: A, the
        condition numbers cond_2(D) and the Dyson scales, (N_E, N_k) each
        (_green_state_production, production_operators.jl:1387-1415)."""
        pr = self.problem
        A = np.zeros(pr.shape, dtype=_CDT[self.precision], order="F")
        kappa = np.zeros((pr.NE, pr.Nk), order="F")
        scale = np.zeros((pr.NE, pr.Nk), order="F")
        check(lib().qcl_scba_green_state(self._h, ctypes.c_void_p(A.ctypes.data), ctypes.c_void_p(kappa.ctypes.data),
                                         ctypes.c_void_p(scale.ctypes.data)))
        return dict(A=A, condition_number=kappa, dyson_scale=scale)

    def retarget(self, *, Ep=None, N_LO=None, kBT=None, h=None, q=None):
        """A new operating point on the resident cache and state
        (retarget_problem + retarget_production_cache,
        composition/operating_point.jl:25-170).  Unspecified values are kept;
        self.problem is replaced by the retargeted copy."""
        import dataclasses

        pr = self.problem
        mechs = list(pr.mechanisms)
        if q is not None:
            q = [float(v) for v in q]
            if len(q) != len(mechs):
                raise ValueError("one kernel scale per mechanism is required")
            mechs = [dataclasses.replace(m, q=v) for m, v in zip(mechs, q)]
        new = dataclasses.replace(pr, Ep=pr.Ep if Ep is None else float(Ep),
                                  N_LO=pr.N_LO if N_LO is None else float(N_LO),
                                  kBT=pr.kBT if kBT is None else float(kBT),
                                  h=pr.h if h is None else _c(h), mechanisms=mechs)
        harr = None if h is None else _c(h)
        qarr = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        check(lib().qcl_scba_retarget(self._h, float(new.Ep), float(new.N_LO), float(new.kBT),
                                      None if harr is None else ctypes.c_void_p(harr.ctypes.data),
                                      None if qarr is None else ctypes.c_void_p(qarr.ctypes.data)))
        self.problem = new
        return new

    def density_matrix(self):
        """rho_ab = sum wE wk G<_ab of the last Dyson solve (N_b x N_b)."""
        n = self.problem.Nb
        rho = np.zeros((n, n), dtype=np.complex128, order="F")
        check(lib().qcl_scba_density_matrix(self._h, ctypes.c_void_p(rho.ctypes.data)))
        return rho

    def mixer_info(self):
        """Anderson mixer diagnostics of the last step."""
        info = AndersonInfo()
        check(lib().qcl_scba_mixer_info(self._h, ctypes.byref(info)))
        d = {n: getattr(info, n) for n, _ in info._fields_}
        d["reset_reason"] = RESET_REASONS[info.reset_reason]
        return d

    def witness(self):
        """The positivity witness of the last step's residual suite."""
        from .operators import PsdWitness

        w = PsdWitness()
        check(lib().qcl_scba_witness(self._h, ctypes.byref(w)))
        return w.as_dict()

    def family(self, f):
        """(SigmaR, Sigma<, Sigma>) of family f: 0..M-1 mechanisms, M plus, M+1 minus."""
        return tuple(self.download(3 + 3 * f + c) for c in range(3))


def estimate_memory(problem, precision="c128", refinement=False, verify_roundoff=True):
    """The device bytes a context for `problem` would allocate
    (qcl_scba_estimate_memory): fields, operators, workspace, anderson,
    resident, peak."""
    tmp = ProductionSCBA.__new__(ProductionSCBA)
    tmp.precision = _prec(precision)
    p, arr = tmp._structs(problem, verify_roundoff, refinement, 0)
    est = MemoryEstimate()
    check(lib().qcl_scba_estimate_memory(ctypes.byref(p), arr, ctypes.byref(est)))
    return {n: int(getattr(est, n)) for n, _ in est._fields_}


def solve_scba_production(problem, iterations, *, precision="c128", verify_roundoff=True, tol_sigma=-1.0,
                          use_graph=False):
    """Seed + up to `iterations` SCBA steps; returns (history, solver)."""
    s = ProductionSCBA(problem, precision=precision, verify_roundoff=verify_roundoff, use_graph=use_graph)
    s.seed()
    return s.run(iterations, tol_sigma), s


class BatchedSweep:
    """A batched sweep of independent operating points (qcl_sweep_*): the
    points that fit the memory budget together are resident at once and one
    iteration of all of them is one CUDA graph launch (their captured
    iterations as child graphs).  The reference solves a bias sweep point by
    point, re-using basis and kernels (retarget_problem,
    composition/operating_point.jl:25-170)."""

    def __init__(self, problems, precision="mixed", verify_roundoff=True, memory_budget_bytes=0):
        self.problems = list(problems)
        self._holders = []
        structs, mech_arrays = [], []
        for pr in self.problems:
            h = ProductionSCBA.__new__(ProductionSCBA)
            h.precision = _prec(precision)
            p, arr = h._structs(pr, verify_roundoff, False, 0)
            self._holders.append((h, p, arr))
            structs.append(p)
            mech_arrays.append(arr)
        n = len(structs)
        self._parr = (_Problem * n)(*structs)
        self._marr = (ctypes.c_void_p * n)(*[ctypes.cast(a, ctypes.c_void_p) if a is not None else None
                                               for a in mech_arrays])
        handle = ctypes.c_void_p()
        check(lib().qcl_sweep_create(n, ctypes.byref(self._parr), ctypes.byref(self._marr),
                                     int(memory_budget_bytes), ctypes.byref(handle)))
        self._h = handle

    def run(self, max_iter, tol_sigma=-1.0):
        """Runs every point; returns (last rows, iteration counts, stats)."""
        n = len(self.problems)
        rows = (Row * n)()
        iters = (ctypes.c_int * n)()
        stats = (ctypes.c_double * 5)()
        check(lib().qcl_sweep_run(self._h, int(max_iter), float(tol_sigma), ctypes.byref(rows), ctypes.byref(iters),
                                  ctypes.byref(stats)))
        st = dict(zip(("wall_s", "iterations", "graph_launches", "max_resident", "graph_builds"), list(stats)))
        return [r.as_dict() for r in rows], list(iters), st

    def close(self):
        if getattr(self, "_h", None):
            lib().qcl_sweep_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
