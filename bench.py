#!/usr/bin/env python
"""Benchmark of the SCBA hot path: the operator-level batch of the
(E, k) Green's-function solves.

Workload (one "step"): N_E x N_k = 4096 x 32 blocks of size N_b = 24 --
the batched retarded Dyson solve G^R = (E - h - Sigma^R)^-1, the Keldysh
product G^< = G^R Sigma^< G^A, and the zero-padded length-8192 FFT Hilbert
transform of Gamma over all N_k N_b^2 columns, in complex128 (FP64).  The
metric is (E, k) Green solves per second.  Inputs are seeded synthetic fields
with the stated distributions (h Hermitian block-tridiagonal, Sigma^R
negative-definite anti-Hermitian part ~1 meV, Sigma^< = i PSD ~0.5 meV);
each field is 1.2 GB, far larger than L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) every rank runs an independent
replica of the batch (the path does not shard) and `value` is the total over
ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "qclnegf.jl_b200"))

NE, NK, NB = 4096, 32, 24
E0_EV = 0.1
# Roofline accounting of the dominant kernel (Dyson + Keldysh, G^R and G^<):
# FP64 flop per block = 8 N^3 (LU + inverse) + 16 N^3 (one triple product);
# bytes per block = read Sigma^R, Sigma^< + write G^R, G^< = 4 * 16 N^2.
FLOP_PER_BLOCK = 24 * NB ** 3
BYTES_PER_BLOCK = 4 * 16 * NB * NB
# DRAM bytes (read + write) of one Dyson launch, from the ncu capture of
# `bench.py --capture dyson` with the two-dimensional elimination, the 3M DMMA
# Keldysh products and 4 blocks per CTA (N_k = 8, a quarter of the blocks:
# 604.4 MB read, 561.2 MB written) scaled by 4 to the bench launch; traffic
# grows with the block count.
DYSON_TRAFFIC_BYTES = 4 * (604.4e6 + 561.2e6)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip the variant and SCBA side measurements")
    ap.add_argument("--capture", choices=["dyson", "step", "hilbert", "scba", "tcgemm", "scba_all_mixed", "scba_all_c128",
                                          "separable", "full_physics_mixed"],
                    help="run one small case of a kernel for an ncu capture (2 launches) and exit")
    ap.add_argument("--study", choices=["full_physics_converged", "full_physics_converged_mixed",
                                        "all_mechanisms_converged", "tutorial_converged", "bias_sweep_64",
                                        "bias_sweep_small_64"],
                    help="run one long study (seconds to minutes of GPU time), print its JSON and exit: the "
                         "full-physics SCBA converged in both precisions, or a 64-point batched bias sweep "
                         "(N_b 16-48, or small structures)")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                mhz.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not mhz:
            return None
        mhz.sort()
        return {"sm_mhz": mhz[len(mhz) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(mhz)}


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------
def grids():
    import numpy as np
    from qclb200.problem import energy_grid

    eps, wE = energy_grid(-0.05 / E0_EV, 0.35 / E0_EV, NE)
    return eps, wE


def device_inputs(torch, dev, N, seed, cdt):
    """Sigma^R, Sigma^<, Gamma as E-fastest (Julia-layout) device fields."""
    import numpy as np
    from qclb200.problem import operator_batch_hamiltonian

    h, wk, _ = operator_batch_hamiltonian(N, NK, seed=seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)

    def psd(scale):
        out = torch.empty((N, N, NK, NE), dtype=cdt, device=dev)
        chunk = 4  # momenta per chunk keeps the temporaries small
        for m0 in range(0, NK, chunk):
            X = torch.randn((chunk * NE, N, N), dtype=torch.complex128, device=dev, generator=g)
            P = (X @ X.mH) * (scale / N)
            # batch index (m, e) -> element (e, m, a, b) at [b, a, m, e]
            out[:, :, m0:m0 + chunk, :] = P.reshape(chunk, NE, N, N).permute(3, 2, 0, 1).to(cdt)
            del X, P
        return out

    PR = psd(0.01)  # ~1 meV broadening (solver units E0 = 0.1 eV)
    SR = (-1j) * PR
    SL = 1j * psd(0.005)
    Gam = (2.0 * PR).contiguous()  # i (SR - SR^H) = 2 P
    hf = torch.from_numpy(np.asfortranarray(h).ravel(order="F").copy()).to(dev)
    return hf, SR.contiguous(), SL.contiguous(), Gam


def cpu_inputs(N, m_count, seed):
    """The same distributions on the host, for m_count momenta."""
    import numpy as np
    from qclb200.problem import operator_batch_hamiltonian

    h, wk, _ = operator_batch_hamiltonian(N, NK, seed=seed)
    h = np.asfortranarray(h[:m_count])
    rng = np.random.default_rng(seed)

    def psd(scale):
        # batch (m, e) of N x N blocks -> Julia layout (e, m, a, b)
        X = rng.standard_normal((m_count, NE, N, N)) + 1j * rng.standard_normal((m_count, NE, N, N))
        P = (X @ np.conj(np.swapaxes(X, -1, -2))) * (scale / N)
        return np.asfortranarray(np.transpose(P, (1, 0, 2, 3)))

    PR = psd(0.01)
    return h, np.asfortranarray(-1j * PR), np.asfortranarray(1j * psd(0.005)), np.asfortranarray(2 * PR)


# ---------------------------------------------------------------------------
# CPU path (the reference algorithm on the host cores: the oracle port)
# ---------------------------------------------------------------------------
def cpu_step(orc, eps, wE, h, SR, SL, Gam, threads):
    """One step of the reference's production path on the host cores:
    LAPACK inverse + lesser sandwich per (E, k) block, pocketfft Hilbert of
    every column (the oracle's production restatements)."""
    orc.production_green_lapack(eps, h, SR, SL, threads=threads)
    orc.production_fft_hilbert_pocketfft(Gam, eps, wE, threads=threads)


CPU_KIND_DETAIL = ("port of the reference production path: per-block inverse and products with LAPACK/BLAS "
                   "(numpy, OpenBLAS), zero-padded FFT Hilbert with pocketfft (scipy.fft), threads over slabs")


def cpu_rate(m_count=NK, reps=1, warm=0):
    """Green solves/s of the CPU baseline on m_count momenta (all energies)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    eps, wE = grids()
    h, SR, SL, Gam = cpu_inputs(NB, m_count, seed=11)
    for _ in range(warm):
        cpu_step(orc, eps, wE, h, SR, SL, Gam, cores())
    t = []
    for _ in range(reps):
        t0 = time.perf_counter()
        cpu_step(orc, eps, wE, h, SR, SL, Gam, cores())
        t.append(time.perf_counter() - t0)
    t.sort()
    sec = t[len(t) // 2]
    return NE * m_count / sec, sec


def cpu_scba_tutorial(iters=2):
    """ms per SCBA iteration of the CPU port (the oracle's SCBA loop: C kernels
    with OpenMP) on the tutorial-scale problem (N_E x N_k = 400 x 16, N_b = 12,
    roundoff check on), after a seed and one iteration."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "qclnegf.jl_b200"))
    import oracle as orc
    from qclb200.problem import tutorial_problem

    pr = tutorial_problem()
    _, st = orc.scba(pr, 1, keep_state=True)
    t0 = time.perf_counter()
    orc.scba(pr, iters, state=st)
    return (time.perf_counter() - t0) / iters * 1e3


def sampled_parity(torch, eps, wE, h, SR, SL, GR, GL, Gam, Lam, nblk=64, ncol=32, seed=0):
    """Parity of a benchmarked batch against the oracle on a fixed random
    sample: `nblk` (e, k) blocks of G^R and G^< (oracle retarded_green /
    keldysh_green on the same, possibly complex64-rounded, inputs) and `ncol`
    Hilbert columns (oracle fft_hilbert).  Device fields are Julia-layout
    tensors of shape (N, N, N_k, N_E); Gam / Lam are (columns, N_E).  Returns
    the largest relative errors (Julia isapprox norm)."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    rng = np.random.default_rng(seed)
    N, nk, ne = SR.shape[1], SR.shape[2], SR.shape[3]
    es = torch.as_tensor(rng.integers(0, ne, nblk), device=SR.device)
    ms = torch.as_tensor(rng.integers(0, nk, nblk), device=SR.device)

    def blocks(X):  # (nblk, a, b) complex128 on the host
        return X[:, :, ms, es].permute(2, 1, 0).to(torch.complex128).cpu().numpy()

    sr, sl, gr, gl = (blocks(X) for X in (SR, SL, GR, GL))

    def rel(x, y):
        d = max(np.linalg.norm(x), np.linalg.norm(y))
        return 0.0 if d == 0 else float(np.linalg.norm(x - y) / d)

    eg, el = 0.0, 0.0
    for i in range(nblk):
        e, m = int(es[i]), int(ms[i])
        f = lambda a: np.asfortranarray(a.reshape((1, 1, N, N)))
        oGR = orc.retarded_green(eps[e:e + 1], np.asfortranarray(h[m:m + 1]), f(sr[i]))[0]
        oGL = orc.keldysh_green(oGR, f(sl[i]))
        eg = max(eg, rel(gr[i], oGR[0, 0]))
        el = max(el, rel(gl[i], oGL[0, 0]))
    cols = torch.as_tensor(rng.integers(0, Gam.shape[0] if Gam.dim() == 2 else Gam.numel() // ne, ncol),
                           device=Gam.device)
    G2, L2 = Gam.reshape(-1, ne), Lam.reshape(-1, ne)
    gam = np.asfortranarray(G2[cols].to(torch.complex128).cpu().numpy().T)
    lam = L2[cols].to(torch.complex128).cpu().numpy().T
    olam = orc.fft_hilbert(gam, eps, wE)
    eh = max(rel(lam[:, j], olam[:, j]) for j in range(ncol))
    return {"GR_max_rel_err": eg, "GL_max_rel_err": el, "hilbert_max_rel_err": eh, "blocks": nblk,
            "hilbert_columns": ncol, "oracle": "oracle.retarded_green / keldysh_green / fft_hilbert (FP64)"}


def cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo", timeout=datetime.timedelta(seconds=120))
        return dist, dist.get_rank(), ws
    return None, 0, 1


def max_over_ranks(dist, value, device=None):
    """The slowest rank's time: the job is done when every replica is."""
    if not dist:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(ws, units_per_rank, ms):
    """Whole-job throughput: units of all ranks over the slowest rank's time."""
    return ws * units_per_rank / (ms / 1e3)


def run_reference(args):
    dist, rank, ws = dist_init(args)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    eps, wE = grids()
    h, SR, SL, Gam = cpu_inputs(NB, NK, seed=11)  # the full batch: 32 momenta x 4096 energies
    th = cores()
    for _ in range(args.warmup):
        cpu_step(orc, eps, wE, h, SR, SL, Gam, th)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_step(orc, eps, wE, h, SR, SL, Gam, th)
    sec = (time.perf_counter() - t0) / args.steps
    rate = NE * NK / sec
    full_ms = sec * 1e3
    sample = f"the full batch ({NK} momenta x {NE} energies, {NK * NB * NB} Hilbert columns) every step; {CPU_KIND_DETAIL}"
    line = {
        "impl": "reference", "metric": "(E,k) Green solves/s", "value": rate, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": full_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 (complex128)",
        "data": "synthetic", "config": {"workload": f"operator batch N_E x N_k = {NE} x {NK}, N_b = {NB}, "
                                                    "Dyson + Keldysh G^< + FFT Hilbert (L = 8192)"},
        "cpu_baseline": {"value": rate, "unit": "solves/s", "cores": th, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import numpy as np
    import torch

    from qclb200 import _lib

    dist, rank, ws = dist_init(args)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = _lib.lib()
    P = ctypes.c_void_p
    prec = _lib.QCL_C128
    cdt = torch.complex128
    eps, wE = grids()
    de = float(eps[1] - eps[0])
    eps_d = torch.tensor(eps, dtype=torch.float64, device=dev)
    wE_d = torch.tensor(wE, dtype=torch.float64, device=dev)
    hf, SR, SL, Gam = device_inputs(torch, dev, NB, seed=7 + rank, cdt=cdt)
    GR = torch.empty_like(SR)
    GL = torch.empty_like(SR)
    Lam = torch.empty_like(Gam)
    status = torch.zeros(2, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = P(stream.cuda_stream)
    ncols = NK * NB * NB
    launches = [0]
    # the project autotuner picks the Dyson kernel's CTA shape for this basis
    # class once per process (untimed, like a library's start-up tuning)
    from qclb200 import operators as _ops

    tune = _ops.autotune(NB, precision="c128", NE=NE, Nk=NK)  # tuned on the workload's own batch

    def dyson():
        st = L.qcl_dev_dyson_keldysh(sp, prec, NE, NK, NB, P(eps_d.data_ptr()), 0.0, P(hf.data_ptr()),
                                     P(SR.data_ptr()), P(SL.data_ptr()), None, P(GR.data_ptr()), P(GL.data_ptr()),
                                     None, None, None, None, P(status.data_ptr()))
        _lib.check(st)
        launches[0] += 1

    def hilbert():
        _lib.check(L.qcl_dev_fft_hilbert_transform(sp, prec, NE, ncols, de, P(wE_d.data_ptr()), P(Gam.data_ptr()),
                                                   P(Lam.data_ptr()), None))
        launches[0] += 1

    clk = ClockSampler(local).__enter__()  # samples warm-up and timed steps (both under load)
    time.sleep(0.3)
    for _ in range(max(args.warmup, 3)):
        dyson()
        hilbert()
    torch.cuda.synchronize()
    if int(status[0]) != 0:
        raise RuntimeError(f"device status {status.tolist()}")
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches[0] = 0
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    if True:
        t0.record(stream)
        for i in range(args.steps):
            ev[i][0].record(stream)
            dyson()
            ev[i][1].record(stream)
            hilbert()
        t1.record(stream)
        torch.cuda.synchronize()
    clk.__exit__(None, None, None)
    total_ms = t0.elapsed_time(t1)
    dyson_ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    step_ms = total_ms / args.steps
    step_ms = max_over_ranks(dist, step_ms, dev)
    value = job_rate(ws, NE * NK, step_ms)
    gpu_launches = launches[0]

    # ---- end to end through the host-buffer C ABI (pinned host arrays) ------------
    e2e = None
    if rank == 0 or True:
        hSR = SR.cpu().pin_memory()
        hSL = SL.cpu().pin_memory()
        hGam = Gam.cpu().pin_memory()
        hGR = torch.empty_like(hSR).pin_memory()
        hGL = torch.empty_like(hSR).pin_memory()
        hLam = torch.empty_like(hGam).pin_memory()
        h_host = hf.cpu().numpy()
        eps_c = np.ascontiguousarray(eps)
        wE_c = np.ascontiguousarray(wE)

        def e2e_step():
            _lib.check(L.qcl_dyson_keldysh(prec, NE, NK, NB, P(eps_c.ctypes.data), 0.0, P(h_host.ctypes.data),
                                           P(hSR.data_ptr()), P(hSL.data_ptr()), None, P(hGR.data_ptr()),
                                           P(hGL.data_ptr()), None, None, None, None))
            _lib.check(L.qcl_fft_hilbert_transform(prec, NE, ncols, P(eps_c.ctypes.data), P(wE_c.ctypes.data),
                                                   P(hGam.data_ptr()), P(hLam.data_ptr()), None))

        e2e_step()
        torch.cuda.synchronize()
        k = max(2, min(args.steps, 5))
        if dist:
            dist.barrier()
        t = time.perf_counter()
        for _ in range(k):
            e2e_step()
        torch.cuda.synchronize()
        e2e_ms = (time.perf_counter() - t) / k * 1e3
        e2e_ms = max_over_ranks(dist, e2e_ms, dev)
        fb = NE * NK * NB * NB * 16
        e2e = {"value": job_rate(ws, NE * NK, e2e_ms), "unit": "solves/s", "h2d_bytes_per_step": 3 * fb,
               "d2h_bytes_per_step": 3 * fb, "ms_per_step": e2e_ms,
               "path": "qcl_dyson_keldysh + qcl_fft_hilbert_transform with pinned host buffers"}
        # the link bound of this path: one field each way at once over PCIe
        # (pinned buffers, two streams), times the 3 fields each way of a step
        dbuf = torch.empty_like(SR)
        s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

        def both_ways():
            with torch.cuda.stream(s_in):
                dbuf.copy_(hSR, non_blocking=True)
            with torch.cuda.stream(s_out):
                hGR.copy_(SR, non_blocking=True)
            torch.cuda.synchronize()

        both_ways()
        t = time.perf_counter()
        for _ in range(2):
            both_ways()
        link_ms = 3 * (time.perf_counter() - t) / 2 * 1e3
        e2e["link_bound_ms_per_step"] = link_ms
        e2e["frac_of_link_bound"] = link_ms / e2e_ms
        del dbuf
        # parity of this very run: GPU G^< equals the device-resident result
        diff = float((hGL.to(dev) - GL).abs().max().item())
        e2e["max_abs_diff_vs_device_run"] = diff
        del hSR, hSL, hGam, hGR, hGL, hLam

    try:
        parity = sampled_parity(torch, eps, wE, hf.cpu().numpy().reshape((NB, NB, NK)).transpose(2, 1, 0), SR, SL,
                                GR, GL, Gam, Lam)
    except Exception as ex:  # noqa: BLE001
        parity = {"error": repr(ex)}
    peak, peak_kind = measured_peaks()
    achieved_gbs = BYTES_PER_BLOCK * NE * NK / (dyson_ms / 1e3) / 1e9
    achieved_tflops = FLOP_PER_BLOCK * NE * NK / (dyson_ms / 1e3) / 1e12
    fp64_nominal = 148 * 64 * 2 * 1.965e9 / 1e12
    line = {
        "metric": "(E,k) Green solves/s", "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (complex128)", "data": "synthetic (seeded)",
        "config": {"workload": f"operator batch N_E x N_k = {NE} x {NK}, N_b = {NB}: Dyson G^R + Keldysh G^< + "
                               f"FFT Hilbert of Gamma (L = 8192, {ncols} columns)",
                   "l2": "inputs larger than L2 (each field 1.2 GB)", "parallelism": f"replicas x{ws}"},
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak, "traffic": DYSON_TRAFFIC_BYTES,
                     "traffic_source": "ncu dram__bytes_read+write of the N_k = 8 capture x 4",
                     "algorithmic_bytes": BYTES_PER_BLOCK * NE * NK, "kernel": "dyson_keldysh_kernel",
                     "kernel_ms": dyson_ms, "peak_kind": peak_kind,
                     "fp64_tflops": achieved_tflops, "fp64_nominal_tflops": fp64_nominal,
                     "fp64_frac_of_nominal": achieved_tflops / fp64_nominal},
        "gpu_launches": gpu_launches,
        "e2e": e2e,
        "parity": parity,
        "autotune": {"dyson_bpc": tune["chosen"], "default_bpc": tune["default"], "ms_per_bpc": tune["ms"]},
    }
    # ---- CPU baseline on the host cores (rank 0, N = 1) ------------------------------
    if ws == 1:
        try:
            rate, sec = cpu_rate(m_count=NK, reps=3, warm=1)
            line["cpu_baseline"] = {"value": rate, "unit": "solves/s", "cores": cores(), "kind": "port",
                                    "sample": f"the full batch ({NK} momenta x {NE} energies), median of 3 "
                                              f"after 1 warm-up, {sec:.2f} s per batch; {CPU_KIND_DETAIL}"}
            line["cpu_baseline"]["scba_tutorial_N12"] = {
                "ms_per_iter": cpu_scba_tutorial(), "kind": "port", "cores": cores(),
                "sample": "2 SCBA iterations of the tutorial problem (N_E x N_k = 400 x 16, N_b = 12, roundoff "
                          "check on) after a seed and 1 iteration; compare extras.scba_tutorial_N12_30iter"}
        except Exception as ex:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "error": str(ex)}
    line["clocks"] = clk.summary()
    if rank == 0:
        if not args.no_extras and ws == 1:
            try:
                line["extras"] = extras(torch, dev, L, _lib)
            except Exception as ex:  # noqa: BLE001
                line["extras"] = {"error": repr(ex)}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def extras(torch, dev, L, _lib):
    """Side measurements: the operator batch (Dyson + Keldysh, and the L = 8192
    Hilbert transform of every column) in complex64 / mixed and at N_b = 48,
    and SCBA iterations/s of the tutorial-scale problem (FP64 vs mixed, J
    error)."""
    import numpy as np

    P = ctypes.c_void_p
    out = {}
    eps, wE = grids()
    eps_d = torch.tensor(eps, dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev)
    sp = P(s.cuda_stream)
    for N, prec, name in ((24, _lib.QCL_C64, "c64_N24"), (24, _lib.QCL_MIXED, "mixed_N24"),
                          (48, _lib.QCL_C128, "c128_N48"), (48, _lib.QCL_MIXED, "mixed_N48")):
        cdt = torch.complex128 if prec == _lib.QCL_C128 else torch.complex64
        hf, SR, SL, _ = device_inputs(torch, dev, N, seed=3, cdt=cdt)
        GR = torch.empty_like(SR)
        GL = torch.empty_like(SR)
        st = torch.zeros(2, dtype=torch.int32, device=dev)

        def call():
            _lib.check(L.qcl_dev_dyson_keldysh(sp, prec, NE, NK, N, P(eps_d.data_ptr()), 0.0, P(hf.data_ptr()),
                                               P(SR.data_ptr()), P(SL.data_ptr()), None, P(GR.data_ptr()),
                                               P(GL.data_ptr()), None, None, None, None, P(st.data_ptr())))

        # the batch's Hilbert transform at the storage precision: Gamma of every
        # (m, a, b) column, L = 8192
        hprec = _lib.QCL_C128 if prec == _lib.QCL_C128 else _lib.QCL_C64
        ncols = NK * N * N
        g = torch.Generator(device=dev)
        g.manual_seed(5)
        Gam = torch.randn((ncols, NE), dtype=cdt, device=dev, generator=g)
        Lam = torch.empty_like(Gam)
        wE_d = torch.tensor(wE, dtype=torch.float64, device=dev)

        def hilbert():
            _lib.check(L.qcl_dev_fft_hilbert_transform(sp, hprec, NE, ncols, float(eps[1] - eps[0]),
                                                       P(wE_d.data_ptr()), P(Gam.data_ptr()), P(Lam.data_ptr()),
                                                       None))

        times = {}
        for key, fn in (("dyson_keldysh_ms", call), ("hilbert_ms", hilbert)):
            for _ in range(3):
                fn()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            for _ in range(5):
                fn()
            b.record(s)
            torch.cuda.synchronize()
            times[key] = a.elapsed_time(b) / 5
        ms = times["dyson_keldysh_ms"]
        out[name] = {"dyson_keldysh_ms": ms, "solves_per_s": NE * NK / (ms / 1e3), "hilbert_ms": times["hilbert_ms"],
                     "step_solves_per_s": NE * NK / ((ms + times["hilbert_ms"]) / 1e3),
                     "hilbert_columns": ncols}
        try:
            hh = hf.cpu().numpy().reshape((N, N, NK)).transpose(2, 1, 0)
            out[name]["parity"] = sampled_parity(torch, eps, wE, hh, SR, SL, GR, GL, Gam, Lam, seed=N + prec)
        except Exception as ex:  # noqa: BLE001
            out[name]["parity"] = {"error": repr(ex)}
        del SR, SL, GR, GL, Gam, Lam
        torch.cuda.empty_cache()
    # SCBA iterations/s at tutorial scale
    from qclb200.problem import tutorial_problem
    from qclb200.scba import ProductionSCBA

    pr = tutorial_problem()
    res = {}
    Jref = None
    for precision in ("c128", "mixed"):
        solver = ProductionSCBA(pr, precision=precision, use_graph=True)
        solver.seed()
        rows = []
        for it in range(3):
            try:
                rows.append(solver.step())
            except Exception as ex:  # noqa: BLE001
                raise RuntimeError(f"tutorial SCBA ({precision}) iteration {it}: {ex!r}") from ex
        torch.cuda.synchronize()
        t = time.perf_counter()
        n = 27
        for _ in range(n):
            rows.append(solver.step())
        sec = (time.perf_counter() - t) / n
        J = [r["J"] for r in rows]
        res[precision] = {"iter_per_s": 1.0 / sec, "ms_per_iter": sec * 1e3, "J_final": J[-1],
                          "r_Sigma_final": rows[-1]["r_Sigma"]}
        if precision == "c128":
            Jref = J
        else:
            res[precision].update(j_error(Jref, J))
        solver.close()
    res["structure"] = ("tutorial-sized synthetic supercell (N_E x N_k = 400 x 16, N_b = 12, seeded levels and "
                        "couplings; the reference's Schroedinger/PzP basis builder is not part of the path)")
    out["scba_tutorial_N12_30iter"] = res
    import traceback

    for key, fn in (("scba_fixed_point_small", lambda: scba_fixed_point_small(torch)),
                    ("scba_all_mechanisms", lambda: scba_all_mechanisms(torch)),
                    ("scba_full_physics_N32", lambda: scba_full_physics(torch)),
                    ("bias_sweep_16", lambda: bias_sweep(torch, npoints=16, iters=12,
                                                         classes=((2, 8), (3, 8), (4, 8)),
                                                         NE_choices=(1024, 1536, 2048))),
                    ("bias_sweep_small_64", lambda: bias_sweep_small(torch))):
        try:
            out[key] = fn()
        except Exception as ex:  # noqa: BLE001
            out[key] = {"error": repr(ex), "where": traceback.format_exc(limit=4)[-600:]}
    return out


def scba_full_physics(torch, timed=(2, 4)):
    """The full-physics mixed-precision configuration at its stated size:
    N_b = 32 (4 periods x 8 states), N_E x N_k = 2048 x 64, LO (separable
    sum of the exact Froehlich kernel on 401 q_z nodes), acoustic, impurity
    (separable sum of the tabulated covariance), IFR and alloy, T = 100 K.
    FP64 and mixed precision from the same seed: seconds per iteration (CUDA
    graphs on; one untimed iteration first), the per-phase device times of
    the last iteration, the relative J difference over the same iterations,
    and the memory estimate of each context."""
    import numpy as np
    from qclb200.problem import full_physics_problem
    from qclb200.scba import ProductionSCBA, estimate_memory

    t = time.perf_counter()
    pr = full_physics_problem()
    res = {"build_s": time.perf_counter() - t,
           "terms": {m.name: int(m.radial.shape[2]) for m in pr.mechanisms if m.kind == "separable_sum"}}
    J = {}
    for precision, n in zip(("c128", "mixed"), timed):
        est = estimate_memory(pr, precision=precision)
        s = ProductionSCBA(pr, precision=precision, use_graph=True, telemetry=True)
        s.seed()
        rows = [s.step()]
        times = []
        for _ in range(n):
            t = time.perf_counter()
            rows.append(s.step())
            times.append(time.perf_counter() - t)
        s.close()
        torch.cuda.synchronize()
        sec = float(np.median(times))
        J[precision] = [r["J"] for r in rows]
        res[precision] = {"s_per_iter": sec, "iter_per_s": 1.0 / sec, "phase_ms": rows[-1]["phase_ms"],
                          "r_Sigma": [r["r_Sigma"] for r in rows], "J": J[precision],
                          "peak_memory_GB": est["peak"] / 1e9}
    res["mixed_speedup_vs_fp64"] = res["mixed"]["iter_per_s"] / res["c128"]["iter_per_s"]
    n = min(len(J["c128"]), len(J["mixed"]))
    res["J_rel_err_mixed_vs_fp64"] = max(abs(a - b) / abs(a) for a, b in zip(J["c128"][:n], J["mixed"][:n]))
    res["config"] = ("N_b = 32, N_E x N_k = 2048 x 64, LO + acoustic + impurity + IFR + alloy, T = 100 K, linear "
                     "mixing 0.5, roundoff check on; iterations after the seed, CUDA graphs on")
    return res


def bias_sweep(torch, npoints=64, iters=5, classes=((2, 8), (3, 8), (4, 8), (6, 8)),
               NE_choices=(1024, 1536, 2048, 2560, 3072, 3584, 4096), Nk=32, Nqz=401, Nphi=64,
               iterations_only=False):
    """The batched bias sweep: `npoints` bias points 20-70 mV per period over
    structure classes (periods x states; by default N_b = 16 ... 48) and
    energy grids N_E from NE_choices, N_k momenta, LO + acoustic + IFR, mixed
    precision, the Dyson CTA shape of every class from the autotuner; `iters`
    iterations per point.  The batched run (qcl_sweep_run: resident points
    in one graph launch per iteration) against the same points one after
    another (qcl_scba_step), in SCBA iterations per second, and the largest J
    difference between the two (the same kernels run, so it is zero).  Both
    wall times run from the first host-side preparation of a point to the
    last row (qcl_sweep_run's own wall time, without the preparation, is in
    batched.wall_s).  With `iterations_only` the iterations are also timed
    without context creation, seeds and graph captures: each sequential
    point runs `iters` more iterations, timed on their own, and the batched
    sweep runs again with 2 `iters` iterations per point, the difference of
    the two batched wall times being its `iters` iterations of every
    point."""
    import numpy as np
    from qclb200 import operators
    from qclb200.problem import bias_sweep_problems
    from qclb200.scba import BatchedSweep, ProductionSCBA

    t = time.perf_counter()
    pts = bias_sweep_problems(npoints=npoints, classes=classes, NE_choices=NE_choices, Nk=Nk, Nqz=Nqz, Nphi=Nphi)
    res = {"build_s": time.perf_counter() - t, "points": npoints,
           "Nb": sorted({p.Nb for p in pts}), "NE": sorted({p.NE for p in pts})}
    tune = {}
    for nb in sorted({p.Nb for p in pts}):
        tune[str(nb)] = operators.autotune(nb, precision="mixed", NE=max(p.NE for p in pts), Nk=Nk)
    res["autotune_mixed"] = tune
    torch.cuda.synchronize()
    t = time.perf_counter()
    Jseq = []
    iter_s = 0.0
    warm_s = 0.0
    for p in pts:
        s = ProductionSCBA(p, precision="mixed", use_graph=True)
        s.seed()
        torch.cuda.synchronize()
        ti = time.perf_counter()
        rows = s.run(iters)
        iter_s += time.perf_counter() - ti
        Jseq.append(rows[-1]["J"])
        if iterations_only:
            ti = time.perf_counter()
            s.run(iters)
            warm_s += time.perf_counter() - ti
        s.close()
    torch.cuda.synchronize()
    seq_s = time.perf_counter() - t
    # the batched wall time includes the host-side preparation of the point
    # structures (BatchedSweep's constructor), as the sequential one does
    torch.cuda.synchronize()
    t = time.perf_counter()
    sw = BatchedSweep(pts, precision="mixed")
    rows, n_it, stats = sw.run(iters)
    sw.close()
    torch.cuda.synchronize()
    bat_s = time.perf_counter() - t
    res["sequential"] = {"wall_s": seq_s, "iter_per_s": npoints * iters / seq_s, "iterations_only_s": iter_s}
    res["batched"] = dict(stats, iter_per_s=stats["iterations"] / bat_s, wall_with_preparation_s=bat_s)
    res["batched_speedup"] = res["batched"]["iter_per_s"] / res["sequential"]["iter_per_s"]
    # lower bound: the batched wall time (context creation and seeds included)
    # against the sequential iterations alone
    res["batched_speedup_vs_sequential_iterations_only"] = iter_s / bat_s
    if iterations_only:
        sw = BatchedSweep(pts, precision="mixed")
        _, n2, stats2 = sw.run(2 * iters)
        sw.close()
        b_s = stats2["wall_s"] - stats["wall_s"]
        res["iterations_only"] = {
            "iterations_per_point": iters, "sequential_s": warm_s, "batched_s": b_s,
            "sequential_ms_per_point_iteration": 1e3 * warm_s / (npoints * iters),
            "batched_ms_per_point_iteration": 1e3 * b_s / (npoints * iters),
            "speedup": warm_s / b_s,
            "how": "sequential: iterations after the first `iters` of each point (graphs captured); batched: "
                   "wall time of a 2 x iters sweep minus that of the iters sweep (creation, seeds and captures "
                   "cancel)"}
    res["J_max_rel_diff_batched_vs_sequential"] = max(abs(r["J"] - j) / abs(j) for r, j in zip(rows, Jseq))
    operators.autotune_reset()
    res["config"] = (f"{npoints} points, bias 20-70 mV/period, N_b in {res['Nb']}, N_E in {res['NE']}, N_k = {Nk}, "
                     f"LO + acoustic + IFR, mixed precision, {iters} iterations per point (seed and context "
                     "creation included in both wall times)")
    return res


def bias_sweep_small(torch, npoints=64, iters=30):
    """The batched sweep at the small end: 64 bias points of small
    structures (N_b = 12 and 16 as 3 x 4, 2 x 6 and 2 x 8 periods x states;
    N_E in 256 ... 512, N_k = 8; LO + acoustic + IFR, mixed), the sizes
    where one point's kernels are shortest and running the points' iteration
    graphs side by side has the most to gain; the iterations are also timed
    apart from the set-up."""
    return bias_sweep(torch, npoints=npoints, iters=iters, classes=((3, 4), (2, 6), (2, 8)),
                      NE_choices=(256, 384, 512), Nk=8, Nqz=101, Nphi=32, iterations_only=True)


def scba_fixed_point_small(torch, tol=1e-10):
    """J at the fixed point in each precision (N_E x N_k = 41 x 3, N_b = 4,
    LO + acoustic + IFR, linear mixing 0.7): FP64 converged to r_Sigma <=
    tol; mixed run to the floor of complex64 storage (the smallest r_Sigma of
    100 iterations past 1e-6); mixed then promoted to FP64 and refined to
    tol.  Relative J errors against the FP64 fixed point."""
    import dataclasses

    from qclb200.problem import small_problem
    from qclb200.scba import ProductionSCBA

    pr = dataclasses.replace(small_problem(NE=41, Nk=3, Nb=4, mechanisms=("LO", "acoustic", "IFR")), alpha=0.7)
    f = ProductionSCBA(pr, precision="c128", use_graph=True)
    f.seed()
    rf = f.run(3000, tol)
    f.close()
    m = ProductionSCBA(pr, precision="mixed", use_graph=True, refinement=True)
    m.seed()
    rm = m.run(3000, 1e-6)
    best = rm[-1]
    for _ in range(100):
        r = m.step()
        rm.append(r)
        if r["r_Sigma"] < best["r_Sigma"]:
            best = r
    m.promote()
    rr = m.run(3000, tol)
    m.close()
    Jf = rf[-1]["J"]
    return {"fp64_iterations": len(rf), "fp64_r_Sigma": rf[-1]["r_Sigma"], "J_fp64": Jf,
            "mixed_iterations": len(rm), "mixed_floor_r_Sigma": best["r_Sigma"],
            "J_rel_err_mixed_floor": abs(best["J"] - Jf) / abs(Jf),
            "refined_fp64_iterations": len(rr), "refined_r_Sigma": rr[-1]["r_Sigma"],
            "J_rel_err_refined": abs(rr[-1]["J"] - Jf) / abs(Jf)}


def j_error(Jref, J):
    """Differences of the current density J of a run against the FP64 run,
    iteration by iteration: the largest relative difference (and where it
    is: a transient J that passes near zero inflates it), the largest
    difference relative to the run's J scale max|J_FP64|, and the relative
    difference at the last iteration."""
    import numpy as np

    Jref, J = np.asarray(Jref, float), np.asarray(J, float)
    rel = np.abs(J - Jref) / np.abs(Jref)
    i = int(np.argmax(rel))
    return {"J_rel_err_vs_fp64": float(rel[i]), "J_rel_err_at_iteration": i + 1, "J_fp64_there": float(Jref[i]),
            "J_err_vs_fp64_over_J_scale": float(np.max(np.abs(J - Jref)) / np.max(np.abs(Jref))),
            "J_rel_err_vs_fp64_last": float(rel[-1])}


def scba_all_mechanisms(torch, NE_=1024, Nk_=32, Nb_=16, warm=2, timed=7):
    """SCBA iterations/s with every scattering mechanism (LO with its four
    shifts, acoustic, impurity, IFR, alloy): plain FP64 against mixed
    precision (complex64 storage, FP64 elimination and reductions, dense
    contractions on the tensor cores as scaled FP16 hi/lo pairs), and the largest relative
    difference of the current density J over the same iterations."""
    import numpy as np
    from qclb200.problem import small_problem
    from qclb200.scba import ProductionSCBA

    pr = small_problem(NE=NE_, Nk=Nk_, Nb=Nb_, mechanisms=("LO", "acoustic", "impurity", "IFR", "alloy"))
    res, J = {}, {}
    for precision in ("c128", "mixed"):
        solver = ProductionSCBA(pr, precision=precision, use_graph=True)
        solver.seed()
        rows = [solver.step() for _ in range(warm)]
        torch.cuda.synchronize()
        times = []
        for _ in range(timed):  # each step ends with its row's device-to-host copy
            t = time.perf_counter()
            rows.append(solver.step())
            times.append(time.perf_counter() - t)
        sec = float(np.median(times))
        J[precision] = np.array([r["J"] for r in rows])
        res[precision] = {"iter_per_s": 1.0 / sec, "ms_per_iter": sec * 1e3,
                          "ms_per_iter_min_max": [min(times) * 1e3, max(times) * 1e3]}
        solver.close()
    res["mixed_speedup_vs_fp64"] = res["mixed"]["iter_per_s"] / res["c128"]["iter_per_s"]
    err = j_error(J["c128"], J["mixed"])
    res["J_rel_err_mixed_vs_fp64"] = err.pop("J_rel_err_vs_fp64")
    res.update({k.replace("_vs_fp64", "_mixed_vs_fp64"): v for k, v in err.items()})
    res["config"] = (f"N_E x N_k = {NE_} x {Nk_}, N_b = {Nb_}, LO+acoustic+impurity+IFR+alloy, "
                     f"{warm} + {timed} timed iterations per precision (median), CUDA graph on, roundoff check on")
    return res


def run_capture(kind):
    """Cases for ncu: the same kernels as the timed step on a quarter of the
    momenta (dyson: N_E x N_k = 4096 x 8, N_b = 24, c128, G^R + G^<), the full
    step three times (step: for a one-metric launch list only), 4096 Hilbert
    columns at L = 8192, or 3 tutorial SCBA iterations."""
    import torch

    from qclb200 import _lib

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    P = ctypes.c_void_p
    sp = P(torch.cuda.current_stream(dev).cuda_stream)
    eps, wE = grids()
    eps_d = torch.tensor(eps, dtype=torch.float64, device=dev)
    if kind == "dyson":
        global NK
        NK = 8
        hf, SR, SL, _ = device_inputs(torch, dev, NB, seed=1, cdt=torch.complex128)
        GR, GL = torch.empty_like(SR), torch.empty_like(SR)
        st = torch.zeros(2, dtype=torch.int32, device=dev)
        for _ in range(2):
            _lib.check(L.qcl_dev_dyson_keldysh(sp, _lib.QCL_C128, NE, NK, NB, P(eps_d.data_ptr()), 0.0,
                                               P(hf.data_ptr()), P(SR.data_ptr()), P(SL.data_ptr()), None,
                                               P(GR.data_ptr()), P(GL.data_ptr()), None, None, None, None,
                                               P(st.data_ptr())))
    elif kind == "step":
        # the bench step itself at full size (Dyson + Keldysh on 4096 x 32 blocks
        # with the built-in CTA shape, which the autotuner also picks on this
        # batch, then the Hilbert transform of all 18 432 columns), 3 times
        hf, SR, SL, Gam = device_inputs(torch, dev, NB, seed=7, cdt=torch.complex128)
        GR, GL, Lam = torch.empty_like(SR), torch.empty_like(SR), torch.empty_like(Gam)
        st = torch.zeros(2, dtype=torch.int32, device=dev)
        wE_d = torch.tensor(wE, dtype=torch.float64, device=dev)
        for _ in range(3):
            _lib.check(L.qcl_dev_dyson_keldysh(sp, _lib.QCL_C128, NE, NK, NB, P(eps_d.data_ptr()), 0.0,
                                               P(hf.data_ptr()), P(SR.data_ptr()), P(SL.data_ptr()), None,
                                               P(GR.data_ptr()), P(GL.data_ptr()), None, None, None, None,
                                               P(st.data_ptr())))
            _lib.check(L.qcl_dev_fft_hilbert_transform(sp, _lib.QCL_C128, NE, NK * NB * NB, float(eps[1] - eps[0]),
                                                       P(wE_d.data_ptr()), P(Gam.data_ptr()), P(Lam.data_ptr()),
                                                       None))
    elif kind == "hilbert":
        ncols = 4096
        g = torch.Generator(device=dev)
        g.manual_seed(1)
        Gam = torch.randn((ncols, NE), dtype=torch.complex128, device=dev, generator=g)
        Lam = torch.empty_like(Gam)
        wE_d = torch.tensor(wE, dtype=torch.float64, device=dev)
        for _ in range(2):
            _lib.check(L.qcl_dev_fft_hilbert_transform(sp, _lib.QCL_C128, NE, ncols, float(eps[1] - eps[0]),
                                                       P(wE_d.data_ptr()), P(Gam.data_ptr()), P(Lam.data_ptr()),
                                                       None))
    elif kind == "tcgemm":
        # complex64 dense contraction on the tensor cores: N_E = 1024 rows,
        # N_k N_b^2 = 16 x 16^2 = 4096 complex columns (a 1024 x 8192 x 8192
        # real GEMM of scaled FP16 hi/lo pairs, three MMA passes)
        import numpy as np
        from qclb200 import operators
        from qclb200.problem import Mechanism

        rng = np.random.default_rng(1)
        ne, nk, nb = 1024, 16, 16
        nc = nk * nb * nb
        M = np.asfortranarray(rng.standard_normal((nc, nc)) + 1j * rng.standard_normal((nc, nc)))
        G = np.asfortranarray(rng.standard_normal((ne, nk, nb, nb)) + 1j * rng.standard_normal((ne, nk, nb, nb)))
        mech = Mechanism("impurity", "dense", 1.0, matrix=M)
        for _ in range(2):
            operators.production_static_contraction(mech, G, np.ones(nk), precision="c64")
    elif kind == "separable":
        # one separable-sum contraction at a quarter of the full-physics energies:
        # N_E x N_k = 512 x 64, N_b = 32, one chunk of 8 terms, complex64 then complex128
        import numpy as np
        from qclb200 import operators
        from qclb200.problem import Mechanism

        rng = np.random.default_rng(0)
        ne, nk, nb, J = 512, 64, 32, 8
        radial = np.asfortranarray(rng.standard_normal((nk, nk, J)) + 1j * rng.standard_normal((nk, nk, J)))
        block = np.asfortranarray(rng.standard_normal((nb * nb, nb * nb, J)) + 1j * rng.standard_normal((nb * nb, nb * nb, J)))
        mech = Mechanism("impurity", "separable_sum", 1.0, radial=radial, block=block)
        G = np.asfortranarray(rng.standard_normal((ne, nk, nb, nb)) + 1j * rng.standard_normal((ne, nk, nb, nb)))
        for prec in ("c64", "c128"):
            operators.production_static_contraction(mech, G, np.ones(nk), precision=prec)
    elif kind == "full_physics_mixed":
        # the full-physics configuration (N_b = 32, N_E x N_k = 2048 x 64, five
        # mechanisms) in mixed precision: seed + 1 eager iteration, for a
        # per-kernel launch list of an iteration at the stated size (73 GB on
        # the device; for a one-pass metric list only)
        from qclb200.problem import full_physics_problem
        from qclb200.scba import ProductionSCBA

        s = ProductionSCBA(full_physics_problem(), precision="mixed", use_graph=False)
        s.seed()
        s.step()
        s.close()
    elif kind.startswith("scba_all"):
        # the all-mechanism SCBA workload of the extras (N_E x N_k = 1024 x 32,
        # N_b = 16, LO + acoustic + impurity + IFR + alloy): seed + 3 eager
        # iterations, for a per-kernel launch list of an iteration
        from qclb200.problem import small_problem
        from qclb200.scba import ProductionSCBA

        pr = small_problem(NE=1024, Nk=32, Nb=16, mechanisms=("LO", "acoustic", "impurity", "IFR", "alloy"))
        s = ProductionSCBA(pr, precision="mixed" if kind.endswith("mixed") else "c128", use_graph=False)
        s.seed()
        for _ in range(3):
            s.step()
        s.close()
    else:
        from qclb200.problem import tutorial_problem
        from qclb200.scba import ProductionSCBA

        s = ProductionSCBA(tutorial_problem(), precision="c128")
        s.seed()
        for _ in range(3):
            s.step()
        s.close()
    torch.cuda.synchronize()
    print("ok", kind)


def run_study(kind):
    import torch

    if kind == "bias_sweep_64":
        out = bias_sweep(torch)
    elif kind == "bias_sweep_small_64":
        out = bias_sweep_small(torch)
    elif kind == "tutorial_converged":
        out = tutorial_converged(torch)
    elif kind == "all_mechanisms_converged":
        out = all_mechanisms_converged(torch)
    elif kind == "full_physics_converged_mixed":
        out = full_physics_converged(torch, plain_fp64=False)
    else:
        out = full_physics_converged(torch)
    print(json.dumps(out), flush=True)


def converged_comparison(torch, pr, tol=1e-8, max_mixed=3000, max_fp64=3000, max_wall_s=2400.0,
                         max_refine_s=1200.0, plain_fp64=True, verbose=True):
    """One problem converged to r_Sigma <= tol both ways.  (1) mixed
    precision from the seed until r_Sigma stops falling (its complex64
    floor: the last 100 iterations did not get 10 % below the best before
    them), then promoted on the device
    to complex128 (qcl_scba_promote) and refined in FP64 to tol: the FP64
    fixed point J_fp.  (2) plain FP64 from the seed to tol, bounded by
    max_wall_s.  Iterations, device-synchronised wall seconds, r_Sigma
    traces, and the relative J differences against J_fp of the mixed floor
    and of plain FP64.  `verbose`: progress lines on stderr and the first
    leg's JSON on stdout before the second leg starts (the long studies)."""
    from qclb200.scba import ProductionSCBA

    out = {}

    def progress(leg, n, r):
        if verbose and n % 25 == 0:
            print(json.dumps({"leg": leg, "iteration": n, "r_Sigma": r["r_Sigma"], "J": r["J"]}), file=sys.stderr,
                  flush=True)

    t = time.perf_counter()
    m = ProductionSCBA(pr, precision="mixed", use_graph=True, refinement=True)
    m.seed()
    rm = []
    best = None
    while len(rm) < max_mixed:
        r = m.step()
        rm.append(r)
        progress("mixed", len(rm), r)
        if best is None or r["r_Sigma"] < best["r_Sigma"]:
            best = r
        if len(rm) > 100 and min(x["r_Sigma"] for x in rm[-100:]) > 0.9 * min(x["r_Sigma"] for x in rm[:-100]):
            break
    torch.cuda.synchronize()
    tm = time.perf_counter() - t
    m.promote()
    rr = []
    t1 = time.perf_counter()
    while len(rr) < max_fp64 and time.perf_counter() - t1 < max_refine_s:
        rr.append(m.step())
        progress("refine", len(rr), rr[-1])
        if rr[-1]["r_Sigma"] <= tol:
            break
    m.close()
    torch.cuda.synchronize()
    Jfp = rr[-1]["J"]
    out["mixed_then_fp64"] = {"mixed_iterations": len(rm), "mixed_wall_s": tm, "mixed_floor_r_Sigma": best["r_Sigma"],
                              "mixed_floor_J": best["J"], "fp64_iterations": len(rr),
                              "wall_s": time.perf_counter() - t, "r_Sigma": rr[-1]["r_Sigma"], "J": Jfp,
                              "converged": rr[-1]["r_Sigma"] <= tol,
                              "mixed_r_Sigma_trace": [x["r_Sigma"] for x in rm[::10]],
                              "fp64_r_Sigma_trace": [x["r_Sigma"] for x in rr[::5]]}
    out["J_rel_err_mixed_floor_vs_fp64_fixed_point"] = abs(best["J"] - Jfp) / abs(Jfp)
    out["mixed_s_per_iter"] = tm / len(rm)
    if verbose:
        print(json.dumps(out), flush=True)  # the first leg, in case the second is cut short
    if not plain_fp64:
        return out
    t = time.perf_counter()
    f = ProductionSCBA(pr, precision="c128", use_graph=True)
    f.seed()
    rf = []
    while len(rf) < max_fp64 and time.perf_counter() - t < max_wall_s:
        rf.append(f.step())
        progress("fp64", len(rf), rf[-1])
        if rf[-1]["r_Sigma"] <= tol:
            break
    f.close()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t
    out["fp64"] = {"iterations": len(rf), "wall_s": wall, "r_Sigma": rf[-1]["r_Sigma"], "J": rf[-1]["J"],
                   "converged": rf[-1]["r_Sigma"] <= tol, "s_per_iter": wall / len(rf),
                   "r_Sigma_trace": [r["r_Sigma"] for r in rf[::10]]}
    out["J_rel_diff_fp64_vs_fp64_fixed_point"] = abs(rf[-1]["J"] - Jfp) / abs(Jfp)
    if out["fp64"]["converged"]:
        out["time_to_solution_speedup"] = wall / out["mixed_then_fp64"]["wall_s"]
    return out


def full_physics_converged(torch, tol=1e-8, periods=2, states=16, alpha=0.8, coupling_ev=0.02,
                           temperature_K=300.0, max_wall_s=2700.0, **kw):
    """The full-physics configuration at its stated size and mechanisms
    (N_b = 32, N_E x N_k = 2048 x 64, all five mechanisms), converged both
    ways (converged_comparison).  The default supercell (4 periods x 8
    states, 4 meV couplings, 100 K) stalls near r_Sigma ~ 7e-3 under linear
    mixing and the 4 x 8 cell with 20 meV couplings at 300 K falls only by
    0.996 per iteration, so the study uses 2 periods x 16 states with 20 meV
    couplings at 300 K (about 0.97 per iteration at alpha = 0.8)."""
    from qclb200.problem import full_physics_problem

    pr = full_physics_problem(periods=periods, states=states, alpha=alpha, coupling_ev=coupling_ev,
                              temperature_K=temperature_K)
    out = converged_comparison(torch, pr, tol=tol, max_wall_s=max_wall_s, **kw)
    out["config"] = (f"N_b = {pr.Nb} ({periods} periods x {states} states), N_E x N_k = {pr.NE} x {pr.Nk}, "
                     f"LO + acoustic + impurity + IFR + alloy, couplings {coupling_ev * 1e3:g} meV, "
                     f"T = {temperature_K:g} K, linear mixing alpha = {alpha}, tolerance r_Sigma <= {tol}")
    return out


def tutorial_converged(torch, tol=1e-8, mixing="anderson", **kw):
    """The tutorial-scale problem (N_E x N_k = 400 x 16, N_b = 12, acoustic
    phonons, mixing 0.3) converged both ways (converged_comparison): the
    converged J of the mixed-precision floor, of the mixed run refined in
    FP64, and of plain FP64.  Under linear mixing this structure still had
    r_Sigma = 8.4e-5 after 15 000 iterations (J drifting by 1 % per 25
    iterations), so the study mixes with Anderson (history depth 5) by
    default."""
    import dataclasses

    from qclb200.problem import tutorial_problem

    pr = dataclasses.replace(tutorial_problem(), mixing=mixing)
    kw.setdefault("max_mixed", 4000)
    kw.setdefault("max_fp64", 15000)
    kw.setdefault("max_wall_s", 15.0)
    kw.setdefault("max_refine_s", 15.0)
    out = converged_comparison(torch, pr, tol=tol, **kw)
    out["config"] = ("tutorial-sized synthetic supercell, N_E x N_k = 400 x 16, N_b = 12, acoustic phonons, "
                     f"{mixing} mixing alpha = {pr.alpha}, tolerance r_Sigma <= {tol}, CUDA graphs on")
    return out


def all_mechanisms_converged(torch, tol=1e-8, alpha=0.6, **kw):
    """The all-mechanism case of the extras (N_E x N_k = 1024 x 32, N_b = 16,
    LO + acoustic + impurity + IFR + alloy, dense LO and impurity maps)
    converged both ways (converged_comparison)."""
    import dataclasses

    from qclb200.problem import small_problem

    pr = dataclasses.replace(small_problem(NE=1024, Nk=32, Nb=16,
                                           mechanisms=("LO", "acoustic", "impurity", "IFR", "alloy")), alpha=alpha)
    out = converged_comparison(torch, pr, tol=tol, **kw)
    out["config"] = ("N_E x N_k = 1024 x 32, N_b = 16, LO + acoustic + impurity + IFR + alloy (dense LO and "
                     f"impurity maps), linear mixing alpha = {alpha}, tolerance r_Sigma <= {tol}")
    return out


def main():
    args = parse()
    if args.capture:
        run_capture(args.capture)
        return
    if args.study:
        run_study(args.study)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
