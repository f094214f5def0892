#!/usr/bin/env python
"""Benchmark of the SBE propagation: k-point x RK4-step throughput of one B200 (or N, one process each).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c0|c1|c3|c4] [--precision mixed|fp64]
                    [--batch B] [--impl ours|reference]

A *step* is one full solve of the workload: nt RK4 steps of every k-point plus the current J(t).
The default workload is "c2" in the mixed form: the 11-orbital TMD-like model (seed 7, 49 R cells)
on a 150 x 150 k-grid under the full pulse (nt = 4096), with complex-FP32 Wannier sums and
commutators and an FP64 state, RK4 accumulation, window velocity and k-sum.  Beside it the same
line carries the plain-FP64 solve of the same configuration (time, J error of the mixed form
against it, per-odd-harmonic intensity errors up to the cutoff) and B = 4 mixed solves (polarisation
0, 45, 90 and 135 degrees) run as one SWEBatch: per-solve time, throughput against the FP64 solo
solve, and time against FP64 solo solves of the same four angles.  --workload c1 --precision
fp64 is the 2-orbital 200 x 200 drop-in configuration.

Printed JSON line (rank 0):
  value         k-pt*RK4-steps/s of the whole job, from CUDA events around the propagation kernels
                (library stream), inputs already on the device; L2 flushed between solves.
  e2e           the same metric through the reference-facing C ABI: SWESim_restart (TB parse,
                placement, host->device tables, rho0 on the GPU) + SWESim_run_simulation +
                SWESim_get_current into host arrays, wall-clocked.
  roofline      the propagation kernel's algorithmic rate against the FP64 (plain form) or blended
                FP64+FP32 (mixed form) FMA peak measured live on the same GPU (the driver's peaks
                file has HBM and bf16 only).
  mixed_vs_fp64 (mixed form) the plain-FP64 solve's time, the speed-up, J rel-L2 and the largest
                per-odd-harmonic intensity error of the mixed form against it, and the batched figure.
  cpu_baseline  the reference's own CPU build (oracle/_ref/libwannier.so: its unmodified sources,
                with an FFT shim standing in for the absent FFTW3) on the host cores, one
                single-threaded process per core (the reference's pol_scan model); a few RK4 steps
                are timed and the rate per k-point step is extrapolated to the full pulse.

With --impl reference the line instead times that reference CPU build alone on all host cores.
For N > 1 (torchrun), every rank runs its own solve at its own polarisation angle (replicas, no
data-path collective); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "hhg-solids_b200")
sys.path.insert(0, PKG)

PULSE = dict(tmax=90.0, dt=21.97e-3, intensity=1e12, tmax_field=80.0, phi_vec=[0.0, 0.0, 0.0], **{"lambda": 3000.0})
WORKLOADS = {
    "c0": dict(model="haldane", n=60, window=5,
               desc="2-orbital Haldane-like TB (a=2.5 A, 25 R cells), 60x60 k-grid, full pulse"),
    "c1": dict(model="haldane", n=200, window=5,
               desc="2-orbital Haldane-like TB (a=2.5 A, 25 R cells), 200x200 k-grid, full pulse"),
    "c2": dict(model="tmd11_s7", n=150, window=7,
               desc="11-orbital TMD-like TB (seed 7, 49 R cells), 150x150 k-grid, full pulse"),
    "c3": dict(model=None, n=None, window=None,
               desc="batched scan: 64 solves, nw in {2,6,11} (seeds 1-3), grids {60,100,150,200}^2, 16 angles "
                    "0-180 deg, I in {0.5,1,1.5,2}e12, lambda in {2000,3000} nm (draws: seed 0)"),
    "spectrum": dict(model=None, n=None, window=None, desc="HHG spectra of 1024 solves x 3 axes (HHG_spectrum)"),
    "c4": dict(model=None, n=None, window=None,
               desc="serving: Poisson arrivals at 20 req/s (seed 0), nw in {2,6,11,12} (seeds 1-3), k-grid side "
                    "even in 60-200, polarisation uniform on the circle, I log-uniform in [3e11,3e12] W/cm^2, "
                    "C0 pulse, mixed precision, continuous batching (SWEServer)"),
}


def scan_params(n_solves: int = 64, seed: int = 0):
    """The batched-scan draws (the BASELINE batched-scan configuration)."""
    import numpy as np
    import tbgen

    rng = np.random.default_rng(seed)
    models = {2: ["haldane"], 6: ["tmd6_s1", "tmd6_s2", "tmd6_s3"], 11: ["tmd11_s1", "tmd11_s2", "tmd11_s3"]}
    out = []
    for _ in range(n_solves):
        nw = int(rng.choice([2, 6, 11]))
        model = models[nw][int(rng.integers(len(models[nw])))]
        n = int(rng.choice([60, 100, 150, 200]))
        ang = math.radians(12.0 * int(rng.integers(16)))
        p = dict(PULSE, nr1=n, nr2=n, nr3=1, path_tb=tbgen.model_path(model))
        p["intensity"] = float(rng.choice([0.5e12, 1e12, 1.5e12, 2e12]))
        p["lambda"] = float(rng.choice([2000.0, 3000.0]))
        p["pol_vec"] = np.array([math.sin(ang), math.cos(ang), 0.0])
        p["phi_vec"] = np.zeros(3)
        out.append((model, nw, p))
    return out


def serve_requests(n: int, rate: float = 20.0, seed: int = 0):
    """The serving draws: (arrival s, model, nw, param) for n Poisson arrivals."""
    import numpy as np
    import tbgen

    rng = np.random.default_rng(seed)
    models = {2: ["haldane"], 6: ["tmd6_s1", "tmd6_s2", "tmd6_s3"], 11: ["tmd11_s1", "tmd11_s2", "tmd11_s3"],
              12: ["tmd12_s1", "tmd12_s2", "tmd12_s3"]}
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for i in range(n):
        nw = int(rng.choice([2, 6, 11, 12]))
        model = models[nw][int(rng.integers(len(models[nw])))]
        side = 2 * int(rng.integers(30, 101))
        th = rng.uniform(0.0, 2.0 * math.pi)
        p = dict(PULSE, nr1=side, nr2=side, nr3=1, path_tb=tbgen.model_path(model))
        p["intensity"] = float(math.exp(rng.uniform(math.log(3e11), math.log(3e12))))
        p["pol_vec"] = np.array([math.cos(th), math.sin(th), 0.0])
        p["phi_vec"] = np.zeros(3)
        out.append((float(t[i]), model, nw, p))
    return out


def serve_stream(srv, reqs, autotune: bool, local: int):
    """Submits `reqs` to the server at their arrival times and waits for all; returns the solves, their
    (submit, admit, start, done) times, the span and the sampled clocks."""
    from pySWE import pyswe

    solves = [None] * len(reqs)
    tickets = [None] * len(reqs)
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    for i, (t_arr, model, nw, p) in enumerate(reqs):
        delay = t0 + t_arr - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        solves[i] = pyswe.SWE(pyswe.Settings(p), precision="mixed", defer_init=True, autotune=autotune)
        tickets[i] = srv.submit(solves[i])
    for tk in tickets:
        srv.wait(tk)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    times = [srv.times(tk) for tk in tickets]
    first, last = min(tm["submit"] for tm in times), max(tm["done"] for tm in times)
    return solves, times, last - first, wall, clk


def latency_report(times, reqs, span):
    """Latency (done - submit), split into queue wait (admit - submit) and service (done - admit)."""
    import numpy as np

    lat = np.array([tm["done"] - tm["submit"] for tm in times])
    wait = np.array([tm["admit"] - tm["submit"] for tm in times])
    service = np.array([tm["done"] - tm["admit"] for tm in times])

    def pct(a):
        return {"p50": float(np.percentile(a, 50)), "p95": float(np.percentile(a, 95)),
                "p99": float(np.percentile(a, 99)), "max": float(a.max()), "mean": float(a.mean())}

    n = len(times)
    return {"requests": n, "offered_load_req_per_s": n / reqs[-1][0], "solves_per_hour": 3600.0 * n / span,
            "span_s": span, "latency_s": pct(lat), "queue_wait_s": pct(wait), "service_s": pct(service)}


def run_serve(args, local: int):
    """Serving: requests submitted at their Poisson arrival times to one SWEServer (mixed form,
    continuous batching); latency = completion - submission, split into queue wait (admission -
    submission) and service (completion - admission).  Two load points: the configuration's arrival
    rate (args.rate, 20 req/s, several times what one GPU serves, so latency there is queueing) and a
    sub-capacity rate of args.low_load x the throughput measured at the first point.  Beside them the
    plain FP64 form run sequentially (setup + propagation, one solve after another) on a sample of the
    same requests."""
    import numpy as np
    import tbgen
    from pySWE import pyswe

    reqs = serve_requests(args.requests, rate=args.rate)  # generates the model files before the clock starts
    srv = pyswe.SWEServer(device=local, max_active=args.max_active, chunk_steps=args.chunk)
    # Warm-up: small requests of every orbital count.
    warm = []
    for _ in range(max(1, args.warmup // 3)):
        for model in ("haldane", "tmd6_s1", "tmd11_s1", "tmd12_s1"):
            p = dict(reqs[0][3], nr1=20, nr2=20, path_tb=tbgen.model_path(model))
            s = pyswe.SWE(pyswe.Settings(p), precision="mixed", defer_init=True)
            warm.append((s, srv.submit(s)))
    for s, tk in warm:
        srv.wait(tk)
        s.delete()
    base = srv.stats()
    solves, times, span, wall, clk = serve_stream(srv, reqs, args.autotune, local)
    high = latency_report(times, reqs, span)
    st = srv.stats()
    nt = int(PULSE["tmax"] / PULSE["dt"])
    ksteps = sum(p["nr1"] * p["nr2"] * nt for _, _, _, p in reqs)
    # The FP64 sample: requests spread evenly over the stream (its model, grid and field mix).
    m = max(1, min(args.baseline_sample, len(reqs)))
    sample = sorted({(i * len(reqs)) // m for i in range(m)})
    J_mixed = [solves[i].get_current()[1:] for i in sample]
    for s in solves:
        s.delete()
    # Sub-capacity load point: the same request mix (its own seeded draw) at low_load x the measured rate.
    low = None
    if args.low_requests > 0:
        low_rate = args.low_load * high["solves_per_hour"] / 3600.0
        reqs_low = serve_requests(args.low_requests, rate=low_rate, seed=1)
        solves_low, times_low, span_low, _, clk_low = serve_stream(srv, reqs_low, args.autotune, local)
        low = latency_report(times_low, reqs_low, span_low)
        low.update(rate_req_per_s=low_rate, seed=1, clocks=clk_low,
                   largest_solve_service_s=float(max(tm["done"] - tm["admit"] for tm in times_low)))
        for s in solves_low:
            s.delete()
    srv.close()
    # Plain FP64, sequential, on the sample.
    seq_s, seq_k, errs = 0.0, 0, []
    for (t_arr, model, nw, p), Jm in zip([reqs[i] for i in sample], J_mixed):
        a = time.perf_counter()
        s = pyswe.SWE(pyswe.Settings(dict(p)), device=local, autotune=args.autotune)
        s.run_simulation()
        J = s.get_current()[1:]
        seq_s += time.perf_counter() - a
        seq_k += p["nr1"] * p["nr2"] * nt
        s.delete()
        errs.append(float(np.linalg.norm(Jm - J) / np.linalg.norm(J)))
    n = len(reqs)
    return {
        "metric": "solves/h", "value": 3600.0 * n / span, "unit": "solves/h", "n_gpus": 1, "steps": n,
        "warmup": len(warm), "ms_per_step": 1e3 * span / n, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 commutators/Wannier sums, f64 state/RK/k-sum",
        "data": "synthetic (seeded TB models and request stream, hhg-solids_b200/tbgen.py)", "impl": "hhg-b200",
        "config": {"workload": f"c4: {WORKLOADS['c4']['desc']}", "requests": n, "rate_req_per_s": args.rate, "nt": nt,
                   "max_active": args.max_active, "chunk_steps": args.chunk,
                   "server": "SWEServer: admission by device-memory footprint, chunked continuous batching, "
                             "each running solve's launches on a stream of a pool per chunk"},
        "latency_s": high["latency_s"], "queue_wait_s": high["queue_wait_s"], "service_s": high["service_s"],
        "k_pt_rk4_steps_per_s": ksteps / span, "span_s": span, "wall_s": wall,
        "offered_load_req_per_s": high["offered_load_req_per_s"],
        "sub_capacity": low,
        "server": {k: (st[k] - base.get(k, 0) if k in ("completed", "chunks", "gpu_ms", "gap_ms", "setup_ms", "finish_ms")
                       else st[k]) for k in st},
        "fp64_sequential_sample": {"requests": len(errs), "solves_per_hour": 3600.0 * len(errs) / seq_s,
                                   "k_pt_rk4_steps_per_s": seq_k / seq_s, "s_per_solve": seq_s / len(errs)},
        "J_rel_l2_mixed_vs_fp64": {"max": max(errs), "median": statistics.median(errs)},
        "clocks": clk,
    }


def run_spectrum(args, local: int):
    """HHG spectra of many currents through the reference-facing post-processing call (HHG_spectrum:
    fftshift(fft(ifftshift(gradient(J, dt)))) of scripts/pol_scan.py:34-40): 1024 solves x 3 axes of
    4096 samples, host buffers in and out (wall-clocked)."""
    import numpy as np
    from pySWE import pyswe

    rng = np.random.default_rng(0)
    count, n = 3 * 1024, int(PULSE["tmax"] / PULSE["dt"])
    J = (rng.standard_normal((count, n)) + 1j * rng.standard_normal((count, n))).astype(np.complex128)
    for _ in range(args.warmup):
        pyswe.spectrum(J, PULSE["dt"])
    t0 = time.perf_counter()
    for _ in range(args.steps):
        S = pyswe.spectrum(J, PULSE["dt"])
    dt = (time.perf_counter() - t0) / args.steps
    ref = np.abs(np.fft.fftshift(np.fft.fft(np.fft.ifftshift(np.gradient(J[:4], PULSE["dt"], axis=1), axes=1), axis=1),
                                 axes=1)) ** 2
    err = float(np.abs(np.abs(S[:4]) ** 2 - ref).max() / ref.max())
    return {"metric": "spectra/s", "value": count / dt, "unit": "spectra/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded random currents)", "impl": "hhg-b200",
            "config": {"workload": f"spectrum: {count} currents of {n} samples (1024 solves x 3 axes), HHG_spectrum "
                                   "with host buffers"},
            "e2e": {"value": count / dt, "unit": "spectra/s", "h2d_bytes_per_step": count * n * 16,
                    "d2h_bytes_per_step": count * n * 16},
            "max_rel_err_vs_numpy_first4": err}


def batch_engine_desc() -> str:
    """What SWEBatch runs, as selected by HHG_BATCH (the library reads the same variable)."""
    if os.environ.get("HHG_BATCH") == "persistent":
        return ("SWEBatch, HHG_BATCH=persistent: one persistent work-stealing launch per kernel shape over packed "
                "(solve, virtual CTA) items, longest first (precomputed-sum shapes on their own streams), "
                "captured in one CUDA graph")
    return ("SWEBatch (default engine): every solve's launches on a stream of its own, all captured in one CUDA "
            "graph and replayed")


def run_scan(args, local: int):
    """Batched scan: the mixed form as one SWEBatch against the plain form as sequential solves."""
    import numpy as np
    from pySWE import pyswe

    draws = scan_params()
    kpts = sum(p["nr1"] * p["nr2"] for _, _, p in draws)
    t0 = time.perf_counter()
    mixed = [pyswe.SWE(pyswe.Settings(dict(p)), device=local, precision="mixed", autotune=args.autotune)
             for _, _, p in draws]
    setup_s = time.perf_counter() - t0
    nt = mixed[0].settings.nt
    batch = pyswe.SWEBatch(mixed)
    for _ in range(args.warmup):
        batch.run()
    clocks = ClockSampler(local)
    clocks.start()
    ms = []
    for _ in range(args.steps):
        batch.run()
        ms.append(batch.last_ms())
    clk = clocks.stop()
    J_mixed = [s.get_current()[1:] for s in mixed]
    batch.delete()
    for s in mixed:
        s.delete()
    # Plain FP64, 64 sequential solves.
    seq_ms, errs = 0.0, []
    for (model, nw, p), Jm in zip(draws, J_mixed):
        s = pyswe.SWE(pyswe.Settings(dict(p)), device=local, autotune=args.autotune)
        s.run_simulation()
        seq_ms += s.last_kernel_ms()
        J = s.get_current()[1:]
        errs.append(float(np.linalg.norm(Jm - J) / np.linalg.norm(J)))
        s.delete()
    batch_ms = statistics.mean(ms)
    value = kpts * nt / (batch_ms * 1e-3)
    return {
        "metric": "k-pt*RK4-steps/s", "value": value, "unit": "k-pt*RK4-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": batch_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 commutators/Wannier sums, f64 state/RK/k-sum",
        "data": "synthetic (seeded TB models, generated by hhg-solids_b200/tbgen.py)", "impl": "hhg-b200",
        "config": {"workload": f"c3: {WORKLOADS['c3']['desc']}", "solves": len(draws), "k_points_total": kpts,
                   "nt": nt, "precision": "mixed", "batch": batch_engine_desc()},
        "solves_per_hour": 3600.0 * len(draws) / (batch_ms * 1e-3),
        "fp64_sequential": {"ms": seq_ms, "value": kpts * nt / (seq_ms * 1e-3),
                            "solves_per_hour": 3600.0 * len(draws) / (seq_ms * 1e-3)},
        "speedup_vs_fp64_sequential": seq_ms / batch_ms,
        "J_rel_l2_vs_fp64": {"max": max(errs), "median": statistics.median(errs)},
        "setup_s_64_solves": setup_s, "clocks": clk,
    }



def workload_param(name: str, rank: int = 0, world: int = 1, grid: int | None = None) -> dict:
    import numpy as np
    import tbgen

    w = WORKLOADS[name]
    ang = math.pi * rank / max(world, 1)  # replicas: one polarisation angle per rank
    pol = [math.sin(ang), math.cos(ang), 0.0]
    n = grid or w["n"]
    p = dict(PULSE, nr1=n, nr2=n, nr3=1, path_tb=tbgen.model_path(w["model"]))
    p["pol_vec"] = np.array(pol)
    p["phi_vec"] = np.array(p["phi_vec"])
    return p


def flops_per_kstep(nw: int, window: int, n: int, n_op: int, n_j: int, kspace: bool = False) -> float:
    """Algorithmic FP64 flops of one k-point x RK4 step (minimal form):
    4 stages x one complex nw^3 product (Hermitian commutator), the Wannier sum of H0 and the
    field-coupled r as a separable pruned DFT over the window x window cells, the windowed velocity
    (4x4 pruned DFT) and Tr(W rho), and the RK axpys.  The k-space solver evaluates H at two new
    points per step (t + dt/2, t + dt) and its window velocity is constant (only Tr(W rho) per step)."""
    f_comm = 32.0 * nw ** 3
    f_w = 8.0 * nw * nw * n_op * window * (1.0 + window / n) * (2.0 if kspace else 1.0)
    f_j = n_j * 8.0 * nw * nw * ((0.0 if kspace else 4.0 * (1.0 + 4.0 / n)) + 1.0)
    f_rk = 12.0 * nw * nw
    return f_comm + f_w + f_j + f_rk


def flops_split_mixed(nw: int, window: int, n: int, n_op: int, n_j: int, kspace: bool = False):
    """(FP64, FP32) parts of flops_per_kstep in the mixed form: the commutators and the Wannier sums
    run in FP32; the windowed velocity, Tr(W rho) and the RK accumulation stay in FP64.  (For nw <= 2
    the mixed form runs the FP64 kernels, so everything counts as FP64.)"""
    total = flops_per_kstep(nw, window, n, n_op, n_j, kspace)
    if nw <= 2:
        return total, 0.0
    f32 = 32.0 * nw ** 3 + 8.0 * nw * nw * n_op * window * (1.0 + window / n) * (2.0 if kspace else 1.0)
    return total - f32, f32


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power)}


# ---------------------------------------------------------------- the reference's CPU build


def _ref_worker_kspace(conn, probe_path, tb, param, nt_sample):
    """One single-threaded process running the reference's own k-space solver (its compiled
    Solver_kspace, driven step by step by oracle/ref_probe.cpp: the reference has no entry point for it)."""
    import ctypes as ct

    import numpy as np

    P = ct.CDLL(probe_path)
    dp = ct.POINTER(ct.c_double)
    P.probe_kspace_new.restype = ct.c_void_p
    P.probe_kspace_new.argtypes = [ct.c_char_p, ct.c_int, ct.c_int] + [ct.c_double] * 5 + [dp, dp]
    P.probe_kspace_steps.argtypes = [ct.c_void_p, ct.c_int]
    P.probe_kspace_delete.argtypes = [ct.c_void_p]
    pol = np.ascontiguousarray(param["pol_vec"], dtype=np.float64)
    phi = np.ascontiguousarray(param["phi_vec"], dtype=np.float64)
    h = P.probe_kspace_new(tb.encode(), int(param["nr1"]), int(param["nr2"]), float(param["tmax"]), float(param["dt"]),
                           float(param["intensity"]), float(param["lambda"]), float(param["tmax_field"]),
                           pol.ctypes.data_as(dp), phi.ctypes.data_as(dp))
    conn.send("ready")
    while True:
        msg = conn.recv()
        if msg != "run":
            break
        t0 = time.perf_counter()
        P.probe_kspace_steps(h, int(nt_sample))
        conn.send(time.perf_counter() - t0)
    P.probe_kspace_delete(h)


def _ref_worker(conn, lib_path, tb, param, nt_sample):
    """One single-threaded reference process (its own SWESim), driven through the reference C ABI."""
    import ctypes as ct

    import numpy as np

    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)  # the reference prints progress to stdout
    L = ct.CDLL(lib_path)
    vp = ct.c_void_p
    L.SWESim_new.restype = vp
    L.Settings_new.restype = vp
    for name in ("SWESim_run_simulation", "SWESim_init", "SWESim_delete"):
        getattr(L, name).argtypes = [vp]
    L.SWESim_set_path_tb.argtypes = [vp, ct.c_char_p]
    L.SWESim_set_settings.argtypes = [vp, vp]
    for name in ("nr1", "nr2", "nr3"):
        getattr(L, f"Settings_set_{name}").argtypes = [vp, ct.c_int]
    for name in ("tmax", "dt", "intensity", "lambda", "tmax_field"):
        getattr(L, f"Settings_set_{name}").argtypes = [vp, ct.c_double]
    dp = ct.POINTER(ct.c_double)
    L.Settings_set_pol_vec.argtypes = [vp, dp]
    L.Settings_set_phi_vec.argtypes = [vp, dp]
    s = L.Settings_new()
    L.Settings_set_nr1(s, int(param["nr1"]))
    L.Settings_set_nr2(s, int(param["nr2"]))
    L.Settings_set_nr3(s, 1)
    L.Settings_set_tmax(s, (nt_sample + 0.5) * param["dt"])
    L.Settings_set_dt(s, param["dt"])
    L.Settings_set_intensity(s, param["intensity"])
    L.Settings_set_lambda(s, param["lambda"])
    L.Settings_set_tmax_field(s, param["tmax_field"])
    pol = np.ascontiguousarray(param["pol_vec"], dtype=np.float64)
    phi = np.ascontiguousarray(param["phi_vec"], dtype=np.float64)
    L.Settings_set_pol_vec(s, pol.ctypes.data_as(dp))
    L.Settings_set_phi_vec(s, phi.ctypes.data_as(dp))
    sim = L.SWESim_new()
    L.SWESim_set_path_tb(sim, tb.encode())
    L.SWESim_set_settings(sim, s)
    L.SWESim_init(sim)
    conn.send("ready")
    while True:
        msg = conn.recv()
        if msg != "run":
            break
        t0 = time.perf_counter()
        L.SWESim_run_simulation(sim)  # nt_sample RK4 steps (the state keeps evolving; the cost per step does not change)
        conn.send(time.perf_counter() - t0)
    L.SWESim_delete(sim)


class ReferencePool:
    """`cores` concurrent single-threaded reference solves of the workload's grid and model."""

    def __init__(self, param: dict, nt_sample: int, cores: int, solver: str = "rspace"):
        import multiprocessing as mp

        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle

        lib = oracle.ref_paths()[0 if solver == "rspace" else 1]
        if not os.path.exists(lib):
            raise FileNotFoundError(f"{os.path.relpath(lib, REPO)} (build: make -C oracle with the reference checkout)")
        os.environ["OPENBLAS_NUM_THREADS"] = "1"
        os.environ["OMP_NUM_THREADS"] = "1"
        ctx = mp.get_context("spawn")
        self.nt_sample, self.cores, self.param = nt_sample, cores, param
        self.conns, self.procs = [], []
        for _ in range(cores):
            a, b = ctx.Pipe()
            target = _ref_worker if solver == "rspace" else _ref_worker_kspace
            p = ctx.Process(target=target, args=(b, lib, param["path_tb"], param, nt_sample), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        for c in self.conns:
            if c.recv() != "ready":
                raise RuntimeError("reference worker failed")

    def step(self) -> float:
        t0 = time.perf_counter()
        for c in self.conns:
            c.send("run")
        for c in self.conns:
            c.recv()
        return time.perf_counter() - t0

    def kpoint_steps(self) -> int:
        return self.cores * self.param["nr1"] * self.param["nr2"] * self.nt_sample

    def close(self):
        for c in self.conns:
            try:
                c.send("stop")
            except Exception:
                pass
        for p in self.procs:
            p.join(timeout=10)
            if p.is_alive():
                p.terminate()


def reference_sample_steps(workload: str) -> int:
    # about 2-4 s of wall time per sample on one core of a current Xeon (measured here: 0.11 s per
    # RK4 step for c1, 6 ms for c0, 2.2 s for c2)
    return {"c0": 400, "c1": 24, "c2": 2}[workload]


REFERENCE_FFT = ("the reference's unmodified sources (oracle/_ref/libwannier.so) linked against this repository's "
                 "FP64 Stockham FFT (oracle/shim/fft_shim.c) in place of FFTW3, which is absent from this image")


def reference_sample_desc(cores: int, nt_sample: int, param: dict) -> str:
    nt = int(param["tmax"] / param["dt"])
    return (f"{cores} concurrent single-threaded processes x {nt_sample} RK4 steps of the same grid and model "
            f"(the reference's pol_scan model, one solve per core); rate per k-point step extrapolated from the "
            f"{nt_sample}-step sample to the {nt}-step pulse")


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return
    if args.workload in ("c3", "c4", "spectrum"):
        print(json.dumps({"impl": "reference", "unavailable": "the batched-scan, serving and spectrum workloads have "
                          "no reference C/C++ implementation; their CPU comparison is the c0-c2 arms"}))
        return
    param = workload_param(args.workload)
    cores = os.cpu_count() or 1
    nt_sample = reference_sample_steps(args.workload)
    line = {"metric": "k-pt*RK4-steps/s", "impl": "reference", "unit": "k-pt*RK4-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded TB model)",
            "config": {"workload": f"{args.workload}: {WORKLOADS[args.workload]['desc']}"
                       + (", mixed form (complex-FP32 Wannier sums and commutators; FP64 state, RK4 accumulation, "
                          "window velocity and k-sum)" if args.precision == "mixed" else ", plain FP64"),
                       "k_grid": [param["nr1"], param["nr2"]], "nt": int(param["tmax"] / param["dt"]),
                       "solver": args.solver,
                       "reference_arithmetic": "FP64 throughout (the reference has one form)",
                       "sample": reference_sample_desc(cores, nt_sample, param),
                       "l2": "n/a (CPU)"}}
    try:
        pool = ReferencePool(param, nt_sample, cores, args.solver)
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build not runnable: {e}"}))
        return
    try:
        for _ in range(args.warmup):
            pool.step()
        times = [pool.step() for _ in range(args.steps)]
    finally:
        pool.close()
    total = sum(times)
    value = pool.kpoint_steps() * len(times) / total
    line.update(value=value, ms_per_step=1e3 * total / len(times),
                cpu_baseline={"value": value, "unit": "k-pt*RK4-steps/s", "cores": cores, "kind": "reference",
                              "sample": line["config"]["sample"], "fft": REFERENCE_FFT},
                e2e={"value": value, "unit": "k-pt*RK4-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(line), flush=True)


def cpu_baseline(workload: str, solver: str = "rspace") -> dict:
    """Reference CPU build on the host cores, bounded sample (one warm and one timed round)."""
    param = workload_param(workload)
    cores = os.cpu_count() or 1
    nt_sample = reference_sample_steps(workload)
    try:
        pool = ReferencePool(param, nt_sample, cores, solver)
    except Exception as e:  # noqa: BLE001
        return {"value": None, "unit": "k-pt*RK4-steps/s", "cores": cores, "kind": "reference",
                "sample": f"unavailable: {e}"}
    try:
        pool.step()
        t = pool.step()
    finally:
        pool.close()
    return {"value": pool.kpoint_steps() / t, "unit": "k-pt*RK4-steps/s", "cores": cores, "kind": "reference",
            "sample": reference_sample_desc(cores, nt_sample, param) + f" ({t:.1f} s wall)", "fft": REFERENCE_FFT}


# ---------------------------------------------------------------- our arm


def harmonic_errors(J, J_ref, param):
    """Per odd harmonic (up to the cutoff, 1e-12 of the fundamental): relative error of the intensity
    of |FFT(dJ/dt)|^2, with the spectrum and order axis of the reference's scripts/pol_scan.py."""
    import numpy as np

    def spec(x):
        return np.abs(np.fft.fftshift(np.fft.fft(np.fft.ifftshift(np.gradient(x, param["dt"]))))) ** 2

    nt = len(J)
    S, S_ref = spec(J), spec(J_ref)
    dw = 2.0 * np.pi / param["tmax"]
    order = np.linspace(-nt * dw / 2.0, nt * dw / 2.0, nt) / (2.0 * np.pi * 300 / param["lambda"])
    fund = S_ref[(order > 0.5) & (order < 1.5)].sum()
    out = []
    for h in range(1, 400, 2):
        win = (order > h - 0.5) & (order < h + 0.5)
        I_ref = S_ref[win].sum()
        if not win.any() or I_ref < 1e-12 * fund:
            break
        out.append(abs(S[win].sum() - I_ref) / I_ref)
    return out


def mixed_report(J_mixed, J_fp64, param, fp64_ms, mixed_ms):
    import numpy as np

    rel = {"vector": float(np.linalg.norm(J_mixed - J_fp64) / np.linalg.norm(J_fp64))}
    for a, ax in enumerate("xyz"):
        n = np.linalg.norm(J_fp64[a])
        if n > 0:
            rel[ax] = float(np.linalg.norm(J_mixed[a] - J_fp64[a]) / n)
    axis = int(np.argmax([np.linalg.norm(J_fp64[a]) for a in range(3)]))
    errs = harmonic_errors(J_mixed[axis], J_fp64[axis], param)
    return {"J_rel_l2_vs_fp64": rel, "harmonics_checked": len(errs),
            "harmonic_intensity_max_rel_err": max(errs) if errs else None,
            "fp64_ms_per_solve": fp64_ms, "mixed_ms_per_solve": mixed_ms, "speedup_vs_fp64": fp64_ms / mixed_ms}


def kcol_executed_flops(window: int, n_op: int, n_j: int, rows_per_tile: int, kspace: bool) -> float:
    """Flops per k-point step that the column kernel (sbe_kcol.cu) executes for nw = 2 with a Hermitian
    placement and a symmetric box: the closed-form commutator (15 flops per stage); the box rows n1 > 0
    only, each pair t G(n1) + conj(t) G(n1)^+ as 2 Re(t G_ii) plus a S + i b D (16 flops per row and
    operator); the column sums G(n1 >= 0) of the tile's points (4 + 6 per row pair of window-long
    complex sums per operator), shared by the tile's rows; the current contracted after the k-sum (32
    products of a twiddle and a state value per k-point, the column's window sums and the contraction
    with them per tile and step); and the RK axpys.  The k-space solver evaluates the box at two new
    points per step and keeps its window sums."""
    h = (window - 1) // 2
    pts = 2 if kspace else 1
    box = pts * n_op * h * 16.0
    col = pts * n_op * (4 + 6 * h) * window * 8.0 / rows_per_tile
    win = 0.0 if kspace else 4 * n_j * 4 * (4 * 8.0 + 6.0) / rows_per_tile
    cur = 64.0 + win + n_j * 4 * 4 * 8.0 / rows_per_tile
    return 4 * 15.0 + box + col + cur + 12.0 * 4


def executed_form(nw: int, kernel: str, fpk: float, ms: float, nk: int, nt: int, peak: float,
                  window: int = 0, n_op: int = 0, n_j: int = 0, rows_per_tile: int = 0, kspace: bool = False):
    """The flop count of the form the kernel actually executes, where it differs from the minimal one:
    for nw = 2 the column kernel's form (kcol_executed_flops) or, in the thread-per-k-point kernel, the
    closed-form commutator of two Hermitian 2x2 matrices (sbe_herm2.cuh: 15 flops per stage instead of
    8 nw^3 = 64); or the 16 x 16 frame of the FP64 tensor-core kernel (3 k-steps x 4 blocks x 3 real
    m8n8k4 products = 18 432 flops per stage instead of 8 nw^3)."""
    if nw == 2 and kernel == "propagate_kcol_kernel" and window % 2 == 1 and rows_per_tile > 0:
        f = kcol_executed_flops(window, n_op, n_j, rows_per_tile, kspace)
        form = ("column kernel: closed-form Hermitian 2x2 commutator, Hermitian-halved box rows, current "
                "contracted after the k-sum")
    elif nw == 2 and kernel in ("propagate_kcol_kernel", "propagate_kpt_kernel"):
        f = fpk - 32.0 * nw ** 3 + 4 * 15.0
        form = "closed-form Hermitian 2x2 commutator (15 flops per stage)"
    elif kernel == "propagate_dfrag_kernel":
        f = fpk - 32.0 * nw ** 3 + 4 * 36 * 512.0
        form = "commutator on the FP64 tensor cores: 16x16 frame, 3 k-steps x 4 blocks x 3 real m8n8k4 products per stage"
    else:
        return None
    achieved = f * nk * nt / (ms * 1e-3) / 1e12
    return {"form": form, "flops_per_kstep": f, "achieved": achieved, "frac": achieved / peak if peak > 0 else None}


def load_profile_counters(workload: str, kernel: str):
    """Pipe-activity counters of this kernel on this workload from the committed ncu summary, if any."""
    name = (kernel or "").split("<")[0].replace("_kernel", "")
    path = os.path.join(REPO, "profiles", f"{name}_{workload}_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get("counters")


def load_traffic(workload: str, kernel: str):
    """DRAM bytes per launch of this kernel on this workload, from a committed ncu capture summary."""
    name = kernel or ""
    short = name.split("<")[0].replace("_kernel", "")
    if "<" in name:  # element-group kernels: one file per arithmetic type
        short += "_" + name.split("<")[1].split(",")[0].rstrip(">").strip()
    path = os.path.join(REPO, "profiles", f"{short}_{workload}_traffic.json")
    if not os.path.exists(path):
        return None, None
    with open(path) as f:
        d = json.load(f)
    return d.get("dram_bytes_per_launch"), d.get("source")


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="mixed: FP32 Wannier sums and commutators, FP64 state / RK accumulation / k-sum")
    ap.add_argument("--solver", default="rspace", choices=["rspace", "kspace"],
                    help="kspace: the reference's k-space solver (src/solver_kspace.cpp) instead of its real-space one")
    ap.add_argument("--batch", type=int, default=4, help="mixed: also time this many solves of the workload as one SWEBatch")
    ap.add_argument("--fp64-steps", type=int, default=3, help="mixed: timed plain-FP64 solves beside the mixed ones")
    ap.add_argument("--batch-steps", type=int, default=3, help="mixed: timed runs of the --batch SWEBatch")
    ap.add_argument("--autotune", action="store_true", help="time candidate tile shapes at setup (SWESim_set_autotune)")
    ap.add_argument("--requests", type=int, default=200, help="c4: requests in the arrival stream")
    ap.add_argument("--max-active", type=int, default=32, help="c4: most solves running at once")
    ap.add_argument("--chunk", type=int, default=256, help="c4: RK4 steps per scheduling chunk")
    ap.add_argument("--rate", type=float, default=20.0, help="c4: arrival rate (req/s) of the configuration")
    ap.add_argument("--low-load", type=float, default=0.8,
                    help="c4: second load point, as a fraction of the throughput measured at --rate")
    ap.add_argument("--low-requests", type=int, default=100, help="c4: requests at the second load point (0: skip)")
    ap.add_argument("--baseline-sample", type=int, default=24,
                    help="c4: requests (spread evenly over the stream) run sequentially in FP64")
    ap.add_argument("--grid", type=int, default=None,
                    help="override the k-grid side (profiling a smaller case of the same kernel)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    import numpy as np
    from pySWE import pyswe

    import ctypes as ct

    lib = ct.CDLL(pyswe.default_library())
    lib.HHG_measure_peaks.argtypes = [ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)]
    fp64_peak, fp32_peak = ct.c_double(), ct.c_double()

    if args.workload in ("c3", "c4", "spectrum"):
        if rank == 0:
            fn = {"c3": run_scan, "c4": run_serve, "spectrum": run_spectrum}[args.workload]
            print(json.dumps(fn(args, local)), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    param = workload_param(args.workload, rank, world, args.grid)
    w = WORKLOADS[args.workload]
    settings = pyswe.Settings(dict(param))
    swe = pyswe.SWE(settings, device=local, precision=args.precision, solver=args.solver, autotune=args.autotune)
    nk = param["nr1"] * param["nr2"]
    nt = settings.nt
    nw = swe.num_orb()
    n_op = 1 + sum(1 for v in param["pol_vec"] if v != 0.0)
    n_j = 2  # v_z = 0 for these 2D models; jz is returned as exact zeros

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2

    for _ in range(args.warmup):
        swe.reset()
        swe.run_simulation()
    lib.HHG_measure_peaks(ct.byref(fp64_peak), ct.byref(fp32_peak))

    clocks = ClockSampler(local)
    barrier()
    if rank == 0:
        clocks.start()
    dev_ms, prop_ms, launches = [], [], 0
    t_wall0 = time.perf_counter()
    for i in range(args.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        swe.reset()
        swe.run_simulation()
        dev_ms.append(swe.last_kernel_ms())
        prop_ms.append(swe.last_propagate_ms())
        launches += swe.last_launches()
    barrier()
    t_wall = time.perf_counter() - t_wall0
    clk = clocks.stop() if rank == 0 else None
    total_ms = max_over_ranks(sum(dev_ms))
    value = world * nk * nt * args.steps / (total_ms * 1e-3)

    # End to end through the reference-facing API with host buffers.
    e2e = None
    if not args.no_e2e:
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            swe.restart()
            swe.run_simulation()
            t_, jx, jy, jz = swe.get_current()
        barrier()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": world * nk * nt * args.steps / e2e_s, "unit": "k-pt*RK4-steps/s",
               "h2d_bytes_per_step": swe.h2d_bytes(), "d2h_bytes_per_step": 3 * nt * 16,
               "calls": "SWESim_restart + SWESim_run_simulation + SWESim_get_current", "ms_per_step": 1e3 * e2e_s / args.steps}

    shape = swe.launch_shape()
    mixed = None
    if args.precision == "mixed" and rank == 0:
        # Error and speed against the plain FP64 form of the same solve: one warm-up solve (its
        # current is the comparison), then args.fp64_steps timed solves with L2 flushed before each.
        swe.reset()
        swe.run_simulation()
        J_mixed = swe.get_current()[1:]
        ref = pyswe.SWE(pyswe.Settings(dict(param)), device=local, solver=args.solver, autotune=args.autotune)
        ref.run_simulation()
        J_fp64 = ref.get_current()[1:]
        fms = []
        for i in range(args.fp64_steps):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            ref.reset()
            ref.run_simulation()
            fms.append(ref.last_kernel_ms())
        fp64_ms = statistics.mean(fms)
        fp64_shape = ref.launch_shape()
        ref.delete()
        mixed = mixed_report(J_mixed, J_fp64, param, fp64_ms, total_ms / args.steps)
        mixed["fp64_timed_solves"] = len(fms)
        mixed["fp64_kernel"] = fp64_shape.get("kernel_name")
        if fp64_shape.get("kernel_name") == "propagate_dfrag_kernel":
            # The plain form on the FP64 pipe as well (the element-group kernel the FP64 tensor-core
            # kernel replaced for these shapes), for the mixed form's speed-up over FP64 arithmetic
            # on the same pipes.
            os.environ["HHG_DFRAG"] = "0"
            try:
                ref2 = pyswe.SWE(pyswe.Settings(dict(param)), device=local, solver=args.solver)
            finally:
                os.environ.pop("HHG_DFRAG", None)
            ref2.run_simulation()
            fms2 = []
            for i in range(args.fp64_steps):
                flush.fill_(float(i))
                torch.cuda.synchronize()
                ref2.reset()
                ref2.run_simulation()
                fms2.append(ref2.last_kernel_ms())
            mixed["fp64_pipe_kernel"] = {"kernel": ref2.launch_shape().get("kernel_name"),
                                         "ms_per_solve": statistics.mean(fms2),
                                         "mixed_speedup": statistics.mean(fms2) / (total_ms / args.steps)}
            ref2.delete()
        if args.batch > 1:
            # The batched mixed form: args.batch solves of this configuration (polarisation angles
            # spread over the half circle) in one SWEBatch, against the plain FP64 solve's throughput.
            solves = []
            for i in range(args.batch):
                pi = dict(param)
                ang = math.pi * i / args.batch
                # (components below 1e-12 are zero: 90 degrees is the x axis alone, not x plus 6e-17 y)
                pi["pol_vec"] = np.array([v if abs(v) > 1e-12 else 0.0 for v in (math.sin(ang), math.cos(ang))] + [0.0])
                solves.append(pyswe.SWE(pyswe.Settings(pi), device=local, precision="mixed", solver=args.solver,
                                        autotune=args.autotune))
            batch = pyswe.SWEBatch(solves)
            batch.run()
            bms = []
            for i in range(args.batch_steps):
                flush.fill_(float(i))
                torch.cuda.synchronize()
                batch.run()
                bms.append(batch.last_ms())
            # The batch against FP64 solo solves of the same angles (one or two field axes): their device
            # time (a second run, L2 flushed before it) and the batch's error against their currents.
            berr, fms_same = [], []
            for i in range(args.batch):
                Jb = solves[i].get_current()[1:]
                f = pyswe.SWE(pyswe.Settings(dict(solves[i].settings.param)), device=local, solver=args.solver)
                f.run_simulation()
                f.reset()
                flush.fill_(float(i))
                torch.cuda.synchronize()
                f.run_simulation()
                fms_same.append(f.last_kernel_ms())
                Jf = f.get_current()[1:]
                f.delete()
                berr.append(float(np.linalg.norm(Jb - Jf) / np.linalg.norm(Jf)))
            batch.delete()
            for s in solves:
                s.delete()
            per_solve = statistics.mean(bms) / args.batch
            mixed["batched"] = {"solves": args.batch, "timed_batches": len(bms), "ms_per_batch": statistics.mean(bms),
                                "ms_per_solve": per_solve, "k_pt_rk4_steps_per_s": nk * nt / (per_solve * 1e-3),
                                "throughput_vs_fp64_solo": fp64_ms / per_solve,
                                "pol_angles_deg": [180.0 * i / args.batch for i in range(args.batch)],
                                "fp64_same_solves_ms": sum(fms_same),
                                "speedup_vs_fp64_same_solves": sum(fms_same) / statistics.mean(bms),
                                "throughput_vs_fp64_pipe_solo": (mixed["fp64_pipe_kernel"]["ms_per_solve"] / per_solve
                                                                 if "fp64_pipe_kernel" in mixed else None),
                                "J_rel_l2_vs_fp64": berr,
                                "engine": batch_engine_desc()}
    swe.delete()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return

    fpk = flops_per_kstep(nw, w["window"], param["nr1"], n_op, n_j, kspace=args.solver == "kspace")
    prop_mean = statistics.mean(prop_ms)
    achieved = fpk * nk * nt / (prop_mean * 1e-3) / 1e12
    traffic, traffic_src = (load_traffic(args.workload, shape.get("kernel_name"))
                            if args.solver == "rspace" and not args.grid else (None, None))
    # The peak the kernel is held to: the FP64 FMA-chain peak, or in the mixed form the rate at which
    # both pipes would finish their own parts (FP64 flops at the FP64 peak plus FP32 flops at the
    # FP32 peak, one after the other).
    bound, peak, split = "fp64", fp64_peak.value, None
    if args.precision == "mixed":
        f64, f32 = flops_split_mixed(nw, w["window"], param["nr1"], n_op, n_j, kspace=args.solver == "kspace")
        if f32 > 0 and fp64_peak.value > 0 and fp32_peak.value > 0:
            bound = "fp64+fp32"
            peak = (f64 + f32) / (f64 / fp64_peak.value + f32 / fp32_peak.value)
            split = {"fp64_flops_per_kstep": f64, "fp32_flops_per_kstep": f32}
    line = {
        "metric": "k-pt*RK4-steps/s",
        "value": value,
        "unit": "k-pt*RK4-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "c64 commutators/Wannier sums, f64 state/RK/k-sum",
        "data": "synthetic (seeded TB model, generated by hhg-solids_b200/tbgen.py)",
        "impl": "hhg-b200",
        "config": {"workload": f"{args.workload}: {WORKLOADS[args.workload]['desc']}"
                   + (f" (grid overridden to {args.grid}x{args.grid})" if args.grid else "")
                   + (", mixed form (complex-FP32 Wannier sums and commutators; FP64 state, RK4 accumulation, "
                      "window velocity and k-sum)" if args.precision == "mixed" else ", plain FP64"),
                   "k_grid": [param["nr1"], param["nr2"]],
                   "nt": nt, "num_orb": nw, "precision": args.precision, "solver": args.solver,
                   "autotune": args.autotune, "parallelism": f"replicas x{world}" if world > 1 else "single",
                   "l2": "flushed between timed solves (256 MiB write)", "launch": shape},
        "solves_per_hour": 3600.0 * world * args.steps / (total_ms * 1e-3),
        "roofline": {"bound": bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak > 0 else None, "traffic": traffic,
                     "kernel": shape.get("kernel_name"), "flops_per_kstep": fpk, "flops_split": split,
                     "peak_source": "live FP64 / FP32 FMA-chain probes on this GPU (HHG_measure_peaks); "
                                    "MEASURED_PEAKS.json has no FP64 or FP32 figure",
                     "fp32_peak": fp32_peak.value, "kernel_ms": prop_mean, "traffic_source": traffic_src,
                     "executed_form": executed_form(nw, shape.get("kernel_name"), fpk, prop_mean, nk, nt, peak,
                                                    w["window"], n_op, n_j, shape.get("k_per_cta", 0),
                                                    args.solver == "kspace"),
                     "ncu_counters": load_profile_counters(args.workload, shape.get("kernel_name"))},
        "gpu_launches": launches,
        "clocks": clk,
        "wall_s_timed_region": t_wall,
    }
    if e2e:
        line["e2e"] = e2e
    if mixed:
        line["mixed_vs_fp64"] = mixed
    if world == 1 and not args.no_cpu_baseline and not args.grid:
        line["cpu_baseline"] = cpu_baseline(args.workload, args.solver)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
