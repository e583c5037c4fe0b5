#!/usr/bin/env python
"""Throughput of the JIMWLK Langevin evolution on B200.

Workload (one "step" = one Langevin step of the whole batch): 64 independent
events on 512 x 512 lattices, MV initial condition with g^2 mu a = 0.5,
m a = 0.02 and 50 slices, running coupling (the reference's
SQRT_COUPLING_CONSTANT, momentum evolution, SIN kernel) with ds = 1e-4
(step = ds / pi^2), advanced by the batched engine in mixed precision (FP32
noise, rotation and transforms; FP64 exponentials, V, per-step
reunitarisation and dipole sums).  Seeded synthetic inputs; no dataset is
involved.  The per-event fields (V 144 B/site, workspaces 192 B/site) total
~5.6 GB, far above the 126 MB L2, so no flush is needed between steps.

Arms
  default            the engine through the C ABI (softx-d-21-00092_b200/lib/libjimwlk.so)
  --impl reference   the reference's own main_optimized (oracle/_ref, OpenMP on all
                     host cores, single-rank MPI and FFTW shims) on one 512^2 event of
                     the same configuration (the reference steps one event at a time)

Launch: python bench.py [--gpus N --steps K --warmup W]; for N > 1 under
torchrun, one rank per GPU, each rank advancing its own 64 events (weak
scaling; the events are independent, so the only collective is the max of the
ranks' timings).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import signal
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "softx-d-21-00092_b200")
REF_MAIN = os.path.join(REPO, "oracle", "_ref", "main_optimized_omp_512")

EVENTS = 64
N = 512
NY_SLICES = 50
MU = 0.5 * N          # g^2 mu a = 0.5 with g = 1 -> config mu = 0.5 N
MASS = 0.04           # m a = 0.02 = mass * mu_MV
ALPHA_S, DS = 0.15, 1e-4
FIXED_STEP = ALPHA_S * DS / math.pi ** 2  # fixed coupling: step = alpha_s ds / pi^2
STEP = DS / math.pi ** 2                  # running (SQRT) coupling: alpha_s(k) sits in the kernel
REUNITARIZE = True                        # the mixed form reunitarises V after every step
METRIC = "lattice site-steps/s"
# algorithmic HBM bytes per site of each kernel kind (mixed precision):
#   pass 1: read V (9 complex FP64 = 144 B) + write 16 FP32 complex planes (128 B)
#   pass 2: read 16 planes (128 B) + write 8 planes (64 B)
#   pass 3: read 8 planes (64 B) + read and write V (288 B)
#   pass 3 + next pass 1: read 8 planes (64 B), read and write V (288 B), write 16 planes (128 B)
# A run of K steps is pass 1, K - 1 times (pass 2, pass 3 + next pass 1), pass 2, pass 3.
KIND_BYTES = {"pass1": 272, "pass2": 192, "pass3": 352, "pass31": 480}
KIND_KERNEL = {"pass1": "k_mix_pass1", "pass2": "k_mix_pass2", "pass3": "k_mix_pass3", "pass31": "k_mix_pass31"}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init_dist(backend: str = "nccl", timeout_s: int = 120) -> None:
    """One process per GPU (torchrun sets RANK/WORLD_SIZE/MASTER_*); a short
    timeout ends ranks that wait for a rank that died."""
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def max_over_ranks(x: float) -> float:
    """The slowest rank's time (every rank calls it at the same point)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def event_seeds(rank: int, events: int) -> list:
    """Each rank evolves its own events (weak scaling): seeds never repeat across ranks."""
    return [1_000_003 * (rank + 1) + i for i in range(events)]


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """Per-launch DRAM bytes of each fused kernel from the committed ncu summary
    (profiles/step_kernels_512x64.md, a line `traffic <kernel> <bytes_per_site>`)."""
    p = os.path.join(REPO, "profiles", "step_kernels_512x64.md")
    out = {}
    if os.path.exists(p):
        for line in open(p):
            m = re.match(r"\s*traffic\s+(\S+)\s+([0-9.]+)", line)
            if m:
                out[m.group(1)] = float(m.group(2))
    return out


class ClockSampler:
    """SM clocks and throttle reasons while the timed region runs, read through
    NVML every 2 ms on a host thread (the timed region lasts ~50-100 ms, too
    short for nvidia-smi's 200 ms loop); nvidia-smi is the fallback when NVML
    cannot be opened.  The GPU is found by its PCI bus id, so the sample is of
    the device the run uses whatever CUDA_VISIBLE_DEVICES maps."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap"}
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, period_s: float = 0.002):
        self.device = device
        self.period = period_s
        self.rows = []
        self.max_mhz = None
        self.handle = None
        self.thread = None
        self.stop = None
        self.proc = None
        self.path = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.device)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        return pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())

    def _poll(self):
        import pynvml
        get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop.is_set():
            try:
                self.rows.append((pynvml.nvmlDeviceGetClockInfo(self.handle, pynvml.NVML_CLOCK_SM),
                                  get_reasons(self.handle)))
            except Exception:
                break
            self.stop.wait(self.period)

    def __enter__(self):
        import threading
        try:
            import pynvml
            self.handle = self._nvml_handle()
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        except Exception:
            self.handle = None
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                              "--format=csv,noheader,nounits", "-lms", "200"],
                                             stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            except OSError:
                self.proc = None
            time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.send_signal(signal.SIGTERM)
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.handle is not None:
            if not self.rows:
                return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "source": "nvml"}
            reasons = sorted({name for _, r in self.rows for bit, name in self.REASONS.items() if r & bit})
            return {"sm_mhz": statistics.median(m for m, _ in self.rows), "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(self.rows), "source": "nvml, 2 ms"}
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].isdigit():
                    rows.append(f)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [int(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi, 200 ms"}


def parse_evolution_times(text: str):
    return [float(x) for x in re.findall(r"Evolution time:\s*([0-9.eE+-]+)", text)]


def run_reference_main(steps: int, warmup: int, nthreads: int | None = None, n_side: int = N,
                       evolution: str = "MOMENTUM_EVOLUTION", coupling: str = "SQRT_COUPLING_CONSTANT",
                       with_wall: bool = False, slices: int = 1, step: float = STEP):
    """The reference's main_optimized on one n_side^2 event: returns seconds per
    Langevin step (mean over the last `steps` of warmup + steps) and, with
    with_wall, the run's wall time outside the initial condition and the
    steps (the set-up, which holds the Cholesky decomposition)."""
    exe = os.path.join(REPO, "oracle", "_ref", f"main_optimized_omp_{n_side}")
    if not os.path.exists(exe):
        return None, f"reference binary oracle/_ref/main_optimized_omp_{n_side} not built"
    with tempfile.TemporaryDirectory() as d:
        cfg = os.path.join(d, "config")
        with open(cfg, "w") as fh:
            # the initial condition is outside the per-step timing (1 MV slice
            # unless asked); SQRT coupling takes the reference's parallel
            # generate_gaussian
            fh.write(f"stat = 1\nmu = {0.5 * n_side}\nmass = {MASS}\nelementaryWilsonLines = {slices}\n"
                     f"file_name = bench\nlangevin_steps = {warmup + steps}\nmeasurements = 1\nstep = {step}\n"
                     f"EvolutionChoice = {evolution}\nCouplingChoice = {coupling}\nKernelChoice = SIN_KERNEL\n")
        env = dict(os.environ)
        env["OMP_NUM_THREADS"] = str(nthreads or os.cpu_count())
        t0 = time.perf_counter()
        r = subprocess.run([exe, "1", "1", cfg], cwd=d, capture_output=True, text=True, env=env, timeout=3600)
        wall = time.perf_counter() - t0
        t = parse_evolution_times(r.stdout)
        if len(t) < warmup + steps:
            return None, f"reference run produced {len(t)} step timings (rc={r.returncode})"
        if with_wall:
            ic = [float(x) for x in re.findall(r"Initial condition time:\s*([0-9.eE+-]+)", r.stdout)]
            return (statistics.mean(t[warmup:]), wall - sum(t) - sum(ic)), None
        return statistics.mean(t[warmup:]), None


# serving: each tick advances the requests with the least remaining work first,
# up to 64 x 512^2 lattice sites (one bench batch)
SERVE_TICK_SITES = 64 * 512 * 512
POS_N, POS_SLICES, POS_STEPS, POS_EVERY = 256, 100, 500, 50
POS_STEP = DS / math.pi ** 2  # running coupling: alpha_s(r) enters through the correlated noise
POS_CPU_N = 32


def position_leg(jw, device: int, steps: int = POS_STEPS, every: int = POS_EVERY):
    """Position-space evolution with Cholesky-correlated noise (the reference's
    POSITION_EVOLUTION + NOISE_COUPLING_CONSTANT path, main_optimized.cpp:
    145-157, 271-304) on one 256^2 event in FP64: MV initial condition with
    Ny = 100 slices, the 68.7 GB factor, `steps` steps measured every `every`
    (C(k), S(r), Q_s).  The factor apply streams the lower triangle of L once
    per step: 16 n (n + 1) / 2 bytes, n = N^2."""
    import torch
    cfg = jw.config_defaults(Nx=POS_N, Ny=POS_N, seed=11, mu=0.5 * POS_N, mass=MASS,
                             elementaryWilsonLines=POS_SLICES, step=POS_STEP, EvolutionChoice=jw.POSITION_EVOLUTION,
                             CouplingChoice=jw.NOISE_COUPLING_CONSTANT, KernelChoice=jw.SIN_KERNEL)
    ctx = jw.Context(cfg, device)
    s = torch.cuda.ExternalStream(jw.lib().jw_context_stream(ctx._h))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    V = ctx.field()
    a.record(s)
    ctx.initial_condition(V)
    b.record(s)
    b.synchronize()
    ic_ms = a.elapsed_time(b)
    corr = ctx.field(1)
    ctx.set_correlations_for_coupling_constant(corr)
    ctx.execute2D(corr, 0)
    ctx.sync()
    t0 = time.perf_counter()
    L = ctx.cholesky(corr)  # returns after the decomposition has finished
    dec_s = time.perf_counter() - t0
    ctx.evolve_position(V, 0, 0, 0, L)  # allocates the step's work fields
    Vk, c = ctx.field(), ctx.field(1)
    evo_ms, qs, done = 0.0, [], 0
    while done < steps:
        k = min(every, steps - done)
        a.record(s)
        ctx.evolve_position(V, done, k, 0, L)
        b.record(s)
        b.synchronize()
        evo_ms += a.elapsed_time(b)
        done += k
        Vk.copy_from(V)
        ctx.execute2D(Vk, 1)
        ctx.trace(Vk, c)
        ctx.average_and_symmetrize(c)
        qs.append(ctx.dipole(c)[3])
    status = ctx.sync()
    Vh = V.get().reshape(-1, 3, 3)
    drift = float(np.abs(Vh @ np.conj(np.transpose(Vh, (0, 2, 1))) - np.eye(3)).max())
    ctx.close()
    n = POS_N * POS_N
    lbytes = 16.0 * n * (n + 1) / 2
    step_ms = evo_ms / steps
    # one apply streams L's lower triangle once for the noise of two steps:
    # 32 real right-hand sides, 2 real FMAs per complex entry and right-hand side
    apply_flops = 2.0 * 2 * 32 * n * (n + 1) / 2
    out = {"workload": f"1 event {POS_N}^2, POSITION_EVOLUTION + NOISE_COUPLING_CONSTANT (Cholesky-correlated "
                       f"noise), SIN kernel, FP64, Ny = {POS_SLICES}, {steps} steps, measured every {every}",
           "status": status, "initial_condition_ms": ic_ms, "cholesky_decompose_s": dec_s,
           "cholesky_tflops_fp64": 4.0 * n ** 3 / 3.0 / dec_s / 1e12,
           "cholesky_decompose_note": "own kernels: diagonal blocks, warp-per-row panel solves, FP64 tensor-core "
                                      "(mma.sync m8n8k4) trailing updates; 4 n^3 / 3 real flops",
           "cholesky_bytes": 16.0 * n * n,
           "step_ms": step_ms, "site_steps_per_s": n / (step_ms / 1e3),
           "factor_stream_gbs": lbytes / (2 * step_ms / 1e3) / 1e9,
           "factor_apply_tflops_fp64": apply_flops / (2 * step_ms / 1e3) / 1e12,
           "factor_stream_note": "the apply reads L's lower triangle once per two steps (both steps' noise): "
                                 "bytes and FP64 tensor flops of one apply / two whole steps' time; the FP64 "
                                 "tensor pipe, not HBM, bounds it (nominal B200 FP64 tensor peak 40 TFLOP/s)",
           "Qs_every_50": qs, "unitarity_drift": drift}
    # the reference's own position path on a bounded sample (32^2), extrapolated by V^2 per step and V^3
    # for the decomposition; 256^2 itself is out of reach on the CPU
    r, why = run_reference_main(2, 0, n_side=POS_CPU_N, evolution="POSITION_EVOLUTION",
                                coupling="NOISE_COUPLING_CONSTANT", with_wall=True)
    if r is not None:
        t_step, t_setup = r
        scale = (POS_N / POS_CPU_N) ** 2
        out["cpu_baseline"] = {"value": POS_CPU_N ** 2 / t_step, "unit": "site-steps/s", "cores": os.cpu_count(),
                               "kind": "reference",
                               "sample": f"main_optimized at {POS_CPU_N}^2, POSITION + NOISE, 2 steps; set-up "
                                         f"(Cholesky) {t_setup:.2f} s",
                               "extrapolated_256_step_s": t_step * scale ** 2,
                               "extrapolated_256_decompose_s": t_setup * scale ** 3}
    else:
        out["cpu_baseline"] = {"value": None, "unit": "site-steps/s", "cores": 0, "kind": "reference", "sample": why}
    return out


def quantize_n(n: float) -> int:
    """Lattice sides are powers of two: the nearest one in log2."""
    return int(2 ** int(round(math.log2(n))))


def serve_leg(jw, device: int, n_requests: int, rate: float, seed: int, tick_sites: int = 0):
    """Continuous batching under Poisson arrivals: requests (N log-uniform on
    [64, 2048] rounded to a power of two, Ny in {50, 100}, steps uniform on
    [10, 2000], g^2 mu a uniform on [0.3, 0.8], per-request seed) submitted at
    their arrival times; latency = finished - arrived."""
    import threading

    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    reqs = []
    for i in range(n_requests):
        N = quantize_n(math.exp(rng.uniform(math.log(64), math.log(2048))))
        reqs.append(dict(N=N, ny_slices=int(rng.choice([50, 100])), steps=int(rng.integers(10, 2001)),
                         mu=float(rng.uniform(0.3, 0.8)) * N, seed=10_000 + i))
    srv = jw.Server(precision=jw.PRECISION_MIXED, max_steps_per_tick=16, device=device, tick_sites=tick_sites,
                    reunitarize=REUNITARIZE)
    rids = [None] * n_requests

    def feeder():
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            dt = arrivals[i] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            rids[i] = srv.submit(r["N"], r["steps"], ny_slices=r["ny_slices"], mu=r["mu"], mass=MASS,
                                 step=FIXED_STEP, coupling=jw.FIXED_COUPLING_CONSTANT, seed=r["seed"])

    th = threading.Thread(target=feeder)
    th.start()
    th.join()
    lat, t_first, t_last, ok = [], None, 0.0, 0
    for rid in rids:
        st, res, _, _ = srv.wait(rid, timeout=3600)
        ok += st == jw.OK
        lat.append(res.t_done - res.t_submit)
        t_first = res.t_submit if t_first is None else min(t_first, res.t_submit)
        t_last = max(t_last, res.t_done)
    stats = srv.stats()
    sizes = srv.size_stats()
    srv.close()
    site_steps = sum(r["N"] ** 2 * r["steps"] for r in reqs)
    mix = [(r["N"], r["ny_slices"], r["steps"]) for r in reqs]
    # where the device time goes: per lattice size, the site-steps it advanced,
    # the device time of its step launches and MV slices (CUDA events on the
    # engine stream), and its own rate
    dev_ms = sum(v["step_ms"] + v["mv_ms"] for v in sizes.values())
    per_n = {str(n): {"requests": sum(1 for r in reqs if r["N"] == n), "site_steps": v["site_steps"],
                      "step_ms": v["step_ms"], "mv_ms": v["mv_ms"], "ticks": v["ticks"],
                      "share_of_device_time": (v["step_ms"] + v["mv_ms"]) / dev_ms if dev_ms else None,
                      "site_steps_per_s_while_stepping": v["site_steps"] / (v["step_ms"] / 1e3) if v["step_ms"] else None}
             for n, v in sorted(sizes.items())}
    return {"requests": n_requests, "ok": ok, "rate_req_per_s": rate, "_mix": mix,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "site_steps_per_s": site_steps / (t_last - t_first), "wall_s": t_last - t_first,
            "window": f"{n_requests} arrivals over {arrivals[-1]:.2f} s (Poisson, {rate:g}/s); latency and "
                      f"throughput over the {t_last - t_first:.1f} s from the first submission to the last "
                      "completion",
            "max_resident": stats.max_active,
            "per_n": per_n,
            "phases_s": {"admit": stats.t_admit, "mv": stats.t_mv, "step": stats.t_step, "retire": stats.t_retire},
            "device_busy_fraction": dev_ms / 1e3 / (t_last - t_first),
            "offered_site_steps_per_s": site_steps / arrivals[-1],
            "tick_sites": tick_sites,
            "what": "Poisson arrivals, N log-uniform 64..2048 rounded to powers of two, steps U[10,2000], "
                    "Ny in {50,100}, mixed precision, continuous batching"
                    + (", least remaining work first per tick" if tick_sites else "")}


def plain_fp64_times(jw, device: int, sizes) -> dict:
    """The plain FP64 form per lattice size: one event at a time through the
    call-for-call layer (the reference's call structure), ms per MV slice and
    per Langevin step, timed with CUDA events."""
    import torch
    out = {}
    for n in sizes:
        cfg = jw.config_defaults(Nx=n, Ny=n, seed=3, mu=0.5 * n, mass=MASS, elementaryWilsonLines=2,
                                 step=FIXED_STEP, CouplingChoice=jw.FIXED_COUPLING_CONSTANT)
        ctx = jw.Context(cfg, device)
        s = torch.cuda.ExternalStream(jw.lib().jw_context_stream(ctx._h))
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        V = ctx.field()
        ctx.initial_condition(V)
        ctx.evolve_momentum(V, 0, 1)
        ctx.sync()
        k = 3 if n >= 1024 else 10
        a.record(s)
        ctx.initial_condition(V)
        b.record(s)
        ctx.evolve_momentum(V, 1, k)
        c.record(s)
        c.synchronize()
        out[n] = {"slice_ms": a.elapsed_time(b) / 2, "step_ms": b.elapsed_time(c) / k}
        ctx.close()
    return out


def uneven_leg(jw, device: int, seed: int):
    """48 events N in {128,256,512,1024} (16/16/12/4), Ny = 50, steps U[200,2000],
    fixed and running coupling mixed, all submitted at once to the server."""
    rng = np.random.default_rng(seed)
    sizes = [128] * 16 + [256] * 16 + [512] * 12 + [1024] * 4
    srv = jw.Server(precision=jw.PRECISION_MIXED, max_steps_per_tick=32, device=device, reunitarize=REUNITARIZE)
    reqs = [dict(N=n, steps=int(rng.integers(200, 2001)), coupling=[jw.FIXED_COUPLING_CONSTANT,
                                                                    jw.SQRT_COUPLING_CONSTANT][i % 2])
            for i, n in enumerate(sizes)]
    t0 = time.perf_counter()
    rids = [srv.submit(r["N"], r["steps"], ny_slices=50,
                       step=FIXED_STEP if r["coupling"] == jw.FIXED_COUPLING_CONSTANT else STEP,
                       coupling=r["coupling"], seed=500 + i)
            for i, r in enumerate(reqs)]
    ok = sum(srv.wait(rid, timeout=3600)[0] == jw.OK for rid in rids)
    wall = time.perf_counter() - t0
    sizes = srv.size_stats()
    srv.close()
    ss = sum(r["N"] ** 2 * r["steps"] for r in reqs)
    per_n = {str(n): {"site_steps": v["site_steps"], "step_ms": v["step_ms"], "mv_ms": v["mv_ms"],
                      "site_steps_per_s_while_stepping": v["site_steps"] / (v["step_ms"] / 1e3) if v["step_ms"] else None}
             for n, v in sorted(sizes.items())}
    return {"events": len(reqs), "ok": ok, "site_steps": ss, "wall_s": wall, "site_steps_per_s": ss / wall,
            "per_n": per_n,
            "what": "48 events N in {128,256,512,1024} (16/16/12/4), steps U[200,2000], mixed couplings, "
                    "one server, MV initial conditions included"}


def uneven_streams_leg(jw, device: int, steps: int = 40) -> dict:
    """The C4 batch's kernels without the server: 48 events N in {128, 256,
    512, 1024} (16/16/12/4), K steps each, (a) as per-size runs back to back on
    one stream (one engine), (b) the four size groups on four concurrent
    streams (one engine per size), (c) each size alone.  Whether one launch
    over mixed sizes could gain: only if a size's own launches leave the GPU
    idle, which (a) against (b) and the sum of (c) measure."""
    import torch
    sizes = [128] * 16 + [256] * 16 + [512] * 12 + [1024] * 4

    def add(eng, i, n):
        c = [jw.FIXED_COUPLING_CONSTANT, jw.SQRT_COUPLING_CONSTANT][i % 2]
        return eng.add_event(n, ny_slices=2, mu=0.5 * n, mass=MASS, coupling=c, seed=500 + i,
                             step=FIXED_STEP if c == jw.FIXED_COUPLING_CONSTANT else STEP)

    def timed(runs):
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for eng, ids in runs:
            eng.step(ids, steps)
        for eng, _ in runs:
            if eng.sync() != jw.OK:
                raise RuntimeError("device error in the uneven-streams leg")
        torch.cuda.synchronize(device)
        return time.perf_counter() - t0

    ss = sum(n * n for n in sizes) * steps
    one = jw.Engine(precision=jw.PRECISION_MIXED, device=device, reunitarize=REUNITARIZE, autotune=True)
    ids = [add(one, i, n) for i, n in enumerate(sizes)]
    one.init_mv(ids)
    one.step(ids, 3)
    t_one = min(timed([(one, ids)]) for _ in range(3))
    one.close()
    per = {}
    for n in (128, 256, 512, 1024):
        e = jw.Engine(precision=jw.PRECISION_MIXED, device=device, reunitarize=REUNITARIZE, autotune=True)
        per[n] = (e, [add(e, i, m) for i, m in enumerate(sizes) if m == n])
        per[n][0].init_mv(per[n][1])
        per[n][0].step(per[n][1], 3)
    t_streams = min(timed(list(per.values())) for _ in range(3))
    alone = {n: min(timed([per[n]]) for _ in range(3)) for n in per}
    for e, _ in per.values():
        e.close()
    return {"steps": steps, "site_steps": ss,
            "one_stream_s": t_one, "one_stream_site_steps_per_s": ss / t_one,
            "concurrent_streams_s": t_streams, "concurrent_streams_site_steps_per_s": ss / t_streams,
            "alone_s": {str(n): t for n, t in alone.items()}, "sum_alone_s": sum(alone.values()),
            "alone_site_steps_per_s": {str(n): len(per[n][1]) * n * n * steps / t for n, t in alone.items()},
            "what": "C4's 48 events without the server: per-size runs on one stream, the size groups on four "
                    "concurrent streams, each size alone (wall time, device synchronised)"}


def c1_leg(jw, device: int):
    """C1, the reference's CPU-runnable case: one FP64 event at 64^2, MV initial
    condition (g^2 mu a = 0.5, m a = 0.02, Ny = 50), 100 fixed-coupling steps
    (alpha_s = 0.15, ds = 1e-4) through the call-for-call layer, then C(k), S(r)
    and Q_s.  Beside it the reference's main_optimized at 64^2 (all host
    threads), per Langevin step."""
    import torch
    n = 64
    cfg = jw.config_defaults(Nx=n, Ny=n, seed=1, mu=0.5 * n, mass=MASS, elementaryWilsonLines=NY_SLICES,
                             step=FIXED_STEP, CouplingChoice=jw.FIXED_COUPLING_CONSTANT)
    ctx = jw.Context(cfg, device)
    s = torch.cuda.ExternalStream(jw.lib().jw_context_stream(ctx._h))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    V, Vk, c = ctx.field(), ctx.field(), ctx.field(1)
    ctx.evolve_momentum(V, 0, 0)
    torch.cuda.synchronize()
    ev[0].record(s)
    ctx.initial_condition(V)
    ev[1].record(s)
    ctx.evolve_momentum(V, 0, 100)
    ev[2].record(s)
    Vk.copy_from(V)
    ctx.execute2D(Vk, 1)
    ctx.trace(Vk, c)
    ctx.average_and_symmetrize(c)
    ev[3].record(s)
    ev[3].synchronize()
    qs = ctx.dipole(c)[3]
    status = ctx.sync()
    ctx.close()
    ic, steps, meas = (ev[i].elapsed_time(ev[i + 1]) for i in range(3))
    out = {"workload": "1 event 64^2 FP64, MV Ny = 50, 100 fixed-coupling steps, measurement (call-for-call layer)",
           "status": status, "total_ms": ic + steps + meas, "initial_condition_ms": ic, "steps_ms": steps,
           "measure_ms": meas, "site_steps_per_s": n * n * 100 / (steps / 1e3), "Qs": qs}
    # the same event through the FP64 batched engine (fused kernels, graph replay)
    eng = jw.Engine(precision=jw.PRECISION_FP64, device=device)
    warm = eng.add_event(n, ny_slices=NY_SLICES, mu=0.5 * n, mass=MASS, step=FIXED_STEP,
                         coupling=jw.FIXED_COUPLING_CONSTANT, seed=2)
    eng.init_mv([warm])
    eng.step([warm], 3)
    eng.measure([warm])
    eid = eng.add_event(n, ny_slices=NY_SLICES, mu=0.5 * n, mass=MASS, step=FIXED_STEP,
                        coupling=jw.FIXED_COUPLING_CONSTANT, seed=1)
    es = torch.cuda.ExternalStream(eng.stream)
    torch.cuda.synchronize()
    ev[0].record(es)
    eng.init_mv([eid])
    ev[1].record(es)
    eng.step([eid], 100)
    ev[2].record(es)
    eng.measure([eid])
    ev[3].record(es)
    ev[3].synchronize()
    estatus = eng.sync()
    eng.close()
    ic, steps, meas = (ev[i].elapsed_time(ev[i + 1]) for i in range(3))
    out["engine_fp64"] = {"status": estatus, "total_ms": ic + steps + meas, "initial_condition_ms": ic,
                          "steps_ms": steps, "measure_ms": meas, "site_steps_per_s": n * n * 100 / (steps / 1e3)}
    t, why = run_reference_main(10, 2, n_side=n)
    out["cpu_baseline"] = ({"value": n * n / t, "unit": "site-steps/s", "cores": os.cpu_count(), "kind": "reference",
                            "sample": f"main_optimized at {n}^2, 10 steps after 2 warm-up, SQRT coupling"}
                           if t is not None else {"value": None, "unit": "site-steps/s", "cores": 0,
                                                  "kind": "reference", "sample": why})
    return out


def fp64_engine_leg(jw, device: int, events: int, mixed_value: float, steps: int = 10) -> dict:
    """The same workload through the FP64 batched engine (FP64 transforms,
    k_step_pass1/2/3), timed with CUDA events over `steps` steps."""
    import torch
    eng = jw.Engine(precision=jw.PRECISION_FP64, device=device)
    ids = [eng.add_event(N, ny_slices=NY_SLICES, mu=MU, mass=MASS, step=STEP, coupling=jw.SQRT_COUPLING_CONSTANT,
                         seed=sd) for sd in event_seeds(0, events)]
    eng.init_mv(ids)
    eng.step(ids, 3)
    s = torch.cuda.ExternalStream(eng.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(s)
    eng.step(ids, steps)
    b.record(s)
    b.synchronize()
    status = eng.sync()
    eng.close()
    ms = a.elapsed_time(b) / steps
    v = events * N * N / (ms / 1e3)
    return {"value": v, "unit": "site-steps/s", "ms_per_step": ms, "steps": steps, "status": status,
            "mixed_over_fp64_batched": mixed_value / v,
            "what": f"{events} events x {N}^2, FP64 batched engine (3 fused passes per step, graph replay)"}


def mixed_error_leg(jw, device: int) -> dict:
    """Mixed precision against the FP64 engine (pinned to the reference's V at
    1e-12 by the parity tests) with the same seeds: max |dS(r)|, |dQ_s|/Q_s and
    the unitarity drift, for the batched workload's size (4 of its events, 1000
    steps), the uneven batch (one event per N, its step counts and couplings)
    and a sample of the serving mix."""
    from jimwlk.precision import compare_mixed_fp64

    def sp(n, steps, seed, coupling, ny=NY_SLICES, g2mu=0.5):
        fixed = coupling == jw.FIXED_COUPLING_CONSTANT
        return dict(N=n, ny_slices=ny, mu=g2mu * n, mass=MASS, step=FIXED_STEP if fixed else STEP,
                    coupling=coupling, seed=seed, steps=steps)

    def summary(res, what):
        return {"what": what, "dS_max": res["dS_max"], "Qs_rel_err_max": res["Qs_rel_err_max"],
                "drift_mixed_max": res["drift_mixed_max"], "drift_fp64_max": res["drift_fp64_max"],
                "ensembles": {str(k): v for k, v in res["ensembles"].items()}, "status": res["status"],
                "per_event": [{k: e[k] for k in ("N", "steps", "dS_max", "Qs", "Qs_rel_err", "drift_mixed")}
                              for e in res["per_event"]]}

    t0 = time.perf_counter()
    out = {"bars": {"dS_max": 1e-5, "Qs_rel_err": 1e-4}, "comparator": "FP64 batched engine, same seeds"}
    out["C3"] = summary(compare_mixed_fp64(jw, [sp(N, 1000, 7000 + i, jw.SQRT_COUPLING_CONSTANT)
                                                for i in range(4)], device),
                        f"4 events x {N}^2, Ny = {NY_SLICES}, 1000 steps, running coupling (the benched workload)")
    rng = np.random.default_rng(48)
    c4 = [sp(n, int(rng.integers(200, 2001)), 600 + i,
             [jw.FIXED_COUPLING_CONSTANT, jw.SQRT_COUPLING_CONSTANT][i % 2]) for i, n in enumerate((128, 256, 512, 1024))]
    out["C4"] = summary(compare_mixed_fp64(jw, c4, device),
                        "one event per N in {128, 256, 512, 1024}, steps U[200, 2000], fixed/running couplings")
    rng = np.random.default_rng(2026)
    c5 = []
    for i in range(4):
        n = quantize_n(math.exp(rng.uniform(math.log(64), math.log(2048))))
        c5.append(sp(n, int(rng.integers(10, 2001)), 10_000 + i, jw.FIXED_COUPLING_CONSTANT,
                     ny=int(rng.choice([50, 100])), g2mu=float(rng.uniform(0.3, 0.8))))
    out["C5"] = summary(compare_mixed_fp64(jw, c5, device),
                        "4 requests drawn from the serving mix (N = 128, 256, 2048, 128; the FP64 comparator "
                        "above 1024^2 is the call-for-call layer)")
    out["seconds"] = time.perf_counter() - t0
    return out


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def workload_config(events: int = EVENTS, n_side: int = N) -> dict:
    """The benched workload, the same dictionary in both arms."""
    return {"workload": f"{events} events x {n_side}^2 Langevin evolution, MV initial condition, running coupling",
            "N": n_side, "events": events, "ny_slices": NY_SLICES, "g2mu_a": 0.5, "m_a": 0.02, "ds": DS,
            "step": STEP, "evolution": "momentum", "kernel": "SIN", "coupling": "running (SQRT_COUPLING_CONSTANT)",
            "l2": "inputs ~5.6 GB per GPU > L2 (no flush needed)"}


def reference_arm(args):
    """The reference's main_optimized on one event of the benched configuration
    (the reference steps one event at a time): the same N, MV slices, coupling,
    kernel and step, K timed Langevin steps after W untimed ones (at most 100
    and 10, a bounded sample of the 64-event workload)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cores = os.cpu_count()
    steps = max(1, min(args.steps, 100))
    warm = max(1, min(args.warmup, 10))
    t, why = run_reference_main(steps, warm, slices=NY_SLICES)
    if t is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    value = N * N / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "site-steps/s", "n_gpus": 0,
        "steps": steps, "warmup": warm, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": "site-steps/s", "cores": cores, "kind": "reference",
                         "sample": f"1 of the {EVENTS} events ({N}^2, {NY_SLICES} MV slices), {steps} Langevin "
                                   f"steps after {warm} warm-up; main_optimized with OpenMP ({cores} threads, "
                                   f"{cpu_model()}), FFTW replaced by the project's radix-2 FFT shim"},
        "e2e": {"value": value, "unit": "site-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main_arm(args):
    rank, world, local = dist_env()
    sys.path.insert(0, PKG)
    import torch
    import jimwlk as jw

    torch.cuda.set_device(local)
    if world > 1:
        init_dist("nccl")
    barrier_max = max_over_ranks

    events = args.events
    n_side = args.n
    eng = jw.Engine(precision=jw.PRECISION_MIXED, device=local, max_batch=args.max_batch,
                    autotune=args.column_form == 0, reunitarize=REUNITARIZE)
    ids = [eng.add_event(n_side, ny_slices=NY_SLICES, mu=0.5 * n_side, mass=MASS, step=STEP,
                         coupling=jw.SQRT_COUPLING_CONSTANT, seed=sd) for sd in event_seeds(rank, events)]
    if args.column_form:
        eng.set_tuning(n_side, args.column_form)
    eng.init_mv(ids)
    eng.step(ids, args.warmup)
    if eng.sync() != jw.OK:
        raise RuntimeError("device error during warm-up")
    sites = events * n_side * n_side

    # ---- timed region: K steps, a CUDA event around every kernel
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        kernels, total_ms = eng.step_timed(ids, args.steps)
    torch.cuda.synchronize()
    status = eng.sync()
    if status != jw.OK:
        raise RuntimeError(f"device status {status} in the timed region")
    total_ms = barrier_max(total_ms)
    clocks = clk.summary()
    value = world * sites * args.steps / (total_ms / 1e3)

    # ---- end to end through the C ABI with host buffers: per step one call
    # of jw_engine_step_measure_ensemble (the event id list in, one step, the
    # ensemble dipole measurement read back to host memory), as main_optimized
    # runs with measurements == langevin_steps.  The same loop as two calls
    # (jw_engine_step, then jw_engine_measure_ensemble) is timed beside it.
    k_e2e = max(3, min(args.steps, 10))
    # page-locked result arrays, as a serving client would keep them
    sum_h = torch.empty((n_side, n_side), dtype=torch.complex128, pin_memory=True).numpy()
    err_h = torch.empty((n_side, n_side), dtype=torch.complex128, pin_memory=True).numpy()
    eng.measure_ensemble(ids, sum_h, err_h)
    stream = torch.cuda.ExternalStream(eng.stream)

    def timed_loop(body):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(k_e2e):
            body()
        e1.record(stream)
        e1.synchronize()
        return barrier_max(e0.elapsed_time(e1))

    e2e_ms = timed_loop(lambda: eng.step_measure_ensemble(ids, 1, sum_h, err_h))
    two_ms = timed_loop(lambda: (eng.step(ids, 1), eng.measure_ensemble(ids, sum_h, err_h)))
    # with several ranks, the ensemble of all ranks' events: one sum of the
    # ranks' fields (the run's only collective), outside the timed loops
    allreduce_ms = None
    if world > 1:
        from jimwlk.dist import allreduce_ensemble
        barrier()
        t0 = time.perf_counter()
        allreduce_ensemble(sum_h, err_h)
        allreduce_ms = max_over_ranks((time.perf_counter() - t0) * 1e3)
    e2e_value = world * sites * k_e2e / (e2e_ms / 1e3)
    h2d = 4 * events                   # the event id list
    d2h = 2 * n_side * n_side * 16     # sum and err, complex

    # ---- roofline of the dominant kernel (the largest share of the timed region)
    peak, peak_kind = measured_peaks()
    launched = {k: v for k, v in kernels.items() if v[1] > 0}
    dom = max(launched, key=lambda k: launched[k][0])
    tuned = eng.tuning(n_side)
    kernel_of = dict(KIND_KERNEL)
    if tuned in (16, 20, 24) or (tuned == 0 and 64 <= n_side <= 1024):  # the persistent TMA column pass
        kernel_of["pass2"] = "k_mix_pass2_tma"
    name = f"{kernel_of[dom]}<{n_side}>"
    per_launch = {k: ms / cnt for k, (ms, cnt) in launched.items()}
    alg_bytes = KIND_BYTES[dom] * sites
    achieved = alg_bytes / (per_launch[dom] / 1e3) / 1e9
    measured = profiled_traffic()
    traffic = measured.get(name)
    kernel_time = sum(ms for ms, _ in launched.values())
    roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": achieved / peak, "traffic": traffic * sites if traffic else None,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per site at 16 events x 512^2 "
                              "(working set >> L2), times this launch's sites (profiles/step_kernels_512x64.md)",
            "algorithmic_bytes": alg_bytes,
            "traffic_over_algorithmic": traffic * sites / alg_bytes if traffic else None,
            "kernels": {f"{kernel_of[k]}<{n_side}>": {
                "launches": cnt, "ms_per_launch": per_launch[k], "share": ms / kernel_time,
                "hbm_frac": KIND_BYTES[k] * sites / (per_launch[k] / 1e3) / 1e9 / peak,
                "traffic_bytes_per_site": measured.get(f"{kernel_of[k]}<{n_side}>")}
                for k, (ms, cnt) in launched.items()}}

    line = {
        "metric": METRIC, "value": value, "unit": "site-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 transforms / f64 exponentials and V", "data": "synthetic",
        "config": workload_config(events, n_side),
        "engine": {"precision": "mixed", "reunitarize": REUNITARIZE, "max_batch": args.max_batch,
                   "parallelism": f"events sharded over {world} rank(s), {events} per rank",
                   "autotuned_column_tile": eng.tuning(n_side)},
        "e2e": {"value": e2e_value, "unit": "site-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": k_e2e, "ms_per_step": e2e_ms / k_e2e,
                "what": "jw_engine_step_measure_ensemble per step (one step + ensemble measurement to host arrays)",
                "two_calls": {"value": world * sites * k_e2e / (two_ms / 1e3), "ms_per_step": two_ms / k_e2e,
                              "what": "jw_engine_step + jw_engine_measure_ensemble per step"},
                "ensemble_allreduce_ms": allreduce_ms},
        "gpu_launches": sum(cnt for _, cnt in launched.values()),
        "clocks": clocks,
        "roofline": roof,
    }

    if rank == 0 and world == 1 and not args.no_extras and n_side == N:
        # plain FP64 form: the call-for-call layer (reference structure), one event at a time
        cfg = jw.config_defaults(Nx=N, Ny=N, seed=7, mu=MU, mass=MASS, elementaryWilsonLines=1, step=STEP,
                                 CouplingChoice=jw.SQRT_COUPLING_CONSTANT)
        ctx = jw.Context(cfg)
        V = ctx.field()
        ctx.initial_condition(V)
        ctx.evolve_momentum(V, 0, 2)
        ctx.sync()
        s0 = torch.cuda.ExternalStream(jw.lib().jw_context_stream(ctx._h))
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        kp = 10
        a0.record(s0)
        ctx.evolve_momentum(V, 2, kp)
        a1.record(s0)
        a1.synchronize()
        plain = N * N * kp / (a0.elapsed_time(a1) / 1e3)
        line["fp64_plain"] = {"value": plain, "unit": "site-steps/s", "steps": kp,
                              "what": "jw_evolve_momentum, reference call structure, FP64, one 512^2 event",
                              "mixed_batched_over_plain": value / plain}
        ctx.close()
        # the FP64 batched engine on the same 64 events: what batching and fusion give
        # without the FP32 transforms (the rest of the ratio above is precision)
        line["fp64_engine"] = fp64_engine_leg(jw, local, events, value)
        line["fp64_plain"]["fp64_batched_over_plain"] = line["fp64_engine"]["value"] / plain
        # mixed-precision error against the FP64 engine at the quoted sizes and step counts
        line["mixed_error"] = mixed_error_leg(jw, local)
        line["serve"] = serve_leg(jw, local, args.serve_requests, 200.0, 2026, tick_sites=SERVE_TICK_SITES)
        line["serve"]["vs_fp64_plain"] = line["serve"]["site_steps_per_s"] / plain
        # the plain FP64 form one request at a time on the same mix: MV slices and steps per request
        mix = line["serve"].pop("_mix")
        per_n = plain_fp64_times(jw, local, sorted({m[0] for m in mix}))
        t_plain = sum(ny * per_n[n]["slice_ms"] + steps * per_n[n]["step_ms"] for n, ny, steps in mix) / 1e3
        mix_rate = sum(n * n * steps for n, _, steps in mix) / t_plain
        line["serve"]["fp64_plain_mix"] = {
            "site_steps_per_s": mix_rate, "seconds": t_plain,
            "per_n_ms": {str(n): v for n, v in per_n.items()},
            "what": "each request of the same mix alone, MV slices + steps through the call-for-call FP64 layer"}
        line["serve"]["vs_fp64_plain_mix"] = line["serve"]["site_steps_per_s"] / mix_rate
        line["uneven"] = uneven_leg(jw, local, 48)
        line["uneven"]["streams"] = uneven_streams_leg(jw, local)
        # served and uneven throughput as a fraction of the HBM roofline, by the
        # compulsory traffic of a mixed site-step (V read and written in FP64,
        # A and B written and read in FP32: 576 B)
        for leg in ("serve", "uneven"):
            line[leg]["hbm_frac"] = line[leg]["site_steps_per_s"] * 576 / (peak * 1e9)
            line[leg]["hbm_frac_basis"] = "576 B per site-step of compulsory traffic / measured HBM peak"
        line["position"] = position_leg(jw, local)
        line["c1"] = c1_leg(jw, local)
        # CPU baseline: the reference's own main on a bounded sample
        t, why = run_reference_main(2, 1)
        if t is not None:
            line["cpu_baseline"] = {"value": N * N / t, "unit": "site-steps/s", "cores": os.cpu_count(),
                                    "kind": "reference",
                                    "sample": f"1 event {N}^2, 2 Langevin steps after 1 warm-up; main_optimized "
                                              f"with OpenMP ({os.cpu_count()} threads, {cpu_model()}), FFT shim"}
        else:
            line["cpu_baseline"] = {"value": None, "unit": "site-steps/s", "cores": 0, "kind": "reference",
                                    "sample": why}
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip the FP64-plain and CPU-baseline legs")
    ap.add_argument("--events", type=int, default=EVENTS, help="events per GPU (profiling runs use fewer)")
    ap.add_argument("--max-batch", type=int, default=0, help="events per launch group (0 = engine default)")
    ap.add_argument("--serve-requests", type=int, default=1000, help="requests in the serving window")
    ap.add_argument("--n", type=int, default=N, help="lattice side (profiling runs; the workload is 512)")
    ap.add_argument("--column-form", type=int, default=0,
                    help="fix the column pass's tuning choice instead of autotuning (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "engine":
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
    else:
        main_arm(args)


if __name__ == "__main__":
    main()
