"""Benchmark of the Fire-X simulation step on B200 (one JSON line on stdout, rank 0).

Workload (the HD tier the headline metric is quoted on): grid 128x192x128 (3,145,728
cells), plain FP32, sphere emitter r=14 cells at (64,12,64) injecting fuel 1.0 and
1500 K with a seeded +-10 % per-step jitter, velocity noise +-0.05, dt = 1/60 s,
96 primary + 96 residual Jacobi sweeps per step. Inputs are synthetic (no dataset).

A bench "step" is one full simulation step. ``value`` = cells x steps x ranks / device
seconds (max over ranks) with all state resident in HBM; ``e2e`` is the same metric
through the C ABI with, every step, the per-step parameter block going host -> device and
the resulting flow field (16 B/cell) read back into pinned host memory. The roofline
object is for the dominant kernel (the Jacobi sweep), timed with CUDA events on the
simulation's own stream inside the timed region.

``--impl reference`` times the CPU restatement of the reference step (oracle/, OpenMP on
all host cores) on the same workload: the reference itself is WGSL for WebGPU and cannot
run on this machine (no WebGPU implementation, no graphics stack, no JS runtime).

Multi-GPU (torchrun): each rank steps its own independent replica (weak scaling; the
step has no cross-rank exchange); barrier + synchronize around the timed region and the
max time over ranks.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

DIMS = (128, 192, 128)
P_ITERS = R_ITERS = 96
DT = 1.0 / 60.0
SPHERE = dict(center=(64.0, 12.0, 64.0), radius=14.0, fuel=1.0, temperature=1500.0)
SEED = 20251203
METRIC = "Gcell-steps/s"
WORKLOAD = "fire-x step, HD tier 128x192x128, plain FP32, sphere r=14 @ (64,12,64), +-10% jitter, 96+96 Jacobi, dt=1/60"
JACOBI_BYTES_PER_CELL = 12  # read p + read div + write p, f32 (algorithmic, per sweep)
L2_BYTES = 126 * 1024 * 1024
E2E_MIN_STEPS = 200


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of each Jacobi
# kernel on this workload, from one ncu capture of that kernel (the same command as this
# benchmark's default run, one launch captured).
# DRAM bytes per launch from captures at HD. The resident kernel: the mean of the step's two
# launches, the primary phase (25.26 MB + 1.34 MB) and the residual phase with its projection
# epilogue (63.03 MB + 33.37 MB: the flow read and written once).
JACOBI_TRAFFIC_PER_LAUNCH: dict = {"fxk_jacobi<float>": 25113088 + 768,
                                   "fxk_jacobi_res<float>": (25264640 + 1340928 + 63026944 + 33365504) // 2}
# The two-sweep pass at 508^3 (too large for a capture): one pass (2 sweeps) of a 508x508x128
# capture moved 266.7 MB + 104.2 MB of DRAM for 33,032,192 cells; the 508^3 figure scales it by
# the cell count (its traffic grows in proportion: the same tiles and chunks over more planes).
ZM2_CAPTURE_BYTES, ZM2_CAPTURE_CELLS = 266.7e6 + 104.2e6, 508 * 508 * 128

JACOBI_KERNEL_NAMES = {1: "fxk_jacobi<float>", 2: "fxk_jacobi_zm<float>", 3: "fxk_jacobi_zm2<float>",
                       4: "fxk_jacobi_res<float>"}


def zm2_roofline(jac: dict, cells: int, peak: float, peak_kind: str) -> dict:
    """The two-sweep pass at 508^3 against the copy bandwidth: algorithmic bytes per launch
    (2 sweeps x 12 B x cells) over the average launch time from the per-pass events, and the
    DRAM traffic of a launch scaled from the 508x508x128 capture."""
    launches = jac.get("launches_per_step") or 0
    if not launches or not jac.get("ms_per_step"):
        return {}
    us = jac["ms_per_step"] / launches * 1e3
    alg = 2 * JACOBI_BYTES_PER_CELL * cells
    achieved = alg / (us / 1e6) / 1e9
    return {"roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "avg_launch_us": us, "algorithmic_bytes_per_launch": alg,
                         "traffic": ZM2_CAPTURE_BYTES * cells / ZM2_CAPTURE_CELLS,
                         "traffic_note": "dram bytes of one launch at 508x508x128 (ncu), scaled by the cell count"}}


def jacobi_kernel_name(diag: dict) -> str:
    if diag.get("jacobi_kernel") == 3 and diag.get("jacobi_block") == 2:
        return "fxk_jacobi_zm2<float>"  # two sweeps per pass
    return JACOBI_KERNEL_NAMES.get(diag.get("jacobi_kernel"), "fxk_jacobi<float>")


def cells() -> int:
    return DIMS[0] * DIMS[1] * DIMS[2]


def options(make_options):
    return make_options(pressure_iterations=P_ITERS, correction_iterations=R_ITERS, seed=SEED, velocity_noise=0.05,
                        emission_jitter=0.1, spheres=[SPHERE])


def config(extra=None) -> dict:
    c = {"workload": WORKLOAD, "grid": list(DIMS), "cells": cells(), "jacobi": [P_ITERS, R_ITERS], "dt": DT,
         "l2": "inputs larger than L2: 365 MB of resident step state per replica vs 126 MB L2",
         "parallelism": "replicas (one independent simulation per GPU)"}
    if extra:
        c.update(extra)
    return c


_NVML_HANDLES: dict = {}


class ClockSampler:
    """Samples SM clocks and clock-event (throttle) reasons during a timed region, through
    NVML every 5 ms (reads only; nvidia-smi every 200 ms where NVML is unavailable). NVML is
    opened when the sampler is made, so a short timed region starts sampling at once."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*)
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40}

    def __init__(self, device_index: int, interval_s: float = 0.005):
        self.idx = device_index
        self.pci = None  # the CUDA device's PCI address: NVML indices need not follow CUDA's
        try:
            import torch
            p = torch.cuda.get_device_properties(device_index)
            self.pci = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        except Exception:
            pass
        self.interval = interval_s
        self.samples = []  # (sm_mhz, max_mhz, set of active reason names)
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        self._h = self._open()
        # the maximum SM clock is a constant and its query takes milliseconds (the current
        # clock and the reasons about 0.3 ms together): read it once, outside the timed region
        self._max_mhz = None
        if self._h is not None:
            try:
                import pynvml as N
                self._max_mhz = float(N.nvmlDeviceGetMaxClockInfo(self._h, N.NVML_CLOCK_SM))
            except Exception:
                self._h = None

    def _sample_nvml(self, h):
        import pynvml as N
        sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
        bits = N.nvmlDeviceGetCurrentClocksEventReasons(h)
        return float(sm), self._max_mhz, {k for k, b in self.REASON_BITS.items() if bits & b}

    def _sample_smi(self):
        out = subprocess.run(["nvidia-smi", "-i", self.pci or str(self.idx), f"--query-gpu={self.QUERY}",
                              "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
        parts = [p.strip() for p in out.stdout.strip().split(",")]
        if len(parts) < 9:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        return float(parts[1]), float(parts[2]), {names[i] for i in range(4) if parts[5 + i].lower() == "active"}

    def _open(self):
        """NVML handle of the CUDA device (opened once per process, before any timed region)."""
        global _NVML_HANDLES
        if self.idx in _NVML_HANDLES:
            return _NVML_HANDLES[self.idx]
        h = None
        try:
            import pynvml as N
            N.nvmlInit()
            try:
                h = N.nvmlDeviceGetHandleByPciBusId(self.pci) if self.pci else None
            except Exception:
                h = None
            if h is None:
                h = N.nvmlDeviceGetHandleByIndex(self.idx)
        except Exception:
            h = None
        _NVML_HANDLES[self.idx] = h
        return h

    def _run(self):
        h = self._h
        self._nvml = h
        while True:
            try:
                s = self._sample_nvml(h) if h is not None else self._sample_smi()
                if s:
                    self.samples.append(s)
            except Exception:
                pass
            if self._stop.wait(self.interval if h is not None else 0.2):
                break

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": sorted(set().union(*(s[2] for s in self.samples))), "samples": len(self.samples),
                "source": "nvml" if self._nvml is not None else "nvidia-smi"}


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline_sample(budget_s: float = 20.0) -> dict:
    """The CPU oracle (restatement of the reference step) on this host's cores: one warm-up
    step, then as many full HD steps as fit in about budget_s seconds (at least one)."""
    from fire_b200.sim import make_options
    from oracle import oracle as O
    O.build()
    sim = O.OracleSim(DIMS, options(make_options))
    sim.step(1, DT)
    n, t0 = 0, time.perf_counter()
    while True:
        sim.step(1, DT)
        n += 1
        el = time.perf_counter() - t0
        if el + el / n > budget_s:
            break
    sim.close()
    return {"value": cells() * n / el / 1e9, "unit": METRIC, "cores": O.num_threads(), "kind": "port",
            "sample": f"{n} full HD steps (96+96) after 1 warm-up, {el:.1f} s, OpenMP over z-slabs",
            "ms_per_step": el / n * 1e3}


def run_reference(args) -> None:
    """--impl reference: the CPU restatement of the reference path on this host."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from fire_b200.sim import make_options
    from oracle import oracle as O
    O.build()
    sim = O.OracleSim(DIMS, options(make_options))
    for _ in range(args.warmup):
        sim.step(1, DT)
    budget = float(os.environ.get("FIREX_REFERENCE_BUDGET_S", "90"))
    times = []
    t_start = time.perf_counter()
    for i in range(args.steps):
        t0 = time.perf_counter()
        sim.step(1, DT)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start + times[-1] > budget:
            break
    el = sum(times)
    n = len(times)
    value = cells() * n / el / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": n, "warmup": args.warmup, "ms_per_step": el / n * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config(),
        "reference_path": "CPU restatement of the src/sim/firex WGSL step (oracle/firex_oracle.cpp), OpenMP",
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": O.num_threads(), "kind": "port",
                         "sample": f"{n} of {args.steps} requested HD steps (budget {budget:.0f} s)"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_step_ms": statistics.median(times) * 1e3,
        "p99_step_ms": sorted(times)[min(n - 1, int(math.ceil(0.99 * n)) - 1)] * 1e3,
    }
    print(json.dumps(line), flush=True)


def percentile(xs, q):
    s = sorted(xs)
    return s[min(len(s) - 1, max(0, int(math.ceil(q * len(s))) - 1))]


def run_gpu(args) -> None:
    import numpy as np
    import torch

    from fire_b200.sim import FireXSim, make_options

    from fire_b200.replicas import Replicas

    reps = Replicas("nccl")
    world, rank = reps.world, reps.rank
    dev = torch.cuda.current_device()
    barrier, max_over_ranks = reps.barrier, reps.max

    sim = FireXSim(DIMS, options(make_options))
    stream = torch.cuda.ExternalStream(sim.stream)
    n_cells = cells()
    ClockSampler(dev)  # opens NVML now, outside every timed region

    # ---- warm-up ----
    sim.step(args.warmup, DT)
    sim.sync()

    # ---- device-resident timed region (each step replays the captured CUDA graph) ----
    sim.pass_times()  # clear the launch counters
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        evs[0].record(stream)
        for i in range(args.steps):
            sim.step(1, DT)
            evs[i + 1].record(stream)
        sim.sync()
        torch.cuda.synchronize()
    barrier()
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    total_ms = evs[0].elapsed_time(evs[-1])
    diag = sim.diagnostics
    launches = diag["launches_per_step"] * args.steps  # kernel nodes of the replayed step graph
    total_ms_max = max_over_ranks(total_ms)
    value = n_cells * args.steps * world / (total_ms_max / 1e3) / 1e9

    # ---- per-pass device times: the same steps launched pass by pass with CUDA events
    # recorded on the simulation's stream between passes (a graph hides its nodes) ----
    prof_steps = max(3, min(args.steps, 20))
    sim.set_profiling(True)
    sim.pass_times()
    barrier()
    sim.step(prof_steps, DT)
    passes = sim.pass_times()
    sim.set_profiling(False)

    # ---- end-to-end through the C ABI with host buffers: every step's flow field is
    # copied into pinned host memory (firex_read_field_async: staged on the device in
    # stream order, then copied while the next step runs); the clock stops after the last
    # copy has landed; at least E2E_MIN_STEPS steps (a window of a few tens of ms on the
    # host clock is dominated by its own start and stop) ----
    pinned = [torch.empty((DIMS[2], DIMS[1], DIMS[0], 4), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    hosts = [p.numpy() for p in pinned]
    e2e_steps = max(E2E_MIN_STEPS, args.steps)
    sim.step(1, DT)
    sim.read_async("flow", hosts[0])
    sim.sync()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        sim.step(1, DT)
        sim.read_async("flow", hosts[i % 2])
    sim.sync()
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e_value = n_cells * e2e_steps * world / t_e2e / 1e9
    assert np.isfinite(hosts[0]).all() and np.isfinite(hosts[1]).all()

    # ---- roofline of the dominant kernel ----
    jac_ms, jac_n = passes["jacobi"]
    jac_avg_ms = jac_ms / max(1, jac_n)
    # sweeps one launch performs: 1 for single-sweep kernels, a whole phase (P = R sweeps)
    # for the resident kernel, K for the fused one
    sweeps_per_launch = (P_ITERS + R_ITERS) * prof_steps / max(1, jac_n)
    peak, peak_kind = measured_peak_hbm()
    # the resident residual launch may also project the flow (36 B per cell: flow read and
    # written, the correction read), once per step, spread here over the step's launches
    epi_bytes = 36 * n_cells * prof_steps / max(1, jac_n) if diag.get("project_resident") else 0
    alg_bytes = JACOBI_BYTES_PER_CELL * n_cells * sweeps_per_launch + epi_bytes
    achieved = alg_bytes / (jac_avg_ms / 1e3) / 1e9
    kernel = jacobi_kernel_name(diag)
    traffic = JACOBI_TRAFFIC_PER_LAUNCH.get(kernel)

    sim.close()
    extra = {}
    if world == 1 and not args.hd_only:
        extra["config3_508"] = measure_508()
        extra["batch48"] = measure_batch48(steps=BATCH48_DEFAULT_STEPS, warmup=3)

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_sample(float(os.environ.get("FIREX_CPU_BASELINE_S", "20")))
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config(),
            "p50_step_ms": percentile(step_ms, 0.5), "p99_step_ms": percentile(step_ms, 0.99),
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 384,
                    "d2h_bytes_per_step": n_cells * 16, "steps": e2e_steps,
                    "what": "firex_step (384 B parameter block host->device) + firex_read_field_async(FLOW) into pinned host memory every step, overlapped with the next step; timed to the last copy"},
            "roofline": {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "traffic": traffic, "bytes_per_cell": JACOBI_BYTES_PER_CELL, "avg_launch_us": jac_avg_ms * 1e3,
                         "launches": jac_n, "sweeps_per_launch": sweeps_per_launch,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "projection_epilogue_bytes_per_launch": epi_bytes},
            "passes_ms_per_step": {k: v[0] / prof_steps for k, v in passes.items()},
            "profiled_steps": prof_steps,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            **extra,
        }
        print(json.dumps(line), flush=True)
    reps.close()


# ---- batched mixed precision: 48 uneven simulations stepped by shared launches --------------
BATCH_FAMILY = [(64, 96, 64), (96, 144, 96), (128, 192, 128), (160, 240, 160)]


def batch48_scenes(seed: int = 4242, count: int = 48):
    """48 scenes drawn by seed: grid from the family, 1-3 sphere emitters of radius 6-24
    cells at random positions near the floor, seeded noise and jitter."""
    import random
    rng = random.Random(seed)
    out = []
    for i in range(count):
        dims = rng.choice(BATCH_FAMILY)
        X, Y, Z = dims
        spheres = []
        for _ in range(rng.randint(1, 3)):
            r = rng.uniform(6.0, min(24.0, X / 4))
            spheres.append(dict(center=(rng.uniform(r, X - r), rng.uniform(2 + r / 2, Y / 5), rng.uniform(r, Z - r)),
                                radius=r, fuel=1.0, temperature=1500.0))
        out.append((dims, dict(pressure_iterations=96, correction_iterations=96, seed=rng.randrange(1 << 30),
                               velocity_noise=0.05, emission_jitter=0.1, spheres=spheres)))
    return out


def measure_batch48(steps: int, warmup: int = 3) -> dict:
    """Gcell-steps/s of the 48-simulation batch in mixed precision (one set of launches per
    step for all members, graph-replayed) against the same 48 simulations stepped one at a
    time in plain FP32, plus the post-projection divergence of every mixed member against
    its plain FP32 twin (relative to the twin's post-projection norm). The accuracy bar
    itself (one step from the FP64 oracle's state, <= 1e-4 of the pre-projection norm) is
    held by the GPU tests, which may run the oracle; this program times the GPU only."""
    import numpy as np
    import torch

    from fire_b200 import _abi as A
    from fire_b200.sim import FireXBatch, FireXSim, make_options

    dev = torch.cuda.current_device()
    scenes = batch48_scenes()
    cells = [d[0] * d[1] * d[2] for d, _ in scenes]
    total_cells = sum(cells)

    # plain FP32, one simulation at a time (each on its own stream, its own step graph)
    plain_ms = 0.0
    plain_norms = []
    with ClockSampler(dev) as clk_plain:
        for dims, o in scenes:
            s = FireXSim(dims, make_options(**o))
            st = torch.cuda.ExternalStream(s.stream)
            s.step(warmup, DT)
            s.sync()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            s.step(steps, DT)
            e1.record(st)
            s.sync()
            plain_ms += e0.elapsed_time(e1)
            plain_norms.append(s.read("final_divergence"))
            s.close()
    plain = total_cells * steps / (plain_ms / 1e3) / 1e9

    # batched, mixed precision; the Jacobi kernel and tiles are picked by the autotuner on a
    # scratch batch of the same workload, so the measured batch starts at the same state as
    # the plain runs
    from fire_b200.autotune import JacobiTuner

    def mixed_batch():
        bb = FireXBatch()
        ms = [FireXSim(dims, make_options(**{**o, "precision": A.PRECISION_MIXED})) for dims, o in scenes]
        for m in ms:
            bb.add(m)
        return bb, ms

    tuner = JacobiTuner(steps=1, warmup=1)
    scratch, scratch_members = mixed_batch()
    tuner.tune(scratch, DT)
    scratch.close()
    for m in scratch_members:
        m.close()
    b, members = mixed_batch()
    choice = tuner.tune(b, DT)  # cached: applied without stepping
    st = torch.cuda.ExternalStream(b.stream)
    b.step(warmup, DT)
    b.sync()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    with ClockSampler(dev) as clk:
        evs[0].record(st)
        for i in range(steps):
            b.step(1, DT)
            evs[i + 1].record(st)
        b.sync()
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
    batch_ms = evs[0].elapsed_time(evs[-1])
    batched = total_cells * steps / (batch_ms / 1e3) / 1e9
    diag = members[0].diagnostics
    # drift: each mixed member's post-projection divergence field after the run against its
    # plain FP32 twin's, relative to the twin's (post-projection) norm; it shows how far FP16
    # species rounding moves a multi-step trajectory
    worst = 0.0
    for m, ref in zip(members, plain_norms):
        d = m.read("final_divergence")[1:-1, 1:-1, 1:-1].astype(np.float64)
        r = ref[1:-1, 1:-1, 1:-1].astype(np.float64)
        worst = max(worst, float(np.linalg.norm((d - r).ravel()) / max(np.linalg.norm(r.ravel()), 1e-300)))
    b.close()
    for m in members:
        m.close()
    return {
        "workload": "48 simulations, grids by seed from 64x96x64 / 96x144x96 / 128x192x128 / 160x240x160, "
                    "1-3 spheres r 6-24, 96+96 Jacobi, dt=1/60, species stored FP16 (batched) vs plain FP32 "
                    "one simulation at a time, Jacobi kernel and tiles autotuned",
        "cells": total_cells, "grids": {str(d): sum(1 for x, _ in scenes if x == d) for d in BATCH_FAMILY},
        "steps": steps, "warmup": warmup,
        "value": batched, "unit": METRIC, "ms_per_step": batch_ms / steps,
        "plain_fp32_sequential": plain, "plain_ms_per_step": plain_ms / steps, "speedup_vs_plain": batched / plain,
        "p50_step_ms": percentile(step_ms, 0.5), "p99_step_ms": percentile(step_ms, 0.99),
        "jacobi_kernel": diag.get("jacobi_kernel"), "launches_per_step": diag.get("launches_per_step"),
        "jacobi_autotune": {"choice": choice.as_list(), "ms_per_step_by_candidate": tuner.last_timings},
        "final_divergence_drift_vs_plain_max": worst,
        "accuracy_bar": "rel_div <= 1e-4 vs the FP64 oracle, one step from its state (tests/test_mixed_gpu.py)",
        "clocks": clk.summary(), "clocks_plain": clk_plain.summary(),
    }


def run_batch48(args) -> None:
    import torch

    torch.cuda.set_device(0)
    r = measure_batch48(args.steps, args.warmup)
    line = {
        "metric": "Gcell-steps/s batched mixed vs plain FP32", "value": r["value"], "unit": METRIC, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (species stored f16)", "data": "synthetic",
        "config": {"workload": r["workload"], "cells": r["cells"], "grids": r["grids"], "l2": "inputs larger than L2"},
        **{k: v for k, v in r.items() if k not in ("workload", "cells", "grids", "value", "steps", "warmup",
                                                  "ms_per_step", "unit")},
    }
    print(json.dumps(line), flush=True)


# ---- the 508^3 grid: plain FP32 (branch A), three seeded spheres near the floor ------------
DIMS_508 = (508, 508, 508)
STEPS_508 = 20
# algorithmic bytes per cell of each pass of a 96 + 96 step (plain FP32, AoS flow, one sweep
# per Jacobi iteration, copyFlow replaced by a parity flip): simulate 72, two divergences of
# 20, 192 sweeps of 12, two projections of 36 = 2488 B per cell-step
PASS_BYTES_PER_CELL = {"simulate": 72, "divergence": 2 * 20, "jacobi": 192 * 12, "project": 2 * 36}
STEP_BYTES_PER_CELL = sum(PASS_BYTES_PER_CELL.values())
BATCH48_DEFAULT_STEPS = 50


def config3_spheres(seed: int = 0, n: int = 3):
    """Three seeded spheres of radius 20-40 cells resting near the floor of the 508^3 grid,
    away from the side walls."""
    import numpy as np
    rng = np.random.default_rng(seed)
    X, Y, Z = DIMS_508
    out = []
    for _ in range(n):
        r = float(rng.uniform(20.0, 40.0))
        out.append(dict(center=(float(rng.uniform(r + 8, X - r - 8)), r + 4.0, float(rng.uniform(r + 8, Z - r - 8))),
                        radius=r, fuel=1.0, temperature=1500.0))
    return out


def measure_508(warmup: int = 3, steps: int = STEPS_508) -> dict:
    """The 508^3 configuration in plain FP32 (branch A, warm-started FP32 pressure): device
    time of `steps` graph-replayed steps with the HBM-roofline fraction of the whole step,
    then the same steps pass by pass (CUDA events between passes) for the per-pass table."""
    import torch

    from fire_b200 import _abi as A
    from fire_b200.sim import FireXSim, make_options

    dev = torch.cuda.current_device()
    sim = FireXSim(DIMS_508, make_options(pressure_iterations=96, correction_iterations=96, seed=0, velocity_noise=0.05,
                                          emission_jitter=0.0, spheres=config3_spheres(),
                                          pressure_mode=A.PRESSURE_WARM_F32))
    st = torch.cuda.ExternalStream(sim.stream)
    sim.step(warmup, DT)
    sim.sync()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    with ClockSampler(dev) as clk:
        evs[0].record(st)
        for i in range(steps):
            sim.step(1, DT)
            evs[i + 1].record(st)
        sim.sync()
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
    total_ms = evs[0].elapsed_time(evs[-1])
    diag = sim.diagnostics
    prof = 3
    sim.set_profiling(True)
    sim.pass_times()
    sim.step(prof, DT)
    passes = sim.pass_times()
    sim.set_profiling(False)
    sim.close()
    n = DIMS_508[0] * DIMS_508[1] * DIMS_508[2]
    peak, peak_kind = measured_peak_hbm()
    ms = total_ms / steps
    achieved = STEP_BYTES_PER_CELL * n / (ms / 1e3) / 1e9
    per_pass = {}
    for k, b in PASS_BYTES_PER_CELL.items():
        t = passes[k][0] / prof
        a = b * n / (t / 1e3) / 1e9 if t > 0 else None
        per_pass[k] = {"ms_per_step": t, "launches_per_step": passes[k][1] / prof, "algorithmic_bytes_per_cell": b,
                       "achieved_gbs": a, "frac": a / peak if a else None}
    return {
        "workload": "fire-x step, 508x508x508 (131,096,512 cells), plain FP32 (branch A), 3 seeded spheres r 20-40 "
                    "near the floor, velocity noise +-0.05, 96+96 Jacobi, dt=1/60",
        "cells": n, "steps": steps, "warmup": warmup,
        "value": n * steps / (total_ms / 1e3) / 1e9, "unit": METRIC, "ms_per_step": ms,
        "p50_step_ms": percentile(step_ms, 0.5), "p99_step_ms": percentile(step_ms, 0.99),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "bytes_per_cell_step": STEP_BYTES_PER_CELL,
                     "target_frac": 0.70},
        "passes": per_pass, "profiled_steps": prof,
        "jacobi": {"kernel": jacobi_kernel_name(diag), "block": diag.get("jacobi_block"),
                   "zchunk": diag.get("jacobi_zchunk"), **zm2_roofline(per_pass["jacobi"], n, peak, peak_kind)},
        "launches_per_step": diag.get("launches_per_step"),
        "clocks": clk.summary(),
    }


# ---- served stream: Poisson arrivals, admission by HBM budget, continuous batching -----------
SERVE_FAMILY = [(64, 96, 64), (96, 144, 96), (128, 192, 128), (160, 240, 160), (192, 288, 192)]


def run_serve(args) -> None:
    """The served stream: Poisson arrivals at 40 requests/s, grids uniform over the family,
    60-600 steps each, 150 GB budget, mixed precision, continuous batching; the arrival
    window and the run are bounded by --serve-seconds. The same stream served plainly (one
    request at a time, FP32, FIFO) for the same time is reported beside it."""
    import torch

    from fire_b200 import _abi as A
    from fire_b200.serve import FireXServer, poisson_stream
    from fire_b200.sim import FireXSim, make_options

    torch.cuda.set_device(0)
    window = float(args.serve_seconds)
    stream = poisson_stream(40.0, window, SERVE_FAMILY, (60, 600), seed=777)
    srv = FireXServer(budget_bytes=150 * 10**9, precision=A.PRECISION_MIXED)
    srv.run_until_idle(list(stream), time_limit=window)
    served = srv.stats()
    srv.close()

    # plain: FIFO, one request at a time in FP32, same arrivals, same wall budget
    stream = poisson_stream(40.0, window, SERVE_FAMILY, (60, 600), seed=777)
    t0 = time.perf_counter()
    cell_steps, dev_ms, waits, steps_ms, lat = 0, 0.0, [], [], []
    done = 0
    for r in stream:
        now = time.perf_counter() - t0
        if now > window:
            break
        if r.arrival > now:
            time.sleep(r.arrival - now)
        waits.append(max(0.0, time.perf_counter() - t0 - r.arrival))
        s = FireXSim(r.dims, make_options(**r.options))
        st = torch.cuda.ExternalStream(s.stream)
        n = 0
        while n < r.steps and time.perf_counter() - t0 < window:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            s.step(1, r.dt)
            e1.record(st)
            s.sync()
            ms = e0.elapsed_time(e1)
            steps_ms.append(ms)
            dev_ms += ms
            n += 1
        cell_steps += n * r.dims[0] * r.dims[1] * r.dims[2]
        done += n == r.steps
        if n == r.steps:
            lat.append(time.perf_counter() - t0 - r.arrival)
        s.close()
    plain_wall = time.perf_counter() - t0
    plain = {"gcell_steps_per_s_device": cell_steps / (dev_ms / 1e3) / 1e9 if dev_ms else None,
             "gcell_steps_per_s_run_wall": cell_steps / plain_wall / 1e9, "run_wall_s": plain_wall,
             "p50_step_ms": percentile(steps_ms, 0.5) if steps_ms else None,
             "p99_step_ms": percentile(steps_ms, 0.99) if steps_ms else None,
             "p50_queue_wait_s": percentile(waits, 0.5) if waits else None,
             "p99_queue_wait_s": percentile(waits, 0.99) if waits else None, "completed": done,
             "completed_per_s": done / plain_wall,
             "p50_latency_s": percentile(lat, 0.5) if lat else None,
             "p99_latency_s": percentile(lat, 0.99) if lat else None}
    line = {
        "metric": "served Gcell-steps/s (wall clock of the run), p50/p99 step ms", "value": served["gcell_steps_per_s_run_wall"],
        "unit": METRIC, "n_gpus": 1, "higher_is_better": True, "dtype": "f32 (species stored f16)",
        "data": "synthetic", "config": {"workload": f"Poisson 40 req/s over {window:.0f} s, grids uniform over "
                                                    "64x96x64 .. 192x288x192, 60-600 steps, 150 GB budget, "
                                                    f"tick target {served['tick_target_ms']} ms",
                                         "requests": len(stream)},
        "served": served, "plain_fifo_fp32": plain,
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 300 for the HD step, as the reference's HD configuration; "
                         "10 for batch48)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fire_b200", choices=["fire_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--hd-only", action="store_true",
                    help="the HD line alone, without the 508^3 and 48-simulation objects")
    ap.add_argument("--workload", default="hd", choices=["hd", "batch48", "serve"],
                    help="hd: the headline HD step (default); batch48: 48 uneven simulations, batched mixed "
                         "vs plain FP32; serve: Poisson-arrival serving")
    ap.add_argument("--serve-seconds", type=float, default=30.0)
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 10 if args.workload == "batch48" else 300
    if args.warmup < 3 and args.impl != "reference":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch48":
        run_batch48(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
