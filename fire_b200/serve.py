"""Continuous-batching server of independent Fire-X simulations on one GPU.

No reference counterpart: the reference steps one simulation per WebGPU device from a
requestAnimationFrame loop (FireXEngine.frame, FireXEngine.ts:651-697). Here many
simulation requests share the GPU:

* ``submit`` queues a request (grid, step count, scene); nothing is allocated yet;
* every ``tick`` first admits queued requests, oldest first, while their planned device
  bytes (``firex_planned_device_bytes``) fit the HBM budget, the batch has a free slot and
  the tick's estimated device time stays within the tick target (``TickBudget``: work in
  cell-sweep equivalents over the throughput measured on the ticks so far), so a tick never
  grows without bound and admitted requests keep finishing; an admitted request gets a
  resident simulation that joins the batch;
* the tick then advances every member by one step with the batch's shared launches
  (one launch per pass for all members), so requests that arrived while others were
  running overlap with them on the device;
* members that reached their step count are read back, leave the batch and free their
  memory before the next tick admits more.

Stepping a simulation inside the batch gives bit-identical fields to stepping it alone
(every kernel computes each cell with the same operations whichever members share the
launch), which ``tests/test_serve.py`` checks.

Per-tick device time comes from CUDA events on the batch stream; ``stats`` reports
p50/p99 step latency (device and wall), queue wait, request completion latency (arrival to
result), completed requests per second and throughput in Gcell-steps/s (device and wall).
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field

from . import _abi as A
from .sim import FireXBatch, FireXSim, make_options, planned_device_bytes

DEFAULT_BUDGET = 150 * 10**9
DEFAULT_TICK_MS = 40.0
# Device cost of one member step outside the Jacobi sweeps (simulate, divergence, both
# projections), in Jacobi cell-sweep equivalents; measured on B200 at 508^3: simulate 8.7 ms,
# divergence and projections 3.3 ms against 1.79 ns per cell-sweep of the two-sweep pass.
FIXED_SWEEP_EQUIVALENTS = 50


class TickBudget:
    """Bounds the device time of a tick. A member's work per tick is cells x (P + R +
    FIXED_SWEEP_EQUIVALENTS) cell-sweep equivalents; the device rate (equivalents per ms) is
    an exponential average over measured ticks, starting from `initial_rate`. A request is
    admitted when the batch is empty or the estimated tick time with it stays within
    `target_ms`."""

    def __init__(self, target_ms: float = DEFAULT_TICK_MS, initial_rate: float = 4.0e8, smoothing: float = 0.3):
        self.target_ms = float(target_ms)
        self.rate = float(initial_rate)
        self.smoothing = float(smoothing)

    @staticmethod
    def work(dims, options) -> float:
        cells = dims[0] * dims[1] * dims[2]
        return float(cells) * (int(options.pressure_iterations) + int(options.correction_iterations) +
                               FIXED_SWEEP_EQUIVALENTS)

    def estimate_ms(self, work: float) -> float:
        return work / self.rate

    def fits(self, current_work: float, candidate_work: float, members: int) -> bool:
        return members == 0 or self.estimate_ms(current_work + candidate_work) <= self.target_ms

    def observe(self, work: float, ms: float) -> None:
        if work > 0 and ms > 0:
            self.rate += self.smoothing * (work / ms - self.rate)


@dataclass
class Request:
    """One simulation request: `steps` steps of a `dims` grid from reset."""
    dims: tuple
    steps: int
    options: dict = field(default_factory=dict)   # make_options keywords (scene, iterations, precision)
    dt: float = 1.0 / 60.0
    keep: tuple = ("flow",)                      # fields read back when the request completes
    arrival: float | None = None                  # server clock seconds (None: at submit)


@dataclass
class _Slot:
    rid: int
    req: Request
    sim: FireXSim
    bytes: int
    done: int = 0
    admitted: float = 0.0
    work: float = 0.0


def _percentile(xs, q):
    if not xs:
        return None
    s = sorted(xs)
    return s[min(len(s) - 1, max(0, int(math.ceil(q * len(s))) - 1))]


class FireXServer:
    """Admission by HBM budget + one shared batch stepped per tick."""

    def __init__(self, budget_bytes: int = DEFAULT_BUDGET, max_members: int = 512, clock=time.perf_counter,
                 device_timing: bool = True, dt: float = 1.0 / 60.0, precision: int = A.PRECISION_MIXED,
                 pressure_mode: int = A.PRESSURE_WARM_F32, tick_target_ms: float | None = DEFAULT_TICK_MS):
        # one batch shares the storage precision, the pressure storage and dt
        self.dt = float(dt)
        self.precision = int(precision)
        self.pressure_mode = int(pressure_mode)
        self.budget = int(budget_bytes)
        self.max_members = int(max_members)
        self.batch = FireXBatch()
        self.queue: collections.deque = collections.deque()
        self.slots: dict[int, _Slot] = {}
        self.results: dict[int, dict] = {}
        self.used = 0
        self._next = 0
        self._clock = clock
        self._t0 = clock()
        self.tick_ms: list[float] = []
        self.tick_wall_ms: list[float] = []
        self.tick_cells: list[int] = []
        self.waits: list[float] = []
        self.latencies: list[float] = []  # arrival to result, completed requests
        self.tick_budget = TickBudget(tick_target_ms) if tick_target_ms else None
        self.work = 0.0  # cell-sweep equivalents of the members per tick
        self._events = None
        self._stream = None
        if device_timing:
            import torch
            self._torch = torch
            self._stream = torch.cuda.ExternalStream(self.batch.stream)

    # ---- clock ----------------------------------------------------------------------------
    def now(self) -> float:
        return self._clock() - self._t0

    # ---- requests -------------------------------------------------------------------------
    def submit(self, req: Request) -> int:
        rid = self._next
        self._next += 1
        if req.arrival is None:
            req.arrival = self.now()
        if req.dt != self.dt:
            self.results[rid] = {"status": "rejected", "reason": f"dt {req.dt} differs from the server's {self.dt}"}
            return rid
        opts = make_options(**{**req.options, "precision": self.precision, "pressure_mode": self.pressure_mode})
        need = planned_device_bytes(req.dims, opts)
        if need > self.budget:
            self.results[rid] = {"status": "rejected", "reason": f"needs {need} bytes, budget {self.budget}"}
            return rid
        self.queue.append((rid, req, opts, need))
        return rid

    def poll(self, rid: int) -> dict:
        if rid in self.results:
            return self.results[rid]
        if rid in self.slots:
            s = self.slots[rid]
            return {"status": "running", "done": s.done, "steps": s.req.steps}
        return {"status": "queued"}

    def idle(self) -> bool:
        return not self.queue and not self.slots

    # ---- one tick -------------------------------------------------------------------------
    def _admit(self) -> None:
        while self.queue and len(self.slots) < self.max_members:
            rid, req, opts, need = self.queue[0]
            if req.arrival > self.now() or self.used + need > self.budget:
                break  # FIFO: the oldest request waits for memory rather than being overtaken
            work = TickBudget.work(req.dims, opts)
            if self.tick_budget is not None and not self.tick_budget.fits(self.work, work, len(self.slots)):
                break  # ... and for the tick's time budget
            self.queue.popleft()
            sim = FireXSim(req.dims, opts)
            self.batch.add(sim)
            self.used += need
            self.work += work
            t = self.now()
            self.slots[rid] = _Slot(rid, req, sim, need, 0, t, work)
            self.waits.append(t - req.arrival)

    def _finish(self) -> None:
        for rid in [r for r, s in self.slots.items() if s.done >= s.req.steps]:
            s = self.slots.pop(rid)
            out = {f: s.sim.read(f) for f in s.req.keep}
            l2, linf, n = s.sim.divergence_norm()
            self.batch.remove(s.sim)
            s.sim.close()
            self.used -= s.bytes
            self.work -= s.work
            t = self.now()
            self.latencies.append(t - s.req.arrival)
            self.results[rid] = {"status": "done", "fields": out, "divergence_norm": (l2, linf, n),
                                 "queue_wait_s": s.admitted - s.req.arrival, "finished_s": t,
                                 "latency_s": t - s.req.arrival}

    def tick(self) -> bool:
        """Admits, steps every member once, retires finished members. False when idle."""
        self._admit()
        if not self.slots:
            return False
        cells = sum(s.req.dims[0] * s.req.dims[1] * s.req.dims[2] for s in self.slots.values())
        w0 = self._clock()
        if self._stream is not None:
            e0 = self._torch.cuda.Event(enable_timing=True)
            e1 = self._torch.cuda.Event(enable_timing=True)
            e0.record(self._stream)
        self.batch.step(1, self.dt)
        if self._stream is not None:
            e1.record(self._stream)
        self.batch.sync()
        self.tick_wall_ms.append((self._clock() - w0) * 1e3)
        if self._stream is not None:
            self.tick_ms.append(e0.elapsed_time(e1))
            if self.tick_budget is not None:
                self.tick_budget.observe(self.work, self.tick_ms[-1])
        self.tick_cells.append(cells)
        for s in self.slots.values():
            s.done += 1
        self._finish()
        return True

    def run_until_idle(self, arrivals: list[Request] | None = None, time_limit: float | None = None) -> None:
        """Feeds `arrivals` (by their arrival times) and ticks until everything finished."""
        self._run_start = self.now()
        pending = collections.deque(sorted(arrivals or [], key=lambda r: r.arrival))
        while True:
            while pending and pending[0].arrival <= self.now():
                self.submit(pending.popleft())
            if time_limit is not None and self.now() > time_limit:
                break
            if not self.tick():
                if not pending and not self.queue:
                    break
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - self.now())))
        self._run_wall = self.now() - self._run_start

    # ---- reporting -----------------------------------------------------------------------
    def stats(self) -> dict:
        dev_ms = sum(self.tick_ms) if self.tick_ms else None
        cells = sum(self.tick_cells)
        completed = sum(1 for r in self.results.values() if r.get("status") == "done")
        run_wall = getattr(self, "_run_wall", None)
        return {
            "p50_latency_s": _percentile(self.latencies, 0.5), "p99_latency_s": _percentile(self.latencies, 0.99),
            "completed_per_s": completed / run_wall if run_wall else None,
            "gcell_steps_per_s_run_wall": cells / run_wall / 1e9 if run_wall else None,
            "run_wall_s": run_wall, "queued_at_end": len(self.queue), "running_at_end": len(self.slots),
            "tick_target_ms": self.tick_budget.target_ms if self.tick_budget else None,
            "ticks": len(self.tick_wall_ms),
            "cell_steps": cells,
            "gcell_steps_per_s_device": cells / (dev_ms / 1e3) / 1e9 if dev_ms else None,
            "gcell_steps_per_s_wall": cells / (sum(self.tick_wall_ms) / 1e3) / 1e9 if self.tick_wall_ms else None,
            "p50_step_ms": _percentile(self.tick_ms, 0.5), "p99_step_ms": _percentile(self.tick_ms, 0.99),
            "p50_step_wall_ms": _percentile(self.tick_wall_ms, 0.5), "p99_step_wall_ms": _percentile(self.tick_wall_ms, 0.99),
            "p50_queue_wait_s": _percentile(self.waits, 0.5), "p99_queue_wait_s": _percentile(self.waits, 0.99),
            "completed": completed,
            "rejected": sum(1 for r in self.results.values() if r.get("status") == "rejected"),
        }

    def close(self) -> None:
        for s in list(self.slots.values()):
            self.batch.remove(s.sim)
            s.sim.close()
        self.slots.clear()
        self.batch.close()


def poisson_stream(rate: float, duration: float, families, step_range, seed: int, options=None) -> list[Request]:
    """Seeded Poisson arrivals (exponential gaps at `rate` per second over `duration`
    seconds); each request draws its grid uniformly from `families` and its step count
    uniformly from `step_range`, with one sphere emitter placed by the same generator."""
    import random
    rng = random.Random(seed)
    t, out = 0.0, []
    while True:
        t += rng.expovariate(rate)
        if t > duration:
            return out
        dims = tuple(rng.choice(families))
        steps = rng.randint(step_range[0], step_range[1])
        X, Y, Z = dims
        r = rng.uniform(6.0, min(24.0, X / 4))
        sphere = dict(center=(rng.uniform(r, X - r), rng.uniform(r * 0.5 + 2, Y / 6 + r), rng.uniform(r, Z - r)),
                      radius=r, fuel=1.0, temperature=1500.0)
        opts = dict(options or {})
        opts.setdefault("pressure_iterations", 96)
        opts.setdefault("correction_iterations", 96)
        opts.update(seed=rng.randrange(1 << 30), velocity_noise=0.05, emission_jitter=0.1, spheres=[sphere])
        out.append(Request(dims=dims, steps=steps, options=opts, arrival=t, keep=()))
