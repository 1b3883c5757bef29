"""Autotuner of the step's launch shapes: picks the Jacobi kernel with its tile parameters
and plane staging, then the source pass's brick shape, for a simulation or a batch, by timing
real steps on the device.

Every Jacobi kernel of the library computes each sweep with the same FP32 operations in
the same order (the GPU tests hold them bit-identical), so the steps taken while tuning are
ordinary steps of the run: the trajectory is the same whichever candidate ran them. The
candidates are the resident kernel in each box variant that fits, the single-sweep kernels
(unblocked, and z-marching with 8, 16 or 32 planes per CTA) and the two-sweep pass with 16-,
32- or 64-plane chunks, its planes staged by TMA or by cp.async. With the fastest Jacobi
applied, the source pass's bricks (32 x 4 x 2, 32 x 2 x 4, 32 x 8 x 1 cells), each with the
primary projection fused with the residual divergence or run as two passes, are timed the same
way; every choice computes each cell with the same operations. The winner is applied
(set_jacobi, set_staging, set_tiles) and remembered per workload signature (grid sizes,
sweep counts, precision, pressure branch), optionally in a JSON file so that a later process
starts tuned.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from pathlib import Path

from . import _abi as A

KERNEL_NAMES = {A.JACOBI_UNBLOCKED: "unblocked", A.JACOBI_ZMARCH: "zmarch", A.JACOBI_FUSED: "fused",
                A.JACOBI_RESIDENT: "resident"}


@dataclass(frozen=True)
class Candidate:
    kernel: str
    block: int = 0
    zchunk: int = 0
    staging: int = A.STAGING_AUTO  # two-sweep pass: cp.async (AUTO) or TMA (FP32 pressure)
    simulate_by: int = 0           # source-pass bricks: 32 x by x (8 / by); 0 = default
    project: int = A.PROJECT_AUTO  # primary projection fused with the residual divergence or not

    def as_list(self) -> list:
        return [self.kernel, self.block, self.zchunk, self.staging, self.simulate_by, self.project]


def default_candidates() -> list:
    out = [Candidate("resident", v + 1) for v in (4, 3, 2, 1, 0)]
    out += [Candidate("unblocked")]
    out += [Candidate("zmarch", 0, zc) for zc in (8, 16, 32)]
    out += [Candidate("fused", 2, zc, st) for zc in (16, 32, 64) for st in (A.STAGING_CPASYNC, A.STAGING_TMA)]
    return out


SIMULATE_SHAPES = (4, 2, 8)


def _members(target) -> list:
    return list(getattr(target, "members", None) or [target])


def signature(target) -> str:
    """Workload key: sorted member shapes with their sweep counts, precision and branch."""
    parts = []
    for m in _members(target):
        o = m.options
        parts.append((tuple(m.dims), int(o.pressure_iterations), int(o.correction_iterations), int(o.precision),
                      int(m.pressure_mode)))
    return json.dumps(sorted(parts))


@dataclass
class JacobiTuner:
    cache_path: str | os.PathLike | None = None
    steps: int = 2    # timed steps per candidate
    warmup: int = 1   # untimed steps per candidate (plan change, graph capture)
    candidates: list = field(default_factory=default_candidates)
    cache: dict = field(default_factory=dict)
    last_timings: dict = field(default_factory=dict)

    def __post_init__(self):
        if self.cache_path and Path(self.cache_path).exists():
            self.cache = json.loads(Path(self.cache_path).read_text())

    def _save(self) -> None:
        if self.cache_path:
            Path(self.cache_path).write_text(json.dumps(self.cache, indent=1, sort_keys=True) + "\n")

    @staticmethod
    def _ran(target, c: Candidate) -> bool:
        """Whether the last step ran candidate c (a resident variant that does not fit falls
        back to the single-sweep default)."""
        d = _members(target)[0].diagnostics
        if c.kernel == "resident":
            return d["jacobi_kernel"] == A.JACOBI_RESIDENT and (c.block == 0 or d["jacobi_variant"] == c.block - 1)
        if c.kernel == "fused":
            return d["jacobi_kernel"] == A.JACOBI_FUSED
        return KERNEL_NAMES.get(d["jacobi_kernel"]) == c.kernel

    def _time(self, target, dt: float) -> float:
        import torch

        stream = torch.cuda.ExternalStream(target.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        target.sync()
        e0.record(stream)
        target.step(self.steps, dt)
        e1.record(stream)
        target.sync()
        return e0.elapsed_time(e1) / self.steps

    @staticmethod
    def apply(target, c: Candidate) -> None:
        target.set_jacobi(c.kernel, c.block, c.zchunk)
        target.set_staging(c.staging)
        target.set_tiles(c.simulate_by, c.project)

    def tune(self, target, dt: float = 1.0 / 60.0, force: bool = False) -> Candidate:
        """Times every Jacobi candidate on `target` (a FireXSim or FireXBatch) for warmup +
        steps real steps each, then the source pass's brick shapes with the fastest Jacobi;
        applies the fastest combination and returns it. A cached workload is applied without
        stepping."""
        key = signature(target)
        if key in self.cache and not force:
            best = Candidate(*self.cache[key]["choice"])
            self.apply(target, best)
            return best
        timings = {}
        for c in self.candidates:
            self.apply(target, c)
            target.step(self.warmup, dt)
            if not self._ran(target, c):
                continue
            timings[c] = self._time(target, dt)
        if not timings:
            self.apply(target, Candidate("auto"))
            return Candidate("auto")
        best = min(timings, key=timings.get)
        for by in SIMULATE_SHAPES:
            for proj in (A.PROJECT_FUSED, A.PROJECT_SEPARATE):
                c = Candidate(best.kernel, best.block, best.zchunk, best.staging, by, proj)
                self.apply(target, c)
                target.step(self.warmup, dt)
                timings[c] = self._time(target, dt)
        best = min(timings, key=timings.get)
        self.apply(target, best)
        self.last_timings = {json.dumps(c.as_list()): ms for c, ms in timings.items()}
        self.cache[key] = {"choice": best.as_list(), "ms_per_step": timings[best], "timings": self.last_timings}
        self._save()
        return best
