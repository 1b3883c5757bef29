"""FireXEngine — the reference engine's host API over the CUDA library.

Mirrors SimulationEngine / FireXEngine (src/sim/types.ts:34-63,
src/sim/firex/FireXEngine.ts:370-1032) for the simulation path: quality and offline-tier
tables, named parameters, transactional grid rebuilds, the fixed-step clock, the exact
offline timeline, reset, and — added for the drop-in — field readback. Presentation
members (canvas, render passes, video frames) are out of scope and absent.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np

from . import _abi as A
from . import grid as G
from .sim import FireXError, FireXSim, make_options


@dataclass(frozen=True)
class QualityConfiguration:
    dimensions: tuple
    pressureIterations: int
    correctionIterations: int
    maximumSubsteps: int
    timeStep: float
    raySteps: int
    renderScale: float
    particleCount: int
    minimumMemoryGuardBytes: int = 0
    opticalDetailTarget: int = 0


# FIREX_QUALITY (FireXEngine.ts:187-238)
FIREX_QUALITY = {
    "low": QualityConfiguration((32, 48, 32), 14, 14, 1, 1 / 30, 80, 0.82, 384),
    "balanced": QualityConfiguration((40, 64, 40), 24, 24, 1, 1 / 30, 112, 1, 640),
    "high": QualityConfiguration((64, 96, 64), 36, 36, 1, 1 / 30, 144, 1, 1024),
    "maximum": QualityConfiguration((80, 120, 80), 48, 48, 1, 1 / 30, 192, 1.25, 1536),
    "cinematic": QualityConfiguration((80, 120, 80), 48, 48, 1, 1 / 30, 192, 1, 1536),
}
# FIREX_OFFLINE_QUALITY (FireXEngine.ts:240-277)
FIREX_OFFLINE_QUALITY = {
    "hd": QualityConfiguration((128, 192, 128), 64, 64, 1, 1 / 60, 256, 1, 2048, 512 * 1024 * 1024, 512),
    "qhd": QualityConfiguration((160, 240, 160), 80, 80, 1, 1 / 60, 320, 1, 3072, 1024 * 1024 * 1024, 768),
    "uhd": QualityConfiguration((192, 288, 192), 96, 96, 1, 1 / 60, 384, 1, 4096, 2 * 1024 * 1024 * 1024, 1024),
}

# Named parameters and their reference defaults (FireXEngine.ts:422-451)
PARAMETER_NAMES = (
    "burnerSize", "burnerDepth", "sourceThickness", "firePower", "sourceLift", "buoyancyScale",
    "flamePersistence", "airEntrainment", "fuelRate", "oxygenRate", "heatEfficiency", "vorticity",
    "waterFlow", "sprayAngle", "waterEnabled", "cameraYaw", "cameraPitch", "cameraDistance", "viewMode",
    "aimHeight", "nozzleType", "exposure", "frontDefinition", "opticalDetailTarget", "domainWidth",
    "domainHeight", "domainDepth", "displayImperial", "viewZoom",
)


def resolveFireXOfflineDimensions(tier: str, override):
    """FireXEngine.ts:279-290: the tier preset, raised per axis by an override."""
    preset = FIREX_OFFLINE_QUALITY[tier].dimensions
    if not override:
        return preset
    return tuple(max(preset[i], override[i]) for i in range(3))


class FixedStepClock:
    """src/sim/FixedStepClock.ts: accumulator stepping with a per-frame cap."""

    def __init__(self, stepSeconds: float, maximumStepsPerFrame: int):
        if not (math.isfinite(stepSeconds) and stepSeconds > 0):
            raise ValueError("Fixed step must be finite and positive.")
        if not (isinstance(maximumStepsPerFrame, int) and maximumStepsPerFrame > 0):
            raise ValueError("Maximum step count must be a positive integer.")
        self.stepSeconds = stepSeconds
        self.maximumStepsPerFrame = maximumStepsPerFrame
        self.accumulator = 0.0

    def advance(self, deltaSeconds: float, step) -> int:
        if not math.isfinite(deltaSeconds):
            return 0
        bounded = max(0.0, min(deltaSeconds, self.stepSeconds * self.maximumStepsPerFrame))
        self.accumulator += bounded
        count = 0
        while self.accumulator >= self.stepSeconds and count < self.maximumStepsPerFrame:
            step(self.stepSeconds)
            self.accumulator -= self.stepSeconds
            count += 1
        if count == self.maximumStepsPerFrame and self.accumulator >= self.stepSeconds:
            self.accumulator = math.fmod(self.accumulator, self.stepSeconds)
        return count

    def reset(self) -> None:
        self.accumulator = 0.0


def splitOfflineSimulationDelta(deltaSeconds: float, maximumStepSeconds: float) -> tuple:
    """src/sim/offlineTimeline.ts:5-20: exact equal solver steps for one output frame."""
    if not math.isfinite(deltaSeconds) or deltaSeconds < 0:
        raise ValueError("Offline frame delta must be finite and non-negative.")
    if not math.isfinite(maximumStepSeconds) or maximumStepSeconds <= 0:
        raise ValueError("Offline maximum step must be positive and finite.")
    if deltaSeconds == 0:
        return ()
    n = max(1, math.ceil(deltaSeconds / maximumStepSeconds - 1e-12))
    return tuple([deltaSeconds / n] * n)


class FireXEngine:
    """Drop-in for the reference FireXEngine's simulation API (no presentation)."""

    backend = "CUDA sm_100a · 3D thermochemical grid"

    def __init__(self, quality: str = "balanced", sim_factory=FireXSim):
        self._factory = sim_factory
        self.quality = quality
        self.offlineRenderTier: str | None = None
        self.gridOverride = None
        self.gridMemoryBudgetBytes = 512 * 1024 * 1024
        self._params: dict[str, object] = {}
        self._sim = None
        self._extra_options: dict = {}
        self.clock = FixedStepClock(FIREX_QUALITY[quality].timeStep, FIREX_QUALITY[quality].maximumSubsteps)
        self.initialized = False
        self.disposed = False
        self.paused = False
        self.renderPacking = False

    # -- configuration ------------------------------------------------------------------------
    def activeConfiguration(self) -> QualityConfiguration:
        if self.offlineRenderTier is not None:
            return FIREX_OFFLINE_QUALITY[self.offlineRenderTier]
        return FIREX_QUALITY[self.quality]

    def effectiveGridDimensions(self):
        if self.offlineRenderTier is not None:
            return resolveFireXOfflineDimensions(self.offlineRenderTier, self.gridOverride)
        return tuple(self.gridOverride) if self.gridOverride else FIREX_QUALITY[self.quality].dimensions

    def usesCinematicPresentation(self) -> bool:
        return self.offlineRenderTier is not None or self.quality == "cinematic"

    def configure_simulation(self, **options) -> None:
        """Extra firex_options for the next (re)build: spheres, seed, velocity_noise,
        emission_jitter, precision, pressure_mode, jacobi_block (extensions)."""
        self._extra_options = dict(options)

    # -- lifecycle ----------------------------------------------------------------------------
    def initialize(self) -> None:
        if self.initialized:
            return
        if self.disposed:
            raise RuntimeError("The Fire-X engine has already been disposed.")
        self._rebuild(self.effectiveGridDimensions())
        self.initialized = True

    def dispose(self) -> None:
        if self.disposed:
            return
        self.disposed = True
        if self._sim is not None:
            self._sim.close()
            self._sim = None

    def _rebuild(self, dimensions, guard_bytes: int | None = None) -> None:
        """Transactional rebuild (FireXEngine.ts:1891-1931): the replacement is created
        first and the previous simulation is kept if that fails."""
        guard = self.gridMemoryBudgetBytes if guard_bytes is None else guard_bytes
        limits = {"maxTextureDimension3D": 2048, "maxStorageBufferBindingSize": 1 << 62, "maxBufferSize": 1 << 62}
        pre = G.preflightFireXGrid(tuple(dimensions), limits,
                                   particleCount=self.activeConfiguration().particleCount, memoryBudgetBytes=None)
        issues = [i.message for i in pre.issues]
        current = G.estimateFireXGridMemory(self._sim.dims, self.activeConfiguration().particleCount).totalBytes if self._sim else 0
        if current + pre.estimate.totalBytes > guard:
            issues.append(f"Transactional rebuild peak requires about {current + pre.estimate.totalBytes} bytes, above the selected {guard} guard.")
        if issues:
            raise FireXError(A.ERR_BUDGET, " ".join(issues))
        cfg = self.activeConfiguration()
        opts = make_options(pressure_iterations=cfg.pressureIterations, correction_iterations=cfg.correctionIterations,
                            cinematic=self.usesCinematicPresentation(), particle_count=cfg.particleCount,
                            **self._extra_options)
        replacement = self._factory(tuple(dimensions), opts)
        for name, value in self._params.items():
            replacement.set_parameter(name, value)
        if self.renderPacking and hasattr(replacement, "set_render_packing"):
            replacement.set_render_packing(True)
        replacement.reset()  # installResourceSet -> initializeFields with the current parameters
        previous, self._sim = self._sim, replacement
        self.clock.reset()
        if previous is not None:
            previous.close()

    def reset(self) -> None:
        self.clock.reset()
        if self._sim is not None:
            self._sim.reset()

    def setPaused(self, paused: bool) -> None:
        self.paused = paused
        if paused:
            self.clock.reset()

    def setParameter(self, name: str, value) -> None:
        if name in PARAMETER_NAMES:
            if self._sim is not None:
                self._sim.set_parameter(name, value)
                self._params[name] = self._sim.get_parameter(name) if name not in ("waterEnabled", "displayImperial") else value
            else:
                self._params[name] = value

    def getParameter(self, name: str) -> float:
        if self._sim is None:
            raise RuntimeError("engine is not initialised")
        return self._sim.get_parameter(name)

    def setQuality(self, quality: str) -> None:
        if quality not in FIREX_QUALITY:
            raise ValueError(f"Unknown quality level: {quality}")
        if self.offlineRenderTier is not None:
            raise RuntimeError("Compute quality cannot change while an exact offline solver bundle is active.")
        if quality == self.quality:
            return
        previous = self.quality
        self.quality = quality
        try:
            if self.initialized:
                self._rebuild(self.effectiveGridDimensions())
        except Exception:
            self.quality = previous
            raise
        cfg = FIREX_QUALITY[quality]
        self.clock = FixedStepClock(cfg.timeStep, cfg.maximumSubsteps)

    def setOfflineRenderTier(self, tier: str | None) -> None:
        if tier == self.offlineRenderTier:
            return
        if tier is not None and tier not in FIREX_OFFLINE_QUALITY:
            raise ValueError(f"Unknown offline tier: {tier}")
        previous = self.offlineRenderTier
        guard = max(self.gridMemoryBudgetBytes,
                    FIREX_OFFLINE_QUALITY[previous].minimumMemoryGuardBytes if previous else 0,
                    FIREX_OFFLINE_QUALITY[tier].minimumMemoryGuardBytes if tier else 0)
        self.offlineRenderTier = tier
        try:
            if self.initialized:
                self._rebuild(self.effectiveGridDimensions(), guard)
        except Exception:
            self.offlineRenderTier = previous
            raise
        cfg = self.activeConfiguration()
        self.clock = FixedStepClock(cfg.timeStep, cfg.maximumSubsteps)

    def setGridDimensions(self, dimensions) -> None:
        if self.offlineRenderTier is not None:
            raise RuntimeError("Grid dimensions cannot change while an exact offline solver bundle is active.")
        nxt = tuple(int(d) for d in dimensions) if dimensions else None
        if nxt == self.gridOverride:
            return
        target = nxt or FIREX_QUALITY[self.quality].dimensions
        if self._sim is not None and tuple(self._sim.dims) == tuple(target):
            self.gridOverride = nxt
            return
        if self.initialized:
            self._rebuild(target)
        self.gridOverride = nxt

    def setGridMemoryBudget(self, nbytes: float) -> None:
        if not math.isfinite(nbytes) or nbytes <= 0:
            return
        self.gridMemoryBudgetBytes = max(256 * 1024 * 1024, min(G.FIREX_MAX_GRID_MEMORY_BUDGET_BYTES, math.floor(nbytes)))

    def getGridInfo(self) -> dict:
        dims = tuple(self._sim.dims) if self._sim else self.effectiveGridDimensions()
        domain = tuple(self._params.get(n, d) for n, d in (("domainWidth", 1.15), ("domainHeight", 1.35), ("domainDepth", 1.15)))
        est = G.estimateFireXGridMemory(dims, self.activeConfiguration().particleCount)
        return {
            "dimensions": dims,
            "domainMeters": domain,
            "cellSizeMeters": tuple(domain[i] / dims[i] for i in range(3)),
            "cellCount": est.cellCount,
            "estimatedBytes": est.totalBytes,
            "deviceBytes": self._sim.device_bytes if self._sim is not None and hasattr(self._sim, "device_bytes") else None,
            "custom": self.offlineRenderTier is None and self.gridOverride is not None,
        }

    def getGridCapabilities(self) -> dict | None:
        if self._sim is None:
            return None
        limits = {"maxTextureDimension3D": 2048, "maxStorageBufferBindingSize": 1 << 40, "maxBufferSize": 1 << 40}
        return {**limits, "maximumDenseCubeAxis": G.maximumFireXDeviceDenseCubeAxis(limits)}

    # -- stepping -------------------------------------------------------------------------------
    def frame(self, timeSeconds: float, deltaSeconds: float) -> float:
        """Live path (FireXEngine.ts:629-641, submitReadyFrame :1064-1101): the fixed-step
        clock decides how many steps run; returns host milliseconds spent queueing."""
        if self._sim is None or self.disposed:
            return 0.0
        start = time.perf_counter()
        steps = [0]
        if not self.paused:
            self.clock.advance(deltaSeconds, lambda dt: steps.__setitem__(0, steps[0] + 1))
        if steps[0]:
            self._sim.step(steps[0], self.activeConfiguration().timeStep)
        return (time.perf_counter() - start) * 1e3

    def renderOfflineFrame(self, deltaSeconds: float, present: bool = True, signal=None) -> None:
        """Offline path (FireXEngine.ts:651-697): exact equal sub-steps, then wait. With
        `present`, the last sub-step also packs the render volumes (the headless stand-in for
        the presentation pass and its beauty volumes, qualityShaders.ts:77-87); a CPU
        simulation without device volumes packs on read instead."""
        if not math.isfinite(deltaSeconds) or deltaSeconds < 0:
            raise ValueError("Offline frame delta must be finite and non-negative.")
        if self._sim is None:
            raise RuntimeError("engine is not initialised")
        self.clock.reset()
        steps = splitOfflineSimulationDelta(deltaSeconds, self.activeConfiguration().timeStep)
        packs = present and hasattr(self._sim, "set_render_packing")
        for i, dt in enumerate(steps):
            if signal is not None and getattr(signal, "aborted", False):
                raise InterruptedError("Offline render canceled.")
            last = packs and i == len(steps) - 1 and not self.renderPacking
            if last:
                self._sim.set_render_packing(True)
            try:
                self._sim.step(1, dt)
            finally:
                if last:
                    self._sim.set_render_packing(False)
        if hasattr(self._sim, "sync"):
            self._sim.sync()

    def setRenderPacking(self, on: bool) -> None:
        """Pack the render volumes at the end of every step (a renderer on the same device
        reads them through renderVolumes())."""
        self.renderPacking = bool(on)
        if self._sim is not None and hasattr(self._sim, "set_render_packing"):
            self._sim.set_render_packing(self.renderPacking)

    def renderVolumes(self) -> list:
        """Device addresses of the flow, chemistry and media volumes (0 before first use)."""
        return self._sim.render_volumes() if hasattr(self._sim, "render_volumes") else [0, 0, 0]

    # -- readback (added for the drop-in) -------------------------------------------------------
    def readField(self, name: str) -> np.ndarray:
        if self._sim is None:
            raise RuntimeError("engine is not initialised")
        return self._sim.read(name)

    def readParticles(self) -> np.ndarray:
        """Droplets as (particleCount, 2, 4) float32: (x, y, z, age), (vx, vy, vz, mass)."""
        if self._sim is None:
            raise RuntimeError("engine is not initialised")
        return self._sim.read_particles()

    def divergenceNorm(self) -> tuple:
        return self._sim.divergence_norm()

    @property
    def simulation(self):
        return self._sim
