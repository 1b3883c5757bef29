"""Grid configuration, memory model and preflight (gridConfiguration.ts).

Mirrors the reference's pure functions with the same names, constants and issue codes
so admission decisions can be checked against the reference's own unit tests
(gridConfiguration.test.ts). ``device_bytes_per_cell`` gives this library's actual
residency for the same grid, which the serving layer admits against.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

from . import _abi as A

FIREX_GRID_AXIS_QUANTUM = 4                      # gridConfiguration.ts:98
FIREX_GRID_MINIMUM_AXIS = 16                     # :99
FIREX_GRID_MAXIMUM_AXIS = 1024                   # :100
FIREX_HEAVY_GRID_CELL_THRESHOLD = 64 * 1024 * 1024   # :105
FIREX_GRID_BYTES_PER_CELL = 116                  # :106
FIREX_HEAVY_GRID_BYTES_PER_CELL = 108            # :107
FIREX_PARTICLE_BYTES = 80                        # :108
FIREX_LARGEST_STORAGE_BYTES_PER_CELL = 16        # :109
FIREX_DETAIL_TEXTURE_BYTES = 64 * 64 * 64 * 4    # :110
FIREX_DEFAULT_GRID_MEMORY_BUDGET_BYTES = 512 * 1024 * 1024   # :111
FIREX_MAX_NEGOTIATED_STORAGE_BYTES = 512 ** 3 * FIREX_LARGEST_STORAGE_BYTES_PER_CELL  # :112
GIB = 1024 ** 3
FIREX_GRID_MEMORY_GUARDS = [                     # :116-125
    (512 * 1024 * 1024, "Safe · 512 MiB"), (GIB, "Heavy · 1 GiB"), (2 * GIB, "Expert · 2 GiB"),
    (4 * GIB, "Workstation · 4 GiB"), (8 * GIB, "Studio · 8 GiB"), (16 * GIB, "Reference · 16 GiB"),
    (24 * GIB, "Reference swap · 24 GiB"), (32 * GIB, "Maximum opt-in · 32 GiB"),
]
FIREX_MAX_GRID_MEMORY_BUDGET_BYTES = FIREX_GRID_MEMORY_GUARDS[-1][0]

# Grid presets (gridConfiguration.ts:135-184)
FIREX_GRID_PRESETS = {
    "maximum": (80, 120, 80), "ultra": (96, 144, 96), "experimental": (128, 192, 128),
    "extreme": (160, 160, 160), "expert": (256, 256, 256), "workstation": (320, 320, 320),
    "studio": (384, 384, 384), "reference": (508, 508, 508),
}


@dataclass
class MemoryEstimate:
    cellCount: int
    gridBytes: int
    particleBytes: int
    fixedBytes: int
    totalBytes: int
    largestStorageBufferBytes: int


@dataclass
class PreflightIssue:
    code: str
    message: str


@dataclass
class PreflightResult:
    ok: bool
    dimensions: tuple
    estimate: MemoryEstimate
    issues: list = field(default_factory=list)


def fireXGridCellCount(dimensions) -> int:
    return int(dimensions[0]) * int(dimensions[1]) * int(dimensions[2])


def estimateFireXGridMemory(dimensions, particleCount: int = 0) -> MemoryEstimate:
    """Reference persistent-memory model (gridConfiguration.ts:272-291)."""
    cells = fireXGridCellCount(dimensions)
    per = FIREX_HEAVY_GRID_BYTES_PER_CELL if cells >= FIREX_HEAVY_GRID_CELL_THRESHOLD else FIREX_GRID_BYTES_PER_CELL
    grid = cells * per
    pc = particleCount if isinstance(particleCount, (int, float)) and math.isfinite(particleCount) else 0
    particles = max(0, math.floor(pc)) * FIREX_PARTICLE_BYTES
    fixed = FIREX_DETAIL_TEXTURE_BYTES
    return MemoryEstimate(cells, grid, particles, fixed, grid + particles + fixed,
                          cells * FIREX_LARGEST_STORAGE_BYTES_PER_CELL)


def _normalize_axis(value, fallback, minimum, maximum):
    v = value if isinstance(value, (int, float)) and math.isfinite(value) else fallback
    snapped = _js_round(v / FIREX_GRID_AXIS_QUANTUM) * FIREX_GRID_AXIS_QUANTUM
    return max(minimum, min(maximum, snapped))


def _js_round(v: float) -> int:
    """JavaScript Math.round: halves round toward +infinity."""
    return math.floor(v + 0.5)


def normalizeFireXGridDimensions(dimensions, minimumAxis=FIREX_GRID_MINIMUM_AXIS,
                                 maximumAxis=FIREX_GRID_MAXIMUM_AXIS, fallback=(64, 96, 64)):
    """Snap to multiples of four and clamp (gridConfiguration.ts:232-265)."""
    lo = math.ceil(minimumAxis / FIREX_GRID_AXIS_QUANTUM) * FIREX_GRID_AXIS_QUANTUM
    hi = math.floor(maximumAxis / FIREX_GRID_AXIS_QUANTUM) * FIREX_GRID_AXIS_QUANTUM
    if lo <= 0 or hi < lo:
        raise ValueError("Fire-X grid bounds must contain at least one positive multiple of four.")
    return tuple(_normalize_axis(dimensions[i], fallback[i], lo, hi) for i in range(3))


def preflightFireXGrid(dimensions, limits: dict, particleCount: int = 0,
                       memoryBudgetBytes: int | None = FIREX_DEFAULT_GRID_MEMORY_BUDGET_BYTES) -> PreflightResult:
    """Limit and budget checks with the reference's issue codes (gridConfiguration.ts:297-350)."""
    est = estimateFireXGridMemory(dimensions, particleCount)
    issues = []
    for label, d in zip("XYZ", dimensions):
        if not isinstance(d, int) or d <= 0:
            issues.append(PreflightIssue("invalid-dimension", f"{label} must be a positive integer."))
        elif d % FIREX_GRID_AXIS_QUANTUM != 0:
            issues.append(PreflightIssue("unaligned-dimension", f"{label} must be a multiple of {FIREX_GRID_AXIS_QUANTUM}."))
        if isinstance(d, (int, float)) and d > limits["maxTextureDimension3D"]:
            issues.append(PreflightIssue("texture-dimension-limit",
                                         f"{label}={d} exceeds this device's 3D-texture limit of {limits['maxTextureDimension3D']}."))
    if est.largestStorageBufferBytes > limits["maxStorageBufferBindingSize"]:
        issues.append(PreflightIssue("storage-binding-limit", "A Fire-X vector field exceeds the storage-binding limit."))
    if est.largestStorageBufferBytes > limits["maxBufferSize"]:
        issues.append(PreflightIssue("buffer-size-limit", "A Fire-X vector field exceeds the buffer limit."))
    if memoryBudgetBytes is not None and est.totalBytes > memoryBudgetBytes:
        issues.append(PreflightIssue("memory-budget",
                                     f"Estimated persistent Fire-X resources require {est.totalBytes} bytes, above the configured {memoryBudgetBytes} budget."))
    return PreflightResult(not issues, tuple(dimensions), est, issues)


def maximumFireXDeviceDenseCubeAxis(limits: dict) -> int:
    """gridConfiguration.ts:207-226."""
    cand = min(limits["maxStorageBufferBindingSize"], limits["maxBufferSize"])
    largest = max(0, cand) if math.isfinite(cand) else 0
    axis = math.floor((largest / FIREX_LARGEST_STORAGE_BYTES_PER_CELL) ** (1 / 3))
    while (axis + 1) ** 3 * FIREX_LARGEST_STORAGE_BYTES_PER_CELL <= largest:
        axis += 1
    while axis ** 3 * FIREX_LARGEST_STORAGE_BYTES_PER_CELL > largest:
        axis -= 1
    m = min(FIREX_GRID_MAXIMUM_AXIS, max(0, math.floor(limits["maxTextureDimension3D"])), axis)
    aligned = (m // FIREX_GRID_AXIS_QUANTUM) * FIREX_GRID_AXIS_QUANTUM
    return aligned if aligned >= FIREX_GRID_MINIMUM_AXIS else 0


def device_bytes_per_cell(precision: int = A.PRECISION_F32, pressure_mode: int = A.PRESSURE_WARM_F32) -> int:
    """Bytes per cell this library allocates for one simulation (the engine's planned_bytes
    without its per-simulation constant): flow ping-pong, species ping-pong (FP16 when
    mixed), pressure + residual pressure buffers (FP16 in branch B; the cold branch shares
    one pair), divergence, reaction, liquid and one scratch field."""
    species = 8 if precision == A.PRECISION_MIXED else 16
    pbytes = 2 if pressure_mode == A.PRESSURE_F16 else 4
    npress = 2 if pressure_mode == A.PRESSURE_COLD_F32 else 4
    return 16 * 2 + species * 2 + pbytes * npress + 4 * 4


def library_preflight(dimensions, options=None, limits: dict | None = None) -> PreflightResult:
    """firex_preflight through the C ABI: the same checks and codes, evaluated natively
    (limits None: the library's own). options carry particle_count and
    memory_budget_bytes (0 = no budget)."""
    import ctypes as C

    from .sim import load_library, make_options

    lib = load_library()
    opts = options if options is not None else make_options()
    lim = None
    if limits is not None:
        lim = A.DeviceLimits(int(limits["maxTextureDimension3D"]), int(limits["maxStorageBufferBindingSize"]),
                             int(limits["maxBufferSize"]))
    r = A.PreflightResult()
    rc = lib.firex_preflight(A.DIMS(*dimensions), C.byref(opts), C.byref(lim) if lim is not None else None, C.byref(r))
    if rc != A.OK:
        raise ValueError("firex_preflight refused its arguments")
    est = MemoryEstimate(r.cell_count, r.grid_bytes, r.particle_bytes, r.fixed_bytes, r.total_bytes,
                         r.largest_storage_buffer_bytes)
    issues = [PreflightIssue(*part.split(": ", 1)) for part in r.message.decode().split("; ") if part]
    return PreflightResult(r.issues == 0, tuple(dimensions), est, issues)
