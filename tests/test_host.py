"""CPU tests of the host logic: grid model and preflight, fixed-step clock, offline
timeline, FireXEngine orchestration (with the oracle standing in for the device), and
the C-ABI library's exports (loaded, no compute calls)."""
from __future__ import annotations

import ctypes as C
import math
import re
from pathlib import Path

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200 import grid as G
from fire_b200.engine import (FIREX_OFFLINE_QUALITY, FIREX_QUALITY, FireXEngine, FixedStepClock,
                              resolveFireXOfflineDimensions, splitOfflineSimulationDelta)
from fire_b200.sim import FireXError, load_library
from oracle.oracle import OracleSim

ROOT = Path(__file__).resolve().parent.parent


# ---- gridConfiguration.test.ts / record-fire-lib.test.mjs ---------------------------------
def test_reference_508_cubed_memory_formula():
    est = G.estimateFireXGridMemory((508, 508, 508), 4096)
    assert est.cellCount == 131_096_512
    assert est.totalBytes / 1024 ** 3 == pytest.approx(13.187, abs=5e-3)


def test_heavy_threshold_switches_bytes_per_cell():
    below = G.estimateFireXGridMemory((1020, 256, 256))
    at = G.estimateFireXGridMemory((1024, 256, 256))
    assert below.cellCount < G.FIREX_HEAVY_GRID_CELL_THRESHOLD
    assert below.gridBytes == below.cellCount * 116
    assert at.cellCount == G.FIREX_HEAVY_GRID_CELL_THRESHOLD
    assert at.gridBytes == at.cellCount * 108


def test_grid_normalization():
    assert G.normalizeFireXGridDimensions((81, 142, 999)) == (80, 144, 1000)
    assert G.normalizeFireXGridDimensions((-3, 17, 18)) == (16, 16, 20)
    assert G.normalizeFireXGridDimensions((math.nan, math.inf, 66), fallback=(80, 120, 80)) == (80, 120, 68)
    assert G.normalizeFireXGridDimensions((1, 200, 77), minimumAxis=18, maximumAxis=126) == (20, 124, 76)


def test_preflight_issue_codes():
    limits = {"maxTextureDimension3D": 256, "maxStorageBufferBindingSize": 128 * 1024 * 1024,
              "maxBufferSize": 64 * 1024 * 1024}
    r = G.preflightFireXGrid((255, 512, 128), limits)
    codes = {i.code for i in r.issues}
    assert not r.ok
    assert {"unaligned-dimension", "texture-dimension-limit", "storage-binding-limit",
            "buffer-size-limit", "memory-budget"} <= codes
    ok = G.preflightFireXGrid((128, 192, 128), {"maxTextureDimension3D": 2048,
                                                 "maxStorageBufferBindingSize": 1 << 30, "maxBufferSize": 1 << 30})
    assert ok.ok and ok.estimate.totalBytes < G.FIREX_DEFAULT_GRID_MEMORY_BUDGET_BYTES


@pytest.mark.parametrize("dims,limits,particles,budget", [
    ((255, 512, 128), {"maxTextureDimension3D": 256, "maxStorageBufferBindingSize": 128 * 1024 * 1024,
                       "maxBufferSize": 64 * 1024 * 1024}, 0, G.FIREX_DEFAULT_GRID_MEMORY_BUDGET_BYTES),
    ((128, 192, 128), {"maxTextureDimension3D": 2048, "maxStorageBufferBindingSize": 1 << 30,
                       "maxBufferSize": 1 << 30}, 2048, G.FIREX_DEFAULT_GRID_MEMORY_BUDGET_BYTES),
    ((0, -4, 6), {"maxTextureDimension3D": 4, "maxStorageBufferBindingSize": 1 << 40, "maxBufferSize": 1 << 40}, 640, 0),
    ((508, 508, 508), {"maxTextureDimension3D": 2048, "maxStorageBufferBindingSize": 1 << 31,
                       "maxBufferSize": 1 << 32}, 4096, 16 * 1024 ** 3),
    ((1024, 256, 256), {"maxTextureDimension3D": 1024, "maxStorageBufferBindingSize": 1 << 40,
                        "maxBufferSize": 1 << 40}, 4096, 4 * 1024 ** 3),
])
def test_library_preflight_matches_reference_restatement(dims, limits, particles, budget):
    """firex_preflight gives the reference's issue codes, in its order, and its estimate."""
    from fire_b200.sim import make_options

    opts = make_options(particle_count=particles)
    opts.memory_budget_bytes = budget
    native = G.library_preflight(dims, opts, limits)
    ref = G.preflightFireXGrid(dims, limits, particleCount=particles, memoryBudgetBytes=budget or None)
    assert native.ok == ref.ok
    assert [i.code for i in native.issues] == [i.code for i in ref.issues]
    assert [i.message for i in native.issues] == [i.message for i in ref.issues]
    if all(d > 0 for d in dims):
        assert native.estimate == ref.estimate


def test_library_preflight_own_limits_and_create_admission():
    from fire_b200.sim import make_options

    opts = make_options()
    assert G.library_preflight((508, 508, 508), opts).ok
    r = G.library_preflight((2052, 2048, 2048), opts)
    assert [i.code for i in r.issues] == ["texture-dimension-limit", "storage-binding-limit", "buffer-size-limit"]
    lib = load_library()
    h = C.c_void_p()
    assert lib.firex_create(A.DIMS(2048, 1024, 1024), C.byref(opts), C.byref(h)) == A.ERR_BAD_ARG
    assert b"storage-binding-limit" in lib.firex_last_error(None)
    assert lib.firex_create(A.DIMS(64, 0, 64), C.byref(opts), C.byref(h)) == A.ERR_BAD_ARG
    assert b"invalid-dimension" in lib.firex_last_error(None)
    assert not h.value


def test_dense_cube_axis_limit():
    assert G.maximumFireXDeviceDenseCubeAxis({"maxTextureDimension3D": 2048,
                                              "maxStorageBufferBindingSize": 512 ** 3 * 16,
                                              "maxBufferSize": 512 ** 3 * 16}) == 512
    assert G.maximumFireXDeviceDenseCubeAxis({"maxTextureDimension3D": 2048,
                                              "maxStorageBufferBindingSize": 512 ** 3 * 16 - 1,
                                              "maxBufferSize": 512 ** 3 * 16}) == 508


# ---- FixedStepClock.test.ts / offlineTimeline.test.ts ------------------------------------------
def test_fixed_step_clock():
    clock = FixedStepClock(1 / 120, 8)
    elapsed = [0.0]
    clock.advance(1 / 60, lambda dt: elapsed.__setitem__(0, elapsed[0] + dt))
    clock.advance(1 / 60, lambda dt: elapsed.__setitem__(0, elapsed[0] + dt))
    assert elapsed[0] == pytest.approx(1 / 30, abs=1e-8)
    c2 = FixedStepClock(1 / 120, 4)
    assert c2.advance(10, lambda dt: None) == 4
    with pytest.raises(ValueError):
        FixedStepClock(math.nan, 4)
    assert FixedStepClock(1 / 120, 4).advance(math.inf, lambda dt: None) == 0


def test_offline_timeline():
    samples = [splitOfflineSimulationDelta(1 / 60, 1 / 30) for _ in range(60)]
    assert all(len(s) == 1 and s[0] > 0 for s in samples)
    assert sum(x for s in samples for x in s) == pytest.approx(1, abs=1e-12)
    steps = splitOfflineSimulationDelta(1 / 15, 1 / 30)
    assert len(steps) == 2 and max(steps) <= 1 / 30
    assert splitOfflineSimulationDelta(0, 1 / 30) == ()
    with pytest.raises(ValueError):
        splitOfflineSimulationDelta(-1, 1 / 30)


# ---- FireXEngine orchestration, oracle as the device ----------------------------------------
def _engine(quality="low"):
    return FireXEngine(quality=quality, sim_factory=lambda dims, opts: OracleSim(dims, opts))


def test_engine_quality_and_offline_tier_tables():
    assert FIREX_QUALITY["high"].dimensions == (64, 96, 64)
    assert FIREX_OFFLINE_QUALITY["hd"].pressureIterations == 64
    assert resolveFireXOfflineDimensions("hd", (100, 300, 50)) == (128, 300, 128)
    e = _engine()
    e.initialize()
    assert e.simulation.dims == (32, 48, 32)
    assert e.simulation.options.pressure_iterations == 14
    assert e.simulation.options.cinematic == 0
    e.setGridMemoryBudget(1 << 30)
    e.setOfflineRenderTier("hd")
    assert e.simulation.dims == (128, 192, 128)
    assert e.simulation.options.cinematic == 1
    with pytest.raises(RuntimeError):
        e.setQuality("high")
    e.dispose()


def test_engine_offline_frame_advances_time_and_frames():
    e = _engine()
    e.initialize()
    e.setParameter("firePower", 3.0)
    e.renderOfflineFrame(1 / 15)  # two 1/30 steps on the low tier
    st = e.simulation.state
    assert st["frame_index"] == 2 and st["simulation_time"] == pytest.approx(1 / 15)
    assert e.simulation.get_parameter("firePower") == 3.0
    e.reset()
    assert e.simulation.state["frame_index"] == 0
    e.dispose()


def test_engine_droplets_follow_the_tier_and_the_water_switch():
    e = _engine()
    e.initialize()
    assert e.readParticles().shape == (384, 2, 4)  # the low tier's particleCount
    e.setParameter("waterEnabled", True)
    e.setParameter("waterFlow", 0.7)
    e.renderOfflineFrame(1 / 15)
    assert (e.readParticles()[:, 1, 3] > 0).any() and e.readField("liquid").any()
    e.setParameter("waterEnabled", False)
    e.renderOfflineFrame(1 / 30)
    assert not e.readField("liquid").any()
    e.dispose()


def test_engine_rebuild_is_transactional():
    e = _engine()
    e.initialize()
    before = e.simulation
    e.setGridMemoryBudget(256 * 1024 * 1024)
    with pytest.raises(FireXError):
        e.setGridDimensions((512, 512, 512))  # above the guard: the old grid stays
    assert e.simulation is before and e.simulation.dims == (32, 48, 32)
    e.dispose()


def test_engine_frame_uses_fixed_step_clock():
    e = _engine()
    e.initialize()
    e.frame(0.0, 1 / 60)  # half a 1/30 step: nothing runs yet
    assert e.simulation.state["frame_index"] == 0
    e.frame(0.0, 1 / 60)
    assert e.simulation.state["frame_index"] == 1
    e.dispose()


# ---- the C-ABI library -----------------------------------------------------------------------
def _header_functions():
    text = (ROOT / "include" / "firex.h").read_text()
    return sorted(set(re.findall(r"\b(firex_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = load_library()
    names = _header_functions()
    assert names, "no declarations found"
    for n in names:
        assert hasattr(lib, n), n
    assert set(A.HEADER_SYMBOLS) <= set(names)


def test_library_host_only_entry_points():
    lib = load_library()
    o = A.Options()
    lib.firex_default_options(C.byref(o))
    assert (o.precision, o.pressure_mode, o.pressure_iterations, o.correction_iterations, o.cinematic) == (
        A.PRECISION_F32, A.PRESSURE_AUTO, 64, 64, 1)
    assert [lib.firex_field_element_size(f) for f in range(A.FIELD_COUNT)] == [16, 16, 4, 4, 4, 4, 1, 4, 4, 8, 8, 8]
    assert lib.firex_field_element_size(99) == 0
    for dims in ((508, 508, 508), (1020, 256, 256), (1024, 256, 256), (64, 96, 64)):
        assert lib.firex_reference_memory_estimate(A.DIMS(*dims), 4096) == G.estimateFireXGridMemory(dims, 4096).totalBytes


def test_create_rejects_bad_arguments_without_a_device():
    lib = load_library()
    h = C.c_void_p()
    o = A.Options()
    lib.firex_default_options(C.byref(o))
    assert lib.firex_create(A.DIMS(63, 96, 64), C.byref(o), C.byref(h)) == A.ERR_BAD_ARG
    assert b"unaligned-dimension: X must be a multiple of 4." in lib.firex_last_error(None)
    o.num_spheres = 99
    assert lib.firex_create(A.DIMS(64, 96, 64), C.byref(o), C.byref(h)) == A.ERR_BAD_ARG
    lib.firex_default_options(C.byref(o))
    o.memory_budget_bytes = 1024
    assert lib.firex_create(A.DIMS(64, 96, 64), C.byref(o), C.byref(h)) == A.ERR_BUDGET
    assert not h.value


def test_device_bytes_per_cell_matches_library_plan():
    """The Python memory model (admission by budget) and the library's plan agree up to the
    per-simulation constant (per-step tables, descriptor, scratch)."""
    lib = load_library()
    combos = [(A.PRECISION_F32, A.PRESSURE_WARM_F32), (A.PRECISION_F32, A.PRESSURE_F16),
              (A.PRECISION_F32, A.PRESSURE_COLD_F32), (A.PRECISION_MIXED, A.PRESSURE_WARM_F32),
              (A.PRECISION_MIXED, A.PRESSURE_F16)]
    for precision, mode in combos:
        o = A.Options()
        lib.firex_default_options(C.byref(o))
        o.precision, o.pressure_mode = precision, mode
        for dims in ((64, 96, 64), (128, 192, 128), (508, 508, 508)):
            n = dims[0] * dims[1] * dims[2]
            extra = lib.firex_planned_device_bytes(A.DIMS(*dims), C.byref(o)) - n * G.device_bytes_per_cell(precision, mode)
            assert 0 <= extra < (1 << 24), (precision, mode, dims, extra)
