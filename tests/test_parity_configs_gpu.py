"""GPU parity against the CPU oracle at the configurations the benchmark and AUTO run.

The small-grid parity tests (test_parity_gpu.py) pin every kernel on grids where AUTO picks
the unblocked Jacobi. These tests compare the CUDA path with the oracle directly where AUTO
picks the other kernels:

  * the HD tier (128x192x128, sphere r=14 at (64,12,64), +-10 % jitter, 96+96 sweeps), the
    benchmark's workload, where AUTO runs the resident Jacobi (box variant 4: faces first,
    interior columns, halo rows brought in by a copy warp);
  * 508x508x36 (9,290,304 cells, above the 8 Mi-cell threshold), where AUTO runs two sweeps
    per HBM pass (the z-marching two-sweep kernel with 16-plane chunks; 36 planes leave a
    partial chunk), in branch A (FP32) and branch B (FP16 pressure, pressureShaders.ts:62-117).

Each starts from a developed state the oracle computed (a few steps with few sweeps), copied
into both sides, and checks a dt = 0 step bit for bit (every transcendental is multiplied by
dt = 0) and a dt = 1/60 step within the tolerances of test_parity_gpu (ATOL: the few-ULP
differences of CUDA's sinf/cosf/expf/powf against the C library's). The dispatch graph is
FireXEngine.ts:2172-2276.
"""
from __future__ import annotations

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXSim
from oracle.oracle import OracleSim
from tests.helpers import DT, copy_state, max_abs, sphere_options
from tests.test_parity_gpu import compare_step, fields_equal

pytestmark = pytest.mark.gpu

HD = (128, 192, 128)
HD_SPHERE = [dict(center=(64.0, 12.0, 64.0), radius=14.0, fuel=1.0, temperature=1500.0)]
WIDE = (508, 508, 36)
WIDE_SPHERES = [dict(center=(120.0, 16.0, 18.0), radius=12.0, fuel=1.0, temperature=1500.0),
                dict(center=(380.0, 20.0, 17.0), radius=15.0, fuel=1.0, temperature=1500.0)]


def developed(dims, spheres, steps, **kw):
    """An oracle state after `steps` steps of 8 + 8 sweeps (hot, burning, moving)."""
    o = OracleSim(dims, sphere_options(dims, P=8, R=8, seed=20251203, spheres=spheres, **kw))
    o.step(steps, DT)
    return o


@pytest.fixture(scope="module")
def hd_state():
    o = developed(HD, HD_SPHERE, 5)
    yield o
    o.close()


@pytest.mark.parametrize("dt", [0.0, DT])
def test_hd_step_against_the_oracle(hd_state, dt):
    opts = sphere_options(HD, P=96, R=96, seed=20251203, spheres=HD_SPHERE)
    g, o = FireXSim(HD, opts), OracleSim(HD, opts)
    for s in (g, o):
        copy_state(hd_state, s)
    g.step(1, dt)
    o.step(1, dt)
    d = g.diagnostics
    assert d["jacobi_kernel"] == A.JACOBI_RESIDENT and d["jacobi_variant"] == 4, d
    assert g.state == o.state
    if dt == 0.0:
        fields_equal(g, o)
    else:
        compare_step(g, o, "hd_one_step")
        ng, no = g.divergence_norm(), o.divergence_norm()
        assert ng[2] == no[2]
        assert abs(ng[0] - no[0]) <= 1e-4 * no[0] + 1e-9, (ng, no)
    g.close()
    o.close()


def fp16_pressure_errors(pg, po, fg, fo, uniforms):
    """FP16 pressure storage (branch B) one step from identical state. The few-ULP differences
    of the transcendentals reach the FP16 pressure stores, where a value that lies that close
    to a rounding boundary of FP16 rounds the other way on one side, and later sweeps average
    that into the neighbours: the pressures then differ by a few FP16 ULPs of the largest
    pressure (bound: 4), the projected velocity by the forward-difference gradient of that
    (bound: 8 ULPs x the largest metric)."""
    pmax = float(np.abs(po).max())
    ulp16 = 2.0 ** (np.floor(np.log2(pmax)) - 10) if pmax > 0 else 0.0
    metric = max(float(uniforms[k]) / max(float(uniforms[32 + k]), 0.001) for k in range(3))
    assert max_abs(pg, po) <= 4 * ulp16, (max_abs(pg, po), ulp16)
    assert max_abs(fg[..., :3], fo[..., :3]) <= 8 * ulp16 * metric + 1e-6, (max_abs(fg[..., :3], fo[..., :3]), ulp16,
                                                                           metric)


def compare_fp16_pressure_step(g, o):
    """Branch B with dt = 1/60: the simulate outputs (temperature, species, reaction) keep
    test_parity_gpu's ATOL; pressure and velocity get the FP16 allowance above."""
    fg, fo = g.read("flow"), o.read("flow")
    assert max_abs(fg[..., 3], fo[..., 3]) <= 2e-3
    assert max_abs(g.read("species"), o.read("species")) <= 2e-6
    assert max_abs(g.read("reaction"), o.read("reaction")) <= 4e-6
    fp16_pressure_errors(g.read("pressure"), o.read("pressure"), fg, fo, g.uniforms(DT))


@pytest.fixture(scope="module")
def wide_state():
    o = developed(WIDE, WIDE_SPHERES, 3)
    yield o
    o.close()


@pytest.mark.parametrize("mode", [A.PRESSURE_WARM_F32, A.PRESSURE_F16])
@pytest.mark.parametrize("dt", [0.0, DT])
def test_two_sweep_pass_against_the_oracle(wide_state, mode, dt):
    opts = sphere_options(WIDE, P=96, R=96, seed=20251203, spheres=WIDE_SPHERES, pressure_mode=mode)
    g, o = FireXSim(WIDE, opts), OracleSim(WIDE, opts)
    for s in (g, o):
        copy_state(wide_state, s)
    g.step(1, dt)
    o.step(1, dt)
    d = g.diagnostics
    assert d["jacobi_kernel"] == A.JACOBI_FUSED and d["jacobi_block"] == 2 and d["jacobi_zchunk"] == 16, d
    assert g.state == o.state
    if dt == 0.0:
        fields_equal(g, o)
    elif mode == A.PRESSURE_WARM_F32:
        compare_step(g, o, "wide_one_step_f32")
    else:
        compare_fp16_pressure_step(g, o)
    g.close()
    o.close()
