"""GPU tests of the resident Jacobi (every sweep of a phase in one cooperative launch,
pressure held in shared memory, box faces exchanged through L2): its fields must be
bit-identical to one sweep per launch in every branch (warm f32, cold f32, f16 storage
rounded every sweep, mixed storage), for any sweep counts, grids that do and do not
divide into boxes, and batches whose members share the launch. The grids cover every
variant the planner picks: faces first (small boxes), faces first with interior columns
(FP16 pressure, or on request), one column per thread (128x192x128, 80x120x80) or columns
split in z parts (96x144x96), and the same with a copy warp (FP32 pressure under AUTO)."""
from __future__ import annotations

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXBatch, FireXSim
from oracle.oracle import OracleSim
from tests.helpers import DT, sphere_options

pytestmark = pytest.mark.gpu

FIELDS = ("flow", "species", "pressure", "reaction", "divergence", "correction")


def same(a, b):
    assert a.state == b.state
    for f in FIELDS:
        x, y = a.read(f), b.read(f)
        assert np.array_equal(x, y), (f, float(np.abs(x.astype(np.float64) - y).max()))


def pair(dims, opts, steps=3):
    one, res = FireXSim(dims, opts), FireXSim(dims, opts)
    one.set_jacobi("unblocked")
    res.set_jacobi("resident")
    one.step(steps, DT)
    res.step(steps, DT)
    assert res.diagnostics["jacobi_kernel"] == A.JACOBI_RESIDENT
    assert one.diagnostics["jacobi_kernel"] == A.JACOBI_UNBLOCKED
    return one, res


@pytest.mark.parametrize("mode", [A.PRESSURE_WARM_F32, A.PRESSURE_COLD_F32, A.PRESSURE_F16])
@pytest.mark.parametrize("dims", [(16, 20, 24), (36, 44, 28), (132, 20, 40), (64, 96, 64), (96, 144, 96), (80, 120, 80)])
def test_resident_equals_single_sweeps(dims, mode):
    one, res = pair(dims, sphere_options(dims, P=12, R=9, pressure_mode=mode))
    same(one, res)


@pytest.mark.parametrize("mode", [A.PRESSURE_WARM_F32, A.PRESSURE_COLD_F32])
@pytest.mark.parametrize("dims", [(96, 144, 96), (80, 120, 80), (128, 192, 128)])
def test_variant3_fp32_equals_single_sweeps(dims, mode):
    """FP32 pressure takes variant 4 under AUTO; variant 3 (block 4) stays selectable."""
    opts = sphere_options(dims, P=12, R=9, pressure_mode=mode)
    one, res = FireXSim(dims, opts), FireXSim(dims, opts)
    one.set_jacobi("unblocked")
    res.set_jacobi("resident", 4)
    one.step(2, DT)
    res.step(2, DT)
    assert res.diagnostics["jacobi_variant"] == 3
    same(one, res)


@pytest.mark.parametrize("P,R", [(0, 3), (1, 2), (2, 1), (7, 0), (5, 6)])
def test_resident_small_and_odd_sweep_counts(P, R):
    dims = (36, 44, 28)
    one, res = FireXSim(dims, sphere_options(dims, P=P, R=R)), FireXSim(dims, sphere_options(dims, P=P, R=R))
    one.set_jacobi("unblocked")
    res.set_jacobi("resident")
    one.step(3, DT)
    res.step(3, DT)
    same(one, res)


def test_resident_hd_grid_96_96():
    """The HD tier (3,145,728 cells) fits on chip: 96 + 96 sweeps, two steps."""
    dims = (128, 192, 128)
    one, res = pair(dims, sphere_options(dims, P=96, R=96), steps=2)
    same(one, res)


def test_resident_mixed_storage():
    dims = (64, 96, 64)
    one, res = pair(dims, sphere_options(dims, P=16, R=16, precision=A.PRECISION_MIXED))
    same(one, res)


def test_resident_zero_dt_step_matches_oracle_bit_exact():
    dims = (36, 44, 28)
    opts = sphere_options(dims, P=16, R=12)
    g, o = FireXSim(dims, opts), OracleSim(dims, opts)
    g.set_jacobi("resident")
    g.step(3, 0.0)
    o.step(3, 0.0)
    assert g.diagnostics["jacobi_kernel"] == A.JACOBI_RESIDENT
    same(g, o)


def test_resident_batch_equals_single_sweep_alone():
    dims_list = [(16, 20, 24), (36, 44, 28), (64, 96, 64), (32, 48, 32)]
    alone = []
    for i, dims in enumerate(dims_list):
        s = FireXSim(dims, sphere_options(dims, P=10 + i, R=8, seed=11 + i))
        s.set_jacobi("unblocked")
        s.step(3, DT)
        alone.append(s)
    b = FireXBatch()
    members = [FireXSim(d, sphere_options(d, P=10 + i, R=8, seed=11 + i)) for i, d in enumerate(dims_list)]
    for m in members:
        b.add(m)
    b.set_jacobi("resident")
    b.step(3, DT)
    b.sync()
    for m, s in zip(members, alone):
        assert m.diagnostics["jacobi_kernel"] == A.JACOBI_RESIDENT
        same(m, s)


def test_grid_beyond_chip_falls_back_to_single_sweeps():
    dims = (256, 128, 128)  # 4.2 Mi cells: more than the CTAs' shared memory and registers hold
    s = FireXSim(dims, sphere_options(dims, P=4, R=4))
    s.set_jacobi("resident")
    s.step(1, DT)
    s.sync()
    assert s.diagnostics["jacobi_kernel"] != A.JACOBI_RESIDENT
