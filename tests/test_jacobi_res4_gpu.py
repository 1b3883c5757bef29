"""GPU tests of variant 4 of the resident Jacobi: the faces-first sweep with interior columns
(variant 3) on all warps but the last, whose lanes wait for the neighbours' faces and bring the
halo rows in with bulk asynchronous copies completing on an mbarrier (fx_jacobi_res.cuh,
fx_res_copier). Its fields must be bit-identical to one sweep per launch in the FP32 branches
(warm and cold start): grids whose boxes do and do not divide the grid, rows of 25 and 33
groups (rows across warps), boxes with one to four neighbours, small and odd sweep counts, the
HD tier at 96 + 96, a batch sharing the launch, and a zero-dt step against the oracle. FP16
pressure keeps the other variants. Its bounded waits expire like the other variants' when a
box withholds its faces."""
from __future__ import annotations

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXBatch, FireXError, FireXSim
from oracle.oracle import OracleSim
from tests.helpers import DT, sphere_options

pytestmark = pytest.mark.gpu

FIELDS = ("flow", "species", "pressure", "reaction", "divergence", "correction")
V4 = 5  # set_jacobi block = variant + 1


def same(a, b):
    assert a.state == b.state
    for f in FIELDS:
        x, y = a.read(f), b.read(f)
        assert np.array_equal(x, y), (f, float(np.abs(x.astype(np.float64) - y).max()))


def pair(dims, opts, steps=3):
    one, res = FireXSim(dims, opts), FireXSim(dims, opts)
    one.set_jacobi("unblocked")
    res.set_jacobi("resident", V4)
    one.step(steps, DT)
    res.step(steps, DT)
    d = res.diagnostics
    assert d["jacobi_kernel"] == A.JACOBI_RESIDENT and d["jacobi_variant"] == 4, d
    return one, res


@pytest.mark.parametrize("mode", [A.PRESSURE_WARM_F32, A.PRESSURE_COLD_F32])
@pytest.mark.parametrize("dims", [(96, 144, 96), (80, 120, 80), (64, 96, 128), (132, 96, 64), (100, 120, 88)])
def test_variant4_equals_single_sweeps(dims, mode):
    one, res = pair(dims, sphere_options(dims, P=12, R=9, pressure_mode=mode))
    same(one, res)


@pytest.mark.parametrize("P,R", [(0, 3), (1, 2), (2, 1), (7, 0), (5, 6)])
def test_variant4_small_and_odd_sweep_counts(P, R):
    dims = (80, 120, 80)
    one, res = pair(dims, sphere_options(dims, P=P, R=R))
    same(one, res)


def test_variant4_hd_grid_96_96():
    dims = (128, 192, 128)
    one, res = pair(dims, sphere_options(dims, P=96, R=96), steps=2)
    same(one, res)


def test_variant4_zero_dt_step_matches_oracle_bit_exact():
    dims = (80, 120, 80)
    opts = sphere_options(dims, P=16, R=12)
    g, o = FireXSim(dims, opts), OracleSim(dims, opts)
    g.set_jacobi("resident", V4)
    g.step(3, 0.0)
    o.step(3, 0.0)
    assert g.diagnostics["jacobi_variant"] == 4
    same(g, o)


def test_variant4_batch_equals_single_sweeps_alone():
    dims_list = [(80, 120, 80), (64, 96, 128), (96, 96, 96)]
    alone = []
    for i, dims in enumerate(dims_list):
        s = FireXSim(dims, sphere_options(dims, P=10 + i, R=8, seed=11 + i))
        s.set_jacobi("unblocked")
        s.step(3, DT)
        alone.append(s)
    members = [FireXSim(d, sphere_options(d, P=10 + i, R=8, seed=11 + i)) for i, d in enumerate(dims_list)]
    with FireXBatch() as b:
        for m in members:
            b.add(m)
        b.set_jacobi("resident", V4)
        b.step(3, DT)
        b.sync()
        assert members[0].diagnostics["jacobi_variant"] == 4
    for m, s in zip(members, alone):
        same(m, s)


def test_fp16_pressure_takes_another_variant():
    dims = (80, 120, 80)
    g = FireXSim(dims, sphere_options(dims, P=8, R=8, pressure_mode=A.PRESSURE_F16))
    g.set_jacobi("resident", V4)
    g.step(1, DT)
    g.sync()
    assert g.diagnostics["jacobi_variant"] != 4
    g.close()


def test_variant4_withheld_face_expires_the_waits():
    dims = (80, 120, 80)
    opts = sphere_options(dims, P=12, R=12)
    g = FireXSim(dims, opts)
    g.set_jacobi("resident", V4)
    g.step(1, DT)
    g.sync()
    assert g.diagnostics["jacobi_variant"] == 4
    g.set_wait_limit(4096)
    g.test_hold_face(0, 3)
    g.step(1, DT)
    with pytest.raises(FireXError) as e:
        g.sync()
    assert e.value.code == A.ERR_TIMEOUT
    g.close()
    h, o = FireXSim(dims, opts), OracleSim(dims, opts)
    h.set_jacobi("resident", V4)
    h.step(2, 0.0)
    o.step(2, 0.0)
    same(h, o)
    h.close()


# ---- the residual projection as the resident launch's epilogue (fx_res_project_epi) ----------

@pytest.mark.parametrize("dims,P,R", [((128, 192, 128), 96, 96), ((96, 144, 96), 12, 1), ((64, 96, 128), 5, 6)])
def test_variant4_projection_epilogue_equals_separate_pass(dims, P, R):
    opts = sphere_options(dims, P=P, R=R)
    epi, sep = FireXSim(dims, opts), FireXSim(dims, opts)
    for s in (epi, sep):
        s.set_jacobi("resident", V4)
    sep.set_tiles(0, A.PROJECT_SEPARATE)
    epi.step(2, DT)
    sep.step(2, DT)
    de, ds = epi.diagnostics, sep.diagnostics
    assert de["jacobi_variant"] == 4 and ds["jacobi_variant"] == 4
    assert de["project_resident"] == 1 and ds["project_resident"] == 0
    assert de["launches_per_step"] == ds["launches_per_step"] - 2  # no projection, no divergence launch
    same(epi, sep)


def test_no_projection_epilogue_without_residual_sweeps():
    dims = (80, 120, 80)
    g = FireXSim(dims, sphere_options(dims, P=8, R=0))
    g.set_jacobi("resident", V4)
    g.step(1, DT)
    g.sync()
    assert g.diagnostics["project_resident"] == 0
    g.close()


def test_projection_epilogue_zero_dt_matches_oracle_bit_exact():
    dims = (96, 144, 96)
    opts = sphere_options(dims, P=10, R=7)
    g, o = FireXSim(dims, opts), OracleSim(dims, opts)
    g.step(3, 0.0)
    o.step(3, 0.0)
    assert g.diagnostics["project_resident"] == 1
    same(g, o)


def test_withheld_last_face_expires_the_epilogue_wait():
    # box 0 withholds its faces from the residual phase's last sweep on: only the epilogue's
    # halo fetch waits for them
    dims = (80, 120, 80)
    opts = sphere_options(dims, P=12, R=12)
    g = FireXSim(dims, opts)
    g.set_jacobi("resident", V4)
    g.step(1, DT)
    g.sync()
    assert g.diagnostics["project_resident"] == 1
    g.set_wait_limit(4096)
    g.test_hold_face(0, 11)
    g.step(1, DT)
    with pytest.raises(FireXError) as e:
        g.sync()
    assert e.value.code == A.ERR_TIMEOUT
    g.close()


def test_projection_epilogue_batch_with_uneven_residual_counts():
    # each member's boxes run their own residual count, then the epilogue
    dims_list = [(80, 120, 80), (64, 96, 128), (96, 96, 96)]
    Rs = [1, 5, 8]
    alone = []
    for i, dims in enumerate(dims_list):
        s = FireXSim(dims, sphere_options(dims, P=9, R=Rs[i], seed=21 + i))
        s.set_jacobi("unblocked")
        s.step(2, DT)
        alone.append(s)
    members = [FireXSim(d, sphere_options(d, P=9, R=Rs[i], seed=21 + i)) for i, d in enumerate(dims_list)]
    with FireXBatch() as b:
        for m in members:
            b.add(m)
        b.set_jacobi("resident", V4)
        b.step(2, DT)
        b.sync()
        d = members[0].diagnostics
        assert d["jacobi_variant"] == 4 and d["project_resident"] == 1
    for m, s in zip(members, alone):
        same(m, s)
