"""The two-sweep Jacobi pass with its planes staged by TMA (cp.async.bulk.tensor tile loads on
mbarriers, fx_jacobi_zm2t.cuh; selected with STAGING_TMA) against the same pass staged by
per-thread cp.async copies (AUTO) and against single sweeps: bit-identical fields in the FP32 branches (warm-started A, cold-started
C, whose first launches of each solve read no input pressure), for grids below, at and above
one 32 x 30 tile, x extents that end inside a tile, the first and last rows and planes of the
grid inside the tensor boxes (their out-of-grid rows arrive as zeros and must not be read),
chunks of 1 plane up to more than the grid, and batches of uneven grids. FP16 pressure keeps
the cp.async staging (its rows are not 16-byte multiples for every X)."""
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


def pair(dims, opts, zc):
    tma, cp = FireXSim(dims, opts), FireXSim(dims, opts)
    for s in (tma, cp):
        s.set_jacobi("fused", 2, zc)
    tma.set_staging(A.STAGING_TMA)
    return tma, cp


@pytest.mark.parametrize("mode", [A.PRESSURE_WARM_F32, A.PRESSURE_COLD_F32])
@pytest.mark.parametrize("zc", [1, 5, 16, 40])
@pytest.mark.parametrize("dims", [(16, 20, 24), (36, 44, 28), (64, 96, 64), (132, 20, 40), (100, 32, 8)])
def test_tma_staging_equals_cp_async_staging(dims, zc, mode):
    opts = sphere_options(dims, P=12, R=8, pressure_mode=mode)
    tma, cp = pair(dims, opts, zc)
    tma.step(3, DT)
    cp.step(3, DT)
    assert tma.diagnostics["jacobi_staging"] == A.STAGING_TMA, tma.diagnostics
    assert cp.diagnostics["jacobi_staging"] == A.STAGING_CPASYNC, cp.diagnostics
    same(tma, cp)
    tma.close()
    cp.close()


def test_tma_staging_zero_dt_matches_the_oracle():
    dims = (68, 64, 36)
    opts = sphere_options(dims, P=16, R=12)
    g, o = FireXSim(dims, opts), OracleSim(dims, opts)
    g.set_jacobi("fused", 2, 8)
    g.set_staging(A.STAGING_TMA)
    g.step(3, 0.0)
    o.step(3, 0.0)
    assert g.diagnostics["jacobi_staging"] == A.STAGING_TMA
    same(g, o)


def test_fp16_pressure_keeps_cp_async_staging():
    dims = (36, 44, 28)
    g = FireXSim(dims, sphere_options(dims, P=8, R=8, pressure_mode=A.PRESSURE_F16))
    g.set_jacobi("fused", 2, 8)
    g.set_staging(A.STAGING_TMA)
    g.step(1, DT)
    assert g.diagnostics["jacobi_staging"] == A.STAGING_CPASYNC
    g.close()


def test_tma_batch_of_uneven_grids_equals_each_alone():
    dims = [(64, 96, 64), (32, 48, 32), (36, 44, 28), (132, 20, 40)]
    alone = [FireXSim(d, sphere_options(d, P=12, R=12, seed=i)) for i, d in enumerate(dims)]
    members = [FireXSim(d, sphere_options(d, P=12, R=12, seed=i)) for i, d in enumerate(dims)]
    for s in alone:
        s.set_jacobi("unblocked")
        s.step(3, DT)
    with FireXBatch() as b:
        b.set_jacobi("fused", 2, 16)
        b.set_staging(A.STAGING_TMA)
        for s in members:
            b.add(s)
        b.step(3, DT)
        b.sync()
        assert members[0].diagnostics["jacobi_staging"] == A.STAGING_TMA
    for a, m in zip(alone, members):
        same(a, m)
