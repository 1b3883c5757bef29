"""GPU tests of the temporally blocked Jacobi: two sweeps fused per launch (the two-sweep
z-marching kernel: 32 x 30 tiles with a one-cell ring) must give bit-identical fields to two
single-sweep launches in every FP32-arithmetic branch (warm f32, cold f32, f16 storage
rounded every sweep), for grids below, at and above one tile in x and y, chunks of 1 plane
up to more than the grid, and inside batches."""
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


@pytest.mark.parametrize("mode", [A.PRESSURE_WARM_F32, A.PRESSURE_COLD_F32, A.PRESSURE_F16])
@pytest.mark.parametrize("k,zc", [(2, 1), (2, 5), (2, 16), (2, 33)])
@pytest.mark.parametrize("dims", [(16, 20, 24), (36, 44, 28), (64, 96, 64), (132, 20, 40)])
def test_fused_sweeps_equal_single_sweeps(dims, k, zc, mode):
    P = R = 12
    opts = sphere_options(dims, P=P, R=R, pressure_mode=mode)
    one, fused = FireXSim(dims, opts), FireXSim(dims, opts)
    one.set_jacobi("zmarch")
    fused.set_jacobi("fused", k, zc)
    one.step(4, DT)
    fused.step(4, DT)
    same(one, fused)


@pytest.mark.parametrize("k", [2])
def test_fused_zero_dt_step_matches_oracle_bit_exact(k):
    dims = (36, 44, 28)
    opts = sphere_options(dims, P=16, R=12)
    g, o = FireXSim(dims, opts), OracleSim(dims, opts)
    g.set_jacobi("fused", k, 8)
    g.step(3, 0.0)
    o.step(3, 0.0)
    same(g, o)


def test_parity_rule_falls_back_to_single_sweeps():
    """P = 6 with two sweeps per launch (three launches) would end the solve in the other
    buffer: the engine must not fuse that phase, and the results stay those of single
    sweeps."""
    dims = (32, 48, 32)
    opts = sphere_options(dims, P=6, R=8)
    one, fused = FireXSim(dims, opts), FireXSim(dims, opts)
    one.set_jacobi("unblocked")
    fused.set_jacobi("fused", 2, 16)
    one.step(3, DT)
    fused.step(3, DT)
    same(one, fused)


def test_fused_blocks_other_than_two_are_refused():
    from fire_b200.sim import FireXError
    g = FireXSim((16, 20, 24), sphere_options((16, 20, 24)))
    for k in (3, 4, 6):
        with pytest.raises(FireXError) as e:
            g.set_jacobi("fused", k, 8)
        assert e.value.code == A.ERR_BAD_ARG
    g.close()


@pytest.mark.parametrize("k", [2])
def test_fused_batch_equals_single_sweep_alone(k):
    dims = [(64, 96, 64), (32, 48, 32), (36, 44, 28)]
    alone = [FireXSim(d, sphere_options(d, P=12, R=12, seed=i)) for i, d in enumerate(dims)]
    mixed = [FireXSim(d, sphere_options(d, P=12, R=12, seed=i)) for i, d in enumerate(dims)]
    for s in alone:
        s.set_jacobi("unblocked")
        s.step(3, DT)
    with FireXBatch() as b:
        b.set_jacobi("fused", k, 16)
        for s in mixed:
            b.add(s)
        b.step(3, DT)
    for a, m in zip(alone, mixed):
        same(a, m)


@pytest.mark.parametrize("zc", [3, 8, 32])
def test_z_marching_and_unblocked_single_sweeps_agree(zc):
    """The single-sweep kernels (z-marching shared-memory tiles; one thread per four cells
    reading neighbours through L1) compute the same sweep, for any z chunking."""
    for dims in ((36, 44, 28), (132, 20, 40)):
        opts = sphere_options(dims, P=7, R=5)
        a, b = FireXSim(dims, opts), FireXSim(dims, opts)
        a.set_jacobi("zmarch", 1, zc)
        b.set_jacobi("unblocked")
        a.step(3, DT)
        b.step(3, DT)
        same(a, b)


def test_auto_runs_two_sweeps_per_pass_with_short_chunks_between_8_and_16_mi_cells():
    """From 8 Mi cells (past L2) to 16 Mi AUTO streams two sweeps per HBM pass in 16-plane
    chunks; the result equals the unblocked kernel's bit for bit."""
    dims = (192, 288, 192)
    opts = sphere_options(dims, P=6, R=5)
    auto, one = FireXSim(dims, opts), FireXSim(dims, opts)
    one.set_jacobi("unblocked")
    auto.step(2, DT)
    one.step(2, DT)
    d = auto.diagnostics
    assert d["jacobi_kernel"] == A.JACOBI_FUSED and d["jacobi_block"] == 2 and d["jacobi_zchunk"] == 16, d
    same(auto, one)


def test_auto_runs_two_sweeps_per_pass_on_large_grids():
    """At 16 Mi cells and above AUTO streams two sweeps per HBM pass (64-plane chunks);
    the result equals single sweeps bit for bit."""
    dims = (256, 256, 256)
    opts = sphere_options(dims, P=8, R=4)
    auto, one = FireXSim(dims, opts), FireXSim(dims, opts)
    one.set_jacobi("zmarch")
    auto.step(2, DT)
    one.step(2, DT)
    d = auto.diagnostics
    assert d["jacobi_kernel"] == A.JACOBI_FUSED and d["jacobi_block"] == 2 and d["jacobi_zchunk"] == 64, d
    same(auto, one)
