"""GPU tests of batched stepping: simulations of different sizes and iteration counts
stepped by the same launches give bit-identical results to each stepped alone, and the
graph-replayed step equals direct launches."""
from __future__ import annotations

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXBatch, FireXError, FireXSim, make_options
from tests.helpers import DT, sphere_options

pytestmark = pytest.mark.gpu

FIELDS = ("flow", "species", "pressure", "reaction", "divergence", "correction")


def scene(dims, seed, P=12, R=10, **kw):
    X, Y, Z = dims
    spheres = [dict(center=(X * 0.4 + seed % 5, Y * 0.15, Z * 0.55), radius=max(3.0, X / 10)),
               dict(center=(X * 0.65, Y * 0.1, Z * 0.35), radius=max(2.5, X / 14))]
    return sphere_options(dims, P=P, R=R, seed=seed, spheres=spheres[: 1 + seed % 2], **kw)


def assert_same(a, b):
    assert a.state == b.state
    for f in FIELDS:
        assert np.array_equal(a.read(f), b.read(f)), f


def test_batch_of_uneven_grids_equals_each_alone():
    dims = [(16, 20, 24), (32, 48, 32), (64, 96, 64), (24, 36, 20)]
    iters = [(12, 10), (8, 14), (12, 10), (5, 3)]
    alone = [FireXSim(d, scene(d, i, *iters[i])) for i, d in enumerate(dims)]
    mixed = [FireXSim(d, scene(d, i, *iters[i])) for i, d in enumerate(dims)]
    for s in alone:
        s.step(5, DT)
    with FireXBatch() as b:
        for s in mixed:
            b.add(s)
        assert len(b) == 4
        b.step(3, DT)
        b.remove(mixed[1])  # leaves mid-run, continues alone
        mixed[1].step(2, DT)
        b.step(2, DT)
    for a, m in zip(alone, mixed):
        assert_same(a, m)


def test_member_joining_late_continues_exactly():
    d = (32, 48, 32)
    a, m = FireXSim(d, scene(d, 3)), FireXSim(d, scene(d, 3))
    a.step(6, DT)
    m.step(2, DT)
    other = FireXSim((16, 20, 24), scene((16, 20, 24), 1))
    with FireXBatch() as b:
        b.add(other)
        b.step(1, DT)
        b.add(m)
        b.step(4, DT)
        with pytest.raises(FireXError):
            m.step(1, DT)  # members step through their batch only
    assert_same(a, m)


def test_graph_and_direct_launches_agree():
    d = (64, 96, 64)
    g, n = FireXSim(d, scene(d, 2)), FireXSim(d, scene(d, 2))
    n.set_graphs(False)
    g.step(7, DT)
    n.step(7, DT)
    assert_same(g, n)


def test_batch_rejects_mixed_storage():
    a = FireXSim((16, 20, 24), make_options(pressure_iterations=2, correction_iterations=2))
    b16 = FireXSim((16, 20, 24), make_options(pressure_iterations=2, correction_iterations=2,
                                              pressure_mode=A.PRESSURE_F16))
    with FireXBatch() as b:
        b.add(a)
        with pytest.raises(FireXError) as e:
            b.add(b16)
        assert e.value.code == A.ERR_UNSUPPORTED
