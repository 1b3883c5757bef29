"""Overlapped readback (firex_read_field_async): copies started after each step, while
the next steps run, hold exactly what a synchronous read at that point returns."""
from __future__ import annotations

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXBatch, FireXError, FireXSim
from tests.helpers import DT, sphere_options

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("field", ["flow", "species", "pressure", "divergence", "reaction", "correction"])
def test_async_reads_equal_sync_reads_of_a_twin(field):
    dims = (64, 96, 64)
    a, b = FireXSim(dims, sphere_options(dims, P=16, R=12)), FireXSim(dims, sphere_options(dims, P=16, R=12))
    got, want = [], []
    for _ in range(4):
        a.step(1, DT)
        got.append(a.read_async(field, np.empty_like(a.read(field))))  # the next step overlaps the copy
        b.step(1, DT)
        want.append(b.read(field))
    a.step(2, DT)
    a.sync()
    for g, w in zip(got, want):
        assert np.array_equal(g, w), field


def test_async_read_refuses_converted_fields_and_works_in_a_batch():
    dims = (32, 48, 32)
    m = FireXSim(dims, sphere_options(dims, P=8, R=8, precision=A.PRECISION_MIXED))
    with pytest.raises(FireXError):
        m.read_async("species", np.empty((32, 48, 32, 4), np.float32))
    with pytest.raises(FireXError):
        m.read_async("emitter_mask", np.empty((32, 48, 32), np.uint8))
    twin = FireXSim(dims, sphere_options(dims, P=8, R=8, precision=A.PRECISION_MIXED))
    bt = FireXBatch()
    bt.add(m)
    bt.step(2, DT)
    out = m.read_async("flow", np.empty((32, 48, 32, 4), np.float32))
    bt.step(1, DT)
    bt.sync()
    twin.step(2, DT)
    assert np.array_equal(out, twin.read("flow"))
    bt.close()
