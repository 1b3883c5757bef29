"""Jacobi autotuner (fire_b200/autotune.py): the workload key, the cache, and on the GPU that
tuning steps are ordinary steps (bit-identical to an untuned run), that the chosen
candidate is the one that ran, and that a cached workload is applied without stepping."""
from __future__ import annotations

import json

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.autotune import Candidate, JacobiTuner, default_candidates, signature
from tests.helpers import DT, sphere_options


class _Stub:
    """Stands in for a simulation on the CPU: records set_jacobi, refuses to step."""

    def __init__(self, dims, P=8, R=8):
        self.dims = dims
        self.options = sphere_options(dims, P=P, R=R)
        self.pressure_mode = A.PRESSURE_WARM_F32
        self.applied = []

    def set_jacobi(self, kernel, block=0, zchunk=0):
        self.applied.append((kernel, block, zchunk))

    def set_staging(self, staging):
        self.applied.append(("staging", staging))

    def set_tiles(self, simulate_by, project=0):
        self.applied.append(("tiles", simulate_by, project))

    def step(self, *a):
        raise AssertionError("a cached workload must not step")


def test_signature_is_order_free_and_covers_the_workload():
    a, b = _Stub((64, 96, 64)), _Stub((32, 48, 32), P=12)

    class B:
        members = [a, b]

    class B2:
        members = [b, a]

    assert signature(B) == signature(B2)
    assert signature(a) != signature(_Stub((64, 96, 64), P=9))
    names = {c.kernel for c in default_candidates()}
    assert names == {"resident", "unblocked", "zmarch", "fused"}


def test_cached_choice_is_applied_without_stepping(tmp_path):
    stub = _Stub((64, 96, 64))
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({signature(stub): {"choice": ["zmarch", 0, 16], "ms_per_step": 1.0}}))
    t = JacobiTuner(cache_path=path)
    assert t.tune(stub) == Candidate("zmarch", 0, 16)
    assert stub.applied == [("zmarch", 0, 16), ("staging", A.STAGING_AUTO), ("tiles", 0, A.PROJECT_AUTO)]
    # a choice with staging and brick shape (the current cache format)
    path.write_text(json.dumps({signature(stub): {"choice": ["fused", 2, 32, A.STAGING_CPASYNC, 8,
                                                            A.PROJECT_SEPARATE]}}))
    stub.applied.clear()
    assert JacobiTuner(cache_path=path).tune(stub) == Candidate("fused", 2, 32, A.STAGING_CPASYNC, 8, A.PROJECT_SEPARATE)
    assert stub.applied == [("fused", 2, 32), ("staging", A.STAGING_CPASYNC), ("tiles", 8, A.PROJECT_SEPARATE)]


@pytest.mark.gpu
def test_tuning_steps_are_ordinary_steps(tmp_path):
    from fire_b200.sim import FireXSim

    dims = (64, 96, 64)
    opts = sphere_options(dims, P=12, R=12)
    tuned, plain = FireXSim(dims, opts), FireXSim(dims, opts)
    t = JacobiTuner(cache_path=tmp_path / "tune.json", steps=1, warmup=1)
    best = t.tune(tuned, DT)
    steps = tuned.state["frame_index"]
    assert steps >= 2 and len(t.last_timings) >= 3
    plain.step(steps, DT)
    for f in ("flow", "species", "pressure", "divergence", "correction", "reaction"):
        assert np.array_equal(tuned.read(f), plain.read(f)), f
    tuned.step(1, DT)
    assert JacobiTuner._ran(tuned, best)
    # a second tuner reading the cache applies the choice without stepping
    again = FireXSim(dims, opts)
    t2 = JacobiTuner(cache_path=tmp_path / "tune.json")
    assert t2.tune(again, DT) == best
    assert again.state["frame_index"] == 0


@pytest.mark.gpu
def test_tuning_a_batch():
    from fire_b200.sim import FireXBatch, FireXSim

    dims_list = [(64, 96, 64), (32, 48, 32), (48, 64, 40)]
    b = FireXBatch()
    members = [FireXSim(d, sphere_options(d, P=8, R=8, seed=i)) for i, d in enumerate(dims_list)]
    for m in members:
        b.add(m)
    t = JacobiTuner(steps=1, warmup=1)
    best = t.tune(b, DT)
    b.step(1, DT)
    b.sync()
    assert JacobiTuner._ran(b, best)
    alone = []
    for i, d in enumerate(dims_list):
        s = FireXSim(d, sphere_options(d, P=8, R=8, seed=i))
        s.step(members[0].state["frame_index"], DT)
        alone.append(s)
    for m, s in zip(members, alone):
        assert np.array_equal(m.read("pressure"), s.read("pressure"))
        assert np.array_equal(m.read("flow"), s.read("flow"))


@pytest.mark.gpu
@pytest.mark.parametrize("by,proj", [(2, A.PROJECT_FUSED), (8, A.PROJECT_SEPARATE), (4, A.PROJECT_SEPARATE)])
def test_launch_shapes_are_bit_identical(by, proj):
    """The source pass's brick shapes (32 x by x 8/by cells) and the fused or separate primary
    projection + residual divergence, among which the tuner chooses, compute every cell with
    the same operations: identical fields, on grids that end inside bricks."""
    from fire_b200.sim import FireXSim

    for dims in ((36, 44, 28), (100, 20, 12)):
        for mode in (A.PRESSURE_WARM_F32, A.PRESSURE_F16):
            opts = sphere_options(dims, P=6, R=6, pressure_mode=mode)
            a, b = FireXSim(dims, opts), FireXSim(dims, opts)
            b.set_tiles(by, proj)
            a.step(3, DT)
            b.step(3, DT)
            assert a.diagnostics["simulate_by"] == 4 and b.diagnostics["simulate_by"] == by
            assert a.diagnostics["project_fused"] == 1
            assert b.diagnostics["project_fused"] == (proj != A.PROJECT_SEPARATE)
            for f in ("flow", "species", "pressure", "divergence", "correction", "reaction"):
                assert np.array_equal(a.read(f), b.read(f)), (dims, mode, f)
            a.close()
            b.close()
