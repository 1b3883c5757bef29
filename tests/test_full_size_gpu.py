"""The 508^3 configuration (131,096,512 cells) at full size, through size-independent
properties: the oracle cannot step a grid this large in a test's time, so these tests check
what holds at any size.

  * 20 steps of the configuration (3 seeded spheres of radius 20-40 near the floor, 96 + 96
    Jacobi sweeps, AUTO: the f16-storage branch B above 64 Mi cells, two Jacobi sweeps per
    HBM pass) keep the reference's clamps (shaders.ts:323-341), and the counters advance as
    FireXEngine.ts:2049 / :681-682 advance them;
  * the post-projection divergence field is exactly the backward divergence
    (shaders.ts:344-364) of the resident flow, recomputed here in float32 with the same
    operation order, and the divergence norm is its interior L2 / max norm;
  * every Jacobi form (two sweeps per pass, one sweep per pass by z-marching, unblocked
    single sweeps) gives bit-identical steps from the same state, in branch B and in the
    plain FP32 branch A.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXSim, make_options
from tests.helpers import DT, backward_divergence, config3_spheres, interior

pytestmark = pytest.mark.gpu

DIMS = (508, 508, 508)


def config3_options(pressure_mode=A.PRESSURE_AUTO):
    return make_options(pressure_iterations=96, correction_iterations=96, seed=0, velocity_noise=0.05,
                        emission_jitter=0.0, spheres=config3_spheres(DIMS), pressure_mode=pressure_mode)


@pytest.fixture(scope="module")
def config3():
    s = FireXSim(DIMS, config3_options())
    s.step(20, DT)
    s.sync()
    yield s
    s.close()


def test_config3_counters_branch_and_clamps(config3):
    s = config3
    st = s.state
    assert st["frame_index"] == 20
    assert st["simulation_time"] == pytest.approx(20 * DT, rel=1e-12)
    assert s.pressure_mode == A.PRESSURE_F16  # 131 M cells >= FIREX_HEAVY_GRID_CELL_THRESHOLD
    d = s.diagnostics
    assert d["jacobi_kernel"] == A.JACOBI_FUSED and d["jacobi_block"] == 2
    flow = s.read("flow")
    assert np.all(np.isfinite(flow))
    assert float(np.abs(flow[..., :3]).max()) <= 1.4
    assert float(flow[..., 3].min()) >= 300.0 and float(flow[..., 3].max()) <= 2900.0
    assert float(flow[..., 3].max()) > 300.0  # the emitters heated the air
    sp = s.read("species")
    assert float(sp.min()) >= 0.0 and float(sp.max()) <= 3.0


def test_config3_final_divergence_is_the_backward_divergence_of_flow(config3):
    s = config3
    flow = s.read("flow")
    want = backward_divergence(flow, s.uniforms(DT))
    del flow
    got = s.read("final_divergence")
    assert np.array_equal(got, want)
    l2, linf, n = s.divergence_norm()
    inner = interior(want).astype(np.float64)
    assert n == inner.size
    assert l2 == pytest.approx(float(np.sqrt(np.sum(inner * inner))), rel=1e-9)
    assert linf == float(np.abs(inner).max())


def _digest(s):
    h = hashlib.sha256()
    for name in ("flow", "pressure", "correction"):  # what the pressure solve writes
        h.update(np.ascontiguousarray(s.read(name)).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("mode", [A.PRESSURE_F16, A.PRESSURE_WARM_F32], ids=["branch_B_f16", "branch_A_f32"])
def test_508_jacobi_forms_give_bit_identical_steps(mode):
    s = FireXSim(DIMS, config3_options(mode))
    try:
        s.step(2, DT)
        snap = s.snapshot()
        digests = {}
        for form, block, zc in (("auto", 0, 0), ("zmarch", 0, 32), ("unblocked", 0, 0)):
            s.restore(snap)
            s.set_jacobi(form, block, zc)
            s.step(1, DT)
            s.sync()
            digests[form] = _digest(s)
        assert digests["auto"] == digests["zmarch"] == digests["unblocked"], digests
    finally:
        s.close()
