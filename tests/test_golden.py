"""Golden fixtures (tests/golden, 8x12x8 grids, made by tests/golden/make_golden.py from the oracle):
the oracle must reproduce them bit for bit (CPU), and the CUDA path must match them
within the parity tolerances of test_parity_gpu (GPU; bit-exact where the step has no
transcendental: the emitter mask and the uniform block)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from fire_b200.sim import FireXSim
from oracle.oracle import OracleSim
from tests.golden.make_golden import CASES, DIMS, FIELDS, start
from tests.helpers import DT, max_abs

HERE = Path(__file__).resolve().parent / "golden"
GOLD = np.load(HERE / "oracle_step_8x12x8.npz")
META = json.loads((HERE / "oracle_step_8x12x8.json").read_text())

# max-abs bounds on the GPU against the FP32 oracle after 3 steps (dt = 1/60); pressure,
# correction and divergence relative to the field's max magnitude
ATOL = {"flow": 2e-3, "species": 2e-5, "reaction": 2e-5}
REL = {"pressure": 2e-4, "correction": 2e-4, "divergence": 2e-4, "liquid": 1e-2}
# droplets: positions and velocities within 1e-4 (domain units, domain units per second)
# of the oracle's, ages and masses equal


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", [32, 64])
def test_oracle_reproduces_golden(name, precision):
    sim = start(OracleSim(DIMS, CASES[name]["options"](), precision=precision), CASES[name])
    sim.step(CASES[name]["steps"], DT)
    for f in FIELDS:
        assert np.array_equal(sim.read(f), GOLD[f"{name}/fp{precision}/{f}"]), (name, precision, f)
    assert np.array_equal(sim.read_particles(), GOLD[f"{name}/fp{precision}/particles"]), (name, precision)
    assert sim.state == META["cases"][f"{name}/fp{precision}"]["state"]
    sim.close()


def test_oracle_golden_uniforms_and_mask():
    sim = OracleSim(DIMS, CASES["spheres_warm_f32"]["options"](), precision=32)
    assert np.array_equal(sim.uniforms(DT), GOLD["uniforms_dt_1_60"])
    assert np.array_equal(sim.read("emitter_mask"), GOLD["emitter_mask"])
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_cuda_path_matches_golden(name):
    g = FireXSim(DIMS, CASES[name]["options"]())
    if name == "spheres_warm_f32":
        assert np.array_equal(g.uniforms(DT), GOLD["uniforms_dt_1_60"])
        assert np.array_equal(g.read("emitter_mask"), GOLD["emitter_mask"])
    start(g, CASES[name])
    g.step(CASES[name]["steps"], DT)
    p, q = g.read_particles(), GOLD[f"{name}/fp32/particles"]
    assert np.array_equal(p[:, 0, 3], q[:, 0, 3]) and np.array_equal(p[:, 1, 3], q[:, 1, 3]), name
    assert max_abs(p[:, :, :3], q[:, :, :3]) <= 1e-4, (name, max_abs(p[:, :, :3], q[:, :, :3]))
    for f in FIELDS:
        ref = GOLD[f"{name}/fp32/{f}"]
        got = g.read(f)
        if f in ATOL:
            assert max_abs(got, ref) <= ATOL[f], (name, f, max_abs(got, ref))
        else:
            scale = max(float(np.abs(ref).max()), 1e-30)
            assert max_abs(got, ref) / scale <= REL[f], (name, f, max_abs(got, ref) / scale)
    g.close()
