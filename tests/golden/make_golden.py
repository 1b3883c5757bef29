"""Generates the golden fixtures of tests/golden from the CPU oracle (oracle/), which
restates the reference step (src/sim/firex/shaders.ts, pressureShaders.ts and the
dispatch graph of FireXEngine.ts:2115-2276). The reference itself cannot run here
(WGSL under WebGPU), so these fixtures pin the oracle and the CUDA path against later
changes rather than against the reference's own outputs.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from fire_b200 import _abi as A  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.helpers import DT, burner_options, sphere_options  # noqa: E402

DIMS = (8, 12, 8)
CASES = {
    "spheres_warm_f32": dict(options=lambda: sphere_options(DIMS, P=8, R=6), steps=3),
    "burner_warm_f32": dict(options=lambda: burner_options(P=8, R=6), steps=3),
    "spheres_f16_pressure": dict(options=lambda: sphere_options(DIMS, P=8, R=6, pressure_mode=A.PRESSURE_F16), steps=3),
    "spheres_cold_f32": dict(options=lambda: sphere_options(DIMS, P=8, R=6, pressure_mode=A.PRESSURE_COLD_F32), steps=3),
    # the hose on (full-cone nozzle, 25 degrees): droplets, their liquid deposit and its cooling
    "spheres_water": dict(options=lambda: sphere_options(DIMS, P=8, R=6, particle_count=384), steps=3,
                          params={"waterEnabled": True, "waterFlow": 0.8, "nozzleType": 1, "sprayAngle": 25}),
}
FIELDS = ("flow", "species", "pressure", "reaction", "divergence", "correction", "liquid")


def start(sim, case):
    """Applies a case's parameters to a new simulation and re-initialises it under them."""
    params = case.get("params")
    if params:
        for k, v in params.items():
            sim.set_parameter(k, v)
        sim.reset()
    return sim


def generate():
    O.build()
    meta = {"dims": DIMS, "dt": DT, "cases": {}}
    arrays = {}
    for name, case in CASES.items():
        for precision in (32, 64):
            sim = start(O.OracleSim(DIMS, case["options"](), precision=precision), case)
            sim.step(case["steps"], DT)
            for f in FIELDS:
                arrays[f"{name}/fp{precision}/{f}"] = sim.read(f)
            arrays[f"{name}/fp{precision}/particles"] = sim.read_particles()
            meta["cases"][f"{name}/fp{precision}"] = {"steps": case["steps"], "divergence_norm": list(sim.divergence_norm()),
                                                      "state": sim.state}
            sim.close()
    sim = O.OracleSim(DIMS, CASES["spheres_warm_f32"]["options"](), precision=32)
    arrays["uniforms_dt_1_60"] = sim.uniforms(DT)
    arrays["emitter_mask"] = sim.read("emitter_mask")
    sim.close()
    return meta, arrays


if __name__ == "__main__":
    meta, arrays = generate()
    np.savez_compressed(HERE / "oracle_step_8x12x8.npz", **arrays)
    (HERE / "oracle_step_8x12x8.json").write_text(json.dumps(meta, indent=1, default=float) + "\n")
    print("wrote", len(arrays), "arrays")
