"""Generates tests/golden/reference_steps.npz: the reference's own Fire-X step executed on
the CPU from its WGSL source (tests/golden/reference_step.py over tests/golden/wgsl_eval.py).

Run where the reference tree is present (default: the REFERENCE_ROOT environment variable,
else ../reference beside this repository's root):

    python -m tests.golden.make_reference_golden [reference_root]

Each case starts from a state (the reference's own reset, or a seeded developed state written
into the buffers the way firex_write_field writes them), runs a few steps of
encodeSimulationStep with the engine's default parameters or a stated parameter set, and
records the resident fields after every step. tests/test_reference_golden.py replays the
cases on the oracle (and the GPU tests on the CUDA path) and compares.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from tests.golden.reference_step import ReferenceStep, load_programs  # noqa: E402

OUT = HERE / "reference_steps.npz"

# name, dims, branch, P, R, start, steps (dt per step), parameters, cinematic, droplets,
# parameter changes before given steps
CASES = [
    ("reset_A", (8, 12, 8), "A", 6, 6, "reset", [1 / 60] * 3, {}, 1, 0, {}),
    ("developed_A", (12, 16, 8), "A", 5, 5, "developed", [1 / 60, 1 / 60], {}, 1, 0, {}),
    ("developed_B", (12, 16, 8), "B", 5, 5, "developed", [1 / 60, 1 / 60], {}, 1, 0, {}),
    ("developed_C", (12, 16, 8), "C", 5, 5, "developed", [1 / 60, 1 / 60], {}, 1, 0, {}),
    ("dt_zero_and_large", (8, 12, 12), "A", 4, 3, "developed", [0.0, 1 / 30], {}, 1, 0, {}),
    ("parameters", (8, 16, 12), "A", 4, 4, "developed", [1 / 60, 1 / 60],
     dict(firePower=3.7, vorticity=5.0, buoyancyScale=3.1, sourceLift=2.4, flamePersistence=0.8,
          airEntrainment=2.6, domainWidth=2.0, domainHeight=3.0, domainDepth=1.5, sourceThickness=2.2,
          burnerSize=1.2, burnerDepth=0.9, heatEfficiency=0.5, fuelRate=0.6, oxygenRate=0.8, aimHeight=0.7), 0, 0, {}),
    ("odd_iterations", (12, 8, 16), "A", 3, 1, "developed", [1 / 60, 1 / 60, 1 / 60], {}, 1, 0, {}),
    # droplets: the jet and the spray nozzle (shaders.ts:514-825), spray switched off before
    # the last step (the state machine parks the droplets and clears the liquid field)
    ("water_jet", (12, 16, 16), "A", 4, 4, "developed", [1 / 60] * 3,
     dict(waterEnabled=True, waterFlow=1.0, nozzleType=0), 1, 96, {}),
    ("water_spray_then_off", (12, 16, 16), "A", 4, 4, "developed", [1 / 60] * 3,
     dict(waterEnabled=True, waterFlow=0.6, nozzleType=1, sprayAngle=24, aimHeight=0.55), 1, 128,
     {2: dict(waterEnabled=False)}),
]


def developed_state(dims, seed):
    """A seeded state with motion, heat, fuel, products and deposited liquid everywhere."""
    X, Y, Z = dims
    N = X * Y * Z
    rng = np.random.default_rng(seed)
    flow = np.empty((N, 4), np.float32)
    flow[:, :3] = rng.uniform(-0.4, 0.4, (N, 3))
    flow[:, 3] = rng.uniform(300.0, 1800.0, N)
    species = np.empty((N, 4), np.float32)
    species[:, 0] = rng.uniform(0.0, 1.2, N)
    species[:, 1] = rng.uniform(0.0, 1.0, N)
    species[:, 2] = rng.uniform(0.0, 0.5, N)
    species[:, 3] = rng.uniform(0.0, 0.3, N)
    pressure = rng.uniform(-1e-4, 1e-4, N).astype(np.float32)
    liquid = np.where(rng.uniform(size=N) < 0.2, rng.integers(0, 2 * 4096, N), 0).astype(np.uint32)
    return flow, species, pressure, liquid


def run_case(progs, name, dims, branch, P, R, start, dts, params, cinematic, droplets, changes, seed):
    sim = ReferenceStep(progs, dims, branch=branch, P=P, R=R, parameters=params, cinematic=cinematic,
                        particle_count=droplets)
    rec = {}
    if start == "developed":
        flow, species, pressure, liquid = developed_state(dims, seed)
        sim.flow[0][...] = flow
        sim.species[sim.species_index][...] = species
        sim.pressure[sim.pressure_index][...] = pressure.astype(sim.pressure[0].dtype)
        sim.liquid[...] = liquid
        # the start sits a few steps into a run: the burner's time terms are not at t = 0
        sim.simulation_time = 0.35
        sim.frame_index = 21
    init = sim.current()
    for k, v in init.items():
        rec[f"{name}/in/{k}"] = v
    for i, dt in enumerate(dts):
        sim.par.update(changes.get(i, {}))
        trace = {}
        sim.step(dt, trace)
        cur = sim.current()
        cur["correction"] = trace["residual.pressure"].astype(np.float32)
        for k, v in cur.items():
            rec[f"{name}/step{i}/{k}"] = v
    meta = dict(dims=list(dims), branch=branch, P=P, R=R, start=start, dts=dts, parameters=params,
                cinematic=cinematic, droplets=droplets, changes={str(k): v for k, v in changes.items()},
                start_time=0.35 if start == "developed" else 0.0,
                start_frame=21 if start == "developed" else 0,
                final=dict(simulation_time=sim.simulation_time, frame_index=sim.frame_index,
                           species_index=sim.species_index, pressure_index=sim.pressure_index))
    return rec, meta


def main(reference_root: str) -> None:
    progs = load_programs(reference_root)
    arrays, metas = {}, {}
    for k, (name, dims, branch, P, R, start, dts, params, cinematic, droplets, changes) in enumerate(CASES):
        rec, meta = run_case(progs, name, dims, branch, P, R, start, dts, params, cinematic, droplets, changes,
                             seed=1000 + k)
        arrays.update(rec)
        metas[name] = meta
        print(f"{name}: {dims} branch {branch}, {len(dts)} steps, {droplets} droplets")
    arrays["meta"] = np.frombuffer(json.dumps(metas, sort_keys=True).encode(), np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    default_root = os.environ.get("REFERENCE_ROOT") or str(ROOT.parent / "reference")
    main(sys.argv[1] if len(sys.argv) > 1 else default_root)
