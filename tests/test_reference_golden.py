"""The oracle against the reference's own step, executed from its WGSL source.

tests/golden/reference_steps.npz holds fields the reference's kernels computed: the WGSL
text of src/sim/firex/shaders.ts:1-512 and pressureShaders.ts:1-161, evaluated on the CPU
(tests/golden/wgsl_eval.py) in the dispatch order of FireXEngine.ts:2115-2276
(tests/golden/reference_step.py), by tests/golden/make_reference_golden.py. Each case starts
from the reference's reset or from a seeded developed state (motion, heat, fuel, products,
deposited liquid) and runs 2-3 steps in one of the three pressure branches, with the engine's
default parameters or a stated parameter set, dt = 1/60, 0 or 1/30; two cases run the SPH
droplet passes (shaders.ts:514-825) with the jet and the spray nozzle, one of them switching
the spray off before its last step.

The oracle must reproduce every field, the droplets and the integer liquid field after every
step bit for bit: its f32 restatement performs the same IEEE operations in the same order, and
both sides take sin / cos / exp / pow from the same C library (the droplet passes' sin, cos,
tan and exp in double precision rounded to f32, on both sides). The GPU tests compare the CUDA path with the same fixtures
within the tolerances that CUDA's own transcendentals require.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import make_options
from oracle.oracle import OracleSim

FIXTURE = Path(__file__).resolve().parent / "golden" / "reference_steps.npz"
BRANCH = {"A": A.PRESSURE_WARM_F32, "B": A.PRESSURE_F16, "C": A.PRESSURE_COLD_F32}
FIELDS = ("flow", "species", "pressure", "divergence", "reaction", "correction")


def load_cases():
    data = np.load(FIXTURE)
    meta = json.loads(bytes(data["meta"]).decode())
    return data, meta


DATA, META = load_cases()


def reshape(name, arr, dims):
    X, Y, Z = dims
    if name in ("flow", "species"):
        return arr.reshape(Z, Y, X, 4)
    return arr.reshape(Z, Y, X)


def start_sim(cls, case, **kw):
    """A simulation (oracle or CUDA) holding the case's start state."""
    m = META[case]
    dims = tuple(m["dims"])
    opts = make_options(pressure_iterations=m["P"], correction_iterations=m["R"], pressure_mode=BRANCH[m["branch"]],
                        cinematic=m["cinematic"], particle_count=m.get("droplets", 0))
    sim = cls(dims, opts, **kw)
    for name, value in m["parameters"].items():
        sim.set_parameter(name, value)
    if m["start"] == "developed":
        sim.set_state(m["start_time"], m["start_frame"], 0, 0)
        for f in ("flow", "species", "pressure", "liquid"):
            sim.write(f, reshape(f, DATA[f"{case}/in/{f}"], dims))
    return sim, dims


def apply_changes(sim, case, i):
    """Parameter changes the case makes before step i (e.g. the spray switched off)."""
    for name, value in META[case].get("changes", {}).get(str(i), {}).items():
        sim.set_parameter(name, value)


@pytest.mark.parametrize("case", sorted(META))
def test_oracle_reproduces_the_reference_step(case):
    m = META[case]
    o, dims = start_sim(OracleSim, case)
    for f in ("flow", "species", "pressure", "liquid"):
        assert np.array_equal(o.read(f), reshape(f, DATA[f"{case}/in/{f}"], dims)), f"start state {f}"
    for i, dt in enumerate(m["dts"]):
        apply_changes(o, case, i)
        o.step(1, dt)
        for f in FIELDS + ("liquid",):
            ref = reshape(f, DATA[f"{case}/step{i}/{f}"], dims)
            got = o.read(f)
            assert np.array_equal(got, ref), (f"{case} step {i} {f}: {int((got != ref).sum())} cells differ, "
                                              f"max abs {float(np.abs(got.astype(np.float64) - ref).max())}")
        if m.get("droplets"):
            ref = DATA[f"{case}/step{i}/particles"]
            got = o.read_particles().reshape(ref.shape)
            assert np.array_equal(got, ref), f"{case} step {i} droplets: {int((got != ref).sum())} values differ"
    st = o.state
    fin = m["final"]
    assert st["frame_index"] == fin["frame_index"]
    assert st["simulation_time"] == fin["simulation_time"]
    assert st["species_index"] == fin["species_index"]
    assert st["pressure_index"] == fin["pressure_index"]
    o.close()


def test_fixture_cases_cover_every_branch_and_start():
    branches = {m["branch"] for m in META.values()}
    starts = {m["start"] for m in META.values()}
    dts = {dt for m in META.values() for dt in m["dts"]}
    assert branches == {"A", "B", "C"} and starts == {"reset", "developed"}
    assert 0.0 in dts and len(dts) >= 3
    assert any(m["parameters"] for m in META.values()) and any(m["cinematic"] == 0 for m in META.values())
    # droplets with both nozzles, and the spray switched off mid-run
    nozzles = {m["parameters"].get("nozzleType") for m in META.values() if m.get("droplets")}
    assert nozzles == {0, 1} and any(m.get("changes") for m in META.values() if m.get("droplets"))
