"""GPU parity of the plain FP32 CUDA path against the CPU oracle, through the C ABI.

Tolerances (stated here, measured on B200):
  * bit-exact: initial fields, the sphere emitter mask, the uniform block, and any step
    with dt = 0 in sphere mode (every transcendental is then multiplied by dt = 0, so the
    step is pure IEEE add/mul/div/sqrt in a fixed order on both sides);
  * one step from identical inputs with dt = 1/60: max-abs error per field below
    ATOL[field] — the only differences are the few-ULP results of sinf/cosf/expf/powf
    on the device against the C library on the host, carried through the solve;
  * multi-step runs: the post-projection divergence norms agree to REL_NORM and the
    fields' relative L2 differences stay below REL_FIELD (chaotic growth of ULP
    differences is bounded by the clamps and the contractive pressure solve).
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXError, FireXSim, make_options
from oracle.oracle import OracleSim
from tests.helpers import DT, burner_options, copy_state, max_abs, rel_l2, sphere_options

pytestmark = pytest.mark.gpu

# Observed on B200 (max over cases): flow_uvw 3e-8, flow_T 3.1e-4 (1 ULP at ~2000 K),
# species 1.8e-7, reaction 3.8e-7, pressure_rel 2.7e-7; 60-step config 1: 1.5e-5 (flow),
# 2.9e-5 (pressure), 2.3e-5 (divergence norm).
ATOL = {"flow_uvw": 1e-6, "flow_T": 2e-3, "species": 2e-6, "reaction": 4e-6, "pressure_rel": 4e-6}
REL_FIELD = 3e-4
REL_NORM = 3e-4

REPORT = os.environ.get("FIREX_PARITY_REPORT")


def report(name, **vals):
    if REPORT:
        with open(REPORT, "a") as f:
            f.write(json.dumps({"test": name, **{k: float(v) for k, v in vals.items()}}) + "\n")


def fields_equal(a, b, names=("flow", "species", "pressure", "reaction", "divergence", "correction")):
    for n in names:
        x, y = a.read(n), b.read(n)
        assert np.array_equal(x, y), f"{n}: max abs diff {max_abs(x, y)}"


def compare_step(g, o, tag):
    fg, fo = g.read("flow"), o.read("flow")
    sg, so = g.read("species"), o.read("species")
    pg, po = g.read("pressure"), o.read("pressure")
    rg, ro = g.read("reaction"), o.read("reaction")
    e = {
        "flow_uvw": max_abs(fg[..., :3], fo[..., :3]),
        "flow_T": max_abs(fg[..., 3], fo[..., 3]),
        "species": max_abs(sg, so),
        "reaction": max_abs(rg, ro),
        "pressure_rel": max_abs(pg, po) / max(1e-12, float(np.abs(po).max())),
    }
    report(tag, **e)
    for k, v in e.items():
        assert v <= ATOL[k], f"{tag}: {k} error {v} above {ATOL[k]}"
    return e


@pytest.mark.parametrize("dims", [(16, 20, 24), (64, 96, 64)])
def test_reset_fields_bit_exact(dims):
    opts = sphere_options(dims)
    g, o = FireXSim(dims, opts), OracleSim(dims, opts)
    fields_equal(g, o, ("flow", "species", "pressure", "reaction", "divergence", "liquid"))


def test_emitter_mask_bit_exact():
    dims = (64, 96, 64)
    opts = sphere_options(dims, spheres=[dict(center=(32, 8, 32), radius=8), dict(center=(10.3, 30.7, 50.1), radius=5.5)])
    g, o = FireXSim(dims, opts), OracleSim(dims, opts)
    assert np.array_equal(g.read("emitter_mask"), o.read("emitter_mask"))
    assert g.read("emitter_mask").sum() > 0


def test_uniform_block_bit_exact():
    dims = (16, 20, 24)
    g, o = FireXSim(dims, sphere_options(dims)), OracleSim(dims, sphere_options(dims))
    for s in (g, o):
        s.set_parameter("firePower", 3.3)
        s.set_parameter("domainHeight", 1.7)
        s.step(3, DT)
    assert np.array_equal(g.uniforms(DT), o.uniforms(DT))
    assert g.state == o.state


@pytest.mark.parametrize("mode", [A.PRESSURE_WARM_F32, A.PRESSURE_COLD_F32, A.PRESSURE_F16])
@pytest.mark.parametrize("dims", [(16, 20, 24), (64, 96, 64)])
def test_zero_dt_sphere_steps_bit_exact(dims, mode):
    """dt = 0 removes every transcendental from the step's results: the divergence,
    Jacobi sweeps, projections, boundary conditions, sphere injection and ping-pong
    parity must then agree bit for bit."""
    opts = sphere_options(dims, P=9, R=7, pressure_mode=mode)
    g, o = FireXSim(dims, opts), OracleSim(dims, opts)
    g.step(3, 0.0)
    o.step(3, 0.0)
    assert g.state == o.state
    fields_equal(g, o)


@pytest.mark.parametrize("scene", ["spheres", "burner"])
@pytest.mark.parametrize("dims", [(16, 20, 24), (64, 96, 64)])
def test_one_step_from_identical_state(dims, scene):
    opts = sphere_options(dims, P=20, R=20) if scene == "spheres" else burner_options(P=20, R=20)
    o = OracleSim(dims, opts)
    o.step(6, DT)  # a developed state: hot, burning, moving
    g = FireXSim(dims, opts)
    copy_state(o, g)
    assert g.state == o.state
    g.step(1, DT)
    o.step(1, DT)
    compare_step(g, o, f"one_step_{scene}_{dims[0]}x{dims[1]}x{dims[2]}")


def test_config1_sixty_steps_track_the_oracle():
    """Config 1 (64x96x64, sphere r=8 at (32,8,32), 40+40, seeded noise) over 60 steps."""
    dims = (64, 96, 64)
    opts = sphere_options(dims, P=40, R=40, seed=1, jitter=0.0, spheres=[dict(center=(32, 8, 32), radius=8)])
    g, o = FireXSim(dims, opts), OracleSim(dims, opts)
    g.step(60, DT)
    o.step(60, DT)
    assert g.state == o.state
    ng, no = g.divergence_norm(), o.divergence_norm()
    e = {"rel_norm_l2": abs(ng[0] - no[0]) / no[0]}
    for f in ("flow", "species", "pressure", "reaction"):
        e[f"rel_l2_{f}"] = rel_l2(g.read(f), o.read(f))
    report("config1_60_steps", **e)
    assert e["rel_norm_l2"] <= REL_NORM
    for f in ("flow", "species", "pressure"):
        assert e[f"rel_l2_{f}"] <= REL_FIELD, (f, e)


def test_divergence_norm_matches_oracle_on_identical_flow():
    dims = (64, 96, 64)
    opts = sphere_options(dims, P=10, R=10)
    o = OracleSim(dims, opts)
    o.step(4, DT)
    g = FireXSim(dims, opts)
    copy_state(o, g)
    ng, no = g.divergence_norm(), o.divergence_norm()
    assert ng[2] == no[2]
    assert ng[0] == pytest.approx(no[0], rel=1e-12)
    assert ng[1] == no[1]
    assert np.array_equal(g.read("final_divergence"), o.read("final_divergence"))


def test_field_round_trip_and_errors():
    dims = (16, 20, 24)
    g = FireXSim(dims, sphere_options(dims))
    rng = np.random.default_rng(0)
    for f in ("flow", "species", "pressure", "divergence", "reaction"):
        data = g.read(f)
        new = rng.standard_normal(data.shape).astype(np.float32)
        g.write(f, new)
        assert np.array_equal(g.read(f), new)
    liq = rng.integers(0, 1 << 20, size=g.read("liquid").shape, dtype=np.uint32)
    g.write("liquid", liq)
    assert np.array_equal(g.read("liquid"), liq)
    with pytest.raises(FireXError) as e:
        g.write("emitter_mask", np.zeros(g.cells, np.uint8))
    assert e.value.code == A.ERR_BAD_ARG
    with pytest.raises(FireXError):
        g.read_into("flow", np.zeros(10, np.float32))
    g.step(2, DT)
    g.sync()


def test_liquid_cools_and_extinguishes_like_the_oracle():
    """shaders.ts:212-215,246,292-297: a deposited liquid field (the SPH deposit's
    output) enters simulate; both sides must treat it identically."""
    dims = (16, 20, 24)
    opts = sphere_options(dims, P=6, R=6)
    o = OracleSim(dims, opts)
    o.step(4, DT)
    liq = np.zeros((24, 20, 16), np.uint32)
    liq[8:16, 2:10, 4:12] = 4096 * 2
    o.write("liquid", liq)
    g = FireXSim(dims, opts)
    copy_state(o, g)
    g.step(1, DT)
    o.step(1, DT)
    compare_step(g, o, "liquid_step")


def test_parameters_match_the_oracle():
    dims = (16, 20, 24)
    g, o = FireXSim(dims, burner_options()), OracleSim(dims, burner_options())
    cases = [("firePower", 10), ("firePower", float("nan")), ("waterEnabled", 1), ("waterEnabled", True),
             ("viewMode", 3.6), ("opticalDetailTarget", 500), ("nozzleType", 0.7), ("aimHeight", 0.01),
             ("domainDepth", 9.0), ("vorticity", -2.0)]
    for name, value in cases:
        g.set_parameter(name, value)
        o.set_parameter(name, value)
        assert g.get_parameter(name) == o.get_parameter(name), name
    assert np.array_equal(g.uniforms(DT), o.uniforms(DT))


def test_budget_and_bad_dims_are_refused():
    with pytest.raises(FireXError) as e:
        FireXSim((64, 96, 64), make_options(memory_budget_bytes=1 << 20))
    assert e.value.code == A.ERR_BUDGET
    with pytest.raises(FireXError) as e:
        FireXSim((62, 96, 64), make_options())
    assert e.value.code == A.ERR_BAD_ARG


@pytest.mark.parametrize("R", [0, 1, 2])
@pytest.mark.parametrize("P", [0, 1, 2])
def test_small_iteration_counts_bit_exact(P, R):
    """Ping-pong parity, zero-input first sweeps and the cleared buffers the reference
    leaves behind (FireXEngine.ts:2215-2230, 2258-2259) for P, R in {0, 1, 2}."""
    dims = (16, 20, 24)
    for mode in (A.PRESSURE_WARM_F32, A.PRESSURE_COLD_F32, A.PRESSURE_F16):
        opts = sphere_options(dims, P=P, R=R, pressure_mode=mode)
        g, o = FireXSim(dims, opts), OracleSim(dims, opts)
        g.step(3, 0.0)
        o.step(3, 0.0)
        assert g.state == o.state, mode
        fields_equal(g, o)
