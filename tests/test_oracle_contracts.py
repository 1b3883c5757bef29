"""CPU tests of the oracle against the contracts the reference's own tests assert.

The reference has no numeric golden vectors for the Fire-X step (its shader tests are
source-string contracts, src/sim/firex/shaders.test.ts); these tests restate those
contracts as numeric checks on the oracle, plus the pure-function tests of
src/sim/physics.test.ts, gridConfiguration.test.ts, FixedStepClock.test.ts and
offlineTimeline.test.ts.
"""
from __future__ import annotations

import math
import struct

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import make_options
from oracle.oracle import OracleSim, load
from tests.helpers import DT, interior, sphere_options


def uniform_state(sim, T=2000.0, fuel=1.0, o2=2.0):
    X, Y, Z = sim.dims
    flow = np.zeros((Z, Y, X, 4), np.float32)
    flow[..., 3] = T
    sp = np.zeros((Z, Y, X, 4), np.float32)
    sp[..., 0] = fuel
    sp[..., 1] = o2
    sim.write("flow", flow)
    sim.write("species", sp)


def test_stoichiometric_one_to_four_bound():
    """physics.test.ts:37-41 (boundStoichiometricReaction(1, 2, 1, 4) -> 0.5 fuel, 2 O2),
    which mirrors shaders.ts:234-250: a fully ignited uniform cell burns min(fuel, O2/4)."""
    s = OracleSim((8, 16, 8), make_options(pressure_iterations=0, correction_iterations=0, spheres=[]))
    uniform_state(s)
    s.step(1, 1.0)  # dt = 1 s: 1 - exp(-80 dt) rounds to 1, the burn reaches its bound
    sp = s.read("species")
    c = sp[4, 4, 4]
    assert c[0] == pytest.approx(0.5, abs=1e-7)
    assert c[1] == pytest.approx(0.0, abs=1e-7)
    assert s.read("reaction")[4, 4, 4] == pytest.approx(0.5 * 0.22, rel=1e-6)


def test_open_top_and_wall_boundaries():
    """shaders.test.ts:38-47: Dirichlet open top (pressure 0 in the top row), zero normal
    velocity on walls and floor, non-negative top outflow, top row duplicating the
    projected row below (shaders.ts:481-499)."""
    s = OracleSim((16, 20, 24), sphere_options((16, 20, 24), P=6, R=6))
    s.step(3, DT)
    f = s.read("flow")
    p = s.read("pressure")
    assert np.all(p[:, -1, :] == 0)
    assert np.all(f[:, :, 0, 0] == 0) and np.all(f[:, :, -1, 0] == 0)
    assert np.all(f[0, :, :, 2] == 0) and np.all(f[-1, :, :, 2] == 0)
    assert np.all(f[:, 0, :, 1] == 0)
    assert np.all(f[:, -1, :, 1] >= 0)


def test_backward_divergence_forward_gradient_compose_to_the_jacobi_laplacian():
    """shaders.test.ts:49-57: backward divergence paired with the forward gradient. Their
    composition is the nearest-neighbour Laplacian Jacobi solves, so a converged solve
    removes the divergence away from the walls (no stride-2 mode survives); next to the
    walls the wall-normal zeroing after projection leaves the boundary residual the
    presentation masks (docs/implementation-notes.md:95-102)."""
    dims = (12, 16, 12)
    opts = make_options(pressure_iterations=1500, correction_iterations=1500, seed=3, velocity_noise=0.05, spheres=[])
    s = OracleSim(dims, opts, precision=64)
    pre = s.read("final_divergence")
    s.step(1, 0.0)  # dt = 0: the step only projects the noise field
    post = s.read("final_divergence")
    deep = (slice(2, -2),) * 3
    assert np.linalg.norm(post[deep]) < 1e-4 * np.linalg.norm(pre[deep])
    assert np.linalg.norm(interior(post)) < 0.05 * np.linalg.norm(interior(pre))


def test_domain_extent_sets_the_anisotropic_metric():
    """shaders.test.ts:71-82: metric = grid / domainExtent (shaders.ts:39-41)."""
    dims = (8, 8, 8)
    s = OracleSim(dims, make_options(spheres=[]))
    X, Y, Z = dims
    f = np.zeros((Z, Y, X, 4), np.float32)
    f[..., 0] = np.arange(X, dtype=np.float32)[None, None, :] * 0.01
    s.write("flow", f)
    d1 = s.read("final_divergence")[4, 4, 4]
    s.set_parameter("domainWidth", 2.3)  # 2x the default 1.15 m
    d2 = s.read("final_divergence")[4, 4, 4]
    assert d1 == pytest.approx(0.01 * 8 / 1.15, rel=1e-6)
    assert d2 == pytest.approx(d1 / 2, rel=1e-6)


@pytest.mark.parametrize("value,expected", [
    (1.0, 0x3C00), (65504.0, 0x7BFF), (65520.0, 0x7C00), (2.0 ** -24, 0x0001), (2.0 ** -25, 0x0000),
    (3 * 2.0 ** -25, 0x0002), (1 + 2.0 ** -11, 0x3C00), (1 + 3 * 2.0 ** -11, 0x3C02), (-2.5, 0xC100),
])
def test_f16_storage_rounds_to_nearest_even(value, expected):
    """pressureShaders.ts:116 stores f16(p); the oracle rounds to nearest even."""
    assert load().fxo_f32_to_f16(value) == expected


def test_f16_round_trip_is_exact_for_every_half():
    lib = load()
    for h in range(0, 0x10000, 7):
        if (h & 0x7C00) == 0x7C00 and (h & 0x3FF):
            continue  # NaN payloads
        assert lib.fxo_f32_to_f16(lib.fxo_f16_to_f32(h)) == h


def test_reset_initialises_ambient_fields_and_seeded_noise():
    """initializeFields (shaders.ts:135-149): flow=(0,0,0,300), species=(0,O2,0,0); the
    seeded velocity noise is uniform in [-a, a] and reproducible."""
    dims = (16, 20, 24)
    a = OracleSim(dims, sphere_options(dims, noise=0.05, seed=11))
    b = OracleSim(dims, sphere_options(dims, noise=0.05, seed=11))
    c = OracleSim(dims, sphere_options(dims, noise=0.05, seed=12))
    fa, fb, fc = a.read("flow"), b.read("flow"), c.read("flow")
    assert np.array_equal(fa, fb) and not np.array_equal(fa, fc)
    assert np.all(fa[..., 3] == 300) and np.abs(fa[..., :3]).max() <= 0.05
    assert abs(float(fa[..., :3].mean())) < 0.005
    sp = a.read("species")
    assert np.all(sp[..., 1] == 1.0) and np.all(sp[..., [0, 2, 3]] == 0)


def test_sphere_mask_is_exact_integer_geometry():
    dims = (64, 96, 64)
    s = OracleSim(dims, sphere_options(dims, spheres=[dict(center=(32, 8, 32), radius=8)]))
    m = s.read("emitter_mask")
    z, y, x = np.meshgrid(np.arange(64), np.arange(96), np.arange(64), indexing="ij")
    ref = ((x + 0.5 - 32) ** 2 + (y + 0.5 - 8) ** 2 + (z + 0.5 - 32) ** 2) <= 64
    assert np.array_equal(m.astype(bool), ref)


def test_uniform_block_layout_matches_write_uniforms():
    """FireXEngine.writeUniforms (FireXEngine.ts:2043-2113)."""
    s = OracleSim((16, 20, 24), make_options(cinematic=True))
    s.step(2, DT)
    u = s.uniforms(DT)
    assert list(u[:4]) == [16, 20, 24, 16 * 20 * 24]
    assert u[4] == np.float32(DT) and u[5] == np.float32(2 * DT) and u[6] == 2
    assert u[15] == 300 and u[42] == 1
    assert u[28] == np.float32(3.1) and u[31] == np.float32(2.5) and u[32] == np.float32(1.15)
    assert u[13] == np.float32(10 * math.pi / 180)


def test_set_parameter_clamps_and_fallbacks():
    """FireXEngine.setParameter (FireXEngine.ts:937-1032)."""
    s = OracleSim((8, 8, 8), make_options())
    s.set_parameter("firePower", 10)
    assert s.get_parameter("firePower") == 4
    s.set_parameter("firePower", float("nan"))
    assert s.get_parameter("firePower") == 4
    s.set_parameter("waterEnabled", 1)  # numbers are ignored for the boolean
    assert s.get_parameter("waterEnabled") == 0
    s.set_parameter("waterEnabled", True)
    assert s.get_parameter("waterEnabled") == 1
    s.set_parameter("viewMode", 3.6)
    assert s.get_parameter("viewMode") == 4
    s.set_parameter("opticalDetailTarget", 500)
    assert s.get_parameter("opticalDetailTarget") == 512
    s.set_parameter("nozzleType", 0.7)
    assert s.get_parameter("nozzleType") == 1
    s.set_parameter("noSuchParameter", 1)  # ignored, as in the reference


def test_branches_a_and_c_agree_on_a_cold_start():
    """Branch A (warm f32) and C (cold f32, shared buffers) compute the same first step
    from a cleared pressure; they diverge afterwards only through the warm start."""
    dims = (16, 20, 24)
    a = OracleSim(dims, sphere_options(dims, pressure_mode=A.PRESSURE_WARM_F32))
    c = OracleSim(dims, sphere_options(dims, pressure_mode=A.PRESSURE_COLD_F32))
    a.step(1, DT)
    c.step(1, DT)
    assert np.array_equal(a.read("flow"), c.read("flow"))
    a.step(1, DT)
    c.step(1, DT)
    assert not np.array_equal(a.read("flow"), c.read("flow"))


def test_f16_branch_tracks_the_f32_branch():
    dims = (16, 20, 24)
    a = OracleSim(dims, sphere_options(dims, P=12, R=12, pressure_mode=A.PRESSURE_WARM_F32))
    b = OracleSim(dims, sphere_options(dims, P=12, R=12, pressure_mode=A.PRESSURE_F16))
    a.step(3, DT)
    b.step(3, DT)
    pa, pb = a.read("pressure"), b.read("pressure")
    assert np.max(np.abs(pa - pb)) <= 2e-3 * max(1.0, float(np.max(np.abs(pa))))


def test_fp64_oracle_tracks_fp32():
    dims = (16, 20, 24)
    a = OracleSim(dims, sphere_options(dims))
    b = OracleSim(dims, sphere_options(dims), precision=64)
    a.step(3, DT)
    b.step(3, DT)
    fa, fb = a.read("flow"), b.read("flow")
    assert np.max(np.abs(fa[..., :3] - fb[..., :3])) < 1e-3
    assert np.max(np.abs(fa[..., 3] - fb[..., 3])) < 0.5


def test_oracle_is_deterministic():
    dims = (16, 20, 24)
    a = OracleSim(dims, make_options(pressure_iterations=4, correction_iterations=4))
    b = OracleSim(dims, make_options(pressure_iterations=4, correction_iterations=4))
    a.step(4, DT)
    b.step(4, DT)
    for f in ("flow", "species", "pressure", "reaction", "divergence"):
        assert np.array_equal(a.read(f), b.read(f))
