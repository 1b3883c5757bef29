"""firex_set_params: every parameter at once from a 44-float block in the layout of the
reference's uniform buffer (Parameters, shaders.ts:2-14, written by FireXEngine.writeUniforms,
FireXEngine.ts:2043-2113). The block goes through the same rules as the named setter
(FireXEngine.setParameter's clamps, FireXEngine.ts:937-1032), so a handle given a block and a
handle given the same values by name must produce the same uniforms and the same step, bit
for bit; a block for another grid is refused."""
from __future__ import annotations

import math

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXError, FireXSim
from tests.helpers import DT, sphere_options

pytestmark = pytest.mark.gpu

DIMS = (16, 20, 24)
FIELDS = ("flow", "species", "pressure", "reaction", "divergence", "correction")

# (slot, parameter name, value written into the block, value the named setter receives)
CHANGES = [
    (8, "fuelRate", 0.45, 0.45),
    (11, "vorticity", 2.2, 2.2),
    (13, "sprayAngle", math.radians(25.0), 25.0),
    (24, "viewMode", 3.6, 3.6),           # rounds to 4
    (28, "burnerSize", 0.1, 0.1),         # clamps to 0.35
    (31, "firePower", 10.0, 10.0),        # clamps to 4
    (32, "domainWidth", 1.5, 1.5),
    (37, "buoyancyScale", 1.7, 1.7),
    (40, "airEntrainment", 2.4, 2.4),
    (43, "opticalDetailTarget", 600.0, 600.0),  # -> 512
]


def test_block_equals_named_parameters_and_steps_the_same():
    opts = sphere_options(DIMS, P=8, R=8)
    a, b = FireXSim(DIMS, opts), FireXSim(DIMS, opts)
    block = a.uniforms(DT)
    for slot, _, v, _ in CHANGES:
        block[slot] = np.float32(v)
    a.set_params(block)
    for _, name, _, v in CHANGES:
        b.set_parameter(name, v)
    ua, ub = a.uniforms(DT), b.uniforms(DT)
    assert np.array_equal(ua, ub)
    assert ua[24] == 4.0 and ua[28] == np.float32(0.35) and ua[31] == 4.0 and ua[43] == 512.0
    assert ua[13] == block[13]  # the spray angle goes through degrees and back exactly
    a.step(2, DT)
    b.step(2, DT)
    for f in FIELDS:
        assert np.array_equal(a.read(f), b.read(f)), f
    a.close()
    b.close()


def test_own_block_round_trips():
    s = FireXSim(DIMS, sphere_options(DIMS))
    s.set_parameter("firePower", 3.3)
    s.set_parameter("waterEnabled", True)
    block = s.uniforms(DT)
    s.set_params(block)
    assert np.array_equal(s.uniforms(DT), block)
    s.close()


def test_block_for_another_grid_is_refused():
    s = FireXSim(DIMS, sphere_options(DIMS))
    block = s.uniforms(DT)
    before = block.copy()
    block[0] = 32.0
    block[8] = 0.9
    with pytest.raises(FireXError) as e:
        s.set_params(block)
    assert e.value.code == A.ERR_BAD_ARG
    assert np.array_equal(s.uniforms(DT), before)
    s.close()
