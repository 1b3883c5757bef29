"""The CUDA path against the reference's own step, executed from its WGSL source
(tests/golden/reference_steps.npz; see tests/test_reference_golden.py for how it is made).

Every step of every fixture case is replayed on the GPU from the fixture's state before that
step, so each comparison is one step from identical inputs: the droplets and the integer
liquid field bit for bit (the droplet passes see the same gas state), the fields within the
tolerances of
test_parity_gpu (ATOL: CUDA's sinf / cosf / expf / powf differ from the C library's by a few
ULP) and, in the FP16 pressure branch, the FP16 rounding allowance of
test_parity_configs_gpu.
"""
from __future__ import annotations

import numpy as np
import pytest

from fire_b200.sim import FireXSim
from tests.helpers import max_abs
from tests.test_parity_configs_gpu import fp16_pressure_errors
from tests.test_parity_gpu import ATOL
from tests.test_reference_golden import DATA, META, apply_changes, reshape, start_sim

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", sorted(META))
def test_cuda_step_matches_the_reference_step(case):
    m = META[case]
    g, dims = start_sim(FireXSim, case)
    t, frame = m["start_time"], m["start_frame"]
    for i, dt in enumerate(m["dts"]):
        if i > 0 or m["start"] == "developed":
            src = f"{case}/step{i - 1}" if i > 0 else f"{case}/in"
            g.set_state(t, frame, 0, 0)
            for f in ("flow", "species", "pressure"):
                g.write(f, reshape(f, DATA[f"{src}/{f}"], dims))
            g.write("liquid", reshape("liquid", DATA[f"{src}/liquid"], dims))
            if m.get("droplets") and i > 0:
                g.write_particles(DATA[f"{src}/particles"])
        apply_changes(g, case, i)
        g.step(1, dt)
        t += dt
        frame += 1
        ref = {f: reshape(f, DATA[f"{case}/step{i}/{f}"], dims) for f in ("flow", "species", "pressure", "reaction")}
        if m.get("droplets"):  # the droplet passes read the same gas state: bit-exact
            assert np.array_equal(g.read_particles().reshape(-1, 8), DATA[f"{case}/step{i}/particles"]), (case, i)
            assert np.array_equal(g.read("liquid"), reshape("liquid", DATA[f"{case}/step{i}/liquid"], dims)), (case, i)
        fg = g.read("flow")
        assert max_abs(fg[..., 3], ref["flow"][..., 3]) <= ATOL["flow_T"], (case, i)
        assert max_abs(g.read("species"), ref["species"]) <= ATOL["species"], (case, i)
        assert max_abs(g.read("reaction"), ref["reaction"]) <= ATOL["reaction"], (case, i)
        if m["branch"] == "B":
            fp16_pressure_errors(g.read("pressure"), ref["pressure"], fg, ref["flow"], g.uniforms(dt))
        else:
            assert max_abs(fg[..., :3], ref["flow"][..., :3]) <= ATOL["flow_uvw"], (case, i)
            pr = max_abs(g.read("pressure"), ref["pressure"]) / max(1e-12, float(np.abs(ref["pressure"]).max()))
            assert pr <= ATOL["pressure_rel"], (case, i, pr)
    g.close()
