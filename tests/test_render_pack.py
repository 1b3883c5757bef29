"""Render-field packing (storePackedFields / packFields, qualityShaders.ts:37-87): the three
rgba16float volumes as 4 x FP16 per cell. The oracle's packing is pinned against a numpy
restatement of the WGSL (CPU); the CUDA packing must equal the oracle's bit for bit from the
same state, in the default view and in the divergence view (7), and when packed at the end
of every step (GPU)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXSim
from oracle.oracle import OracleSim
from tests.helpers import DT, copy_state, sphere_options

F32 = np.float32


def smoothstep(e0, e1, x):
    t = np.clip((x - F32(e0)) / (F32(e1) - F32(e0)), F32(0), F32(1)).astype(np.float32)
    return (t * t * (F32(3) - F32(2) * t)).astype(np.float32)


def pack_reference(flow, species, reaction, liquid, final_div, view7):
    """numpy restatement of storePackedFields in FP32, then FP16 (round to nearest even)."""
    sp = np.maximum(species, F32(0))
    rc = np.clip(reaction, F32(0), F32(4))
    richness = np.clip(sp[..., 0] / np.maximum(sp[..., 0] + sp[..., 1] * F32(0.25), F32(0.0001)), F32(0), F32(1))
    soot = (sp[..., 2] * smoothstep(0.25, 0.82, richness)).astype(np.float32)
    liq = (liquid.astype(np.float32) * F32(3.4 / 4096.0)).astype(np.float32)
    disp = np.maximum(np.maximum(rc, soot), np.maximum(liq, np.maximum(sp[..., 3], smoothstep(420.0, 700.0, flow[..., 3]))))
    if view7:
        disp = final_div.copy()
        disp[0, :, :] = disp[-1, :, :] = 0
        disp[:, 0, :] = disp[:, -1, :] = 0
        disp[:, :, 0] = disp[:, :, -1] = 0
    t = np.clip((flow[..., 3] - F32(300)) / F32(2600), F32(0), F32(1))
    h = lambda a: a.astype(np.float16).view(np.uint16)
    return (h(np.stack([flow[..., 0], flow[..., 1], flow[..., 2], t], -1)), h(sp),
            h(np.stack([rc, soot, liq, disp], -1)))


@pytest.mark.parametrize("view", [0, 7])
def test_oracle_packing_matches_numpy_restatement(view):
    dims = (16, 20, 24)
    o = OracleSim(dims, sphere_options(dims, P=8, R=6), precision=32)
    o.set_parameter("viewMode", view)
    o.step(4, DT)
    ref = pack_reference(o.read("flow"), o.read("species"), o.read("reaction"), o.read("liquid"),
                         o.read("final_divergence"), view == 7)
    for name, r in zip(("render_flow", "render_chemistry", "render_media"), ref):
        assert np.array_equal(o.read(name), r), name


def _device_u16(ptr, shape):
    from cuda.bindings import runtime as rt
    out = np.empty(shape, np.uint16)
    err, = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("view", [0, 7])
def test_cuda_packing_equals_oracle(view):
    dims = (32, 48, 32)
    opts = sphere_options(dims, P=10, R=8)
    o = OracleSim(dims, opts, precision=32)
    o.set_parameter("viewMode", view)
    o.step(5, DT)
    g = FireXSim(dims, opts)
    g.set_parameter("viewMode", view)
    copy_state(o, g, fields=("flow", "species", "pressure", "liquid", "reaction"))
    for name in ("render_flow", "render_chemistry", "render_media"):
        assert np.array_equal(g.read(name), o.read(name)), name


@pytest.mark.gpu
def test_packing_at_step_end_equals_packing_on_read():
    dims = (32, 48, 32)
    g = FireXSim(dims, sphere_options(dims, P=10, R=8))
    g.set_render_packing(True)
    g.step(3, DT)
    g.sync()
    ptrs = g.render_volumes()
    assert all(ptrs)
    X, Y, Z = dims
    at_step = [_device_u16(p, (Z, Y, X, 4)) for p in ptrs]
    on_read = [g.read(n) for n in ("render_flow", "render_chemistry", "render_media")]
    for a, b in zip(at_step, on_read):
        assert np.array_equal(a, b)
    d = g.diagnostics  # the packing pass joins the step (the residual projection may run in the resident launch)
    assert d["launches_per_step"] == 10 - d["project_resident"]


@pytest.mark.gpu
def test_offline_frame_presentation_packs_the_last_step():
    """renderOfflineFrame(present=True) leaves the render volumes of the final state on the
    device (the headless presentation); present=False leaves them as they were."""
    from fire_b200.engine import FireXEngine

    e = FireXEngine(quality="low")
    e.initialize()
    e.setParameter("waterEnabled", True)
    e.setParameter("waterFlow", 0.6)
    e.renderOfflineFrame(1 / 15, present=True)
    sim = e.simulation
    X, Y, Z = sim.dims
    ptrs = e.renderVolumes()
    assert all(ptrs)
    packed = [_device_u16(p, (Z, Y, X, 4)) for p in ptrs]
    fresh = [sim.read(n) for n in ("render_flow", "render_chemistry", "render_media")]
    for a, b in zip(packed, fresh):
        assert np.array_equal(a, b)
    assert packed[2][..., 2].any()  # the media volume carries the sprayed liquid
    e.renderOfflineFrame(1 / 30, present=False)
    assert np.array_equal(_device_u16(ptrs[0], (Z, Y, X, 4)), packed[0])
    e.dispose()
