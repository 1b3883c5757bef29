"""firex_divergence_norm_noalloc against firex_divergence_norm, through the C ABI.

The no-allocation entry point serves callers whose device memory belongs to their own
pool or budget, or whose loop must not stall on cudaMalloc/cudaFree: they hand the
library a flow field they own and get its divergence norm without the library
allocating anything. Here the flow of a simulation is copied into a torch tensor (the
"caller-owned" buffer) and both entry points must agree: the per-cell divergence is the
same FP32 expression, so the max abs and the cell count are equal exactly and the L2
norm differs only by the FP64 summation order (relative 1e-12).

Two calls in a row run on grids with different plane counts, larger first, so the
second call runs over scratch that still holds the first call's partial sums.

This file is collected last on purpose, so a run stopped at the first failure has run
every other test before it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXSim, load_library
from tests.helpers import DT, sphere_options

pytestmark = pytest.mark.gpu

REL_L2 = 1e-12


def _metric(sim, dims):
    """grid / domain per axis in FP32, as the engine's cellMetric (shaders.ts:39-41)."""
    names = ("domainWidth", "domainHeight", "domainDepth")
    return [np.float32(n) / max(np.float32(sim.get_parameter(k)), np.float32(0.001)) for n, k in zip(dims, names)]


def _noalloc(lib, flow_dev, dims, metric, stream=None):
    out = (C.c_double * 3)()
    rc = lib.firex_divergence_norm_noalloc(C.c_void_p(flow_dev), A.DIMS(*dims), (C.c_float * 3)(*metric),
                                           C.c_void_p(stream) if stream else None, out)
    return rc, (out[0], out[1], out[2])


def _scene(dims, steps):
    sim = FireXSim(dims, sphere_options(dims, P=8, R=4))
    sim.step(steps, DT)
    sim.sync()
    return sim


def test_noalloc_norm_matches_handle_norm_twice():
    import torch

    lib = load_library()
    cases = [((48, 64, 40), 3), ((32, 40, 24), 2)]  # 38 interior planes, then 22
    for dims, steps in cases:
        sim = _scene(dims, steps)
        try:
            ref = sim.divergence_norm()
            flow = torch.from_numpy(sim.read("flow").reshape(-1)).to("cuda")
            torch.cuda.synchronize()
            rc, got = _noalloc(lib, flow.data_ptr(), dims, _metric(sim, dims))
            assert rc == A.OK, lib.firex_last_error(None)
            assert ref[0] > 0.0
            assert got[2] == ref[2]
            assert got[1] == ref[1]
            assert abs(got[0] - ref[0]) <= REL_L2 * ref[0], (got, ref)
            # the same buffer on the simulation's own stream gives the same answer
            rc, again = _noalloc(lib, flow.data_ptr(), dims, _metric(sim, dims), sim.stream)
            assert rc == A.OK and again == got
        finally:
            sim.close()


def test_noalloc_rejects_beyond_scratch_and_misaligned():
    import torch

    lib = load_library()
    flow = torch.zeros(16 * 4, dtype=torch.float32, device="cuda")
    # more interior planes than the static scratch holds: refused before any launch
    rc, _ = _noalloc(lib, flow.data_ptr(), (4, 4, A.NOALLOC_MAX_PLANES + 3), [1.0, 1.0, 1.0])
    assert rc == A.ERR_BAD_ARG
    assert b"interior planes" in lib.firex_last_error(None)
    # misaligned pointer
    rc, _ = _noalloc(lib, flow.data_ptr() + 4, (2, 2, 2), [1.0, 1.0, 1.0])
    assert rc == A.ERR_BAD_ARG
    # a grid without interior cells launches nothing and reports zeros
    rc, got = _noalloc(lib, flow.data_ptr(), (2, 2, 4), [1.0, 1.0, 1.0])
    assert rc == A.OK and got == (0.0, 0.0, 0.0)


def test_noalloc_rejects_short_buffers_and_host_memory():
    """Dims that need more flow records than the caller's allocation holds, and a host
    pointer, are refused before any launch; the calling thread's current device is left as
    it was."""
    import torch

    lib = load_library()
    dev_before = torch.cuda.current_device()
    small = torch.zeros(64, dtype=torch.float32, device="cuda")  # inside a 2 MiB cached segment
    rc, _ = _noalloc(lib, small.data_ptr(), (256, 256, 64), [1.0, 1.0, 1.0])  # 64 MiB of records
    assert rc == A.ERR_BAD_ARG
    assert b"allocation" in lib.firex_last_error(None)
    host = np.zeros(8 * 8 * 8 * 4, np.float32)
    ptr = host.ctypes.data + (-host.ctypes.data) % 16
    rc, _ = _noalloc(lib, ptr, (4, 4, 4), [1.0, 1.0, 1.0])
    assert rc == A.ERR_BAD_ARG
    assert torch.cuda.current_device() == dev_before
    # a valid call afterwards still works, and leaves the current device alone
    flow = torch.zeros(6 * 6 * 6 * 4, dtype=torch.float32, device="cuda")
    rc, got = _noalloc(lib, flow.data_ptr(), (6, 6, 6), [1.0, 1.0, 1.0])
    assert rc == A.OK and got == (0.0, 0.0, 64.0)
    assert torch.cuda.current_device() == dev_before
