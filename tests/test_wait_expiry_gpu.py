"""The resident Jacobi's bounded waits, made to expire on purpose.

The resident kernel's CTAs wait on their neighbours' published faces with bounded polls
(fx_jacobi_res.cuh). Here one box stops publishing its faces from one sweep on
(firex_test_hold_face: a flag that nothing sets) and the wait limit is short
(firex_set_wait_limit): the neighbours' waits expire, each CTA sets the simulation's error word and returns, the waits of the boxes
behind them expire in turn, and every CTA of the launch returns. The host must then report
FIREX_ERR_TIMEOUT at the next sync and poison the handle, as the reference poisons its engine
after a device loss (FireXEngine.ts:538-542, 2887-2897: later calls throw). The GPU stays
usable: a fresh handle afterwards steps bit-exactly like the oracle.
"""
from __future__ import annotations

import pytest

from fire_b200 import _abi as A
from fire_b200.sim import FireXError, FireXSim
from oracle.oracle import OracleSim
from tests.helpers import DT, sphere_options
from tests.test_parity_gpu import fields_equal

pytestmark = pytest.mark.gpu

DIMS = (64, 96, 64)


def test_withheld_face_expires_the_waits_and_poisons_the_handle():
    opts = sphere_options(DIMS, P=12, R=12)
    g = FireXSim(DIMS, opts)
    g.step(1, DT)
    g.sync()
    assert g.diagnostics["jacobi_kernel"] == A.JACOBI_RESIDENT
    g.set_wait_limit(4096)
    g.test_hold_face(0, 3)
    g.step(1, DT)
    with pytest.raises(FireXError) as e:
        g.sync()
    assert e.value.code == A.ERR_TIMEOUT
    with pytest.raises(FireXError) as e:
        g.step(1, DT)
    assert e.value.code == A.ERR_STATE
    g.close()

    # the device and the library are unharmed: a fresh handle runs the same kernel exactly
    h, o = FireXSim(DIMS, opts), OracleSim(DIMS, opts)
    h.step(2, 0.0)
    o.step(2, 0.0)
    h.sync()
    assert h.diagnostics["jacobi_kernel"] == A.JACOBI_RESIDENT
    fields_equal(h, o)
    h.close()
    o.close()


def test_hold_arguments_are_checked():
    g = FireXSim((16, 20, 24), sphere_options((16, 20, 24)))
    with pytest.raises(FireXError) as e:
        g.test_hold_face(5000, 1)
    assert e.value.code == A.ERR_BAD_ARG
    g.test_hold_face(-1, 0)  # clears
    g.set_wait_limit(0)      # the library's limit
    g.step(1, DT)
    g.sync()
    g.close()
