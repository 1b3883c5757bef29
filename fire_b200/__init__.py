"""fire_b200 — B200-native (sm_100a) Fire-X simulation step behind a C ABI.

The compute path is the CUDA library ``fire_b200/libfirex_b200.so`` (built by
``fire_b200.build``). There is no CPU fallback: importing the engine API loads that
library and fails loudly if it is missing or cannot be loaded.
"""
from __future__ import annotations

from ._abi import (  # noqa: F401
    EMITTER_BURNER, EMITTER_SPHERES, FIELD_NAMES, PRECISION_F32, PRECISION_MIXED, PRESSURE_AUTO,
    PRESSURE_COLD_F32, PRESSURE_F16, PRESSURE_WARM_F32,
)
from .sim import FireXBatch, FireXError, FireXSim, load_library, make_options, planned_device_bytes  # noqa: F401
from .engine import FireXEngine  # noqa: F401

__all__ = ["FireXEngine", "FireXSim", "FireXBatch", "FireXError", "make_options", "load_library", "planned_device_bytes"]
