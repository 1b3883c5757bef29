"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this module. It
exposes ``OracleSim`` with the same methods as ``fire_b200.FireXSim`` so parity tests can
run both side by side; ``precision=32`` is the f32 restatement of the reference step,
``precision=64`` the FP64 accuracy oracle.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

from fire_b200 import _abi as A
from fire_b200.sim import _Handle

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIB_PATH = HERE / "liboracle.so"
_LIB: C.CDLL | None = None


def build() -> Path:
    """Compiles oracle/liboracle.so (g++, OpenMP) if it is missing or stale."""
    src = HERE / "firex_oracle.cpp"
    hdr = ROOT / "include" / "firex.h"
    if LIB_PATH.exists() and LIB_PATH.stat().st_mtime >= max(src.stat().st_mtime, hdr.stat().st_mtime):
        return LIB_PATH
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile"), str(LIB_PATH.relative_to(ROOT))], cwd=ROOT, check=True)
    return LIB_PATH


def load() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            build()
        lib = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        sig = {
            "fxo_create": (C.c_int, [C.c_int, A.DIMS, C.POINTER(A.Options), C.POINTER(vp)]),
            "fxo_destroy": (C.c_int, [vp]),
            "fxo_last_error": (C.c_char_p, [vp]),
            "fxo_set_parameter": (C.c_int, [vp, C.c_char_p, C.c_int32, C.c_double]),
            "fxo_get_parameter": (C.c_int, [vp, C.c_char_p, C.POINTER(C.c_double)]),
            "fxo_reset": (C.c_int, [vp]),
            "fxo_sync": (C.c_int, [vp]),
            "fxo_step": (C.c_int, [vp, C.c_int32, C.c_double]),
            "fxo_read_field": (C.c_int, [vp, C.c_int32, vp, C.c_size_t]),
            "fxo_write_field": (C.c_int, [vp, C.c_int32, vp, C.c_size_t]),
            "fxo_get_state": (C.c_int, [vp, C.POINTER(A.State)]),
            "fxo_set_state": (C.c_int, [vp, C.POINTER(A.State)]),
            "fxo_get_uniforms": (C.c_int, [vp, C.c_double, C.POINTER(C.c_float)]),
            "fxo_divergence_norm": (C.c_int, [vp, C.POINTER(C.c_double)]),
            "fxo_pressure_mode": (C.c_int, [vp]),
            "fxo_pre_projection_norm": (C.c_int, [vp, C.POINTER(C.c_double)]),
            "fxo_read_particles": (C.c_int, [vp, vp, C.c_size_t]),
            "fxo_write_particles": (C.c_int, [vp, vp, C.c_size_t]),
            "fxo_emission_jitter": (C.c_float, [C.c_uint64, C.c_int64, C.c_float]),
            "fxo_velocity_noise": (C.c_float, [C.c_uint64, C.c_uint64, C.c_int, C.c_float]),
            "fxo_f32_to_f16": (C.c_uint16, [C.c_float]),
            "fxo_f16_to_f32": (C.c_float, [C.c_uint16]),
            "fxo_num_threads": (C.c_int, []),
            "fxo_reference_memory_estimate": (C.c_uint64, [A.DIMS, C.c_int64]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


class _PrecisionBound:
    """Adapts fxo_create(precision, ...) to the firex_create(dims, opts, out) shape."""

    def __init__(self, lib: C.CDLL, precision: int):
        self._lib = lib
        self._p = precision

    def __getattr__(self, name):
        if name == "fxo_create":
            return lambda dims, opts, out: self._lib.fxo_create(self._p, dims, opts, out)
        return getattr(self._lib, name)


class OracleSim(_Handle):
    """CPU restatement of the reference step with the FireXSim interface."""

    prefix = "fxo_"

    def __init__(self, dims, options: A.Options | None = None, precision: int = 32, **kw):
        self.precision = precision
        super().__init__(_PrecisionBound(load(), precision), dims, options, **kw)

    @property
    def pressure_mode(self) -> int:
        return self._lib.fxo_pressure_mode(self._h)

    def pre_projection_norm(self) -> tuple[float, float, int]:
        """Interior divergence of the last step's predicted flow: (L2, max abs, cells)."""
        out = (C.c_double * 3)()
        self._lib.fxo_pre_projection_norm(self._h, out)
        return out[0], out[1], int(out[2])


def num_threads() -> int:
    return load().fxo_num_threads()
