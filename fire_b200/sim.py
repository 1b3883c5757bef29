"""Python handle over the C ABI (include/firex.h) of the CUDA library.

``FireXSim`` owns one ``firex_sim*``: create, named parameters, reset, step, field
readback/upload, divergence norm and counters. Fields come back as numpy arrays in the
reference layout, shaped (Z, Y, X, 4) for vec4 fields and (Z, Y, X) for scalars
(cell index x + X*(y + Y*z), shaders.ts:47-51).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Iterable, Mapping, Sequence

import numpy as np

from . import _abi as A

_LIB: C.CDLL | None = None
LIB_PATH = Path(__file__).resolve().parent / "libfirex_b200.so"


class FireXError(RuntimeError):
    """A firex_* call returned a negative status; ``code`` holds it."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads the CUDA library (once): `path`, else the FIREX_LIBRARY environment variable (a
    build of the same sources with other compile-time choices), else the in-tree build.
    Raises if it is missing: there is no fallback."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else Path(os.environ.get("FIREX_LIBRARY") or LIB_PATH)
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build it with `python -m fire_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(str(p))
    A.declare_firex(lib)
    if path is None:
        _LIB = lib
    return lib


def make_options(
    *,
    precision: int = A.PRECISION_F32,
    pressure_mode: int = A.PRESSURE_AUTO,
    pressure_iterations: int = 64,
    correction_iterations: int = 64,
    spheres: Sequence[Mapping[str, object]] | None = None,
    seed: int = 0,
    velocity_noise: float = 0.0,
    emission_jitter: float = 0.0,
    cinematic: bool = True,
    jacobi_block: int = 0,
    memory_budget_bytes: int = 0,
    particle_count: int = 640,
) -> A.Options:
    """Options with the library defaults (firex_default_options) plus overrides.

    ``spheres`` switches the emitter to the sphere list; each entry has ``center``
    (x, y, z in cells), ``radius`` (cells), ``fuel`` and ``temperature`` (K).
    """
    o = A.Options()
    o.precision = precision
    o.pressure_mode = pressure_mode
    o.pressure_iterations = pressure_iterations
    o.correction_iterations = correction_iterations
    o.emitter_mode = A.EMITTER_BURNER
    if spheres is not None:
        if len(spheres) > A.MAX_SPHERES:
            raise ValueError(f"at most {A.MAX_SPHERES} spheres")
        o.emitter_mode = A.EMITTER_SPHERES
        o.num_spheres = len(spheres)
        for i, s in enumerate(spheres):
            c = s["center"]
            o.spheres[i].center[0], o.spheres[i].center[1], o.spheres[i].center[2] = (float(c[0]), float(c[1]), float(c[2]))
            o.spheres[i].radius = float(s["radius"])
            o.spheres[i].fuel = float(s.get("fuel", 1.0))
            o.spheres[i].temperature = float(s.get("temperature", 1500.0))
    o.seed = seed & 0xFFFFFFFFFFFFFFFF
    o.velocity_noise = velocity_noise
    o.emission_jitter = emission_jitter
    o.cinematic = 1 if cinematic else 0
    o.jacobi_block = jacobi_block
    o.memory_budget_bytes = memory_budget_bytes
    o.particle_count = particle_count
    return o


class _Handle:
    """Shared method bodies for any library exporting the firex_* signatures under
    ``prefix``; the CUDA library uses prefix 'firex_'."""

    prefix = "firex_"

    def __init__(self, lib: C.CDLL, dims: Iterable[int], options: A.Options | None = None, **kw):
        self._lib = lib
        self._h = C.c_void_p()
        self.dims = tuple(int(d) for d in dims)
        if len(self.dims) != 3:
            raise ValueError("dims must be (X, Y, Z)")
        opts = options if options is not None else make_options(**kw)
        rc = self._fn("create")(A.DIMS(*self.dims), C.byref(opts), C.byref(self._h))
        if rc != A.OK:
            msg = self._fn("last_error")(None)
            raise FireXError(rc, msg.decode() if msg else "create failed")
        self.options = opts
        self.cells = self.dims[0] * self.dims[1] * self.dims[2]

    def _fn(self, name: str):
        return getattr(self._lib, self.prefix + name)

    def _check(self, rc: int) -> None:
        if rc != A.OK:
            msg = self._fn("last_error")(self._h)
            raise FireXError(rc, msg.decode() if msg else "error")

    # -- lifecycle -----------------------------------------------------------------------
    def close(self) -> None:
        if self._h:
            self._fn("destroy")(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- engine ----------------------------------------------------------------------------
    def set_parameter(self, name: str, value) -> None:
        kind = A.VALUE_BOOLEAN if isinstance(value, bool) else A.VALUE_NUMBER
        self._check(self._fn("set_parameter")(self._h, name.encode(), kind, float(value)))

    def get_parameter(self, name: str) -> float:
        v = C.c_double()
        self._check(self._fn("get_parameter")(self._h, name.encode(), C.byref(v)))
        return v.value

    def reset(self) -> None:
        self._check(self._fn("reset")(self._h))

    def step(self, n: int = 1, dt: float = 1.0 / 60.0) -> None:
        self._check(self._fn("step")(self._h, int(n), float(dt)))

    def sync(self) -> None:
        self._check(self._fn("sync")(self._h))

    # -- fields ------------------------------------------------------------------------------
    def _shape(self, field: int):
        dtype, comps = A.FIELD_LAYOUT[field]
        X, Y, Z = self.dims
        shape = (Z, Y, X, comps) if comps > 1 else (Z, Y, X)
        return np.dtype(dtype), shape

    def read(self, field) -> np.ndarray:
        f = A.FIELD_NAMES[field] if isinstance(field, str) else int(field)
        dtype, shape = self._shape(f)
        out = np.empty(shape, dtype=dtype)
        self._check(self._fn("read_field")(self._h, f, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def read_into(self, field, out: np.ndarray) -> np.ndarray:
        f = A.FIELD_NAMES[field] if isinstance(field, str) else int(field)
        self._check(self._fn("read_field")(self._h, f, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def write(self, field, data: np.ndarray) -> None:
        f = A.FIELD_NAMES[field] if isinstance(field, str) else int(field)
        dtype, shape = self._shape(f)
        arr = np.ascontiguousarray(data, dtype=dtype).reshape(shape)
        self._check(self._fn("write_field")(self._h, f, arr.ctypes.data_as(C.c_void_p), arr.nbytes))

    # -- droplets ----------------------------------------------------------------------------
    @property
    def particle_count(self) -> int:
        return int(self.options.particle_count)

    def read_particles(self) -> np.ndarray:
        """Droplets as (particle_count, 2, 4) float32: (x, y, z, age), (vx, vy, vz, mass)."""
        out = np.empty((self.particle_count, 2, 4), dtype=np.float32)
        self._check(self._fn("read_particles")(self._h, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def write_particles(self, data: np.ndarray) -> None:
        arr = np.ascontiguousarray(data, dtype=np.float32).reshape(self.particle_count, 2, 4)
        self._check(self._fn("write_particles")(self._h, arr.ctypes.data_as(C.c_void_p), arr.nbytes))

    def divergence_norm(self) -> tuple[float, float, int]:
        out = (C.c_double * 3)()
        self._check(self._fn("divergence_norm")(self._h, out))
        return out[0], out[1], int(out[2])

    # -- counters ---------------------------------------------------------------------------
    @property
    def state(self) -> dict:
        st = A.State()
        self._check(self._fn("get_state")(self._h, C.byref(st)))
        return {
            "simulation_time": st.simulation_time,
            "frame_index": st.frame_index,
            "species_index": st.species_index,
            "pressure_index": st.pressure_index,
        }

    def set_state(self, simulation_time: float, frame_index: int, species_index: int, pressure_index: int) -> None:
        st = A.State(simulation_time, frame_index, species_index, pressure_index)
        self._check(self._fn("set_state")(self._h, C.byref(st)))

    def uniforms(self, dt: float = 1.0 / 60.0) -> np.ndarray:
        out = (C.c_float * A.UNIFORM_FLOATS)()
        self._check(self._fn("get_uniforms")(self._h, float(dt), out))
        return np.frombuffer(out, dtype=np.float32).copy()

    def snapshot(self) -> dict:
        """All state needed to resume: counters plus the resident fields."""
        snap = {"state": self.state}
        for name in ("flow", "species", "pressure", "liquid", "reaction", "divergence"):
            snap[name] = self.read(name)
        return snap

    def restore(self, snap: Mapping) -> None:
        st = snap["state"]
        self.set_state(st["simulation_time"], st["frame_index"], st["species_index"], st["pressure_index"])
        for name in ("flow", "species", "pressure", "liquid", "reaction", "divergence"):
            if name in snap:
                self.write(name, snap[name])


class FireXSim(_Handle):
    """One simulation on the GPU through libfirex_b200.so."""

    prefix = "firex_"

    def __init__(self, dims: Iterable[int], options: A.Options | None = None, **kw):
        super().__init__(load_library(), dims, options, **kw)

    def set_params(self, block) -> None:
        """Every parameter from a 44-float uniform block (the layout of `uniforms()` and of
        the reference's writeUniforms); the grid slots must match this simulation."""
        arr = np.ascontiguousarray(np.asarray(block, dtype=np.float32).reshape(A.UNIFORM_FLOATS))
        self._check(self._lib.firex_set_params(self._h, arr.ctypes.data_as(C.POINTER(C.c_float))))

    def set_render_packing(self, on: bool) -> None:
        """Pack the three FP16 render volumes at the end of every step (qualityShaders.ts)."""
        self._check(self._lib.firex_set_render_packing(self._h, 1 if on else 0))

    def render_volumes(self) -> list:
        """Device addresses of the render volumes (flow, chemistry, media); 0 before use."""
        out = (C.c_void_p * 3)()
        self._check(self._lib.firex_render_volumes(self._h, out))
        return [v or 0 for v in out]

    def read_async(self, field, out: np.ndarray) -> np.ndarray:
        """Starts an overlapped copy of `field` (as it stands after the steps enqueued so
        far) into `out`; `out` is complete after sync(). Use pinned memory for overlap."""
        f = A.FIELD_NAMES[field] if isinstance(field, str) else int(field)
        self._check(self._lib.firex_read_field_async(self._h, f, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    @property
    def device_bytes(self) -> int:
        v = C.c_uint64()
        self._check(self._lib.firex_device_bytes(self._h, C.byref(v)))
        return v.value

    @property
    def pressure_mode(self) -> int:
        o, d = A.Options(), A.DIMS()
        self._check(self._lib.firex_get_info(self._h, d, C.byref(o)))
        return o.pressure_mode  # the resolved branch (AUTO picked by grid size)

    @property
    def stream(self) -> int:
        return self._lib.firex_stream(self._h) or 0

    def set_wait_limit(self, polls: int) -> None:
        """Polls before a bounded device wait gives up (0: the library's limit)."""
        self._check(self._lib.firex_set_wait_limit(self._h, int(polls)))

    def test_hold_face(self, box: int, sweep: int) -> None:
        """Test hook: box `box` of the resident Jacobi stops publishing its faces from sweep
        `sweep` on (box < 0 clears it), so that its neighbours' bounded waits expire."""
        self._check(self._lib.firex_test_hold_face(self._h, int(box), int(sweep)))

    def set_jacobi(self, kernel, block: int = 0, zchunk: int = 0) -> None:
        """Jacobi kernel: 'auto', 'unblocked', 'zmarch', 'fused' (with `block` sweeps per
        launch) or 'resident' (`block` = box variant + 1, 0 = planner's choice), and z planes
        per CTA (0 = auto)."""
        self._check(self._lib.firex_set_jacobi(self._h, jacobi_kernel(kernel), int(block), int(zchunk)))

    def set_staging(self, staging: int) -> None:
        """How the two-sweep pass stages its planes: A.STAGING_AUTO (cp.async), A.STAGING_CPASYNC
        or A.STAGING_TMA (tensor tile loads; FP32 pressure only)."""
        self._check(self._lib.firex_set_staging(self._h, int(staging)))

    def set_tiles(self, simulate_by: int, project: int = 0) -> None:
        """Brick shape of the source pass: 32 x simulate_by x (8 / simulate_by) cells (2, 4, 8;
        0: default); `project`: A.PROJECT_FUSED / A.PROJECT_SEPARATE primary projection and
        residual divergence (A.PROJECT_AUTO: fused below 8 Mi cells)."""
        self._check(self._lib.firex_set_tiles(self._h, int(simulate_by), int(project)))

    @property
    def diagnostics(self) -> dict:
        d = A.Diagnostics()
        self._check(self._lib.firex_get_diagnostics(self._h, C.byref(d)))
        return {k: getattr(d, k) for k, _ in A.Diagnostics._fields_ if k != "reserved"}

    def set_graphs(self, on: bool) -> None:
        self._check(self._lib.firex_set_graphs(self._h, 1 if on else 0))

    def set_profiling(self, on: bool) -> None:
        self._check(self._lib.firex_set_profiling(self._h, 1 if on else 0))

    def pass_times(self) -> dict:
        """Accumulated device ms and launch counts per pass since the previous call."""
        ms = (C.c_double * len(A.PASS_NAMES))()
        n = (C.c_int64 * len(A.PASS_NAMES))()
        self._check(self._lib.firex_pass_times(self._h, ms, n))
        return {name: (ms[i], n[i]) for i, name in enumerate(A.PASS_NAMES)}


JACOBI_KERNELS = {"auto": A.JACOBI_AUTO, "unblocked": A.JACOBI_UNBLOCKED, "zmarch": A.JACOBI_ZMARCH,
                  "fused": A.JACOBI_FUSED, "resident": A.JACOBI_RESIDENT}


def jacobi_kernel(kernel) -> int:
    return JACOBI_KERNELS[kernel] if isinstance(kernel, str) else int(kernel)


def planned_device_bytes(dims, options: A.Options) -> int:
    """Device bytes firex_create would allocate (admission control)."""
    return int(load_library().firex_planned_device_bytes(A.DIMS(*dims), C.byref(options)))


class FireXBatch:
    """Simulations stepped together by the same launches (firex_batch_*).

    Members may have different grid sizes and iteration counts; they must share the
    storage precision and the pressure storage type. While a member, a simulation is
    stepped only through the batch; its reads and writes stay valid.
    """

    def __init__(self):
        self._lib = load_library()
        self._h = C.c_void_p()
        rc = self._lib.firex_batch_create(C.byref(self._h))
        if rc != A.OK:
            raise FireXError(rc, (self._lib.firex_batch_last_error(None) or b"").decode())
        self.members: list[FireXSim] = []

    def _check(self, rc: int) -> None:
        if rc != A.OK:
            raise FireXError(rc, (self._lib.firex_batch_last_error(self._h) or b"").decode())

    def add(self, sim: FireXSim) -> None:
        self._check(self._lib.firex_batch_add(self._h, sim._h))
        self.members.append(sim)

    def remove(self, sim: FireXSim) -> None:
        self._check(self._lib.firex_batch_remove(self._h, sim._h))
        self.members.remove(sim)

    def __len__(self) -> int:
        n = C.c_int32()
        self._check(self._lib.firex_batch_size(self._h, C.byref(n)))
        return n.value

    def step(self, n: int = 1, dt: float = 1.0 / 60.0) -> None:
        self._check(self._lib.firex_batch_step(self._h, int(n), float(dt)))

    def set_jacobi(self, kernel, block: int = 0, zchunk: int = 0) -> None:
        self._check(self._lib.firex_batch_set_jacobi(self._h, jacobi_kernel(kernel), int(block), int(zchunk)))

    def set_staging(self, staging: int) -> None:
        self._check(self._lib.firex_batch_set_staging(self._h, int(staging)))

    def set_tiles(self, simulate_by: int, project: int = 0) -> None:
        self._check(self._lib.firex_batch_set_tiles(self._h, int(simulate_by), int(project)))

    def sync(self) -> None:
        self._check(self._lib.firex_batch_sync(self._h))

    @property
    def stream(self) -> int:
        return self._lib.firex_batch_stream(self._h) or 0

    def close(self) -> None:
        if self._h:
            self._lib.firex_batch_destroy(self._h)
            self._h = C.c_void_p()
            self.members = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
