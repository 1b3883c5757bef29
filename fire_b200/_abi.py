"""ctypes mirror of include/firex.h (constants, structs, function prototypes).

The same declarations serve the CUDA library (prefix ``firex_``) and, in tests, the CPU
oracle (prefix ``fxo_``), whose entry points take the same arguments.
"""
from __future__ import annotations

import ctypes as C

ABI_VERSION = 1

OK = 0
ERR_BAD_ARG = -1
ERR_OOM = -2
ERR_BUDGET = -3
ERR_CUDA = -4
ERR_TIMEOUT = -5
ERR_UNSUPPORTED = -6
ERR_STATE = -7

NOALLOC_MAX_PLANES = 2048  # interior z planes the no-allocation norm's static scratch holds

PRECISION_F32 = 0
PRECISION_MIXED = 1

PRESSURE_AUTO = 0
PRESSURE_WARM_F32 = 1
PRESSURE_F16 = 2
PRESSURE_COLD_F32 = 3

HEAVY_GRID_CELL_THRESHOLD = 64 * 1024 * 1024

EMITTER_BURNER = 0
EMITTER_SPHERES = 1
MAX_SPHERES = 8

FIELD_FLOW = 0
FIELD_SPECIES = 1
FIELD_PRESSURE = 2
FIELD_DIVERGENCE = 3
FIELD_REACTION = 4
FIELD_LIQUID = 5
FIELD_EMITTER_MASK = 6
FIELD_CORRECTION = 7
FIELD_FINAL_DIVERGENCE = 8
FIELD_RENDER_FLOW = 9
FIELD_RENDER_CHEMISTRY = 10
FIELD_RENDER_MEDIA = 11
FIELD_COUNT = 12

JACOBI_AUTO = 0
JACOBI_UNBLOCKED = 1
JACOBI_ZMARCH = 2
JACOBI_FUSED = 3
JACOBI_RESIDENT = 4
STAGING_AUTO = 0
STAGING_CPASYNC = 1
STAGING_TMA = 2
PROJECT_AUTO = 0
PROJECT_FUSED = 1
PROJECT_SEPARATE = 2

VALUE_NUMBER = 0
VALUE_BOOLEAN = 1

UNIFORM_FLOATS = 44

# (numpy dtype, components per cell) of each field in the reference layout
FIELD_LAYOUT = {
    FIELD_FLOW: ("float32", 4),
    FIELD_SPECIES: ("float32", 4),
    FIELD_PRESSURE: ("float32", 1),
    FIELD_DIVERGENCE: ("float32", 1),
    FIELD_REACTION: ("float32", 1),
    FIELD_LIQUID: ("uint32", 1),
    FIELD_EMITTER_MASK: ("uint8", 1),
    FIELD_CORRECTION: ("float32", 1),
    FIELD_FINAL_DIVERGENCE: ("float32", 1),
    FIELD_RENDER_FLOW: ("uint16", 4),
    FIELD_RENDER_CHEMISTRY: ("uint16", 4),
    FIELD_RENDER_MEDIA: ("uint16", 4),
}

FIELD_NAMES = {
    "flow": FIELD_FLOW,
    "species": FIELD_SPECIES,
    "pressure": FIELD_PRESSURE,
    "divergence": FIELD_DIVERGENCE,
    "reaction": FIELD_REACTION,
    "liquid": FIELD_LIQUID,
    "emitter_mask": FIELD_EMITTER_MASK,
    "correction": FIELD_CORRECTION,
    "final_divergence": FIELD_FINAL_DIVERGENCE,
    "render_flow": FIELD_RENDER_FLOW,
    "render_chemistry": FIELD_RENDER_CHEMISTRY,
    "render_media": FIELD_RENDER_MEDIA,
}


class Sphere(C.Structure):
    _fields_ = [
        ("center", C.c_float * 3),
        ("radius", C.c_float),
        ("fuel", C.c_float),
        ("temperature", C.c_float),
    ]


class Options(C.Structure):
    _fields_ = [
        ("precision", C.c_int32),
        ("pressure_mode", C.c_int32),
        ("pressure_iterations", C.c_int32),
        ("correction_iterations", C.c_int32),
        ("emitter_mode", C.c_int32),
        ("num_spheres", C.c_int32),
        ("spheres", Sphere * MAX_SPHERES),
        ("seed", C.c_uint64),
        ("velocity_noise", C.c_float),
        ("emission_jitter", C.c_float),
        ("cinematic", C.c_int32),
        ("jacobi_block", C.c_int32),
        ("memory_budget_bytes", C.c_uint64),
        ("jacobi_zchunk", C.c_int32),
        ("particle_count", C.c_int32),
        ("reserved", C.c_int32 * 6),
    ]


class DeviceLimits(C.Structure):
    _fields_ = [("max_texture_dimension_3d", C.c_uint64), ("max_storage_buffer_binding_size", C.c_uint64),
                ("max_buffer_size", C.c_uint64)]


class PreflightResult(C.Structure):
    _fields_ = [("issues", C.c_uint32), ("issue_count", C.c_uint32), ("cell_count", C.c_uint64),
                ("grid_bytes", C.c_uint64), ("particle_bytes", C.c_uint64), ("fixed_bytes", C.c_uint64),
                ("total_bytes", C.c_uint64), ("largest_storage_buffer_bytes", C.c_uint64),
                ("planned_device_bytes", C.c_uint64), ("message", C.c_char * 1024)]


# preflight issue bits and the reference's codes (gridConfiguration.ts:297-350)
ISSUE_CODES = {0x01: "invalid-dimension", 0x02: "unaligned-dimension", 0x04: "texture-dimension-limit",
               0x08: "storage-binding-limit", 0x10: "buffer-size-limit", 0x20: "memory-budget"}


class Diagnostics(C.Structure):
    _fields_ = [
        ("fast_division", C.c_int32),
        ("jacobi_block", C.c_int32),
        ("jacobi_zchunk", C.c_int32),
        ("graph", C.c_int32),
        ("launches_per_step", C.c_int32),
        ("jacobi_kernel", C.c_int32),
        ("jacobi_variant", C.c_int32),
        ("jacobi_staging", C.c_int32),
        ("simulate_by", C.c_int32),
        ("project_fused", C.c_int32),
        ("project_resident", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class State(C.Structure):
    _fields_ = [
        ("simulation_time", C.c_double),
        ("frame_index", C.c_int64),
        ("species_index", C.c_int32),
        ("pressure_index", C.c_int32),
    ]


DIMS = C.c_int32 * 3


def declare_firex(lib: C.CDLL) -> None:
    """Attach argtypes/restype to the library's firex_* entry points."""
    vp = C.c_void_p
    sig = {
        "firex_default_options": (None, [C.POINTER(Options)]),
        "firex_field_element_size": (C.c_size_t, [C.c_int32]),
        "firex_create": (C.c_int, [DIMS, C.POINTER(Options), C.POINTER(vp)]),
        "firex_destroy": (C.c_int, [vp]),
        "firex_last_error": (C.c_char_p, [vp]),
        "firex_set_parameter": (C.c_int, [vp, C.c_char_p, C.c_int32, C.c_double]),
        "firex_set_params": (C.c_int, [vp, C.POINTER(C.c_float)]),
        "firex_get_parameter": (C.c_int, [vp, C.c_char_p, C.POINTER(C.c_double)]),
        "firex_reset": (C.c_int, [vp]),
        "firex_step": (C.c_int, [vp, C.c_int32, C.c_double]),
        "firex_sync": (C.c_int, [vp]),
        "firex_read_field": (C.c_int, [vp, C.c_int32, vp, C.c_size_t]),
        "firex_write_field": (C.c_int, [vp, C.c_int32, vp, C.c_size_t]),
        "firex_divergence_norm": (C.c_int, [vp, C.POINTER(C.c_double)]),
        "firex_read_field_async": (C.c_int, [vp, C.c_int32, vp, C.c_size_t]),
        "firex_set_render_packing": (C.c_int, [vp, C.c_int32]),
        "firex_render_volumes": (C.c_int, [vp, C.POINTER(C.c_void_p)]),
        "firex_read_particles": (C.c_int, [vp, vp, C.c_size_t]),
        "firex_write_particles": (C.c_int, [vp, vp, C.c_size_t]),
        "firex_divergence_norm_noalloc": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_float), vp,
                                                    C.POINTER(C.c_double)]),
        "firex_set_wait_limit": (C.c_int, [vp, C.c_uint32]),
        "firex_test_hold_face": (C.c_int, [vp, C.c_int32, C.c_int32]),
        "firex_get_state": (C.c_int, [vp, C.POINTER(State)]),
        "firex_set_state": (C.c_int, [vp, C.POINTER(State)]),
        "firex_get_uniforms": (C.c_int, [vp, C.c_double, C.POINTER(C.c_float)]),
        "firex_get_info": (C.c_int, [vp, DIMS, C.POINTER(Options)]),
        "firex_device_bytes": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
        "firex_reference_memory_estimate": (C.c_uint64, [DIMS, C.c_int64]),
        "firex_preflight": (C.c_int, [DIMS, C.POINTER(Options), C.POINTER(DeviceLimits), C.POINTER(PreflightResult)]),
        "firex_stream": (vp, [vp]),
        "firex_set_profiling": (C.c_int, [vp, C.c_int32]),
        "firex_pass_times": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
        "firex_planned_device_bytes": (C.c_uint64, [DIMS, C.POINTER(Options)]),
        "firex_set_graphs": (C.c_int, [vp, C.c_int32]),
        "firex_set_jacobi": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32]),
        "firex_get_diagnostics": (C.c_int, [vp, C.POINTER(Diagnostics)]),
        "firex_batch_set_jacobi": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32]),
        "firex_set_staging": (C.c_int, [vp, C.c_int32]),
        "firex_batch_set_staging": (C.c_int, [vp, C.c_int32]),
        "firex_set_tiles": (C.c_int, [vp, C.c_int32, C.c_int32]),
        "firex_batch_set_tiles": (C.c_int, [vp, C.c_int32, C.c_int32]),
        "firex_batch_create": (C.c_int, [C.POINTER(vp)]),
        "firex_batch_destroy": (C.c_int, [vp]),
        "firex_batch_add": (C.c_int, [vp, vp]),
        "firex_batch_remove": (C.c_int, [vp, vp]),
        "firex_batch_size": (C.c_int, [vp, C.POINTER(C.c_int32)]),
        "firex_batch_step": (C.c_int, [vp, C.c_int32, C.c_double]),
        "firex_batch_sync": (C.c_int, [vp]),
        "firex_batch_last_error": (C.c_char_p, [vp]),
        "firex_batch_stream": (vp, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


# Entry points the header declares; the CPU suite checks the built library exports them.
HEADER_SYMBOLS = [
    "firex_default_options", "firex_field_element_size", "firex_create", "firex_destroy",
    "firex_last_error", "firex_set_parameter", "firex_set_params", "firex_get_parameter", "firex_reset", "firex_step",
    "firex_sync", "firex_read_field", "firex_read_field_async", "firex_write_field", "firex_divergence_norm",
    "firex_set_render_packing", "firex_render_volumes", "firex_read_particles", "firex_write_particles",
    "firex_divergence_norm_noalloc", "firex_set_wait_limit", "firex_test_hold_face", "firex_get_state",
    "firex_set_state", "firex_get_uniforms", "firex_get_info", "firex_device_bytes",
    "firex_reference_memory_estimate", "firex_preflight", "firex_stream", "firex_set_profiling", "firex_pass_times",
    "firex_planned_device_bytes", "firex_set_graphs", "firex_set_jacobi", "firex_get_diagnostics", "firex_batch_set_jacobi", "firex_set_staging", "firex_batch_set_staging", "firex_set_tiles", "firex_batch_set_tiles", "firex_batch_create", "firex_batch_destroy",
    "firex_batch_add", "firex_batch_remove", "firex_batch_size", "firex_batch_step", "firex_batch_sync",
    "firex_batch_last_error", "firex_batch_stream",
]

PASS_NAMES = ("simulate", "divergence", "jacobi", "project", "other", "particles")
