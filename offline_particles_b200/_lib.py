"""ctypes binding of liboffline_particles_b200.so (the C ABI in include/opb200.h).

There is no CPU fallback: if the library cannot be loaded, or no CUDA device
is present, every kernel call raises.
"""

from __future__ import annotations

import ctypes
import threading

from ._build import LIB_PATH, build_library

MAX_SLOTS = 8
F64, F32, BF16, F16 = 0, 1, 2, 3
F64_PAIRS, F32_PAIRS = 4, 5
F32_QUADS, F64_XPAIRS = 6, 7
F32_OCTS, F64_YXPAIRS = 8, 9
F32_ZETA_H, F64_IN_ZETA, F64_DX_DY, F64_IN_DX = 10, 11, 12, 13
INLINE_TABLE = 720  # OPB_INLINE_TABLE: opb_time entries a host step table may hold
ABI_VERSION = 5
OK, EINVAL, ECUDA = 0, 1, 2
ERRF_ZERO_DIVISION = 1


class opb_field(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p * MAX_SLOTS),
        ("dtype", ctypes.c_int32),
        ("ndim", ctypes.c_int32),
        ("shape", ctypes.c_int64 * 3),
        ("offset", ctypes.c_double * 3),
        ("is_static", ctypes.c_int32),
        ("nslots", ctypes.c_int32),
        ("scale", ctypes.c_void_p * MAX_SLOTS),
    ]


class opb_roms_fields(ctypes.Structure):
    _fields_ = [(name, opb_field) for name in ("u", "v", "w", "dx", "dy", "h", "zeta", "C")]


class opb_time(ctypes.Structure):
    _fields_ = [("prev", ctypes.c_int32), ("next", ctypes.c_int32), ("ft", ctypes.c_double), ("gt", ctypes.c_double)]


PARTICLE_POINTERS = ("zidx", "yidx", "xidx", "z", "_dxidx0", "_dyidx0", "_dz0", "_dxidx1", "_dyidx1", "_dz1",
                     "_dxidx2", "_dyidx2", "_dz2")


class opb_particles(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("status", ctypes.c_void_p)] + [
        (name.lstrip("_"), ctypes.c_void_p) for name in PARTICLE_POINTERS
    ] + [("err", ctypes.c_void_p), ("rho_t", ctypes.c_void_p)]


class opb_records(ctypes.Structure):
    _fields_ = [("mask", ctypes.c_uint64 * 4), ("stride", ctypes.c_int64), ("zidx", ctypes.c_void_p),
                ("yidx", ctypes.c_void_p), ("xidx", ctypes.c_void_p), ("z", ctypes.c_void_p),
                ("status", ctypes.c_void_p)]


class opb_scalars(ctypes.Structure):
    _fields_ = [
        ("hc", ctypes.c_double),
        ("NZ", ctypes.c_int32),
        ("_pad", ctypes.c_int32),
        ("dt", ctypes.c_double),
        ("alpha", ctypes.c_double),
        ("bounds", ctypes.c_double * 6),
        ("w_max", ctypes.c_double),
        ("rho_scale", ctypes.c_double),
    ]


class opb_experiment(ctypes.Structure):
    _fields_ = [("start", ctypes.c_int64), ("count", ctypes.c_int64), ("first_chunk", ctypes.c_int64),
                ("scheme", ctypes.c_int32), ("nsteps", ctypes.c_int32), ("table_offset", ctypes.c_int32),
                ("validate", ctypes.c_int32), ("dt", ctypes.c_double), ("alpha", ctypes.c_double),
                ("bucket_row", ctypes.c_int32), ("_pad", ctypes.c_int32)]


class opb_batch_header(ctypes.Structure):
    _fields_ = [("nexp", ctypes.c_int32), ("nbuckets", ctypes.c_int32), ("nchunks", ctypes.c_int64),
                ("next_chunk", ctypes.c_uint64)]


SCHEME_RK2, SCHEME_AB3 = 1, 2
BATCH_CHUNK = 32
BATCH_SHAPES = ((256, 16), (256, 24), (256, 32), (128, 16))  # (block, warps per SM)

_P = ctypes.POINTER
_VP = ctypes.c_void_p

# name -> argtypes (every entry point returns int)
SIGNATURES = {
    "opb_finite_indices": [_P(opb_particles), _VP],
    "opb_domain_bounds": [_P(opb_particles), _P(opb_scalars), _VP],
    "opb_validation": [_P(opb_particles), _P(opb_scalars), _VP],
    "opb_compute_z": [_P(opb_particles), _VP, _P(opb_scalars), _P(opb_roms_fields), _P(opb_time), _VP],
    "opb_rk2_w_advection_step_1": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _P(opb_time), _VP],
    "opb_rk2_w_advection_step_2": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _P(opb_time), _VP],
    "opb_rk2_w_advection_update": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _P(opb_time), _VP],
    "opb_ab3_w_advection": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _P(opb_time), _VP],
    "opb_ab3_post_w_advection": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _P(opb_time), _VP],
    "opb_ab3_isopycnal_following": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _P(opb_time), _VP],
    "opb_ab3_isopycnal_following_steps": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _VP,
                                          ctypes.c_int32, ctypes.c_int32, _VP],
    "opb_linear_interpolation": [_P(opb_particles), _VP, _P(opb_field), _P(opb_time), _VP, _VP],
    "opb_bilinear_interpolation": [_P(opb_particles), _VP, _VP, _P(opb_field), _P(opb_time), _VP, _VP],
    "opb_trilinear_interpolation": [_P(opb_particles), _P(opb_field), _P(opb_time), _VP, _VP],
    "opb_rk2_w_advection_steps": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _VP, ctypes.c_int32,
                                  ctypes.c_int32, _VP],
    "opb_ab3_w_advection_steps": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _VP, ctypes.c_int32,
                                  ctypes.c_int32, _VP],
    "opb_rk2_w_advection_steps_rec": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _VP, ctypes.c_int32,
                                      ctypes.c_int32, _VP, _VP],
    "opb_ab3_w_advection_steps_rec": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _VP, ctypes.c_int32,
                                      ctypes.c_int32, _VP, _VP],
    "opb_ab3_isopycnal_following_steps_rec": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _VP,
                                              ctypes.c_int32, ctypes.c_int32, _VP, _VP],
    "opb_rk2_w_advection_steps_fp32": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _VP,
                                       ctypes.c_int32, ctypes.c_int32, _VP],
    "opb_ab3_w_advection_steps_fp32": [_P(opb_particles), _P(opb_scalars), _P(opb_roms_fields), _VP,
                                       ctypes.c_int32, ctypes.c_int32, _VP],
    "opb_batched_steps": [_P(opb_particles), _VP, _VP, _P(opb_scalars), _P(opb_roms_fields), _VP, _VP, _VP,
                          ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _VP],
    "opb_interleave_pairs": [_VP, _VP, _VP, ctypes.c_int64, ctypes.c_int32, _VP],
    "opb_interleave_quads": [_VP, _VP, _VP, ctypes.c_int64, _VP],
    "opb_neighbour_pairs": [_VP, _VP, ctypes.c_int64, _VP],
    "opb_interleave_octets": [_VP, _VP, _VP, ctypes.c_int64, ctypes.c_int64, _VP],
    "opb_neighbour_quads": [_VP, _VP, ctypes.c_int64, ctypes.c_int64, _VP],
    "opb_bundle_zeta_h": [_VP, _VP, _VP, _VP, ctypes.c_int64, _VP],
    "opb_bundle_dx_dy": [_VP, _VP, _VP, ctypes.c_int64, _VP],
    "opb_quantize_levels": [_VP, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, _VP, _VP, _VP],
    "opb_check_div12": [_VP, ctypes.c_int64, _VP, _VP],
}

SIGNATURES_OTHER = {
    "opb_sort_particles": ([_P(opb_particles), _P(ctypes.c_int64 * 3), _VP, _VP, ctypes.c_size_t, _VP], ctypes.c_int),
    "opb_sort_particles_ranges": ([_P(opb_particles), _P(ctypes.c_int64 * 3), _VP, _VP, ctypes.c_int32, _VP,
                                   _VP, ctypes.c_size_t, _VP], ctypes.c_int),
    "opb_gather_particles": ([_P(opb_particles), _P(opb_particles), _VP, _VP, _VP, _VP], ctypes.c_int),
    "opb_sort_workspace_bytes": ([ctypes.c_int64], ctypes.c_size_t),
    "opb_sort_particles_noalloc": ([_P(opb_particles), _P(ctypes.c_int64 * 3), _VP, _VP], ctypes.c_int),
    "opb_sort_segments_workspace_bytes": ([ctypes.c_int64, ctypes.c_int32], ctypes.c_size_t),
    "opb_sort_segments": ([_P(opb_particles), _P(ctypes.c_int64 * 3), _VP, _VP, ctypes.c_int32, _VP,
                           ctypes.c_int32, _VP, _VP, ctypes.c_size_t, _VP], ctypes.c_int),
}
NOALLOC_MAX_PARTICLES = 1 << 20

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def load(build: bool = True) -> ctypes.CDLL:
    """Load the CUDA library (building it first if it is missing or stale)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build:
            build_library()
        if not LIB_PATH.exists():
            raise RuntimeError(f"offline_particles_b200: CUDA library not found at {LIB_PATH}; run build()")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, argtypes in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = ctypes.c_int
        for name, (argtypes, restype) in SIGNATURES_OTHER.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = restype
        lib.opb_last_error.argtypes = []
        lib.opb_last_error.restype = ctypes.c_char_p
        lib.opb_abi_version.argtypes = []
        lib.opb_abi_version.restype = ctypes.c_int
        if lib.opb_abi_version() != ABI_VERSION:
            raise RuntimeError("offline_particles_b200: ABI version mismatch")
        _lib = lib
        return lib


def call(name: str, *args) -> None:
    """Call one C-ABI entry point; raise on a non-zero return code."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != OK:
        msg = lib.opb_last_error().decode(errors="replace")
        if rc == EINVAL:
            raise ValueError(msg)
        raise RuntimeError(msg)
