"""ctypes binding of libacoustic_fdtd_b200.so (the C ABI in include/acoustic_fdtd_b200.h).

There is no fallback: if the library is missing the import fails loudly, and
the engine never routes a computation anywhere but the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB_PATH

FDTD_OK, FDTD_ERR_NULL, FDTD_ERR_DIM, FDTD_ERR_UNSTABLE, FDTD_ERR_CUDA, FDTD_ERR_ARG = 0, -1, -2, -3, -4, -5

vp = C.c_void_p
i32 = C.c_int
f32 = C.c_float
P_i32 = C.POINTER(C.c_int)
P_f32 = C.POINTER(C.c_float)
P_f64 = C.POINTER(C.c_double)
P_u8 = C.POINTER(C.c_uint8)

# name -> (restype, argtypes); the 26 reference entry points first, then extensions
SIGNATURES = {
    "fdtd_create": (vp, [i32, i32, i32, f32, f32, f32, P_u8, i32, P_u8, f32, f32, f32, f32, i32]),
    "fdtd_destroy": (None, [vp]),
    "fdtd_set_bridge_sources": (i32, [vp, i32, P_i32, P_f32]),
    "fdtd_inject_bridge": (i32, [vp, f32, f32, f32]),
    "fdtd_inject_bridge_drive": (i32, [vp, P_f32, f32]),
    "fdtd_inject_plate_force": (i32, [vp, i32, P_i32, P_f32, f32]),
    "fdtd_set_face_fractions": (i32, [vp, P_f32, P_f32, P_f32]),
    "fdtd_sample_plate_weighted": (i32, [vp, i32, P_i32, P_f32, P_f32]),
    "fdtd_precompute_pressure_samplers": (i32, [vp, i32, P_f32, P_i32, P_f32]),
    "fdtd_precompute_velocity_samplers": (i32, [vp, i32, P_f32, P_i32, P_f32, P_i32, P_f32, P_i32, P_f32]),
    "fdtd_sample_pressure_precomputed": (i32, [vp, i32, P_i32, P_f32, P_f32]),
    "fdtd_sample_velocity_precomputed": (i32, [vp, i32, P_i32, P_f32, P_i32, P_f32, P_i32, P_f32,
                                               P_f32, P_f32, P_f32]),
    "fdtd_step": (i32, [vp, i32]),
    "fdtd_get_step_count": (i32, [vp]),
    "fdtd_get_dt": (f32, [vp]),
    "fdtd_reset": (i32, [vp]),
    "fdtd_get_pressure_field": (i32, [vp, P_f32, i32]),
    "fdtd_b200_get_volume_slice": (i32, [vp, i32, i32, P_f32, i32]),
    "fdtd_get_plate_displacement": (i32, [vp, P_f32, i32]),
    "fdtd_sample_plate_displacement_batch": (i32, [vp, i32, P_i32, P_f32, P_f32]),
    "fdtd_sample_pressure": (i32, [vp, i32, P_f32, P_f32]),
    "fdtd_get_velocity_dims": (None, [vp, P_i32, P_i32, P_i32]),
    "fdtd_get_velocity_x": (i32, [vp, P_f32, i32]),
    "fdtd_get_velocity_y": (i32, [vp, P_f32, i32]),
    "fdtd_get_velocity_z": (i32, [vp, P_f32, i32]),
    "fdtd_sample_velocity": (i32, [vp, i32, P_f32, P_f32, P_f32, P_f32]),
    "fdtd_get_surface_emission": (i32, [vp, i32, P_f32, P_f32, P_f32, P_f32]),
    # extensions
    "fdtd_b200_field_layout": (i32, [i32, i32, i32, P_i32, C.POINTER(C.c_size_t)]),
    "fdtd_b200_create_ex": (vp, [i32, i32, i32, f32, f32, f32, P_u8, i32, P_u8, f32, f32, f32, f32,
                                 i32, i32, C.POINTER(vp)]),
    "fdtd_b200_set_face_absorption": (i32, [vp, P_f32]),
    "fdtd_b200_add_pressure": (i32, [vp, i32, f32]),
    "fdtd_b200_set_point_source": (i32, [vp, i32, P_f32, i32]),
    "fdtd_b200_set_receivers": (i32, [vp, i32, P_i32, P_f32, i32]),
    "fdtd_b200_get_traces": (i32, [vp, P_f32, i32, P_i32]),
    "fdtd_b200_set_stream": (i32, [vp, vp]),
    "fdtd_b200_get_stream": (vp, [vp]),
    "fdtd_b200_step_async": (i32, [vp, i32]),
    "fdtd_b200_synchronize": (i32, [vp]),
    "fdtd_b200_set_kernel": (i32, [vp, i32]),
    "fdtd_b200_debug_hold_load": (i32, [vp, i32, i32]),
    "fdtd_b200_get_kernel": (i32, [vp]),
    "fdtd_b200_device_fields": (i32, [vp, C.POINTER(vp)]),
    "fdtd_b200_profile": (i32, [vp, i32]),
    "fdtd_b200_profile_read": (i32, [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                      C.POINTER(C.c_longlong)]),
    "fdtd_b200_sample_pressure_noalloc": (i32, [vp, i32, P_i32, P_f32, P_f32]),
    "fdtd_b200_batch_create": (vp, [i32]),
    "fdtd_b200_batch_destroy": (None, [vp]),
    "fdtd_b200_batch_set": (i32, [vp, C.POINTER(vp), P_i32, i32]),
    "fdtd_b200_batch_set_tile": (i32, [vp, i32]),
    "fdtd_b200_batch_set_segment": (i32, [vp, i32]),
    "fdtd_b200_batch_step": (i32, [vp, i32, i32]),
    "fdtd_b200_batch_sync": (i32, [vp, P_i32, P_i32]),
    "fdtd_b200_batch_launch_count": (C.c_longlong, [vp]),
    "fdtd_b200_prec_create": (vp, [i32, i32, i32, C.c_double, C.c_double, C.c_double, i32, P_f32,
                                   i32, f32, f32, i32]),
    "fdtd_b200_prec_destroy": (None, [vp]),
    "fdtd_b200_prec_dt": (C.c_double, [vp]),
    "fdtd_b200_prec_set_source": (i32, [vp, i32, P_f64, i32]),
    "fdtd_b200_prec_set_receivers": (i32, [vp, i32, P_i32, P_f64, i32, i32]),
    "fdtd_b200_prec_step": (i32, [vp, i32, i32]),
    "fdtd_b200_prec_get_traces": (i32, [vp, P_f64, i32, P_i32]),
    "fdtd_b200_prec_get_energy": (i32, [vp, P_f64, i32, P_i32]),
    "fdtd_b200_prec_get_pressure": (i32, [vp, P_f64, i32]),
    "fdtd_b200_prec_set_kernel": (i32, [vp, i32]),
    "fdtd_b200_prec_get_kernel": (i32, [vp]),
    "fdtd_b200_prec_launch_count": (C.c_longlong, [vp]),
    "fdtd_b200_prec_stream": (vp, [vp]),
    "fdtd_b200_adj_create": (vp, [i32, i32, i32, C.c_double, C.c_double, C.c_double, i32, i32, i32]),
    "fdtd_b200_adj_destroy": (None, [vp]),
    "fdtd_b200_adj_dt": (C.c_double, [vp]),
    "fdtd_b200_adj_launch_count": (C.c_longlong, [vp]),
    "fdtd_b200_adj_set_absorption": (i32, [vp, vp, i32, i32]),
    "fdtd_b200_adj_set_source": (i32, [vp, i32, P_f64, i32]),
    "fdtd_b200_adj_set_receivers": (i32, [vp, i32, P_i32, P_f64, i32]),
    "fdtd_b200_adj_forward": (i32, [vp, i32, i32, P_f64]),
    "fdtd_b200_adj_backward": (i32, [vp, P_f64, vp]),
    "fdtd_b200_slab_layout": (i32, [i32, i32, i32, i32, i32, P_i32, P_i32]),
    "fdtd_b200_slab_create": (vp, [i32, i32, i32, i32, i32, f32, f32, f32, i32, P_f32, C.POINTER(vp), i32]),
    "fdtd_b200_slab_destroy": (None, [vp]),
    "fdtd_b200_slab_set_stream": (i32, [vp, vp]),
    "fdtd_b200_slab_dt": (f32, [vp]),
    "fdtd_b200_slab_current": (i32, [vp]),
    "fdtd_b200_slab_vset": (i32, [vp]),
    "fdtd_b200_slab_step": (i32, [vp]),
    "fdtd_b200_slab_step_part": (i32, [vp, i32]),
    "fdtd_b200_slab_set_peer": (i32, [vp, i32, C.POINTER(vp), i32, i32]),
    "fdtd_b200_slab_launch_count": (C.c_longlong, [vp]),
    "fdtd_b200_slab_set_source": (i32, [vp, i32, P_f32, i32]),
    "fdtd_b200_slab_set_receivers": (i32, [vp, i32, P_i32, P_f32, i32]),
    "fdtd_b200_slab_deposit": (i32, [vp, i32]),
    "fdtd_b200_slab_add_pressure": (i32, [vp, i32, f32]),
    "fdtd_b200_slab_read_last": (i32, [vp, P_f32, i32]),
    "fdtd_b200_slab_velocity": (i32, [vp]),
    "fdtd_b200_slab_pressure": (i32, [vp]),
    "fdtd_b200_slab_record": (i32, [vp]),
    "fdtd_b200_slab_check": (i32, [vp, i32, C.POINTER(C.c_longlong)]),
    "fdtd_b200_slab_get_traces": (i32, [vp, P_f32, i32, P_i32]),
    "fdtd_b200_substep": (i32, [vp, P_f32, f32, i32, P_i32, P_f32, f32, i32, P_i32, P_f32, P_f32]),
    "fdtd_b200_get_progress": (i32, [vp, P_i32, P_i32, P_i32]),
    "fdtd_b200_set_progress": (i32, [vp, i32, i32, i32]),
    "fdtd_b200_launch_count": (C.c_longlong, [vp]),
    "fdtd_b200_last_error": (C.c_char_p, []),
}

REFERENCE_ENTRY_POINTS = [n for n in SIGNATURES if not n.startswith("fdtd_b200_")]

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load (once) and bind the engine library; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"CUDA engine library not found: {path}. Build it with "
            "`python -m spectral_analyzer_b200.build` (nvcc, sm_100a).")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    msg = load().fdtd_b200_last_error()
    return msg.decode() if msg else ""
