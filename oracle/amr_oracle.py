"""ctypes binding of the compiled reference AMR stepper (oracle/_ref/libamr_ref.so).

TEST INFRASTRUCTURE ONLY: the checker for the engine's AMR backend.  The
library is the reference's csrc/kernels/acoustic_amr.cpp compiled unchanged by
oracle/Makefile; ``AMRRef`` wraps its C ABI (csrc/include/acoustic_amr.h) with
NumPy arrays and is set up in the call order of the reference's AMR pressure
backend (csrc/kernels/acoustic_pressure_backend.cpp:461-548: amr_create,
amr_setup_plate, bridge and neck sources, amr_set_border_condition).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
AMR_REF_LIB = os.path.join(HERE, "_ref", "libamr_ref.so")

vp, i32, f32, f64 = C.c_void_p, C.c_int, C.c_float, C.c_double
P = C.c_void_p

# name -> (restype, argtypes), csrc/include/acoustic_amr.h:20-327
SIGNATURES = {
    "amr_create": (vp, [i32, P, P, P, P, i32, P, P, P, P, P, f64, f64, f64, i32]),
    "amr_get_last_create_error_message": (C.c_char_p, []),
    "amr_destroy": (None, [vp]),
    "amr_step": (i32, [vp, i32]),
    "amr_reset": (i32, [vp]),
    "amr_inject_pressure_nearest": (i32, [vp, P, f32]),
    "amr_get_pressure": (i32, [vp, P, i32]),
    "amr_get_velocity": (i32, [vp, P, i32]),
    "amr_get_dt": (f64, [vp]),
    "amr_get_step_count": (i32, [vp]),
    "amr_scatter_pressure_uniform": (i32, [vp, i32, i32, i32, P, P, P]),
    "amr_set_border_condition": (i32, [vp, i32, f32, f32, f32, i32, P, P]),
    "amr_setup_plate": (i32, [vp, i32, i32, f32, P, P, f32, f32, f32, f32, i32, P, P, P, P, P, P, P, P, P]),
    "amr_set_bridge_plate_sources": (i32, [vp, i32, P, P]),
    "amr_set_neck_plate_sources": (i32, [vp, i32, P, P]),
    "amr_inject_bridge_drive": (i32, [vp, P, i32, f32]),
    "amr_inject_plate_force": (i32, [vp, i32, P, P, f32]),
    "amr_sample_plate_displacement_batch": (i32, [vp, i32, P, P, P]),
    "amr_sample_plate_weighted": (i32, [vp, i32, P, P, P]),
    "amr_get_plate_displacement": (i32, [vp, P, i32]),
    "amr_setup_mic_samplers": (i32, [vp, i32, P, P, i32]),
    "amr_sample_mics": (i32, [vp, i32, P, P, P, P]),
}


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


_lib = None


def load_reference() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(AMR_REF_LIB):
            raise RuntimeError(f"compiled reference AMR missing: {AMR_REF_LIB} "
                               "(build it with `make -C oracle REF=<reference checkout>`)")
        lib = C.CDLL(AMR_REF_LIB)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class AMRRef:
    """One reference AMR state built from an AMR co-evolver descriptor.

    Method names follow the engine's ``spectral_analyzer_b200.amr.AcousticAMR``
    so one driving script runs on both."""

    def __init__(self, desc: dict, gradient_order: int = 2, border=None):
        lib = self._lib = load_reference()
        d = self._d = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in desc.items()}
        self.n_cells, self.n_faces = int(d["n_cells"]), int(d["n_faces"])
        h = lib.amr_create(self.n_cells, _p(d["cell_centers"]), _p(d["cell_volumes"]), _p(d["open_volume_frac"]),
                           _p(d["cell_types"]), self.n_faces, _p(d["face_cell_neg"]), _p(d["face_cell_pos"]),
                           _p(d["face_area"]), _p(d["face_open_frac"]), _p(d["face_distance"]), float(d["c"]),
                           float(d["rho_air"]), float(d["min_dx"]), int(gradient_order))
        if not h:
            raise RuntimeError("amr_create failed: " + (lib.amr_get_last_create_error_message() or b"").decode())
        self._h = C.c_void_p(h)
        if "plate_Nx" not in d:           # a grid without a plate (no sources either)
            self._plate_nodes = 0
            if int(d.get("n_pml", 0)) > 0 and border is not None:
                mode, sig, R, Z = border
                rc = lib.amr_set_border_condition(self._h, int(mode), float(sig), float(R), float(Z),
                                                  int(d["n_pml"]), _p(d["bounds_min"]), _p(d["bounds_max"]))
                assert rc == 0, rc
            return
        self._plate_nodes = int(d["plate_Nx"]) * int(d["plate_Ny"])
        rc = lib.amr_setup_plate(
            self._h, int(d["plate_Nx"]), int(d["plate_Ny"]), float(d["plate_dx"]), _p(d["plate_origin"]),
            _p(d["plate_active"]), float(d["plate_mass_density"]), float(d["plate_stiffness_D"]),
            float(d["plate_alpha_M"]), float(d["plate_beta_K"]), int(d["n_active_plate"]),
            _p(d["plate_active_flat_idx"]), _p(d["plate_face_above_starts"]), _p(d["plate_face_above_idx"]),
            _p(d["plate_face_above_wgt"]), _p(d["plate_face_below_starts"]), _p(d["plate_face_below_idx"]),
            _p(d["plate_face_below_wgt"]), _p(d["plate_cell_above"]), _p(d["plate_cell_below"]))
        assert rc == 0, rc
        rc = lib.amr_set_bridge_plate_sources(self._h, int(d["n_bridge_plate"]), _p(d["bridge_plate_idx"]),
                                              _p(d["bridge_plate_wgt"]))
        assert rc == 0, rc
        if int(d.get("n_neck_plate", 0)) > 0:
            rc = lib.amr_set_neck_plate_sources(self._h, int(d["n_neck_plate"]), _p(d["neck_plate_idx"]),
                                                _p(d["neck_plate_wgt"]))
            assert rc == 0, rc
        if int(d.get("n_pml", 0)) > 0 and border is not None:
            mode, sig, R, Z = border
            rc = lib.amr_set_border_condition(self._h, int(mode), float(sig), float(R), float(Z), int(d["n_pml"]),
                                              _p(d["bounds_min"]), _p(d["bounds_max"]))
            assert rc == 0, rc

    def close(self):
        if getattr(self, "_h", None):
            self._lib.amr_destroy(self._h)
            self._h = None

    __del__ = close

    def setup_mic_samplers(self, pos, axis, need_velocity=True) -> int:
        self._mp = np.ascontiguousarray(pos, np.float32).ravel()
        self._ma = np.ascontiguousarray(axis, np.float32).ravel()
        self._n_mics = self._mp.size // 3
        return self._lib.amr_setup_mic_samplers(self._h, self._n_mics, _p(self._mp), _p(self._ma),
                                                1 if need_velocity else 0)

    def step_rc(self, n: int = 1) -> int:
        return self._lib.amr_step(self._h, int(n))

    def reset(self) -> int:
        return self._lib.amr_reset(self._h)

    def inject_pressure_nearest(self, xyz, value):
        x = np.ascontiguousarray(xyz, np.float64).ravel()
        assert self._lib.amr_inject_pressure_nearest(self._h, _p(x), float(value)) == 0

    def inject_bridge_drive(self, drives, scale=1.0) -> int:
        a = np.ascontiguousarray(drives, np.float32)
        return self._lib.amr_inject_bridge_drive(self._h, _p(a), a.size, float(scale))

    def inject_plate_force(self, idx, wgt, total) -> int:
        i = np.ascontiguousarray(idx, np.int32)
        w = np.ascontiguousarray(wgt, np.float32)
        return self._lib.amr_inject_plate_force(self._h, i.size, _p(i), _p(w), float(total))

    @property
    def dt(self) -> float:
        return self._lib.amr_get_dt(self._h)

    @property
    def step_count(self) -> int:
        return self._lib.amr_get_step_count(self._h)

    def get_pressure(self):
        out = np.empty(self.n_cells, np.float32)
        assert self._lib.amr_get_pressure(self._h, _p(out), out.size) == 0
        return out

    def get_velocity(self):
        out = np.empty(self.n_faces, np.float32)
        assert self._lib.amr_get_velocity(self._h, _p(out), out.size) == 0
        return out

    def get_plate_displacement(self):
        out = np.empty(self._plate_nodes, np.float32)
        assert self._lib.amr_get_plate_displacement(self._h, _p(out), out.size) == 0
        return out

    def sample_plate_displacement_batch(self, idx4, wgt4):
        i = np.ascontiguousarray(idx4, np.int32)
        w = np.ascontiguousarray(wgt4, np.float32)
        out = np.empty(i.size // 4, np.float32)
        assert self._lib.amr_sample_plate_displacement_batch(self._h, out.size, _p(i), _p(w), _p(out)) == 0
        return out

    def sample_plate_weighted(self, idx, wgt):
        i = np.ascontiguousarray(idx, np.int32)
        w = np.ascontiguousarray(wgt, np.float32)
        out = np.empty(1, np.float32)
        assert self._lib.amr_sample_plate_weighted(self._h, i.size, _p(i), _p(w), _p(out)) == 0
        return out[0]

    def sample_mics(self):
        outs = [np.empty(self._n_mics, np.float32) for _ in range(4)]
        assert self._lib.amr_sample_mics(self._h, self._n_mics, *[_p(o) for o in outs]) == 0
        return tuple(outs)

    def scatter_pressure_uniform(self, nx, ny, nz, bmin, bmax):
        lo = np.ascontiguousarray(bmin, np.float64)
        hi = np.ascontiguousarray(bmax, np.float64)
        out = np.empty(nx * ny * nz, np.float32)
        assert self._lib.amr_scatter_pressure_uniform(self._h, nx, ny, nz, _p(lo), _p(hi), _p(out)) == 0
        return out.reshape(nx, ny, nz)
