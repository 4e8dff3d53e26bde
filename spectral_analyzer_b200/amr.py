"""AcousticAMR — drop-in for the reference's ``_spectral_kernels.AcousticAMR``.

The reference's AMR pressure stepper (csrc/kernels/acoustic_amr.cpp behind
csrc/include/acoustic_amr.h) is reached from Python through the pybind class
``AcousticAMR`` (csrc/bindings/pybind_kernels.cpp:6506-6603, :8877-8920) used by
acoustic_amr.py ``AcousticAMRFDTD`` (:314-380), and from C++ through the
pressure backend (acoustic_pressure_backend.cpp:388-569).  This class has the
pybind surface (same constructor arguments, methods, properties and
exceptions) over the engine's GPU implementation of the same C ABI
(include/acoustic_amr_b200.h, exported by libacoustic_fdtd_b200.so), plus the
backend's set-up and coupling calls (plate, bridge/neck sources, border,
microphones) so that a caller holding an AMR co-evolver descriptor
(acoustic_amr.py ``build_amr_coevolver_descriptor``) builds the whole backend
with ``from_descriptor``.  There is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native

vp, i32, f32, f64 = C.c_void_p, C.c_int, C.c_float, C.c_double
P = C.c_void_p

# name -> (restype, argtypes): include/acoustic_amr_b200.h (the reference's
# acoustic_amr.h:20-327 plus the engine's amr_b200_* extensions)
AMR_SIGNATURES = {
    "amr_create": (vp, [i32, P, P, P, P, i32, P, P, P, P, P, f64, f64, f64, i32]),
    "amr_get_last_create_error_stage": (C.c_char_p, []),
    "amr_get_last_create_error_message": (C.c_char_p, []),
    "amr_get_create_progress_active": (i32, []),
    "amr_get_create_progress_done_faces": (i32, []),
    "amr_get_create_progress_total_faces": (i32, []),
    "amr_destroy": (None, [vp]),
    "amr_step": (i32, [vp, i32]),
    "amr_reset": (i32, [vp]),
    "amr_inject_pressure_nearest": (i32, [vp, P, f32]),
    "amr_get_pressure": (i32, [vp, P, i32]),
    "amr_get_cell_centers": (i32, [vp, P, i32]),
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
    "amr_b200_last_error": (C.c_char_p, []),
    "amr_b200_launch_count": (C.c_longlong, [vp]),
    "amr_b200_step_async": (i32, [vp, i32]),
    "amr_b200_synchronize": (i32, [vp]),
    "amr_b200_profile": (i32, [vp, i32]),
    "amr_b200_profile_read": (i32, [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
}

SK_OK, SK_ERR_NULL_STATE, SK_ERR_DIM_MISMATCH, SK_ERR_DIVERGED, AMR_ERR_CUDA = 0, -1, -2, -3, -4
BORDER_ANECHOIC, BORDER_ROOM_PANEL, BORDER_TRANSMISSION = 0, 1, 2

_bound = None


def load() -> C.CDLL:
    """The engine library with the AMR entry points bound (raises if not built)."""
    global _bound
    if _bound is None:
        lib = _native.load()
        for name, (res, args) in AMR_SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _bound = lib
    return _bound


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _arr(x, dt):
    return np.ascontiguousarray(x, dtype=dt)


class AcousticAMR:
    """Topology-driven AMR acoustic pressure stepper on a CUDA GPU."""

    def __init__(self, cell_centers, cell_volumes, open_volume_fraction, cell_types, face_cell_neg,
                 face_cell_pos, face_area, face_open_fraction, face_distance, c, rho_air, min_dx,
                 gradient_order):
        import torch
        self._lib = load()
        self._h = None
        cc = _arr(cell_centers, np.float64)
        if cc.ndim != 2 or cc.shape[1] != 3:
            raise RuntimeError("cell_centers must have shape (n_cells, 3)")
        n = int(cc.shape[0])
        cv, ov, ct = _arr(cell_volumes, np.float64), _arr(open_volume_fraction, np.float64), _arr(cell_types, np.uint8)
        if cv.size != n or ov.size != n or ct.size != n:
            raise RuntimeError("cell arrays must have n_cells elements")
        fn = _arr(face_cell_neg, np.int32)
        nf = int(fn.size)
        fp, fa, fo, fd = (_arr(face_cell_pos, np.int32), _arr(face_area, np.float64),
                          _arr(face_open_fraction, np.float64), _arr(face_distance, np.float64))
        if fp.size != nf or fa.size != nf or fo.size != nf or fd.size != nf:
            raise RuntimeError("face arrays must have n_faces elements")
        if not torch.cuda.is_available():
            raise RuntimeError("AcousticAMR needs a CUDA device (no CPU path)")
        torch.cuda.current_device()          # make the CUDA context current
        h = self._lib.amr_create(n, _p(cc), _p(cv), _p(ov), _p(ct), nf, _p(fn), _p(fp), _p(fa), _p(fo), _p(fd),
                                 float(c), float(rho_air), float(min_dx), int(gradient_order))
        if not h:
            raise RuntimeError("amr_create failed: invalid AMR topology or allocation failure")
        self._h = C.c_void_p(h)
        self.n_cells, self.n_faces = n, nf
        self.gradient_order = int(gradient_order)
        self._plate_nodes = 0
        self._n_mics = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.amr_destroy(h)
            self._h = None

    close = __del__

    def _rc(self, rc, what):
        if rc == AMR_ERR_CUDA:
            raise RuntimeError(f"{what}: CUDA error: {(self._lib.amr_b200_last_error() or b'').decode()}")
        if rc != SK_OK:
            raise RuntimeError(f"{what} failed: rc={rc}")
        return rc

    # ---------------------------------------------- the pybind class's surface
    def step(self, n_steps: int = 1) -> int:
        return self._rc(self._lib.amr_step(self._h, int(n_steps)), "amr_step")

    def reset(self):
        self._rc(self._lib.amr_reset(self._h), "amr_reset")

    def inject_pressure_nearest(self, xyz, value):
        x = _arr(xyz, np.float64)
        if x.size != 3:
            raise RuntimeError("xyz must have 3 elements")
        self._rc(self._lib.amr_inject_pressure_nearest(self._h, _p(x), float(value)), "amr_inject_pressure_nearest")

    def get_pressure(self) -> np.ndarray:
        out = np.empty(self.n_cells, np.float32)
        self._rc(self._lib.amr_get_pressure(self._h, _p(out), out.size), "amr_get_pressure")
        return out

    def get_velocity(self) -> np.ndarray:
        out = np.empty(self.n_faces, np.float32)
        self._rc(self._lib.amr_get_velocity(self._h, _p(out), out.size), "amr_get_velocity")
        return out

    @property
    def dt(self) -> float:
        return self._lib.amr_get_dt(self._h)

    @property
    def step_count(self) -> int:
        return self._lib.amr_get_step_count(self._h)

    # ------------------------------------ the pressure backend's other calls
    def step_rc(self, n_steps: int = 1) -> int:
        """amr_step's return code (SK_ERR_DIVERGED = -3 on a diverged step)."""
        return self._lib.amr_step(self._h, int(n_steps))

    def setup_plate(self, plate_Nx, plate_Ny, plate_dx, plate_origin, plate_active, plate_rho_h, plate_D,
                    plate_alpha_M, plate_beta_K, n_active_plate, plate_active_flat_idx, face_above_starts,
                    face_above_idx, face_above_wgt, face_below_starts, face_below_idx, face_below_wgt,
                    cell_above, cell_below) -> int:
        keep = [_arr(plate_origin, np.float32), _arr(plate_active, np.uint8),
                _arr(plate_active_flat_idx, np.int32), _arr(face_above_starts, np.int32),
                _arr(face_above_idx, np.int32), _arr(face_above_wgt, np.float32),
                _arr(face_below_starts, np.int32), _arr(face_below_idx, np.int32),
                _arr(face_below_wgt, np.float32), _arr(cell_above, np.int32), _arr(cell_below, np.int32)]
        rc = self._lib.amr_setup_plate(self._h, int(plate_Nx), int(plate_Ny), float(plate_dx), _p(keep[0]),
                                       _p(keep[1]), float(plate_rho_h), float(plate_D), float(plate_alpha_M),
                                       float(plate_beta_K), int(n_active_plate), *[_p(a) for a in keep[2:]])
        if rc == SK_OK:
            self._plate_nodes = int(plate_Nx) * int(plate_Ny)
        return rc

    def set_bridge_plate_sources(self, idx, wgt) -> int:
        i, w = _arr(idx, np.int32), _arr(wgt, np.float32)
        return self._lib.amr_set_bridge_plate_sources(self._h, i.size, _p(i), _p(w))

    def set_neck_plate_sources(self, idx, wgt) -> int:
        i, w = _arr(idx, np.int32), _arr(wgt, np.float32)
        return self._lib.amr_set_neck_plate_sources(self._h, i.size, _p(i), _p(w))

    def set_border_condition(self, mode, sigma_order, R_reflection, Z_match, n_pml, bounds_min, bounds_max) -> int:
        lo, hi = _arr(bounds_min, np.float64), _arr(bounds_max, np.float64)
        return self._lib.amr_set_border_condition(self._h, int(mode), float(sigma_order), float(R_reflection),
                                                  float(Z_match), int(n_pml), _p(lo), _p(hi))

    def inject_bridge_drive(self, cell_drives, force_scale=1.0) -> int:
        d = _arr(cell_drives, np.float32)
        return self._lib.amr_inject_bridge_drive(self._h, _p(d), d.size, float(force_scale))

    def inject_plate_force(self, plate_idx, wgt, total_force_N) -> int:
        i, w = _arr(plate_idx, np.int32), _arr(wgt, np.float32)
        return self._lib.amr_inject_plate_force(self._h, i.size, _p(i), _p(w), float(total_force_N))

    def sample_plate_displacement_batch(self, idx4, wgt4) -> np.ndarray:
        i, w = _arr(idx4, np.int32), _arr(wgt4, np.float32)
        out = np.empty(i.size // 4, np.float32)
        self._rc(self._lib.amr_sample_plate_displacement_batch(self._h, out.size, _p(i), _p(w), _p(out)),
                 "amr_sample_plate_displacement_batch")
        return out

    def sample_plate_weighted(self, idx, wgt) -> np.float32:
        i, w = _arr(idx, np.int32), _arr(wgt, np.float32)
        out = np.empty(1, np.float32)
        self._rc(self._lib.amr_sample_plate_weighted(self._h, i.size, _p(i), _p(w), _p(out)),
                 "amr_sample_plate_weighted")
        return out[0]

    def get_plate_displacement(self) -> np.ndarray:
        out = np.empty(self._plate_nodes, np.float32)
        self._rc(self._lib.amr_get_plate_displacement(self._h, _p(out), out.size), "amr_get_plate_displacement")
        return out

    def setup_mic_samplers(self, pos_xyz, axis_xyz, need_velocity=True) -> int:
        p, a = _arr(pos_xyz, np.float32), _arr(axis_xyz, np.float32)
        rc = self._lib.amr_setup_mic_samplers(self._h, p.size // 3, _p(p), _p(a), 1 if need_velocity else 0)
        if rc == SK_OK:
            self._n_mics = p.size // 3
        return rc

    def sample_mics(self):
        """(p, vx, vy, vz) at every microphone."""
        outs = [np.empty(self._n_mics, np.float32) for _ in range(4)]
        self._rc(self._lib.amr_sample_mics(self._h, self._n_mics, *[_p(o) for o in outs]), "amr_sample_mics")
        return tuple(outs)

    def scatter_pressure_uniform(self, Nx, Ny, Nz, bounds_min, bounds_max) -> np.ndarray:
        lo, hi = _arr(bounds_min, np.float64), _arr(bounds_max, np.float64)
        out = np.empty(int(Nx) * int(Ny) * int(Nz), np.float32)
        self._rc(self._lib.amr_scatter_pressure_uniform(self._h, int(Nx), int(Ny), int(Nz), _p(lo), _p(hi), _p(out)),
                 "amr_scatter_pressure_uniform")
        return out.reshape(int(Nx), int(Ny), int(Nz))

    # ------------------------------------------------------ engine extensions
    def step_async(self, n_steps: int = 1) -> int:
        return self._rc(self._lib.amr_b200_step_async(self._h, int(n_steps)), "amr_b200_step_async")

    def synchronize(self) -> int:
        """SK_OK, or SK_ERR_DIVERGED if a queued step diverged."""
        return self._lib.amr_b200_synchronize(self._h)

    @property
    def launch_count(self) -> int:
        return self._lib.amr_b200_launch_count(self._h)

    def profile(self, enable: bool = True):
        self._lib.amr_b200_profile(self._h, 1 if enable else 0)

    def profile_read(self):
        ms, n = C.c_double(), C.c_longlong()
        self._lib.amr_b200_profile_read(self._h, C.byref(ms), C.byref(n))
        return ms.value, n.value

    @classmethod
    def from_descriptor(cls, desc: dict, gradient_order=None, border=None) -> "AcousticAMR":
        """The whole backend from an AMR co-evolver descriptor, in the reference
        pressure backend's order (acoustic_pressure_backend.cpp:461-548): create,
        plate, bridge sources, neck sources, border.  ``border`` = (mode,
        sigma_order, R_reflection, Z_match) overrides the descriptor's."""
        d = desc
        go = int(d.get("gradient_order", 2) if gradient_order is None else gradient_order)
        s = cls(d["cell_centers"], d["cell_volumes"], d["open_volume_frac"], d["cell_types"], d["face_cell_neg"],
                d["face_cell_pos"], d["face_area"], d["face_open_frac"], d["face_distance"], d["c"], d["rho_air"],
                d["min_dx"], go)
        if s.setup_plate(d["plate_Nx"], d["plate_Ny"], d["plate_dx"], d["plate_origin"], d["plate_active"],
                         d["plate_mass_density"], d["plate_stiffness_D"], d["plate_alpha_M"], d["plate_beta_K"],
                         d["n_active_plate"], d["plate_active_flat_idx"], d["plate_face_above_starts"],
                         d["plate_face_above_idx"], d["plate_face_above_wgt"], d["plate_face_below_starts"],
                         d["plate_face_below_idx"], d["plate_face_below_wgt"], d["plate_cell_above"],
                         d["plate_cell_below"]) != SK_OK:
            raise RuntimeError("amr_setup_plate failed")
        if s.set_bridge_plate_sources(d["bridge_plate_idx"], d["bridge_plate_wgt"]) != SK_OK:
            raise RuntimeError("amr_set_bridge_plate_sources failed")
        if int(d.get("n_neck_plate", 0)) > 0:
            if s.set_neck_plate_sources(d["neck_plate_idx"], d["neck_plate_wgt"]) != SK_OK:
                raise RuntimeError("amr_set_neck_plate_sources failed")
        if int(d.get("n_pml", 0)) > 0:
            mode, sig, R, Z = border if border is not None else (
                d.get("border_mode", 0), d.get("border_sigma_order", 3.0), d.get("border_R_reflection", 0.0),
                d.get("border_Z_match", 0.0))
            if s.set_border_condition(mode, sig if sig > 0 else 3.0, R, Z, d["n_pml"], d["bounds_min"],
                                      d["bounds_max"]) != SK_OK:
                raise RuntimeError("amr_set_border_condition failed")
        return s
