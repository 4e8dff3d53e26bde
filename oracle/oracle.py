"""oracle.py — TEST INFRASTRUCTURE ONLY: ctypes front-end for the two CPU checkers.

* ``OracleFDTD`` — the C restatement in ``oracle/fdtd_oracle_body.h`` (float, or
  double with ``precision="f64"``), built into ``oracle/liboracle_fdtd.so``.
* ``RefFDTD`` — the reference's own ``csrc/kernels/acoustic_fdtd.cpp`` compiled
  unchanged into ``oracle/_ref/libfdtd_ref.so`` (plus the three hooks of
  ``oracle/ref_shim.cpp``).  Present only where the reference tree was
  available when ``oracle/Makefile`` ran.

Both expose the method surface of the reference's ``_spectral_kernels.AcousticFDTD``
(csrc/bindings/pybind_kernels.cpp:8924-9022) plus ``add_pressure`` (the
deposit rule, acoustic_fdtd.cpp:840-872), ``set_face_absorption`` and ``run``.
Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may use
this module.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle_fdtd.so")
REF_LIB = os.path.join(HERE, "_ref", "libfdtd_ref.so")
REF_LIB_V3 = os.path.join(HERE, "_ref", "libfdtd_ref_v3.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

_lib_cache: dict = {}


def _host_has_avx2_fma() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            txt = f.read()
    except OSError:
        return False
    flags = set()
    for line in txt.splitlines():
        if line.startswith("flags"):
            flags.update(line.split(":", 1)[1].split())
            break
    return {"avx2", "fma", "bmi2"} <= flags


def reference_available() -> bool:
    return os.path.exists(REF_LIB)


def oracle_available() -> bool:
    return os.path.exists(ORACLE_LIB)


def _bind_common(lib, pfx: str, real, realp):
    """Declare the shared entry points of a library with prefix ``pfx``."""
    vp = C.c_void_p
    sig = {
        "create": (vp, [C.c_int, C.c_int, C.c_int, real, real, real, _u8p, C.c_int, _u8p,
                        real, real, real, real, C.c_int]),
        "destroy": (None, [vp]),
        "step": (C.c_int, [vp, C.c_int]),
        "reset": (C.c_int, [vp]),
        "get_step_count": (C.c_int, [vp]),
        "get_dt": (real, [vp]),
        "get_pressure_field": (C.c_int, [vp, realp, C.c_int]),
        "get_velocity_x": (C.c_int, [vp, realp, C.c_int]),
        "get_velocity_y": (C.c_int, [vp, realp, C.c_int]),
        "get_velocity_z": (C.c_int, [vp, realp, C.c_int]),
        "get_plate_displacement": (C.c_int, [vp, realp, C.c_int]),
        "set_face_fractions": (C.c_int, [vp, vp, vp, vp]),
        "set_bridge_sources": (C.c_int, [vp, C.c_int, _i32p, realp]),
        "inject_bridge_drive": (C.c_int, [vp, realp, real]),
        "inject_plate_force": (C.c_int, [vp, C.c_int, _i32p, realp, real]),
        "sample_pressure": (C.c_int, [vp, C.c_int, realp, realp]),
        "sample_velocity": (C.c_int, [vp, C.c_int, realp, realp, realp, realp]),
        "precompute_pressure_samplers": (C.c_int, [vp, C.c_int, realp, _i32p, realp]),
        "precompute_velocity_samplers": (C.c_int, [vp, C.c_int, realp, _i32p, realp, _i32p, realp,
                                                   _i32p, realp]),
        "sample_pressure_precomputed": (C.c_int, [vp, C.c_int, _i32p, realp, realp]),
        "sample_velocity_precomputed": (C.c_int, [vp, C.c_int, _i32p, realp, _i32p, realp, _i32p,
                                                  realp, realp, realp, realp]),
        "get_surface_emission": (C.c_int, [vp, C.c_int, realp, realp, realp, realp]),
        "sample_plate_displacement_batch": (C.c_int, [vp, C.c_int, _i32p, realp, realp]),
        "sample_plate_weighted": (C.c_int, [vp, C.c_int, _i32p, realp, realp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, pfx + name)
        fn.restype = res
        fn.argtypes = args


def _load_oracle():
    if "oracle" not in _lib_cache:
        if not oracle_available():
            raise RuntimeError(f"oracle library missing: {ORACLE_LIB} (run `make -C oracle`)")
        lib = C.CDLL(ORACLE_LIB)
        for pfx, real, realp in (("orc_", C.c_float, _f32p), ("orc64_", C.c_double, _f64p)):
            _bind_common(lib, pfx, real, realp)
            for name, res, args in (
                ("set_face_absorption", C.c_int, [C.c_void_p, realp]),
                ("set_cell_absorption", C.c_int, [C.c_void_p, realp]),
                ("add_pressure", C.c_int, [C.c_void_p, C.c_int, real]),
                ("get_p_damp", C.c_int, [C.c_void_p, realp, C.c_int]),
                ("set_pressure_field", None, [C.c_void_p, realp]),
                ("run", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                  C.c_void_p, C.c_void_p, C.c_void_p]),
            ):
                fn = getattr(lib, pfx + name)
                fn.restype = res
                fn.argtypes = args
        _lib_cache["oracle"] = lib
    return _lib_cache["oracle"]


def _load_ref(fast: bool = False):
    key = "ref_v3" if fast else "ref"
    if key not in _lib_cache:
        path = REF_LIB_V3 if (fast and os.path.exists(REF_LIB_V3) and _host_has_avx2_fma()) else REF_LIB
        if not os.path.exists(path):
            raise RuntimeError(f"compiled reference missing: {path} (build it with `make -C oracle REF=<reference checkout>`)")
        lib = C.CDLL(path)
        # the reference's own names: fdtd_<name>
        _bind_common(lib, "fdtd_", C.c_float, _f32p)
        lib.fdtd_get_velocity_dims.restype = None
        lib.fdtd_get_velocity_dims.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                               C.POINTER(C.c_int)]
        lib.fdtd_inject_bridge.restype = C.c_int
        lib.fdtd_inject_bridge.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float]
        lib.fdtd_ref_add_pressure.restype = C.c_int
        lib.fdtd_ref_add_pressure.argtypes = [C.c_void_p, C.c_int, C.c_float]
        lib.fdtd_ref_set_face_absorption.restype = C.c_int
        lib.fdtd_ref_set_face_absorption.argtypes = [C.c_void_p, C.c_int, _f32p]
        lib.fdtd_ref_get_p_damp.restype = C.c_int
        lib.fdtd_ref_get_p_damp.argtypes = [C.c_void_p, _f32p, C.c_int]
        lib.fdtd_ref_pool_threads.restype = C.c_int
        lib.fdtd_ref_pool_threads.argtypes = []
        lib._path = path
        _lib_cache[key] = lib
    return _lib_cache[key]


class _CpuFDTD:
    """Common method surface; subclasses choose library, prefix and dtype."""

    _pfx = ""
    dtype = np.float32

    def _fn(self, name):
        return getattr(self._lib, self._pfx + name)

    def _init(self, Nx, Ny, Nz, dx, c, rho_air, cell_type, plate_iz, plate_active,
              plate_mass_density, plate_stiffness_D, plate_alpha_M, plate_beta_K, n_pml):
        ct = np.ascontiguousarray(cell_type, dtype=np.uint8).ravel()
        pa = np.ascontiguousarray(plate_active, dtype=np.uint8).ravel()
        if ct.size != Nx * Ny * Nz:
            raise RuntimeError("cell_type: expected Nx*Ny*Nz elements")
        if pa.size != Nx * Ny:
            raise RuntimeError("plate_active: expected Nx*Ny elements")
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.n_pml = int(n_pml)
        h = self._fn("create")(Nx, Ny, Nz, dx, c, rho_air, ct, plate_iz, pa, plate_mass_density,
                              plate_stiffness_D, plate_alpha_M, plate_beta_K, n_pml)
        if not h:
            raise RuntimeError("fdtd_create: allocation failed")
        self._h = C.c_void_p(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._fn("destroy")(h)
            self._h = None

    def _arr(self, x, n=None):
        a = np.ascontiguousarray(x, dtype=self.dtype).ravel()
        if n is not None and a.size != n:
            raise ValueError(f"expected {n} elements, got {a.size}")
        return a

    @property
    def dims(self):
        Nx, Ny, Nz = self.Nx, self.Ny, self.Nz
        return (Nx - 1) * Ny * Nz, Nx * (Ny - 1) * Nz, Nx * Ny * (Nz - 1)

    # stepping
    def step(self, n_steps: int = 1) -> int:
        rc = self._fn("step")(self._h, int(n_steps))
        if rc == -3:
            raise RuntimeError("AcousticFDTD: pressure diverged (FDTD_ERR_UNSTABLE)")
        return rc

    def step_rc(self, n_steps: int = 1) -> int:
        return self._fn("step")(self._h, int(n_steps))

    def reset(self):
        self._fn("reset")(self._h)

    @property
    def dt(self):
        return self._fn("get_dt")(self._h)

    @property
    def step_count(self):
        return self._fn("get_step_count")(self._h)

    # fields
    def get_pressure_field(self):
        out = np.empty(self.Nx * self.Ny * self.Nz, dtype=self.dtype)
        rc = self._fn("get_pressure_field")(self._h, out, out.size)
        assert rc == 0, rc
        return out.reshape(self.Nx, self.Ny, self.Nz)

    def _vel(self, comp, n):
        out = np.empty(n, dtype=self.dtype)
        rc = self._fn("get_velocity_" + comp)(self._h, out, n)
        assert rc == 0, rc
        return out

    def get_velocity_dims(self):
        return self.dims

    def get_velocity_x(self):
        return self._vel("x", self.dims[0])

    def get_velocity_y(self):
        return self._vel("y", self.dims[1])

    def get_velocity_z(self):
        return self._vel("z", self.dims[2])

    def get_plate_displacement(self):
        out = np.empty(self.Nx * self.Ny, dtype=self.dtype)
        rc = self._fn("get_plate_displacement")(self._h, out, out.size)
        assert rc == 0, rc
        return out.reshape(self.Nx, self.Ny)

    # configuration
    def set_face_fractions(self, vx_frac, vy_frac, vz_frac):
        nvx, nvy, nvz = self.dims
        a = self._arr(vx_frac, nvx) if vx_frac is not None else None
        b = self._arr(vy_frac, nvy) if vy_frac is not None else None
        c = self._arr(vz_frac, nvz) if vz_frac is not None else None
        self._keep = (a, b, c)
        ptr = lambda x: x.ctypes.data_as(C.c_void_p) if x is not None else None
        rc = self._fn("set_face_fractions")(self._h, ptr(a), ptr(b), ptr(c))
        assert rc == 0, rc

    def set_bridge_sources(self, cell_indices, weights):
        idx = np.ascontiguousarray(cell_indices, dtype=np.int32).ravel()
        w = self._arr(weights)
        if idx.size != w.size:
            raise RuntimeError("cell_indices and weights must have the same length")
        rc = self._fn("set_bridge_sources")(self._h, idx.size, idx, w)
        if rc != 0:
            raise RuntimeError(f"fdtd_set_bridge_sources error: {rc}")

    def inject_bridge_drive(self, cell_drives, force_scale=1.0):
        return self._fn("inject_bridge_drive")(self._h, self._arr(cell_drives), force_scale)

    def inject_plate_force(self, plate_indices, weights, total_force_N):
        idx = np.ascontiguousarray(plate_indices, dtype=np.int32).ravel()
        return self._fn("inject_plate_force")(self._h, idx.size, idx, self._arr(weights, idx.size),
                                              total_force_N)

    # sampling
    def sample_pressure(self, rec_xyz):
        x = self._arr(rec_xyz)
        n = x.size // 3
        out = np.empty(n, dtype=self.dtype)
        self._fn("sample_pressure")(self._h, n, x, out)
        return out

    def sample_velocity(self, rec_xyz):
        x = self._arr(rec_xyz)
        n = x.size // 3
        vx, vy, vz = (np.empty(n, dtype=self.dtype) for _ in range(3))
        self._fn("sample_velocity")(self._h, n, x, vx, vy, vz)
        return vx, vy, vz

    def get_surface_emission(self, xyz, normals):
        x = self._arr(xyz)
        nr = self._arr(normals)
        n = x.size // 3
        P, vn = np.empty(n, dtype=self.dtype), np.empty(n, dtype=self.dtype)
        self._fn("get_surface_emission")(self._h, n, x, nr, P, vn)
        return P, vn

    def precompute_pressure_samplers(self, rec_xyz):
        x = self._arr(rec_xyz)
        n = x.size // 3
        idx = np.empty(8 * n, dtype=np.int32)
        w = np.empty(8 * n, dtype=self.dtype)
        self._fn("precompute_pressure_samplers")(self._h, n, x, idx, w)
        return idx, w

    def precompute_velocity_samplers(self, rec_xyz):
        x = self._arr(rec_xyz)
        n = x.size // 3
        outs = []
        for _ in range(3):
            outs += [np.empty(8 * n, dtype=np.int32), np.empty(8 * n, dtype=self.dtype)]
        self._fn("precompute_velocity_samplers")(self._h, n, x, *outs)
        return outs

    def sample_pressure_precomputed(self, idx8, wgt8):
        idx = np.ascontiguousarray(idx8, dtype=np.int32).ravel()
        w = self._arr(wgt8)
        n = idx.size // 8
        out = np.empty(n, dtype=self.dtype)
        self._fn("sample_pressure_precomputed")(self._h, n, idx, w, out)
        return out

    def sample_velocity_precomputed(self, xi, xw, yi, yw, zi, zw):
        n = np.asarray(xi).size // 8
        outs = [np.empty(n, dtype=self.dtype) for _ in range(3)]
        self._fn("sample_velocity_precomputed")(
            self._h, n, np.ascontiguousarray(xi, np.int32), self._arr(xw),
            np.ascontiguousarray(yi, np.int32), self._arr(yw),
            np.ascontiguousarray(zi, np.int32), self._arr(zw), *outs)
        return tuple(outs)

    def sample_plate_displacement_batch(self, idx4, wgt4):
        idx = np.ascontiguousarray(idx4, dtype=np.int32).ravel()
        n = idx.size // 4
        out = np.empty(n, dtype=self.dtype)
        self._fn("sample_plate_displacement_batch")(self._h, n, idx, self._arr(wgt4), out)
        return out

    def sample_plate_weighted(self, plate_indices, weights):
        idx = np.ascontiguousarray(plate_indices, dtype=np.int32).ravel()
        out = np.empty(1, dtype=self.dtype)
        self._fn("sample_plate_weighted")(self._h, idx.size, idx, self._arr(weights), out)
        return out[0]

    # room runs: deposit s[n] before step n, record receivers after it
    def run(self, n_steps: int, src_idx: int, signal, idx8, wgt8) -> np.ndarray:
        idx = np.ascontiguousarray(idx8, dtype=np.int32).ravel()
        w = self._arr(wgt8)
        n_rec = idx.size // 8
        trace = np.zeros((n_steps, n_rec), dtype=self.dtype)
        for n in range(n_steps):
            sc = self.step_count
            if signal is not None and sc < len(signal):
                self.add_pressure(src_idx, float(signal[sc]))
            self.step(1)
            trace[n] = self.sample_pressure_precomputed(idx, w)
        return trace


class OracleFDTD(_CpuFDTD):
    """The C restatement; ``precision="f64"`` selects the FP64 instantiation."""

    def __init__(self, Nx, Ny, Nz, dx, c=343.0, rho_air=1.21, cell_type=None, plate_iz=-1,
                 plate_active=None, plate_mass_density=7.0, plate_stiffness_D=0.45,
                 plate_alpha_M=2.0, plate_beta_K=1e-5, n_pml=10, precision="f32"):
        self._lib = _load_oracle()
        self._pfx = "orc_" if precision == "f32" else "orc64_"
        self.dtype = np.float32 if precision == "f32" else np.float64
        if cell_type is None:
            cell_type = np.zeros(Nx * Ny * Nz, np.uint8)
        if plate_active is None:
            plate_active = np.zeros(Nx * Ny, np.uint8)
        self._init(Nx, Ny, Nz, dx, c, rho_air, cell_type, plate_iz, plate_active,
                   plate_mass_density, plate_stiffness_D, plate_alpha_M, plate_beta_K, n_pml)

    def add_pressure(self, idx: int, amp: float) -> int:
        return self._fn("add_pressure")(self._h, int(idx), amp)

    def set_face_absorption(self, a6: Sequence[float]):
        rc = self._fn("set_face_absorption")(self._h, self._arr(a6, 6))
        assert rc == 0

    def set_cell_absorption(self, a_cell):
        rc = self._fn("set_cell_absorption")(self._h, self._arr(a_cell, self.Nx * self.Ny * self.Nz))
        assert rc == 0

    def get_p_damp(self):
        out = np.empty(self.Nx * self.Ny * self.Nz, dtype=self.dtype)
        self._fn("get_p_damp")(self._h, out, out.size)
        return out

    def set_pressure_field(self, p):
        self._pin = self._arr(p, self.Nx * self.Ny * self.Nz)
        self._fn("set_pressure_field")(self._h, self._pin)

    def run(self, n_steps, src_idx, signal, idx8, wgt8):
        """Whole room run inside C (same semantics as the base-class loop)."""
        idx = np.ascontiguousarray(idx8, dtype=np.int32).ravel()
        w = self._arr(wgt8)
        n_rec = idx.size // 8
        sig = self._arr(signal) if signal is not None else None
        trace = np.zeros((n_steps, n_rec), dtype=self.dtype)
        vp = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None
        rc = self._fn("run")(self._h, int(n_steps), int(src_idx), vp(sig),
                             0 if sig is None else sig.size, n_rec, vp(idx), vp(w), vp(trace))
        if rc == -3:
            raise RuntimeError("AcousticFDTD: pressure diverged (FDTD_ERR_UNSTABLE)")
        return trace


class RefFDTD(_CpuFDTD):
    """The reference's acoustic_fdtd.cpp, compiled unchanged (oracle/_ref)."""

    def __init__(self, Nx, Ny, Nz, dx, c=343.0, rho_air=1.21, cell_type=None, plate_iz=-1,
                 plate_active=None, plate_mass_density=7.0, plate_stiffness_D=0.45,
                 plate_alpha_M=2.0, plate_beta_K=1e-5, n_pml=10, fast: bool = False):
        self._lib = _load_ref(fast)
        self._pfx = "fdtd_"
        self.dtype = np.float32
        if cell_type is None:
            cell_type = np.zeros(Nx * Ny * Nz, np.uint8)
        if plate_active is None:
            plate_active = np.zeros(Nx * Ny, np.uint8)
        self._init(Nx, Ny, Nz, dx, c, rho_air, cell_type, plate_iz, plate_active,
                   plate_mass_density, plate_stiffness_D, plate_alpha_M, plate_beta_K, n_pml)

    @property
    def library_path(self) -> str:
        return self._lib._path

    @staticmethod
    def pool_threads() -> int:
        return _load_ref(False).fdtd_ref_pool_threads()

    def add_pressure(self, idx: int, amp: float) -> int:
        return self._lib.fdtd_ref_add_pressure(self._h, int(idx), amp)

    def set_face_absorption(self, a6: Sequence[float]):
        rc = self._lib.fdtd_ref_set_face_absorption(self._h, self.n_pml, self._arr(a6, 6))
        assert rc == 0

    def get_p_damp(self):
        out = np.empty(self.Nx * self.Ny * self.Nz, dtype=np.float32)
        self._lib.fdtd_ref_get_p_damp(self._h, out, out.size)
        return out

    def inject_bridge(self, signal_val, signal_ddt, force_scale=1.0):
        rc = self._lib.fdtd_inject_bridge(self._h, signal_val, signal_ddt, force_scale)
        if rc != 0:
            raise RuntimeError("fdtd_inject_bridge is disabled")
