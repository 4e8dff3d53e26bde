"""AcousticFDTD — drop-in for the reference's ``_spectral_kernels.AcousticFDTD``.

Same constructor keywords and defaults, methods, return shapes, properties and
exceptions as the pybind class (csrc/bindings/pybind_kernels.cpp:5473-5664,
:8924-9022), backed by the CUDA engine through its C ABI.  The pressure and
velocity fields are PyTorch tensors on the GPU (the engine's device buffers);
``pressure_tensor()`` / ``velocity_tensors()`` expose them without a copy.

Beyond the reference's surface the class offers the engine extensions used by
room workloads: point source, receivers with a device trace, per-face
absorption, async stepping and kernel selection.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _native

_REQUIRED = object()


def _f32(x, n: Optional[int] = None) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.float32).ravel()
    if n is not None and a.size != n:
        raise RuntimeError(f"expected {n} float32 elements, got {a.size}")
    return a


def _i32(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.int32).ravel()


def _pf(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_native.P_f32)


def _pi(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_native.P_i32)


class AcousticFDTD:
    """3-D acoustic FDTD solver (staggered p/vx/vy/vz leapfrog) on a CUDA GPU."""

    def __init__(self, Nx, Ny, Nz, dx, c=343.0, rho_air=1.21, cell_type=_REQUIRED,
                 plate_iz=_REQUIRED, plate_active=_REQUIRED, plate_mass_density=7.0,
                 plate_stiffness_D=0.45, plate_alpha_M=2.0, plate_beta_K=1e-5, n_pml=10,
                 *, device=None):
        import torch

        for name, val in (("cell_type", cell_type), ("plate_iz", plate_iz),
                          ("plate_active", plate_active)):
            if val is _REQUIRED:
                raise TypeError(f"AcousticFDTD(): missing required argument '{name}'")
        self._lib = _native.load()
        Nx, Ny, Nz = int(Nx), int(Ny), int(Nz)
        ct = np.ascontiguousarray(cell_type, dtype=np.uint8).ravel()
        pa = np.ascontiguousarray(plate_active, dtype=np.uint8).ravel()
        if ct.size != Nx * Ny * Nz:
            raise RuntimeError("cell_type: expected Nx*Ny*Nz elements")
        if pa.size != Nx * Ny:
            raise RuntimeError("plate_active: expected Nx*Ny elements")
        if not torch.cuda.is_available():
            raise RuntimeError("AcousticFDTD needs a CUDA device (no CPU path)")
        dev = torch.device("cuda", torch.cuda.current_device() if device is None
                           else torch.device(device).index or 0)
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.device = dev
        self._h = None
        self._fields = []
        if Nx > 0 and Ny > 0 and Nz > 0:
            sz = C.c_int()
            nbytes = C.c_size_t()
            self._lib.fdtd_b200_field_layout(Nx, Ny, Nz, C.byref(sz), C.byref(nbytes))
            self.row_stride = sz.value
            n_el = nbytes.value // 4
            # two pressure buffers and two velocity sets, owned by torch
            self._fields = [torch.zeros(n_el, dtype=torch.float32, device=dev) for _ in range(8)]
            ptrs = (C.c_void_p * 8)(*[t.data_ptr() for t in self._fields])
            torch.cuda.synchronize(dev)
            h = self._lib.fdtd_b200_create_ex(
                Nx, Ny, Nz, float(dx), float(c), float(rho_air),
                ct.ctypes.data_as(_native.P_u8), int(plate_iz), pa.ctypes.data_as(_native.P_u8),
                float(plate_mass_density), float(plate_stiffness_D), float(plate_alpha_M),
                float(plate_beta_K), int(n_pml), dev.index,
                C.cast(ptrs, C.POINTER(C.c_void_p)))
        else:
            h = None
        if not h:
            raise RuntimeError("fdtd_create: allocation failed " + _native.last_error())
        self._h = C.c_void_p(h)
        # the solver works on its own non-blocking stream; torch_stream() wraps it

    # ------------------------------------------------------------------ internals
    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.fdtd_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    def _check(self, rc: int, what: str) -> int:
        if rc == _native.FDTD_ERR_CUDA:
            raise RuntimeError(f"{what}: CUDA error: {_native.last_error()}")
        if rc == _native.FDTD_ERR_ARG:
            raise ValueError(f"{what}: invalid argument")
        return rc

    @property
    def _dims(self) -> Tuple[int, int, int]:
        Nx, Ny, Nz = self.Nx, self.Ny, self.Nz
        return (Nx - 1) * Ny * Nz, Nx * (Ny - 1) * Nz, Nx * Ny * (Nz - 1)

    # --------------------------------------------------- reference method surface
    def set_bridge_sources(self, cell_indices, weights):
        idx, w = _i32(cell_indices), _f32(weights)
        if idx.size != w.size:
            raise RuntimeError("cell_indices and weights must have the same length")
        rc = self._lib.fdtd_set_bridge_sources(self._h, idx.size, _pi(idx), _pf(w))
        if rc != 0:
            raise RuntimeError(f"fdtd_set_bridge_sources error: {rc}")

    def set_face_fractions(self, vx_frac, vy_frac, vz_frac):
        nvx, nvy, nvz = self._dims
        a = None if vx_frac is None else _f32(vx_frac, nvx)
        b = None if vy_frac is None else _f32(vy_frac, nvy)
        c = None if vz_frac is None else _f32(vz_frac, nvz)
        rc = self._check(self._lib.fdtd_set_face_fractions(self._h, _pf(a), _pf(b), _pf(c)),
                         "set_face_fractions")
        if rc != 0:
            raise RuntimeError(f"fdtd_set_face_fractions error: {rc}")

    def inject_bridge(self, signal_val, signal_ddt, force_scale=1.0):
        rc = self._lib.fdtd_inject_bridge(self._h, float(signal_val), float(signal_ddt),
                                          float(force_scale))
        if rc != 0:
            raise RuntimeError(
                "fdtd_inject_bridge is disabled: direct pressure bridge injection "
                "bypasses plate impedance; use AcousticCoEvolver structural coupling")

    def step(self, n_steps: int = 1) -> int:
        rc = self._check(self._lib.fdtd_step(self._h, int(n_steps)), "step")
        if rc == _native.FDTD_ERR_UNSTABLE:
            raise RuntimeError("AcousticFDTD: pressure diverged (FDTD_ERR_UNSTABLE)")
        return rc

    def step_rc(self, n_steps: int = 1) -> int:
        """fdtd_step's return code without the exception mapping."""
        return self._check(self._lib.fdtd_step(self._h, int(n_steps)), "step")

    def reset(self):
        self._check(self._lib.fdtd_reset(self._h), "reset")

    def get_pressure_field(self) -> np.ndarray:
        out = np.empty(self.Nx * self.Ny * self.Nz, dtype=np.float32)
        rc = self._check(self._lib.fdtd_get_pressure_field(self._h, _pf(out), out.size),
                         "get_pressure_field")
        if rc != 0:
            raise RuntimeError(f"fdtd_get_pressure_field error: {rc}")
        return out.reshape(self.Nx, self.Ny, self.Nz)

    def get_plate_displacement(self) -> np.ndarray:
        out = np.empty(self.Nx * self.Ny, dtype=np.float32)
        rc = self._check(self._lib.fdtd_get_plate_displacement(self._h, _pf(out), out.size),
                         "get_plate_displacement")
        if rc != 0:
            raise RuntimeError(f"fdtd_get_plate_displacement error: {rc}")
        return out.reshape(self.Nx, self.Ny)

    def sample_pressure(self, rec_xyz) -> np.ndarray:
        x = _f32(rec_xyz)
        n = x.size // 3
        out = np.zeros(n, dtype=np.float32)
        self._check(self._lib.fdtd_sample_pressure(self._h, n, _pf(x), _pf(out)), "sample_pressure")
        return out

    def sample_velocity(self, rec_xyz):
        x = _f32(rec_xyz)
        n = x.size // 3
        vx, vy, vz = (np.zeros(n, dtype=np.float32) for _ in range(3))
        self._check(self._lib.fdtd_sample_velocity(self._h, n, _pf(x), _pf(vx), _pf(vy), _pf(vz)),
                    "sample_velocity")
        return vx, vy, vz

    def get_surface_emission(self, xyz, normals):
        x, nr = _f32(xyz), _f32(normals)
        n = x.size // 3
        P, vn = np.zeros(n, dtype=np.float32), np.zeros(n, dtype=np.float32)
        self._check(self._lib.fdtd_get_surface_emission(self._h, n, _pf(x), _pf(nr), _pf(P), _pf(vn)),
                    "get_surface_emission")
        return P, vn

    def get_velocity_dims(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._lib.fdtd_get_velocity_dims(self._h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def _vel(self, fn, n):
        out = np.empty(n, dtype=np.float32)
        self._check(fn(self._h, _pf(out), n), "get_velocity")
        return out

    def get_velocity_x(self) -> np.ndarray:
        return self._vel(self._lib.fdtd_get_velocity_x, self._dims[0])

    def get_volume_slice(self, axis: int = 2, idx: int = -1) -> np.ndarray:
        """2-D pressure plane as the bridge's get_volume_slice returns it
        (axis 2 -> (Nx, Ny); idx -1 = mid-plane, clamped), gathered on the
        device so only the plane crosses to the host."""
        shape = {0: (self.Ny, self.Nz), 1: (self.Nx, self.Nz), 2: (self.Nx, self.Ny)}.get(int(axis))
        if shape is None:
            raise ValueError("axis must be 0, 1 or 2")
        out = np.empty(shape, dtype=np.float32)
        rc = self._check(self._lib.fdtd_b200_get_volume_slice(self._h, int(axis), int(idx), _pf(out), out.size),
                         "get_volume_slice")
        if rc != 0:
            raise RuntimeError(f"fdtd_b200_get_volume_slice error: {rc}")
        return out

    def get_velocity_y(self) -> np.ndarray:
        return self._vel(self._lib.fdtd_get_velocity_y, self._dims[1])

    def get_velocity_z(self) -> np.ndarray:
        return self._vel(self._lib.fdtd_get_velocity_z, self._dims[2])

    @property
    def dt(self) -> float:
        return self._lib.fdtd_get_dt(self._h)

    @property
    def step_count(self) -> int:
        return self._lib.fdtd_get_step_count(self._h)

    # ------------------------------------------- C-ABI functions used by C callers
    def inject_bridge_drive(self, cell_drives, force_scale=1.0) -> int:
        return self._check(self._lib.fdtd_inject_bridge_drive(self._h, _pf(_f32(cell_drives)),
                                                              float(force_scale)), "inject_bridge_drive")

    def inject_plate_force(self, plate_indices, weights, total_force_N) -> int:
        idx = _i32(plate_indices)
        return self._check(self._lib.fdtd_inject_plate_force(
            self._h, idx.size, _pi(idx), _pf(_f32(weights, idx.size)), float(total_force_N)),
            "inject_plate_force")

    def precompute_pressure_samplers(self, rec_xyz):
        x = _f32(rec_xyz)
        n = x.size // 3
        idx, w = np.empty(8 * n, np.int32), np.empty(8 * n, np.float32)
        self._lib.fdtd_precompute_pressure_samplers(self._h, n, _pf(x), _pi(idx), _pf(w))
        return idx, w

    def precompute_velocity_samplers(self, rec_xyz):
        x = _f32(rec_xyz)
        n = x.size // 3
        outs = []
        for _ in range(3):
            outs += [np.empty(8 * n, np.int32), np.empty(8 * n, np.float32)]
        self._lib.fdtd_precompute_velocity_samplers(
            self._h, n, _pf(x), _pi(outs[0]), _pf(outs[1]), _pi(outs[2]), _pf(outs[3]),
            _pi(outs[4]), _pf(outs[5]))
        return outs

    def sample_pressure_precomputed(self, idx8, wgt8) -> np.ndarray:
        idx, w = _i32(idx8), _f32(wgt8)
        n = idx.size // 8
        out = np.zeros(n, dtype=np.float32)
        self._check(self._lib.fdtd_sample_pressure_precomputed(self._h, n, _pi(idx), _pf(w), _pf(out)),
                    "sample_pressure_precomputed")
        return out

    def sample_velocity_precomputed(self, xi, xw, yi, yw, zi, zw):
        xi, yi, zi = _i32(xi), _i32(yi), _i32(zi)
        xw, yw, zw = _f32(xw), _f32(yw), _f32(zw)
        n = xi.size // 8
        outs = [np.zeros(n, dtype=np.float32) for _ in range(3)]
        self._check(self._lib.fdtd_sample_velocity_precomputed(
            self._h, n, _pi(xi), _pf(xw), _pi(yi), _pf(yw), _pi(zi), _pf(zw),
            _pf(outs[0]), _pf(outs[1]), _pf(outs[2])), "sample_velocity_precomputed")
        return tuple(outs)

    def sample_plate_displacement_batch(self, idx4, wgt4) -> np.ndarray:
        idx, w = _i32(idx4), _f32(wgt4)
        n = idx.size // 4
        out = np.zeros(n, dtype=np.float32)
        self._check(self._lib.fdtd_sample_plate_displacement_batch(self._h, n, _pi(idx), _pf(w), _pf(out)),
                    "sample_plate_displacement_batch")
        return out

    def substep(self, cell_drives=None, drive_scale=1.0, force_idx=None, force_wgt=None,
                force_total_N=0.0, saddle_idx4=None, saddle_wgt4=None) -> np.ndarray:
        """One co-evolver substep in one call (fdtd_b200_substep): bridge drive,
        plate force, one step and the saddle samples, as inject_bridge_drive,
        inject_plate_force, step(1) and sample_plate_displacement_batch would
        give them, with one stream synchronisation.  When no receivers are
        recorded on the device, the substep's device work is replayed as a
        cached CUDA graph.  Returns the saddle samples."""
        drv = _f32(cell_drives) if cell_drives is not None else None
        fi = _i32(force_idx if force_idx is not None else [])
        fw = _f32(force_wgt if force_wgt is not None else np.zeros(fi.size), fi.size)
        si = _i32(saddle_idx4 if saddle_idx4 is not None else [])
        sw = _f32(saddle_wgt4 if saddle_wgt4 is not None else np.zeros(si.size), si.size)
        n = si.size // 4
        out = np.zeros(n, dtype=np.float32)
        rc = self._check(self._lib.fdtd_b200_substep(
            self._h, _pf(drv) if drv is not None else None, float(drive_scale), fi.size, _pi(fi), _pf(fw),
            float(force_total_N), n, _pi(si), _pf(sw), _pf(out)), "substep")
        if rc == _native.FDTD_ERR_UNSTABLE:
            raise RuntimeError("AcousticFDTD: pressure diverged (FDTD_ERR_UNSTABLE)")
        return out

    def sample_plate_weighted(self, plate_indices, weights) -> np.float32:
        idx, w = _i32(plate_indices), _f32(weights)
        out = np.zeros(1, dtype=np.float32)
        self._check(self._lib.fdtd_sample_plate_weighted(self._h, idx.size, _pi(idx), _pf(w), _pf(out)),
                    "sample_plate_weighted")
        return out[0]

    # ------------------------------------------------------------ engine extensions
    def add_pressure(self, cell_index: int, amp: float) -> int:
        """One deposit with the reference's open-cell rule (acoustic_fdtd.cpp:840-872)."""
        return self._check(self._lib.fdtd_b200_add_pressure(self._h, int(cell_index), float(amp)),
                           "add_pressure")

    def set_face_absorption(self, a6: Sequence[float]):
        """Per-face scale (x_lo, x_hi, y_lo, y_hi, z_lo, z_hi) on the PML's sigma_max."""
        self._check(self._lib.fdtd_b200_set_face_absorption(self._h, _pf(_f32(a6, 6))),
                    "set_face_absorption")

    def set_point_source(self, cell_index: int, signal):
        """Deposit signal[n] at cell_index before the step that starts at step count n."""
        s = None if signal is None else _f32(signal)
        self._check(self._lib.fdtd_b200_set_point_source(
            self._h, int(cell_index), _pf(s), 0 if s is None else s.size), "set_point_source")

    def set_receivers(self, idx8, wgt8, capacity: int):
        """Record the 8-tap pressure sample of each receiver after every step."""
        idx, w = _i32(idx8), _f32(wgt8)
        self._check(self._lib.fdtd_b200_set_receivers(self._h, idx.size // 8, _pi(idx), _pf(w),
                                                       int(capacity)), "set_receivers")
        self._n_rec, self._cap = idx.size // 8, int(capacity)

    def get_traces(self) -> np.ndarray:
        """Recorded traces, shape (n_recorded, n_rec); clears them."""
        n_rec = getattr(self, "_n_rec", 0)
        out = np.zeros(max(1, getattr(self, "_cap", 0) * n_rec), dtype=np.float32)
        n = C.c_int()
        self._check(self._lib.fdtd_b200_get_traces(self._h, _pf(out), out.size, C.byref(n)),
                    "get_traces")
        return out[: n.value * n_rec].reshape(n.value, n_rec).copy()

    def run(self, n_steps: int, src_idx: int, signal, idx8, wgt8) -> np.ndarray:
        """Room run: deposit signal[n] before step n, step, record every receiver."""
        self.set_point_source(src_idx, signal)
        self.set_receivers(idx8, wgt8, n_steps)
        self.step(n_steps)
        return self.get_traces()

    def step_async(self, n_steps: int = 1) -> int:
        return self._check(self._lib.fdtd_b200_step_async(self._h, int(n_steps)), "step_async")

    def synchronize(self) -> int:
        return self._check(self._lib.fdtd_b200_synchronize(self._h), "synchronize")

    def debug_hold_load(self, plane: int, wait_us: int = 0):
        """Test hook: the fused step's load of pressure plane ``plane`` is never
        issued, so its bounded wait runs out after ``wait_us`` microseconds
        (0: the normal bound); ``plane=-1`` turns it off."""
        self._check(self._lib.fdtd_b200_debug_hold_load(self._h, int(plane), int(wait_us)), "debug_hold_load")

    def set_kernel(self, mode: str):
        m = {"auto": 0, "two_pass": 1, "fused": 2}[mode]
        self._check(self._lib.fdtd_b200_set_kernel(self._h, m), "set_kernel")

    @property
    def kernel(self) -> str:
        return {1: "two_pass", 2: "fused"}[self._lib.fdtd_b200_get_kernel(self._h)]

    @property
    def launch_count(self) -> int:
        """Kernels launched by this solver since it was created."""
        return self._lib.fdtd_b200_launch_count(self._h)

    @property
    def stream_handle(self) -> int:
        return self._lib.fdtd_b200_get_stream(self._h) or 0

    def torch_stream(self):
        """The solver's CUDA stream as a torch stream (for events and ordering)."""
        import torch
        return torch.cuda.ExternalStream(self.stream_handle, device=self.device)

    def _device_fields(self):
        out = (C.c_void_p * 5)()
        self._lib.fdtd_b200_device_fields(self._h, out)
        return [out[q] for q in range(5)]

    def _view(self, ptr: int):
        for t in self._fields:
            if t.data_ptr() == ptr:
                return t.view(self.Nx, self.Ny, self.row_stride)
        raise RuntimeError("device field not owned by this object")

    def pressure_tensor(self):
        """Zero-copy (Nx, Ny, Nz) view of the current pressure field (float32, CUDA)."""
        self.synchronize()
        return self._view(self._device_fields()[0])[:, :, : self.Nz]

    def velocity_tensors(self):
        """Zero-copy views of the staggered velocities: (Nx-1,Ny,Nz), (Nx,Ny-1,Nz), (Nx,Ny,Nz-1)."""
        self.synchronize()
        f = self._device_fields()
        return (self._view(f[2])[: self.Nx - 1, :, : self.Nz],
                self._view(f[3])[:, : self.Ny - 1, : self.Nz],
                self._view(f[4])[:, :, : self.Nz - 1])

    def snapshot(self) -> dict:
        """The room's state in host memory: the current P and V fields (the
        device layout, padding included), the step count, the stability
        check's phase and the step whose source sample P already holds.  ``restore`` on a handle of the same room configuration
        (source schedule, receivers) continues exactly as this one would."""
        import torch
        self.synchronize()
        f = self._device_fields()
        step, phase, dep = C.c_int(), C.c_int(), C.c_int()
        self._check(self._lib.fdtd_b200_get_progress(self._h, C.byref(step), C.byref(phase), C.byref(dep)),
                    "get_progress")
        fields = [self._view(f[q]).to("cpu") for q in (0, 2, 3, 4)]
        torch.cuda.synchronize(self.device)
        return {"step": step.value, "phase": phase.value, "deposited": dep.value, "fields": fields,
                "dims": (self.Nx, self.Ny, self.Nz)}

    def restore(self, snap: dict):
        """Load a snapshot taken from a handle of the same room (see snapshot)."""
        if tuple(snap["dims"]) != (self.Nx, self.Ny, self.Nz):
            raise ValueError("snapshot of another grid")
        self.synchronize()
        f = self._device_fields()
        for q, t in zip((0, 2, 3, 4), snap["fields"]):
            self._view(f[q]).copy_(t)
        import torch
        torch.cuda.synchronize(self.device)
        self._check(self._lib.fdtd_b200_set_progress(self._h, int(snap["step"]), int(snap["phase"]),
                                                     int(snap["deposited"])), "set_progress")

    def profile(self, enable: bool = True):
        self._check(self._lib.fdtd_b200_profile(self._h, 1 if enable else 0), "profile")

    def profile_read(self):
        ms, n, nk = C.c_double(), C.c_longlong(), C.c_longlong()
        self._check(self._lib.fdtd_b200_profile_read(self._h, C.byref(ms), C.byref(n), C.byref(nk)),
                    "profile_read")
        return ms.value, n.value, nk.value
