"""Storage-precision study of the open-room step (fdtd_b200_prec_*).

The same room is run with its fields stored as FP32, BF16, FP16 and the two
compensated 16-bit forms (value + FP32-formed residual, four bytes per value
in all), each with FP32 update arithmetic, and once with FP64 storage and
FP64 arithmetic, the GPU oracle.  Receivers sum their 8 taps in double in
every mode, and every ``audit_every`` steps the velocity pass also sums the
discrete energy

    E^n = dx^3/2 * ( sum (p^n)^2 / (rho c^2) + rho * sum v^{n-1/2} v^{n+1/2} )

in double.  ``study`` reports, per storage mode, the relative L2 error of the
receiver traces against the FP64 run and the largest deviation of the energy
log from the FP64 one, relative to the FP64 energy at the same step and to
its peak.

The update is the reference's (csrc/kernels/acoustic_fdtd.cpp:1099-1148
velocity, :1176-1234 pressure, :216-222 and :469-476 damping), restricted to
open rooms: no walls, face fractions or plate.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from typing import Dict, Iterable, Optional

import numpy as np

from .rooms import Room, rel_l2

MODES = {"fp32": 0, "fp64": 1, "bf16": 2, "fp16": 3, "bf16c": 4, "fp16c": 5}
BYTES_PER_VALUE = {"fp32": 4, "fp64": 8, "bf16": 2, "fp16": 2, "bf16c": 4, "fp16c": 4}
STUDY_MODES = ("fp32", "bf16", "fp16", "bf16c", "fp16c")


def pressure_taps(nx: int, ny: int, nz: int, xyz) -> tuple:
    """8-tap trilinear samplers of the pressure grid, in float32 as
    fdtd_precompute_pressure_samplers computes them (acoustic_fdtd.cpp:1567-1596):
    clamp to the grid, floor, next index clamped, weights from the fractions."""
    f = np.float32
    pts = np.asarray(xyz, dtype=np.float32).reshape(-1, 3)
    idx = np.empty((len(pts), 8), np.int32)
    w = np.empty((len(pts), 8), np.float32)
    dims = (nx, ny, nz)
    for r, p in enumerate(pts):
        g = []
        for a in range(3):
            v = p[a]
            v = f(0) if v < 0 else v
            v = f(dims[a] - 1) if v > f(dims[a] - 1) else v
            v = f(0) if v != v else v
            g.append(f(v))
        i0, j0, k0 = (int(v) for v in g)
        i1 = i0 + 1 if i0 < nx - 1 else i0
        j1 = j0 + 1 if j0 < ny - 1 else j0
        k1 = k0 + 1 if k0 < nz - 1 else k0
        fx, fy, fz = f(g[0] - f(i0)), f(g[1] - f(j0)), f(g[2] - f(k0))
        one = f(1)
        FI = lambda a, b, c: c + nz * (b + ny * a)
        corners = [(i0, j0, k0), (i1, j0, k0), (i0, j1, k0), (i1, j1, k0),
                   (i0, j0, k1), (i1, j0, k1), (i0, j1, k1), (i1, j1, k1)]
        wx = (one - fx, fx)
        wy = (one - fy, fy)
        wz = (one - fz, fz)
        for t, (a, b, c) in enumerate(corners):
            idx[r, t] = FI(a, b, c)
            w[r, t] = f(f(wx[t & 1] * wy[(t >> 1) & 1]) * wz[t >> 2])
    return idx.ravel(), w.ravel()


def fp16_scales(amp: float) -> tuple:
    """Powers of two for FP16 storage: P times 2^10 and V times 2^19 for unit
    source samples, shifted by the source amplitude's octave.  Pressure near a
    unit source stays below ~40 Pa, velocity ~ p / (rho c) ~ p / 2^9."""
    shift = -int(round(math.log2(abs(amp)))) if amp else 0
    return float(2.0 ** (10 + shift)), float(2.0 ** (19 + shift))


class PrecisionRoom:
    """One room on the GPU with a chosen field storage."""

    def __init__(self, room: Room, mode: str, audit_capacity: int = 64, device: int = 0,
                 trace_capacity: Optional[int] = None, kernel: str = "auto"):
        from . import _native
        if mode not in MODES:
            raise ValueError(f"unknown storage mode {mode!r}; one of {sorted(MODES)}")
        self._native = _native
        self._lib = _native.load()
        self.room, self.mode = room, mode
        a6 = np.ascontiguousarray(room.absorption, dtype=np.float32)
        ps, vs = fp16_scales(room.amp)
        h = self._lib.fdtd_b200_prec_create(room.nx, room.ny, room.nz, float(room.dx), float(room.c),
                                            float(room.rho), room.n_pml,
                                            a6.ctypes.data_as(_native.P_f32), MODES[mode], ps, vs,
                                            device)
        if not h:
            raise RuntimeError("fdtd_b200_prec_create failed: " + _native.last_error())
        self._h = C.c_void_p(h)
        sig = np.ascontiguousarray(room.signal(), dtype=np.float64)
        self._check(self._lib.fdtd_b200_prec_set_source(self._h, room.src_flat,
                                                        sig.ctypes.data_as(_native.P_f64), sig.size),
                    "prec_set_source")
        idx, w = pressure_taps(room.nx, room.ny, room.nz, room.receiver_xyz())
        self.n_rec = idx.size // 8
        self._idx = np.ascontiguousarray(idx, np.int32)
        self._w = np.ascontiguousarray(w, np.float64)
        cap = room.n_steps if trace_capacity is None else trace_capacity
        self._check(self._lib.fdtd_b200_prec_set_receivers(
            self._h, self.n_rec, self._idx.ctypes.data_as(_native.P_i32),
            self._w.ctypes.data_as(_native.P_f64), int(cap), int(audit_capacity)), "prec_set_receivers")
        self.steps = 0
        if kernel not in ("auto", "fused", "two_pass"):
            raise ValueError(f"unknown kernel {kernel!r}; one of auto, fused, two_pass")
        if kernel != "auto":
            self._check(self._lib.fdtd_b200_prec_set_kernel(self._h, 1 if kernel == "fused" else 0),
                        "prec_set_kernel")

    @property
    def kernel(self) -> str:
        """The step kernel: "fused" (single pass, the 16-bit modes' default) or "two_pass"."""
        return "fused" if self._lib.fdtd_b200_prec_get_kernel(self._h) == 1 else "two_pass"

    def torch_stream(self):
        """The handle's stream as a torch stream (CUDA events around steps)."""
        import torch
        return torch.cuda.ExternalStream(self._lib.fdtd_b200_prec_stream(self._h))

    @property
    def launch_count(self) -> int:
        return int(self._lib.fdtd_b200_prec_launch_count(self._h))

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: rc={rc} {self._native.last_error()}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fdtd_b200_prec_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def dt(self) -> float:
        return self._lib.fdtd_b200_prec_dt(self._h)

    @property
    def taps(self):
        return self._idx.copy(), self._w.copy()

    def step(self, n: int, audit_every: int = 0):
        self._check(self._lib.fdtd_b200_prec_step(self._h, int(n), int(audit_every)), "prec_step")
        self.steps += int(n)

    def traces(self) -> np.ndarray:
        out = np.empty(max(self.steps * self.n_rec, 1), np.float64)
        n = C.c_int(0)
        self._check(self._lib.fdtd_b200_prec_get_traces(self._h, out.ctypes.data_as(self._native.P_f64),
                                                        out.size, C.byref(n)), "prec_get_traces")
        return out[: n.value * self.n_rec].reshape(n.value, self.n_rec)

    def energy(self) -> np.ndarray:
        """(rows, 3): step, potential part, E."""
        rows = 4096
        out = np.empty(rows * 3, np.float64)
        n = C.c_int(0)
        self._check(self._lib.fdtd_b200_prec_get_energy(self._h, out.ctypes.data_as(self._native.P_f64),
                                                        rows, C.byref(n)), "prec_get_energy")
        return out[: 3 * n.value].reshape(n.value, 3)

    def pressure(self) -> np.ndarray:
        r = self.room
        out = np.empty(r.nx * r.ny * r.nz, np.float64)
        self._check(self._lib.fdtd_b200_prec_get_pressure(self._h, out.ctypes.data_as(self._native.P_f64),
                                                          out.size), "prec_get_pressure")
        return out.reshape(r.nx, r.ny, r.nz)


def run_mode(room: Room, mode: str, audit_every: int = 500, chunk: int = 500, device: int = 0,
             kernel: str = "auto") -> dict:
    """Run the room in one storage mode; traces, energy log and wall time."""
    import torch
    cap = room.n_steps // audit_every + 2 if audit_every > 0 else 1
    pr = PrecisionRoom(room, mode, audit_capacity=cap, device=device, kernel=kernel)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    left = room.n_steps
    while left > 0:
        n = min(chunk, left)
        pr.step(n, audit_every)
        left -= n
    tr = pr.traces()            # synchronises
    sec = time.perf_counter() - t0
    out = {"mode": mode, "traces": tr, "energy": pr.energy(), "seconds": sec,
           "bytes_per_value": BYTES_PER_VALUE[mode],
           "gcell_per_s": room.cells * room.n_steps / sec / 1e9}
    pr.close()
    return out


def compare(res: dict, ref: dict) -> dict:
    """Errors of one storage mode against the FP64 run."""
    tr, rt = res["traces"], ref["traces"]
    e, re = res["energy"], ref["energy"]
    finite = bool(np.all(np.isfinite(tr)))
    ok_e = e.shape == re.shape and e.size > 0
    e_rel = (np.abs(e[:, 2] - re[:, 2]) / np.maximum(np.abs(re[:, 2]), 1e-300)) if ok_e else np.array([np.nan])
    e_peak = (np.abs(e[:, 2] - re[:, 2]) / np.max(np.abs(re[:, 2]))) if ok_e else np.array([np.nan])
    per_rec = [rel_l2(tr[:, q], rt[:, q]) for q in range(rt.shape[1])]
    return {"mode": res["mode"], "bytes_per_value": res["bytes_per_value"],
            "trace_rel_l2": rel_l2(tr, rt) if finite else float("inf"),
            "trace_rel_l2_per_receiver": per_rec,
            "trace_max_abs_err": float(np.max(np.abs(tr - rt))) if finite else float("inf"),
            "energy_max_rel_dev": float(np.max(e_rel)),
            "energy_max_dev_rel_peak": float(np.max(e_peak)),
            "energy_final_rel_dev": float(e_rel[-1]),
            "seconds": res["seconds"], "gcell_per_s": res["gcell_per_s"]}


def study(room: Room, modes: Iterable[str] = STUDY_MODES, audit_every: int = 500,
          device: int = 0) -> Dict[str, object]:
    """FP64 oracle run, then each storage mode, with errors per mode."""
    ref = run_mode(room, "fp64", audit_every, device=device)
    rows = [compare(run_mode(room, m, audit_every, device=device), ref) for m in modes]
    return {"room": room.describe(), "audit_every": audit_every,
            "fp64": {"seconds": ref["seconds"], "gcell_per_s": ref["gcell_per_s"],
                     "energy": ref["energy"].tolist()},
            "modes": rows}
