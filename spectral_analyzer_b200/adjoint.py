"""Gradient of a receiver-trace loss w.r.t. per-cell boundary absorption.

``AdjointRoom`` wraps the engine's fdtd_b200_adj_* handle: a room whose
absorption is a per-cell field a_c = alpha_c * dt (P damping 1/(1+a_c), face
damping 1 - (a_L+a_R)/2, the reference's update otherwise), a point source
and 8-tap receivers.  ``forward`` runs the room from rest and records the
traces, keeping checkpoints every K steps; ``backward`` runs the hand-written
adjoint kernels backwards over the recomputed segments and returns dL/da.

``TraceLoss`` puts this behind ``torch.autograd.Function``:
``loss = TraceLoss.apply(a, room, targets)`` with ``a`` a CUDA tensor of shape
(Nx, Ny, Nz) and L = sum over steps and receivers of (y - target)^2.

``boundary_absorption`` builds the absorbing layer used for the
differentiation workload: a seeded Gaussian random field (Gaussian kernel,
correlation length in cells) mapped to mean 0.275, standard deviation 0.1125
and clipped to [0.05, 0.5] on the cells within ``n_pml`` of a face, 0 inside.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from .precision import pressure_taps
from .rooms import reference_dt, ricker


def gaussian_random_field(shape: Tuple[int, int, int], corr: float, seed: int) -> np.ndarray:
    """Zero-mean, unit-variance field: white noise filtered by exp(-r^2 / (2 corr^2))."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n) * 2 * np.pi for n in shape]
    kx, ky, kz = np.meshgrid(*k, indexing="ij")
    filt = np.exp(-0.5 * corr ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    f = np.real(np.fft.ifftn(np.fft.fftn(noise) * filt))
    f -= f.mean()
    return f / f.std()


def boundary_mask(shape: Tuple[int, int, int], n_pml: int) -> np.ndarray:
    nx, ny, nz = shape
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    d = np.minimum.reduce([i, nx - 1 - i, j, ny - 1 - j, k, nz - 1 - k])
    return d < n_pml


def boundary_absorption(shape, n_pml: int = 10, corr: float = 8.0, seed: int = 0,
                        lo: float = 0.05, hi: float = 0.5) -> np.ndarray:
    g = gaussian_random_field(shape, corr, seed)
    a = np.clip(0.5 * (lo + hi) + 0.25 * (hi - lo) * g, lo, hi)
    return np.where(boundary_mask(shape, n_pml), a, 0.0).astype(np.float32)


@dataclass
class DiffProblem:
    """Room, source, receivers and the absorption fields of a differentiation run."""
    shape: Tuple[int, int, int]
    n_steps: int
    src: Tuple[int, int, int]
    receivers: List[Tuple[int, int, int]]
    a: np.ndarray           # float32 (Nx, Ny, Nz): where the gradient is taken
    a_target: np.ndarray    # float32: the field the targets come from
    dx: float = 0.01
    c: float = 343.0
    rho: float = 1.21
    f0: float = 1000.0
    n_pml: int = 10

    @property
    def cells(self) -> int:
        return int(np.prod(self.shape))

    def flat(self, p) -> int:
        nx, ny, nz = self.shape
        return int(p[2] + nz * (p[1] + ny * p[0]))

    def signal(self) -> np.ndarray:
        return ricker(self.n_steps, reference_dt(self.dx, self.c), self.f0)

    def describe(self) -> dict:
        return {"shape": list(self.shape), "steps": self.n_steps, "src": list(self.src),
                "receivers": [list(r) for r in self.receivers], "n_pml": self.n_pml}


def differentiation_problem(n=128, n_steps: int = 4000, seed: int = 5, n_rec: int = 4,
                            n_pml: int = 10, corr: float = 8.0, perturb: float = 0.1) -> DiffProblem:
    """n^3 (or n = (Nx, Ny, Nz)) room, Ricker 1 kHz source and n_rec receivers at
    seeded cells at least n_pml + 2 from every face; a from a seeded field,
    targets from the field times (1 + perturb * g') with g' another seeded field."""
    rng = np.random.default_rng(seed)
    shape = (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)
    if min(shape) <= 2 * n_pml + 4:
        raise ValueError("room too small for its absorbing layer")

    def interior():
        return tuple(int(rng.integers(n_pml + 2, d - n_pml - 2)) for d in shape)

    src = interior()
    recs = [interior() for _ in range(n_rec)]
    a = boundary_absorption(shape, n_pml, corr, seed)
    g2 = gaussian_random_field(shape, corr, seed + 1000)
    a_t = np.where(a > 0, np.clip(a * (1.0 + perturb * g2), 0.0, 1.0), 0.0).astype(np.float32)
    return DiffProblem(shape, n_steps, src, recs, a, a_t, n_pml=n_pml)


class AdjointRoom:
    """One handle of the adjoint engine for a DiffProblem's room."""

    def __init__(self, prob: DiffProblem, double: bool = False, checkpoint_every: int = 200,
                 device: int = 0):
        from . import _native
        self._native = _native
        self._lib = _native.load()
        self.prob = prob
        self.double = bool(double)
        nx, ny, nz = prob.shape
        h = self._lib.fdtd_b200_adj_create(nx, ny, nz, prob.dx, prob.c, prob.rho, int(self.double),
                                           int(checkpoint_every), device)
        if not h:
            raise RuntimeError("fdtd_b200_adj_create failed: " + _native.last_error())
        self._h = C.c_void_p(h)
        sig = np.ascontiguousarray(prob.signal(), np.float64)
        self._check(self._lib.fdtd_b200_adj_set_source(self._h, prob.flat(prob.src),
                                                       sig.ctypes.data_as(_native.P_f64), sig.size),
                    "adj_set_source")
        idx, w = pressure_taps(nx, ny, nz, np.asarray(prob.receivers, np.float32))
        self.taps = (np.ascontiguousarray(idx, np.int32), np.ascontiguousarray(w, np.float64))
        self.n_rec = len(prob.receivers)
        self._check(self._lib.fdtd_b200_adj_set_receivers(
            self._h, self.n_rec, self.taps[0].ctypes.data_as(_native.P_i32),
            self.taps[1].ctypes.data_as(_native.P_f64), prob.n_steps), "adj_set_receivers")
        self.steps = 0

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: rc={rc} {self._native.last_error()}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fdtd_b200_adj_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def dt(self) -> float:
        return self._lib.fdtd_b200_adj_dt(self._h)

    @property
    def launch_count(self) -> int:
        return self._lib.fdtd_b200_adj_launch_count(self._h)

    def set_absorption(self, a):
        """a: numpy array or CUDA tensor of Nx*Ny*Nz float32/float64 values in [0, 1]."""
        n = self.prob.cells
        if hasattr(a, "data_ptr"):
            import torch
            t = a.detach().contiguous()
            if t.numel() != n or t.dtype not in (torch.float32, torch.float64):
                raise ValueError("absorption: expected Nx*Ny*Nz float32/float64 values")
            torch.cuda.synchronize(t.device)
            rc = self._lib.fdtd_b200_adj_set_absorption(self._h, C.c_void_p(t.data_ptr()), n, t.element_size())
        else:
            arr = np.ascontiguousarray(a)
            if arr.dtype not in (np.float32, np.float64):
                arr = arr.astype(np.float32)
            if arr.size != n:
                raise ValueError("absorption: expected Nx*Ny*Nz values")
            rc = self._lib.fdtd_b200_adj_set_absorption(self._h, arr.ctypes.data_as(C.c_void_p), n,
                                                        arr.itemsize)
        self._check(rc, "adj_set_absorption")

    def forward(self, n_steps: Optional[int] = None, keep_checkpoints: bool = True) -> np.ndarray:
        n = self.prob.n_steps if n_steps is None else int(n_steps)
        out = np.empty((n, self.n_rec), np.float64)
        self._check(self._lib.fdtd_b200_adj_forward(self._h, n, int(keep_checkpoints),
                                                    out.ctypes.data_as(self._native.P_f64)), "adj_forward")
        self.steps = n
        return out

    def backward(self, dloss_dtrace: np.ndarray, out=None):
        """dL/da for the last checkpointed forward; out: CUDA float64 tensor or None (numpy)."""
        r = np.ascontiguousarray(dloss_dtrace, np.float64)
        if r.shape != (self.steps, self.n_rec):
            raise ValueError(f"dloss_dtrace: expected shape {(self.steps, self.n_rec)}")
        if out is None:
            g = np.empty(self.prob.shape, np.float64)
            ptr = g.ctypes.data_as(C.c_void_p)
        else:
            g = out
            ptr = C.c_void_p(out.data_ptr())
        self._check(self._lib.fdtd_b200_adj_backward(self._h, r.ctypes.data_as(self._native.P_f64), ptr),
                    "adj_backward")
        return g

    def loss(self, a, targets: np.ndarray) -> float:
        """L(a) by a forward without checkpoints (finite differences)."""
        self.set_absorption(a)
        y = self.forward(keep_checkpoints=False)
        return float(np.sum((y - targets) ** 2))


def _function():
    import torch

    class TraceLoss(torch.autograd.Function):
        """L(a) = sum_{n,r} (y_r^n(a) - target_r^n)^2; backward by the adjoint kernels."""

        @staticmethod
        def forward(ctx, a, room: AdjointRoom, targets):
            room.set_absorption(a)
            y = room.forward(keep_checkpoints=True)
            t = np.asarray(targets, np.float64)
            ctx.room, ctx.resid = room, 2.0 * (y - t)
            ctx.a_meta = (a.shape, a.dtype, a.device)
            return torch.tensor(float(np.sum((y - t) ** 2)), dtype=torch.float64, device=a.device)

        @staticmethod
        def backward(ctx, g_out):
            shape, dtype, device = ctx.a_meta
            grad = torch.empty(shape, dtype=torch.float64, device=device)
            torch.cuda.synchronize(device)     # the engine writes grad on its own stream
            ctx.room.backward(ctx.resid * float(g_out), out=grad)
            return grad.to(dtype), None, None

    return TraceLoss


_TRACE_LOSS = None


def trace_loss(a, room: AdjointRoom, targets):
    """Differentiable loss of a CUDA tensor a (Nx, Ny, Nz)."""
    global _TRACE_LOSS
    if _TRACE_LOSS is None:
        _TRACE_LOSS = _function()
    return _TRACE_LOSS.apply(a, room, targets)
