"""Room workloads: grid, absorption, point source and receivers.

A *room* is an open box of air (no walls, no plate) with the reference's graded
PML on all six faces, a point pressure source and integer-coordinate
receivers.  Conventions shared by the engine, the oracle and the benchmark:

* before step n (n = 0, 1, ...) the source sample s[n] is deposited at the
  source cell with the reference's open-cell rule (deposit_pressure_open,
  csrc/kernels/acoustic_fdtd.cpp:840-872);
* after step n every receiver records its 8-tap trilinear sample
  (fdtd_sample_pressure_precomputed, acoustic_fdtd.cpp:1663-1676);
* the time step is the reference's fixed dt = 0.77*dx/(c*sqrt(3))
  (acoustic_fdtd.cpp:348), Courant 0.4446.  A Courant number of 0.99/sqrt(3)
  exceeds the scheme's 6/(7*sqrt(3)) limit and diverges in the reference;
* per-face absorption a_f in (0, 1] scales the PML's sigma_max on that face;
  a_f = 1 on every face is the unmodified reference.

Source signals are computed in float64 and rounded once to float32, so every
implementation injects identical values.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

FDTD_AIR, FDTD_WALL, FDTD_PLATE, FDTD_PML = 0, 1, 2, 3


def reference_dt(dx: float, c: float) -> float:
    """The reference's time step in float32 arithmetic (acoustic_fdtd.cpp:348)."""
    f = np.float32
    return float(f(f(0.77) * f(dx)) / f(f(c) * f(1.732050808)))


def gaussian_pulse(n_steps: int, sigma_steps: float = 8.0, amp: float = 1.0) -> np.ndarray:
    """s[n] = amp * exp(-0.5*((n - 4*sigma)/sigma)^2), n in steps."""
    n = np.arange(n_steps, dtype=np.float64)
    return (amp * np.exp(-0.5 * ((n - 4.0 * sigma_steps) / sigma_steps) ** 2)).astype(np.float32)


def ricker(n_steps: int, dt: float, f0: float = 1000.0, amp: float = 1.0) -> np.ndarray:
    """Ricker wavelet s(t) = amp*(1 - 2 pi^2 f^2 tau^2) exp(-pi^2 f^2 tau^2), tau = t - 1/f, t = n*dt."""
    t = np.arange(n_steps, dtype=np.float64) * float(dt)
    tau = t - 1.0 / f0
    a = (math.pi * f0 * tau) ** 2
    return (amp * (1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32)


@dataclass
class Room:
    nx: int
    ny: int
    nz: int
    n_steps: int
    src: Tuple[int, int, int]
    receivers: List[Tuple[int, int, int]]
    absorption: Tuple[float, ...] = (1.0,) * 6   # x_lo, x_hi, y_lo, y_hi, z_lo, z_hi
    source_kind: str = "gaussian"                 # "gaussian" | "ricker"
    dx: float = 0.01
    c: float = 343.0
    rho: float = 1.21
    n_pml: int = 10
    sigma_steps: float = 8.0
    f0: float = 1000.0
    amp: float = 1.0
    name: str = "room"

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def dt(self) -> float:
        return reference_dt(self.dx, self.c)

    def flat(self, i: int, j: int, k: int) -> int:
        """Reference flat index k + Nz*(j + Ny*i) (acoustic_fdtd.h:67-71)."""
        return k + self.nz * (j + self.ny * i)

    @property
    def src_flat(self) -> int:
        return self.flat(*self.src)

    def receiver_xyz(self) -> np.ndarray:
        return np.asarray(self.receivers, dtype=np.float32).reshape(-1, 3)

    def signal(self, n: Optional[int] = None) -> np.ndarray:
        n = self.n_steps if n is None else n
        if self.source_kind == "gaussian":
            return gaussian_pulse(n, self.sigma_steps, self.amp)
        if self.source_kind == "ricker":
            return ricker(n, self.dt, self.f0, self.amp)
        raise ValueError(self.source_kind)

    def cell_type(self) -> np.ndarray:
        return np.zeros(self.cells, dtype=np.uint8)

    def plate_active(self) -> np.ndarray:
        return np.zeros(self.nx * self.ny, dtype=np.uint8)

    def describe(self) -> dict:
        return {"grid": [self.nx, self.ny, self.nz], "steps": self.n_steps, "src": list(self.src),
                "receivers": [list(r) for r in self.receivers],
                "absorption": [float(a) for a in self.absorption], "source": self.source_kind,
                "dx": self.dx, "n_pml": self.n_pml}


def gaussian_room_64(a: float = 0.1, n_steps: int = 2000) -> Room:
    """64^3 room, Gaussian source (sigma 8 steps) at (16,20,24), receiver at (48,40,32)."""
    return Room(64, 64, 64, n_steps, (16, 20, 24), [(48, 40, 32)], (a,) * 6, "gaussian",
                name="room64_gaussian")


def _interior(rng: np.random.Generator, n: int, n_pml: int) -> int:
    lo, hi = n_pml + 2, n - n_pml - 2
    if lo >= hi:           # grid thinner than its absorbing layers: any cell
        lo, hi = 0, n
    return int(rng.integers(lo, hi))


def seeded_room(nx: int, ny: int, nz: int, n_steps: int, seed: int, n_rec: int = 8,
                source_kind: str = "ricker", n_pml: int = 10,
                a_range: Tuple[float, float] = (0.02, 0.3)) -> Room:
    """Per-face absorption ~ U[a_range], seeded interior source cell and receivers."""
    rng = np.random.default_rng(seed)
    a6 = tuple(float(v) for v in rng.uniform(a_range[0], a_range[1], 6).astype(np.float32))
    src = tuple(_interior(rng, d, n_pml) for d in (nx, ny, nz))
    recs = [tuple(_interior(rng, d, n_pml) for d in (nx, ny, nz)) for _ in range(n_rec)]
    return Room(nx, ny, nz, n_steps, src, recs, a6, source_kind, n_pml=n_pml,
                name=f"room{nx}x{ny}x{nz}_seed{seed}")


def large_room(n_steps: int = 10000, seed: int = 2) -> Room:
    """512x384x256 room (50.3M cells), Ricker 1 kHz, 8 receivers, a_f ~ U[0.02, 0.3]."""
    r = seeded_room(512, 384, 256, n_steps, seed, n_rec=8, source_kind="ricker")
    r.name = "room512x384x256_ricker"
    return r


def rel_l2(x: np.ndarray, ref: np.ndarray) -> float:
    """||x - ref||_2 / ||ref||_2 in float64 (0 when both are zero)."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = float(np.linalg.norm(ref))
    num = float(np.linalg.norm(x - ref))
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return num / den
