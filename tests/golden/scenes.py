"""Deterministic test scenes and the driver that runs them on any implementation.

A scene exercises every branch of the reference path that the open rooms do
not: rigid walls (FDTD_WALL), an active Kirchhoff plate (FDTD_PLATE) with a
soundhole, cut-cell face fractions, bridge sources and drives, plate forces,
point deposits into open and solid cells, fractional-coordinate samplers and
the plate samplers.  ``drive_scene`` calls only the method surface shared by
the reference (oracle/_ref), the restatement (oracle/) and the CUDA engine, so
the same inputs reach all three.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

AIR, WALL, PLATE = 0, 1, 2


@dataclass
class Scene:
    nx: int
    ny: int
    nz: int
    dx: float
    n_pml: int
    plate_iz: int
    cell_type: np.ndarray      # (nx*ny*nz,) uint8
    plate_active: np.ndarray   # (nx*ny,) uint8
    fracs: tuple               # (vx, vy, vz) float32 flat, or None
    bridge_idx: np.ndarray     # int32
    bridge_wgt: np.ndarray     # float32
    point_cells: tuple         # flat cells for point deposits (one open, one solid)
    rec_xyz: np.ndarray        # (n, 3) float32 fractional grid coordinates
    plate_idx4: np.ndarray     # (n*4,) int32
    plate_wgt4: np.ndarray     # (n*4,) float32
    force_idx: np.ndarray      # plate nodes for inject_plate_force
    force_wgt: np.ndarray
    seed: int

    def kwargs(self):
        return dict(Nx=self.nx, Ny=self.ny, Nz=self.nz, dx=self.dx, c=343.0, rho_air=1.21,
                    cell_type=self.cell_type, plate_iz=self.plate_iz,
                    plate_active=self.plate_active, n_pml=self.n_pml)


def body_scene(nx: int = 24, ny: int = 20, nz: int = 16, seed: int = 0, dx: float = 0.01,
               n_pml: int = 3) -> Scene:
    """A closed body below a plate: back wall, rib walls, plate with a soundhole."""
    rng = np.random.default_rng(seed)
    ct = np.zeros((nx, ny, nz), np.uint8)
    back, piz = 3, nz - 5
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    ci, cj = (nx - 1) / 2.0, (ny - 1) / 2.0
    ri, rj = nx * 0.32, ny * 0.32
    inside = ((ii - ci) / ri) ** 2 + ((jj - cj) / rj) ** 2 < 1.0
    for k in range(back, piz + 1):
        ct[:, :, k][~inside & (np.abs(ii - ci) < ri + 2) & (np.abs(jj - cj) < rj + 2)] = WALL
    ct[:, :, back][inside] = WALL
    ct[:, :, piz][inside] = PLATE
    hole = ((ii - ci) ** 2 + (jj - (cj + rj * 0.35)) ** 2) < 2.5 ** 2
    plate_active = (inside & ~hole).astype(np.uint8)
    ct[:, :, piz][hole & inside] = PLATE          # reverted to air by the plate mask rule
    ct_flat = ct.ravel()

    solid = (ct == WALL) | (ct == PLATE)
    solid[:, :, piz] = (ct[:, :, piz] == WALL) | plate_active.astype(bool)

    def face_fracs(a, b, shape_axis):
        f = np.where(a | b, 0.0, 1.0).astype(np.float32)
        bd = a ^ b
        f[bd] = rng.choice(np.array([0.0, 0.25, 0.5, 0.75], np.float32), size=int(bd.sum()))
        return f

    vx = face_fracs(solid[:-1], solid[1:], 0)
    vy = face_fracs(solid[:, :-1], solid[:, 1:], 1)
    vz = face_fracs(solid[:, :, :-1], solid[:, :, 1:], 2)
    pa = plate_active.astype(bool)
    vz[:, :, piz - 1][pa] = 1.0
    vz[:, :, piz][pa] = 1.0

    # bridge kernel: Gaussian weights in the layer just below the plate
    bi, bj = int(ci), int(cj - rj * 0.4)
    b_idx, b_w = [], []
    for i in range(nx):
        for j in range(ny):
            r2 = (i - bi) ** 2 + (j - bj) ** 2
            w = math.exp(-r2 / (2 * 1.5 ** 2))
            if w >= 1e-3:
                b_idx.append((piz - 1) + nz * (j + ny * i))
                b_w.append(w)
    open_cell = (piz + 2) + nz * (int(cj) + ny * int(ci))
    solid_cell = back + nz * (int(cj) + ny * int(ci))
    rec = np.array([[ci + 0.3, cj - 1.7, piz + 2.25], [2.5, 3.75, 1.5], [nx - 1.0, ny + 3.0, -2.0],
                    [ci, cj, piz - 1.5]], np.float32)
    # plate samplers: bilinear at two points
    idx4, w4 = [], []
    for (x, y) in ((ci + 0.4, cj - 0.6), (ci - 2.25, cj + 1.5)):
        i0, j0 = int(x), int(y)
        fi, fj = x - i0, y - j0
        idx4 += [i0 * ny + j0, (i0 + 1) * ny + j0, i0 * ny + j0 + 1, (i0 + 1) * ny + j0 + 1]
        w4 += [(1 - fi) * (1 - fj), fi * (1 - fj), (1 - fi) * fj, fi * fj]
    f_idx = np.array([int(ci + 2) * ny + int(cj), int(ci - 3) * ny + int(cj + 1), -5,
                      int(ci) * ny + int(cj + rj * 0.35)], np.int32)
    f_w = np.array([0.5, 0.3, 0.1, 0.2], np.float32)
    return Scene(nx, ny, nz, dx, n_pml, piz, ct_flat, plate_active.ravel(),
                 (vx.ravel(), vy.ravel(), vz.ravel()),
                 np.array(b_idx, np.int32), np.array(b_w, np.float32), (open_cell, solid_cell),
                 rec, np.array(idx4, np.int32), np.array(w4, np.float32), f_idx, f_w, seed)


def drive_scene(f, sc: Scene, n_steps: int, use_fracs: bool = True):
    """Run ``n_steps`` of the scene; returns a dict of per-step samples."""
    if use_fracs:
        f.set_face_fractions(*sc.fracs)
    f.set_bridge_sources(sc.bridge_idx, sc.bridge_wgt)
    p_idx, p_w = f.precompute_pressure_samplers(sc.rec_xyz)
    v_s = f.precompute_velocity_samplers(sc.rec_xyz)
    n_src = sc.bridge_idx.size
    tr_p, tr_v, tr_w, tr_pw = [], [], [], []
    for n in range(n_steps):
        drv = (0.2 * math.sin(2 * math.pi * n / 37.0) * np.linspace(0.5, 1.5, n_src)).astype(np.float32)
        f.inject_bridge_drive(drv, 1.0)
        if n % 5 == 0:
            f.inject_plate_force(sc.force_idx, sc.force_wgt, 0.05 * math.cos(n / 11.0))
        if n < 40:
            f.add_pressure(sc.point_cells[0], 0.5 * math.exp(-0.5 * ((n - 12) / 4.0) ** 2))
            f.add_pressure(sc.point_cells[1], -0.25 * math.exp(-0.5 * ((n - 20) / 5.0) ** 2))
        f.step(1)
        tr_p.append(f.sample_pressure_precomputed(p_idx, p_w))
        tr_v.append(np.stack(f.sample_velocity_precomputed(*v_s)))
        tr_w.append(f.sample_plate_displacement_batch(sc.plate_idx4, sc.plate_wgt4))
        tr_pw.append(np.float32(f.sample_plate_weighted(sc.force_idx, sc.force_wgt)))
    P_e, vn_e = f.get_surface_emission(sc.rec_xyz, np.tile(np.float32([0.6, 0.0, 0.8]), (len(sc.rec_xyz), 1)))
    vx_s, vy_s, vz_s = f.sample_velocity(sc.rec_xyz)
    return {
        "p_idx8": np.asarray(p_idx, np.int32), "p_wgt8": np.asarray(p_w, np.float32),
        "v_samplers": np.concatenate([np.asarray(a).astype(np.float32).view(np.uint32) if a.dtype != np.int32
                                      else np.asarray(a).view(np.uint32) for a in v_s]),
        "trace_p": np.array(tr_p, np.float32), "trace_v": np.array(tr_v, np.float32),
        "trace_w": np.array(tr_w, np.float32), "trace_pw": np.array(tr_pw, np.float32),
        "P": f.get_pressure_field().ravel().astype(np.float32),
        "Vx": f.get_velocity_x().astype(np.float32), "Vy": f.get_velocity_y().astype(np.float32),
        "Vz": f.get_velocity_z().astype(np.float32),
        "W": f.get_plate_displacement().ravel().astype(np.float32),
        "direct_p": f.sample_pressure(sc.rec_xyz).astype(np.float32),
        "direct_v": np.stack([vx_s, vy_s, vz_s]).astype(np.float32),
        "emission": np.stack([P_e, vn_e]).astype(np.float32),
        "step_count": np.int32(f.step_count),
    }
