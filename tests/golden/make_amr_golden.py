"""Fixture for the AMR backend parity tests: a guitar-body AMR grid built by the
reference's own Python and stepped by the reference's own AMR solver.

The grid and its co-evolver descriptor come from the reference checkout's
``acoustic_amr.build_guitar_amr_grid`` (acoustic_amr.py:642) on the bridge's
default guitar outline (acoustic_fdtd_bridge.py ``_default_guitar_outline``)
with a soundhole, and ``build_amr_coevolver_descriptor`` (acoustic_amr.py:2396)
with the plate geometry the bridge derives for it
(acoustic_fdtd_bridge.py:1305-1328: plate spacing max(base_dx/2, 4 mm), the
outline's bounding box plus two plate cells, bridge saddles at the scene's
default positions).  The stepper is the reference's csrc/kernels/acoustic_amr.cpp
compiled unchanged (oracle/_ref/libamr_ref.so), set up in the order of its
pressure backend (acoustic_pressure_backend.cpp:461-548) plus the microphone
samplers, and driven by tests/amr_script.py.

Cases: gradient order 2 with the anechoic border, order 8 (Fornberg stencil)
with a room-panel border (R = 0.3, quadratic grading), order 2 with the
transmission border; plus a diverging case (a 1e6 Pa deposit) that must stop
at its first check.

    make -C oracle REF=<reference checkout>
    python tests/golden/make_amr_golden.py <reference checkout> [steps]
"""
from __future__ import annotations

import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import amr_script as S  # noqa: E402

GRID_KEYS = ("cell_centers", "cell_volumes", "open_volume_frac", "cell_types", "face_cell_neg",
             "face_cell_pos", "face_area", "face_open_frac", "face_distance", "bounds_min", "bounds_max",
             "plate_origin", "plate_active", "plate_active_flat_idx", "plate_face_above_starts",
             "plate_face_above_idx", "plate_face_above_wgt", "plate_face_below_starts",
             "plate_face_below_idx", "plate_face_below_wgt", "plate_cell_above", "plate_cell_below",
             "bridge_plate_idx", "bridge_plate_wgt", "neck_plate_idx", "neck_plate_wgt")
SCALAR_KEYS = ("n_cells", "n_faces", "c", "rho_air", "min_dx", "plate_Nx", "plate_Ny", "plate_dx",
               "plate_mass_density", "plate_stiffness_D", "plate_alpha_M", "plate_beta_K",
               "n_active_plate", "n_bridge_plate", "n_neck_plate", "n_pml")


def main():
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FDTD_REFERENCE_DIR", "")
    if not ref_dir or not os.path.isfile(os.path.join(ref_dir, "acoustic_amr.py")):
        raise SystemExit("usage: make_amr_golden.py <reference checkout> [steps]")
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else 200
    sys.path.insert(0, ref_dir)
    from amr_oracle import AMRRef
    import acoustic_amr as A
    import acoustic_fdtd_bridge as bridge
    t0 = time.time()
    outline = bridge._default_guitar_outline()
    body_h, soundhole = 0.06, (0.0, 0.05, 0.028)
    base_dx, pad, n_pml = 0.016, 6, 3
    grid = A.build_guitar_amr_grid(outline, body_h, dx=base_dx, pad_cells=pad, n_pml=n_pml,
                                   soundhole=soundhole, max_refinement_level=1)
    plate_dx = max(float(grid.base_dx * 0.5), 0.004)
    margin = 2.0 * plate_dx
    omin, omax = outline.min(axis=0), outline.max(axis=0)
    pmin_x, pmax_x = float(omin[0]) - margin, float(omax[0]) + margin
    pmin_y, pmax_y = float(omin[1]) - margin, float(omax[1]) + margin
    plate_origin = np.array([pmin_x, pmin_y, body_h], np.float32)
    pnx = max(1, math.ceil((pmax_x - pmin_x) / plate_dx))
    pny = max(1, math.ceil((pmax_y - pmin_y) / plate_dx))
    bridge_xyz = np.array([[bx, by, body_h] for bx, by in [(-0.030, -0.070), (0.000, -0.070), (0.030, -0.070)]],
                          np.float32)
    # the descriptor of gradient order 2 (amr_create builds the order-8 stencil itself)
    d = A.build_amr_coevolver_descriptor(
        grid=grid, plate_Nx=pnx, plate_Ny=pny, plate_dx=plate_dx, plate_origin=plate_origin,
        body_h=body_h, plate_mass_density=7.0, plate_stiffness_D=0.45, plate_alpha_M=2.0,
        plate_beta_K=1e-5, bridge_src_xyz=bridge_xyz, bridge_sigma=0.012, gradient_order=2,
        border_spec=A.border_anechoic(3.0), n_pml=n_pml)
    rng = np.random.default_rng(5)
    act = np.asarray(d["plate_active_flat_idx"], np.int32)
    d["neck_plate_idx"] = np.sort(rng.choice(act, 5, replace=False)).astype(np.int32)
    d["neck_plate_wgt"] = rng.uniform(0.1, 0.3, 5).astype(np.float32)
    d["n_neck_plate"] = 5
    print(f"grid: {grid.n_cells} cells, {grid.n_faces} faces, min_dx {grid.min_dx}; plate {pnx}x{pny} "
          f"({int(d['n_active_plate'])} active), {int(d['n_bridge_plate'])} bridge nodes "
          f"({time.time() - t0:.1f} s)", flush=True)
    sc = S.make_script(d, steps)
    # microphones: inside the body, at the soundhole, in the body's side, above the top (clamped by the solver)
    mics = {"pos": np.array([[0.0, -0.02, 0.03], [0.0, 0.05, 0.07], [0.12, -0.1, 0.02], [0.0, 0.0, 0.5]],
                            np.float32),
            "axis": np.array([[0, 0, 1], [0, 0, 1], [1, 0, 0], [0, 0, -1]], np.float32)}
    arrays = {f"grid/{k}": np.ascontiguousarray(d[k]) for k in GRID_KEYS}
    arrays.update({f"script/{k}": v for k, v in sc.items()})
    arrays.update({f"mics/{k}": v for k, v in mics.items()})
    meta = {"steps": steps,
            "grid": {k: (float(d[k]) if isinstance(d[k], float) else int(d[k])) for k in SCALAR_KEYS},
            "builder": {"base_dx": base_dx, "pad_cells": pad, "n_pml": n_pml, "max_refinement_level": 1,
                        "body_h": body_h, "soundhole": list(soundhole)},
            "library": "libamr_ref.so", "cases": {}}
    for name, go, border in S.CASES:
        s = AMRRef(d, gradient_order=go, border=border)
        res = S.run(s, d, sc, mics, steps)
        meta["cases"][name] = {"gradient_order": go, "border": list(border), "dt": s.dt,
                               "step_count": s.step_count,
                               "sha256": {k: S.sha(res[k]) for k in ("P", "V", "W")},
                               "peak_mic_p": float(np.abs(res["mic_p"]).max()),
                               "peak_w": float(np.abs(res["W"]).max())}
        s.close()
        for k in S.RECORDS:
            arrays[f"{name}/{k}"] = res[k]
        print(name, meta["cases"][name], flush=True)
    # divergence: a 1e6 Pa deposit trips the check of the first step
    s = AMRRef(d, gradient_order=2, border=S.CASES[0][2])
    s.inject_pressure_nearest(np.array([0.0, -0.02, 0.03]), 1e6)
    rc = [s.step_rc(1), s.step_rc(1)]
    meta["diverge"] = {"xyz": [0.0, -0.02, 0.03], "value": 1e6, "rc": rc, "step_count": s.step_count,
                       "P_sha256": S.sha(s.get_pressure()), "W_sha256": S.sha(s.get_plate_displacement())}
    s.close()
    print("diverge", meta["diverge"], flush=True)
    np.savez_compressed(S.NPZ, **arrays)
    with open(S.JSON, "w") as fh:
        json.dump(meta, fh, indent=1)
    print(f"wrote {S.NPZ} ({os.path.getsize(S.NPZ) / 1e6:.2f} MB) in {time.time() - t0:.1f} s")


if __name__ == "__main__":
    main()
