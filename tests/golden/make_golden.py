"""Generate the golden fixtures from the reference's own FDTD.

The reference has no test, golden vector or known answer for this path, so the
fixtures are outputs of the reference itself: csrc/kernels/acoustic_fdtd.cpp
compiled unchanged by oracle/Makefile (oracle/_ref/libfdtd_ref.so, plus the
deposit and per-face absorption hooks of oracle/ref_shim.cpp), run here on
seeded inputs.  Run from the repository root:

    make -C oracle REF=<reference checkout> && python tests/golden/make_golden.py

Writes tests/golden/reference_fixtures.npz (arrays) and
tests/golden/reference_fixtures.json (SHA-256 of large final fields, return
codes, step counts).  Small cases keep full final fields; large ones keep the
receiver traces plus field hashes.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from oracle import RefFDTD  # noqa: E402
from scenes import body_scene, drive_scene  # noqa: E402
from spectral_analyzer_b200.rooms import gaussian_room_64, seeded_room  # noqa: E402

OUT_NPZ = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_fixtures.npz")
OUT_JSON = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_fixtures.json")


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def room_case(room, patched: bool):
    f = RefFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, room.cell_type(), -1,
                room.plate_active(), n_pml=room.n_pml)
    if patched:
        f.set_face_absorption(room.absorption)
    idx, w = f.precompute_pressure_samplers(room.receiver_xyz())
    trace = f.run(room.n_steps, room.src_flat, room.signal(), idx, w)
    fields = {"P": f.get_pressure_field().ravel(), "Vx": f.get_velocity_x(),
              "Vy": f.get_velocity_y(), "Vz": f.get_velocity_z(), "pdamp": f.get_p_damp()}
    return trace, fields, idx, w, f.step_count


def main():
    arrays, meta = {}, {}

    # open rooms: the 64^3 Gaussian room, unmodified (a=1) and with a=0.1 on all faces
    for tag, a, patched in (("room64_a1", 1.0, False), ("room64_a01", 0.1, True)):
        room = gaussian_room_64(a)
        trace, fields, idx, w, sc = room_case(room, patched)
        arrays[f"{tag}/trace"] = trace
        arrays[f"{tag}/idx8"] = idx
        arrays[f"{tag}/wgt8"] = w
        meta[tag] = {"room": room.describe(), "step_count": sc,
                     "sha256": {k: sha(v) for k, v in fields.items()},
                     "P_absmax": float(np.abs(fields["P"]).max())}
        print(tag, "trace absmax", float(np.abs(trace).max()), "steps", sc)

    # odd-sized seeded room, n_pml 4, Ricker, 3 receivers
    room = seeded_room(37, 29, 23, 300, seed=7, n_rec=3, n_pml=4)
    trace, fields, idx, w, sc = room_case(room, True)
    arrays["odd37/trace"] = trace
    for k, v in fields.items():
        arrays[f"odd37/{k}"] = v
    meta["odd37"] = {"room": room.describe(), "step_count": sc}

    # overlapping PML zones (N < 2*n_pml on every axis)
    room = seeded_room(7, 5, 6, 120, seed=3, n_rec=1, n_pml=4)
    room.src, room.receivers = (3, 2, 2), [(5, 3, 4)]
    trace, fields, idx, w, sc = room_case(room, True)
    arrays["tiny/trace"] = trace
    for k, v in fields.items():
        arrays[f"tiny/{k}"] = v
    meta["tiny"] = {"room": room.describe(), "step_count": sc}

    # body scenes: walls + plate + soundhole + bridge, with and without cut-cell fractions
    for tag, use_fracs, steps in (("body_fracs", True, 300), ("body_nofrac", False, 200)):
        sc = body_scene()
        f = RefFDTD(**sc.kwargs())
        out = drive_scene(f, sc, steps, use_fracs=use_fracs)
        for k, v in out.items():
            arrays[f"{tag}/{k}"] = np.asarray(v)
        meta[tag] = {"steps": steps, "use_fracs": use_fracs,
                     "trace_p_absmax": float(np.abs(out["trace_p"]).max()),
                     "W_absmax": float(np.abs(out["W"]).max())}
        print(tag, "p absmax", meta[tag]["trace_p_absmax"], "w absmax", meta[tag]["W_absmax"])

    # reset mid-run then continue
    sc = body_scene(seed=1)
    f = RefFDTD(**sc.kwargs())
    drive_scene(f, sc, 50)
    f.reset()
    out = drive_scene(f, sc, 30)
    arrays["body_reset/P"] = out["P"]
    arrays["body_reset/W"] = out["W"]
    arrays["body_reset/trace_p"] = out["trace_p"]
    meta["body_reset"] = {"step_count": int(out["step_count"])}

    # pressure instability: returns -3 at the first 256-step check
    room = seeded_room(16, 16, 16, 300, seed=1, n_rec=1, n_pml=2)
    f = RefFDTD(16, 16, 16, 0.01, n_pml=2)
    f.add_pressure(room.src_flat, 1e9)
    rc = f.step_rc(300)
    meta["unstable_pressure"] = {"src": room.src_flat, "amp": 1e9, "rc": rc, "step_count": f.step_count,
                                 "P_sha256": sha(f.get_pressure_field().ravel())}
    print("unstable pressure rc", rc, "at step", f.step_count)

    # plate guard: a huge bridge drive trips |w| > 0.02 m
    sc = body_scene(seed=2)
    f = RefFDTD(**sc.kwargs())
    f.set_bridge_sources(sc.bridge_idx, sc.bridge_wgt)
    rcs = []
    for n in range(60):
        f.inject_bridge_drive(np.full(sc.bridge_idx.size, 5e4, np.float32), 1.0)
        rc = f.step_rc(1)
        rcs.append(rc)
        if rc:
            break
    meta["unstable_plate"] = {"rc": rcs[-1], "calls": len(rcs), "step_count": f.step_count,
                              "W_sha256": sha(f.get_plate_displacement().ravel())}
    print("plate guard rc", rcs[-1], "after", len(rcs), "calls; step", f.step_count)

    np.savez_compressed(OUT_NPZ, **arrays)
    with open(OUT_JSON, "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)
    print("wrote", OUT_NPZ, os.path.getsize(OUT_NPZ), "bytes")


if __name__ == "__main__":
    main()
