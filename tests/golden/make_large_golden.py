"""Golden prefix of the 512x384x256 room from the reference's own FDTD.

The bench workload (50.3M cells, per-face absorption, Ricker source, 8
receivers) run for 500 steps by csrc/kernels/acoustic_fdtd.cpp compiled
unchanged by oracle/Makefile (oracle/_ref/libfdtd_ref.so with the deposit and
per-face absorption hooks of oracle/ref_shim.cpp), here on the host cores
(about four minutes on 8 threads; the full 10000-step run about 80).  Run
from the repository root:

    make -C oracle REF=<reference checkout> && python tests/golden/make_large_golden.py [steps]

Writes tests/golden/large_room_prefix.npz (the steps x 8 receiver traces and
the sampler taps) and tests/golden/large_room_prefix.json (SHA-256 of the
final P, Vx, Vy, Vz and the room's description) for the default 500 steps,
large_room_<steps>.npz / .json otherwise.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import RefFDTD  # noqa: E402
from spectral_analyzer_b200.rooms import large_room  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
N_STEPS = 500


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def main():
    steps = int(sys.argv[1]) if len(sys.argv) > 1 else N_STEPS
    name = "large_room_prefix" if steps == N_STEPS else f"large_room_{steps}"
    room = large_room(n_steps=steps)
    t0 = time.time()
    f = RefFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, room.cell_type(), -1,
                room.plate_active(), n_pml=room.n_pml)
    f.set_face_absorption(room.absorption)
    idx, w = f.precompute_pressure_samplers(room.receiver_xyz())
    trace = f.run(room.n_steps, room.src_flat, room.signal(), idx, w)
    meta = {"room": room.describe(), "steps": int(f.step_count), "library": os.path.basename(f.library_path),
            "sha256": {"P": sha(f.get_pressure_field()), "Vx": sha(f.get_velocity_x()),
                       "Vy": sha(f.get_velocity_y()), "Vz": sha(f.get_velocity_z())},
            "trace_abs_max": float(np.abs(trace).max()), "seconds": round(time.time() - t0, 1)}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), trace=trace, idx8=idx, wgt8=w)
    with open(os.path.join(HERE, name + ".json"), "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
