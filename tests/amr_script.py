"""The drive script of the AMR parity tests (tests/golden/amr_guitar.*).

One script drives both the compiled reference AMR stepper (oracle/amr_oracle.py)
and the engine's AcousticAMR: per step, per-bridge-node forces (a seeded shape
times a decaying pluck), a neck force, one step, the saddle displacements
(4-tap batch), the neck's weighted displacement and the microphones (pressure
and the three velocity components), as the reference co-evolver's substep
calls its pressure backend (acoustic_coevolver.cpp:2064-2121, :2191-2224).
"""
from __future__ import annotations

import hashlib
import json
import math
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NPZ = os.path.join(HERE, "amr_guitar.npz")
JSON = os.path.join(HERE, "amr_guitar.json")

CASES = [  # name, gradient order, border (mode, sigma order, R, Z)
    ("order2_anechoic", 2, (0, 3.0, 0.0, 0.0)),
    ("order8_room_panel", 8, (1, 2.0, 0.3, 0.0)),
    ("order2_transmission", 2, (2, 3.0, 0.0, 0.0)),
]
RECORDS = ("rc", "mic_p", "mic_vx", "mic_vy", "mic_vz", "saddle", "neck_w")


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make_script(desc, steps, seed=11):
    rng = np.random.default_rng(seed)
    shape = rng.uniform(0.5, 1.5, int(desc["n_bridge_plate"])).astype(np.float32)
    drive = np.zeros(steps, np.float64)
    for n in range(steps):
        t = n * 2.0e-5
        drive[n] = 0.6 * math.exp(-t * 150.0) * (math.sin(2 * math.pi * 196.0 * t) +
                                                 0.5 * math.sin(2 * math.pi * 392.0 * t))
        if n < 30:
            drive[n] += 1.5 * (1.0 - n / 30.0)
    act = np.asarray(desc["plate_active_flat_idx"], np.int32)
    saddle_idx4 = np.sort(rng.choice(act, 8, replace=False)).astype(np.int32)
    return {"bridge_shape": shape, "drive": drive, "saddle_idx4": saddle_idx4,
            "saddle_w4": np.full(8, 0.25, np.float32)}


def run(solver, desc, sc, mics, steps):
    """Drive one solver; returns the per-step records and the final fields."""
    assert solver.setup_mic_samplers(mics["pos"], mics["axis"], True) == 0
    neck_idx = np.asarray(desc["neck_plate_idx"], np.int32)
    neck_wgt = np.asarray(desc["neck_plate_wgt"], np.float32)
    rec = {k: [] for k in RECORDS}
    for n in range(steps):
        d = (sc["drive"][n] * sc["bridge_shape"]).astype(np.float32)
        assert solver.inject_bridge_drive(d, 1.0) == 0
        assert solver.inject_plate_force(neck_idx, neck_wgt, np.float32(0.05 * sc["drive"][n])) == 0
        rec["rc"].append(solver.step_rc(1))
        rec["saddle"].append(solver.sample_plate_displacement_batch(sc["saddle_idx4"], sc["saddle_w4"]))
        rec["neck_w"].append(np.float32(solver.sample_plate_weighted(neck_idx, neck_wgt)))
        for k, v in zip(("mic_p", "mic_vx", "mic_vy", "mic_vz"), solver.sample_mics()):
            rec[k].append(v)
    out = {k: np.asarray(v) for k, v in rec.items()}
    out["P"], out["V"], out["W"] = solver.get_pressure(), solver.get_velocity(), solver.get_plate_displacement()
    return out


def load():
    with open(JSON) as fh:
        meta = json.load(fh)
    with np.load(NPZ) as z:
        arrays = {k: z[k] for k in z.files}
    desc = dict(meta["grid"])
    desc.update({k[5:]: v for k, v in arrays.items() if k.startswith("grid/")})
    sc = {k[7:]: v for k, v in arrays.items() if k.startswith("script/")}
    mics = {k[5:]: v for k, v in arrays.items() if k.startswith("mics/")}
    return meta, arrays, desc, sc, mics
