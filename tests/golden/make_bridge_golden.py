"""Fixture for the bridge replay tests: the reference's own Python bridge driving
the compiled reference solver, every solver call recorded.

The unmodified ``acoustic_fdtd_bridge.py`` of the reference checkout is imported
with a recording ``_spectral_kernels`` module in ``sys.modules``.  Its
``AcousticFDTD`` has the pybind class's surface (csrc/bindings/pybind_kernels.cpp:
8924-9022; fields returned as (Nx, Ny, Nz) / (Nx, Ny) arrays) over the reference's
``acoustic_fdtd.cpp`` compiled unchanged (oracle/_ref/libfdtd_ref.so), and it logs
each call with its arguments and results.  Then:

* ``FDTDCoEvolver.from_body_scene`` (acoustic_fdtd_bridge.py:647-699) on the
  reference's own ``string_plate`` body scene
  (sm_plugins/orchestral_resonance.py ``_build_body_scene``) at the bridge's
  defaults (dx 4 mm, pad 12 cells, n_pml 10): ``_extract_guitar_geometry``,
  ``voxelise_guitar_body`` (:255-359), ``_apply_soundhole_cutout`` (:411-421),
  the solver constructor, ``compute_cut_cell_fractions`` (:456-552) and
  ``set_face_fractions``, ``build_bridge_kernel`` (:559-599) and
  ``set_bridge_sources``;
* a seeded pluck through ``coev.fdtd`` the way the co-evolver's substep drives
  it (acoustic_coevolver.cpp:2064-2121): per-bridge-cell forces
  (``inject_bridge_drive``), a neck force on plate cells
  (``inject_plate_force``), ``step(1)``, the saddle displacement
  (``sample_plate_displacement_batch``); once per audio sample (the bridge's
  ``steps_per_sample`` substeps) the microphones through the bridge's
  ``sample_at_receivers`` (:761-779);
* at the end the bridge's field accessors: ``get_volume_slice`` (:737-757) on
  all three axes, ``get_soundboard_pressure``, ``get_plate_displacement``, and
  the four fields.

The fixture (bridge_replay.npz + bridge_replay.json) holds the call log: the
bridge-made inputs (cell types, plate mask, face fractions, bridge kernel,
receiver grid coordinates, drive vectors) and every result.  The replay tests
run the same calls on the GPU engine through its ``_spectral_kernels`` shim and
on the C restatement.

    make -C oracle REF=<reference checkout>
    python tests/golden/make_bridge_golden.py <reference checkout> [steps]
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT_NPZ = os.path.join(HERE, "bridge_replay.npz")
OUT_JSON = os.path.join(HERE, "bridge_replay.json")


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


class CallLog:
    """Calls in order: name, positional/keyword arguments and the result.

    Arrays go to the npz under a generated key (identical arrays once); the
    JSON entry names the key.  A drive vector is recorded as its scale and base
    vector when ``scaled`` says how it was made."""

    def __init__(self):
        self.calls = []
        self.arrays = {}
        self._seen = {}
        self.scaled = None

    def _enc(self, v, tag):
        if isinstance(v, np.ndarray):
            v = np.ascontiguousarray(v)
            if self.scaled is not None and tag.startswith("inject_bridge_drive_arg0"):
                scale, base = self.scaled
                assert np.array_equal((scale * self.arrays[base]).astype(np.float32).view(np.uint32),
                                      v.astype(np.float32).view(np.uint32))
                return {"scaled": base, "by": scale, "sha256": sha(v)}
            h = hashlib.sha256(v.tobytes() + str((v.dtype, v.shape)).encode()).hexdigest()
            if h in self._seen:
                return {"array": self._seen[h]}
            key = f"a{len(self.arrays):05d}_{tag}"
            self.arrays[key] = v
            self._seen[h] = key
            return {"array": key}
        if isinstance(v, (np.floating, float)):
            return {"float32": float(np.float32(v))}
        if isinstance(v, (np.integer, int)):
            return int(v)
        if isinstance(v, tuple):
            return {"tuple": [self._enc(x, f"{tag}{q}") for q, x in enumerate(v)]}
        if v is None:
            return None
        raise TypeError(f"cannot record {type(v)}")

    def add(self, name, args, kwargs, result, store_result=True):
        entry = {"m": name,
                 "args": [self._enc(a, f"{name}_arg{q}") for q, a in enumerate(args)],
                 "kwargs": {k: self._enc(v, f"{name}_{k}") for k, v in kwargs.items()}}
        if store_result:
            entry["result"] = self._enc(result, f"{name}_out")
        elif isinstance(result, np.ndarray):
            entry["result_sha256"] = sha(result)
            entry["result_shape"] = list(result.shape)
        self.calls.append(entry)


LOG = CallLog()


def make_recording_module(ref_fdtd_cls):
    """A ``_spectral_kernels`` module whose AcousticFDTD records every call."""

    class AcousticFDTD:
        def __init__(self, *args, **kwargs):
            names = ["Nx", "Ny", "Nz", "dx", "c", "rho_air", "cell_type", "plate_iz",
                     "plate_active", "plate_mass_density", "plate_stiffness_D",
                     "plate_alpha_M", "plate_beta_K", "n_pml"]
            kw = dict(zip(names, args))
            kw.update(kwargs)
            rec = {k: (np.ascontiguousarray(v, np.uint8) if k in ("cell_type", "plate_active")
                       else v) for k, v in kw.items()}
            self._s = ref_fdtd_cls(**rec)
            self._plate_active = rec["plate_active"].ravel().copy()
            LOG.add("__init__", args, kwargs, None)

        def __getattr__(self, name):
            if name in ("dt", "step_count", "Nx", "Ny", "Nz"):
                return getattr(self._s, name)
            fn = getattr(self._s, name)

            def call(*args, **kwargs):
                out = fn(*args, **kwargs)
                big = name in ("get_pressure_field", "get_velocity_x", "get_velocity_y",
                               "get_velocity_z")
                LOG.add(name, args, kwargs, out, store_result=not big)
                return out
            return call

    mod = types.ModuleType("_spectral_kernels")
    mod.AcousticFDTD = AcousticFDTD
    return mod


def main():
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FDTD_REFERENCE_DIR", "")
    if not ref_dir or not os.path.isfile(os.path.join(ref_dir, "acoustic_fdtd_bridge.py")):
        raise SystemExit("usage: make_bridge_golden.py <reference checkout> [steps]")
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else 300
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefFDTD
    sys.modules["_spectral_kernels"] = make_recording_module(RefFDTD)
    sys.path.insert(0, ref_dir)
    t0 = time.time()
    import acoustic_fdtd_bridge as bridge
    from sm_plugins.orchestral_resonance import _build_body_scene

    scene = _build_body_scene("string_plate")
    coev = bridge.FDTDCoEvolver.from_body_scene(scene)
    f = coev.fdtd
    info = coev.info
    Nx, Ny, Nz = info["Nx"], info["Ny"], info["Nz"]
    K = coev.steps_per_sample
    print(f"grid {Nx}x{Ny}x{Nz}, plate_iz {info['plate_iz']}, dt {coev.dt:.4e}, "
          f"{K} steps per sample ({time.time() - t0:.1f} s set-up)", flush=True)

    # seeded pluck: per-bridge-cell forces (a decaying 196 Hz partial sum), a neck
    # force on a few plate cells, two saddle read-outs, three microphones in the
    # bridge's world frame (metres)
    rng = np.random.default_rng(42)
    bidx, bwgt = bridge.build_bridge_kernel(coev._bridge_positions, info)
    share = (bwgt / np.sum(np.abs(bwgt))).astype(np.float32)
    share_key = "bridge_share"
    LOG.arrays[share_key] = share
    plate_cells = np.flatnonzero(f._plate_active)       # the mask the bridge built
    neck = np.sort(rng.choice(plate_cells, 6, replace=False)).astype(np.int32)
    neck_w = rng.uniform(0.5, 1.0, neck.size).astype(np.float32)
    saddle_idx4 = (bidx[:8] // Nz).astype(np.int32).reshape(2, 4)
    saddle_w4 = np.full((2, 4), 0.25, np.float32)
    mics = np.array([[0.0, 0.35, 0.03], [0.12, -0.05, 0.15], [-0.05, 0.05, 0.02]], np.float32)
    for n in range(steps):
        t = n * coev.dt
        drive = 0.8 * math.exp(-t * 200.0) * (math.sin(2 * math.pi * 196.0 * t) +
                                               0.5 * math.sin(2 * math.pi * 392.0 * t))
        if n < 40:
            drive += 2.0 * (1.0 - n / 40.0)     # the pluck's release
        LOG.scaled = (drive, share_key)     # recorded as drive x share (float32 product)
        f.inject_bridge_drive((drive * share).astype(np.float32), 1.0)
        LOG.scaled = None
        f.inject_plate_force(neck, neck_w, np.float32(0.05 * drive))
        f.step(1)
        f.sample_plate_displacement_batch(saddle_idx4.ravel(), saddle_w4.ravel())
        if (n + 1) % K == 0:
            coev.sample_at_receivers(mics)
    slices = [coev.get_volume_slice(2, -1), coev.get_volume_slice(0, 10),
              coev.get_volume_slice(1, Ny // 3), coev.get_soundboard_pressure()]
    w = coev.get_plate_displacement()
    fields = {"P": sha(f.get_pressure_field()), "Vx": sha(f.get_velocity_x()),
              "Vy": sha(f.get_velocity_y()), "Vz": sha(f.get_velocity_z())}
    arrays = dict(LOG.arrays)
    for q, s in enumerate(slices):
        arrays[f"bridge_slice{q}"] = np.ascontiguousarray(s, np.float32)
    arrays["bridge_plate_w"] = np.ascontiguousarray(w, np.float32)
    np.savez_compressed(OUT_NPZ, **arrays)
    mic_trace = [c["result"] for c in LOG.calls if c["m"] == "sample_pressure"]
    meta = {"library": "libfdtd_ref.so", "steps": steps, "grid": [Nx, Ny, Nz],
            "dx": info["dx"], "plate_iz": info["plate_iz"], "steps_per_sample": K,
            "bridge_cells": int(bidx.size), "neck_cells": neck.tolist(),
            "slices": ["get_volume_slice(2, -1)", "get_volume_slice(0, 10)",
                       f"get_volume_slice(1, {Ny // 3})", "get_soundboard_pressure()"],
            "fields_sha256": fields, "calls": LOG.calls, "seconds": round(time.time() - t0, 1),
            "mic_samples": len(mic_trace),
            "peak_plate_w": float(np.abs(w).max()),
            "peak_P": float(np.abs(arrays[mic_trace[-1]["array"]]).max()) if mic_trace else 0.0}
    with open(OUT_JSON, "w") as fh:
        json.dump(meta, fh, separators=(",", ":"))
    print(f"{len(LOG.calls)} calls, {len(mic_trace)} microphone samples, peak |w| "
          f"{meta['peak_plate_w']:.3e} m; {time.time() - t0:.1f} s; wrote {OUT_NPZ}", flush=True)


if __name__ == "__main__":
    main()
