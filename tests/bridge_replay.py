"""Replay of the reference bridge's recorded solver calls (tests/golden/bridge_replay.*).

tests/golden/make_bridge_golden.py ran the reference's unmodified
acoustic_fdtd_bridge.py (``FDTDCoEvolver.from_body_scene`` on its string_plate
body scene, a seeded pluck through ``coev.fdtd``, ``sample_at_receivers`` and
the field accessors) over the compiled reference and logged every call the
bridge and the driving loop made on the solver, with the arguments and the
results.  ``replay`` makes the same calls, in the same order and with the same
positional and keyword arguments, on another ``AcousticFDTD`` class and checks
every result against the log.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NPZ = os.path.join(HERE, "bridge_replay.npz")
JSON = os.path.join(HERE, "bridge_replay.json")


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def load():
    with open(JSON) as fh:
        meta = json.load(fh)
    with np.load(NPZ) as z:
        arrays = {k: z[k] for k in z.files}
    return meta, arrays


def decode(v, arrays):
    if isinstance(v, dict):
        if "array" in v:
            return arrays[v["array"]].copy()
        if "scaled" in v:                      # drive vector = float32(scale * base)
            out = (v["by"] * arrays[v["scaled"]]).astype(np.float32)
            assert sha(out) == v["sha256"], "drive vector reconstruction differs"
            return out
        if "float32" in v:
            return np.float32(v["float32"])
        if "tuple" in v:
            return tuple(decode(x, arrays) for x in v["tuple"])
    return v


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def _mismatch(a, b) -> str:
    a = np.ascontiguousarray(a, dtype=np.float32).ravel()
    b = np.ascontiguousarray(b, dtype=np.float32).ravel()
    if a.size != b.size:
        return f"size {a.size} vs {b.size}"
    q = np.nonzero(a.view(np.uint32) != b.view(np.uint32))[0]
    return f"{q.size} of {a.size} differ; first at {q[0]}: {a[q[0]]!r} vs {b[q[0]]!r}"


def replay(cls, meta, arrays, on_result=None):
    """Make the logged calls on ``cls``; returns (solver, list of mismatches).

    ``on_result(entry, result)`` sees every result (e.g. to collect traces)."""
    calls = meta["calls"]
    assert calls[0]["m"] == "__init__"
    ini = calls[0]
    f = cls(*[decode(a, arrays) for a in ini["args"]],
            **{k: decode(v, arrays) for k, v in ini["kwargs"].items()})
    bad = []
    for n, c in enumerate(calls[1:], start=1):
        args = [decode(a, arrays) for a in c["args"]]
        kwargs = {k: decode(v, arrays) for k, v in c["kwargs"].items()}
        out = getattr(f, c["m"])(*args, **kwargs)
        if on_result is not None:
            on_result(c, out)
        if "result_sha256" in c:
            if list(np.shape(out)) != c["result_shape"] or sha(out) != c["result_sha256"]:
                bad.append((n, c["m"], "field hash"))
            continue
        want = decode(c.get("result"), arrays)
        if isinstance(want, np.ndarray):
            if not bits_equal(out, want):
                bad.append((n, c["m"], _mismatch(out, want)))
        elif isinstance(want, np.floating):
            if not bits_equal(np.float32(out), want):
                bad.append((n, c["m"], f"{out!r} vs {want!r}"))
        elif want is not None and out != want:
            bad.append((n, c["m"], f"{out!r} vs {want!r}"))
    return f, bad


def bridge_slices(P, meta):
    """The slices the bridge took of the final field: get_volume_slice(2, -1),
    (0, 10), (1, Ny // 3) and get_soundboard_pressure (acoustic_fdtd_bridge.py:737-759)."""
    ny = P.shape[1]
    return [P[:, :, P.shape[2] // 2], P[10, :, :], P[:, ny // 3, :], P[:, :, meta["plate_iz"]]]
