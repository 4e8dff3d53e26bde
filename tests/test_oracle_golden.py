"""Pin the oracle: the C restatement reproduces the reference's own outputs bit for bit.

The golden fixtures were produced by the reference's acoustic_fdtd.cpp compiled
unchanged (tests/golden/make_golden.py).  Everything here runs on the CPU.
"""
import hashlib

import numpy as np
import pytest

from conftest import bits_equal, first_mismatch
from oracle import OracleFDTD, reference_available, RefFDTD
from scenes import body_scene, drive_scene
from spectral_analyzer_b200.rooms import gaussian_room_64, seeded_room


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def _room_oracle(room, patched, precision="f32"):
    f = OracleFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, room.cell_type(), -1,
                   room.plate_active(), n_pml=room.n_pml, precision=precision)
    if patched:
        f.set_face_absorption(room.absorption)
    idx, w = f.precompute_pressure_samplers(room.receiver_xyz())
    trace = f.run(room.n_steps, room.src_flat, room.signal(), idx, w)
    return f, trace, idx, w


@pytest.mark.parametrize("tag,a,patched", [("room64_a1", 1.0, False), ("room64_a01", 0.1, True)])
def test_room64_bit_exact(golden, tag, a, patched):
    arrays, meta = golden
    f, trace, idx, w = _room_oracle(gaussian_room_64(a), patched)
    assert np.array_equal(idx, arrays[f"{tag}/idx8"])
    assert bits_equal(w, arrays[f"{tag}/wgt8"])
    assert bits_equal(trace, arrays[f"{tag}/trace"]), first_mismatch(trace, arrays[f"{tag}/trace"])
    h = meta[tag]["sha256"]
    assert sha(f.get_pressure_field()) == h["P"]
    assert sha(f.get_velocity_x()) == h["Vx"]
    assert sha(f.get_velocity_y()) == h["Vy"]
    assert sha(f.get_velocity_z()) == h["Vz"]
    assert sha(f.get_p_damp()) == h["pdamp"]
    assert f.step_count == meta[tag]["step_count"] == 2000


@pytest.mark.parametrize("tag,nx,ny,nz,steps,seed,n_rec,n_pml,override", [
    ("odd37", 37, 29, 23, 300, 7, 3, 4, None),
    ("tiny", 7, 5, 6, 120, 3, 1, 4, ((3, 2, 2), [(5, 3, 4)])),
])
def test_small_rooms_bit_exact(golden, tag, nx, ny, nz, steps, seed, n_rec, n_pml, override):
    arrays, _ = golden
    room = seeded_room(nx, ny, nz, steps, seed=seed, n_rec=n_rec, n_pml=n_pml)
    if override:
        room.src, room.receivers = override
    f, trace, _, _ = _room_oracle(room, True)
    assert bits_equal(trace, arrays[f"{tag}/trace"]), first_mismatch(trace, arrays[f"{tag}/trace"])
    for k, got in (("P", f.get_pressure_field()), ("Vx", f.get_velocity_x()),
                   ("Vy", f.get_velocity_y()), ("Vz", f.get_velocity_z()), ("pdamp", f.get_p_damp())):
        assert bits_equal(got.ravel(), arrays[f"{tag}/{k}"]), (k, first_mismatch(got, arrays[f"{tag}/{k}"]))


@pytest.mark.parametrize("tag,use_fracs,steps", [("body_fracs", True, 300), ("body_nofrac", False, 200)])
def test_body_scene_bit_exact(golden, tag, use_fracs, steps):
    arrays, _ = golden
    sc = body_scene()
    f = OracleFDTD(**sc.kwargs())
    out = drive_scene(f, sc, steps, use_fracs=use_fracs)
    for k, got in out.items():
        ref = arrays[f"{tag}/{k}"]
        if k in ("p_idx8", "v_samplers", "step_count"):
            assert np.array_equal(np.asarray(got), ref), k
        else:
            assert bits_equal(got, ref), (k, first_mismatch(got, ref))


def test_reset_then_continue(golden):
    arrays, meta = golden
    sc = body_scene(seed=1)
    f = OracleFDTD(**sc.kwargs())
    drive_scene(f, sc, 50)
    f.reset()
    out = drive_scene(f, sc, 30)
    assert int(out["step_count"]) == meta["body_reset"]["step_count"]
    for k in ("P", "W", "trace_p"):
        assert bits_equal(out[k], arrays[f"body_reset/{k}"]), k


def test_pressure_instability_code(golden):
    _, meta = golden
    m = meta["unstable_pressure"]
    f = OracleFDTD(16, 16, 16, 0.01, n_pml=2)
    f.add_pressure(m["src"], m["amp"])
    rc = f.step_rc(300)
    assert rc == m["rc"] == -3
    assert f.step_count == m["step_count"] == 256
    assert sha(f.get_pressure_field()) == m["P_sha256"]


def test_plate_guard_code(golden):
    _, meta = golden
    m = meta["unstable_plate"]
    sc = body_scene(seed=2)
    f = OracleFDTD(**sc.kwargs())
    f.set_bridge_sources(sc.bridge_idx, sc.bridge_wgt)
    rcs = []
    for _ in range(60):
        f.inject_bridge_drive(np.full(sc.bridge_idx.size, 5e4, np.float32), 1.0)
        rcs.append(f.step_rc(1))
        if rcs[-1]:
            break
    assert rcs[-1] == m["rc"] == -3
    assert len(rcs) == m["calls"]
    assert f.step_count == m["step_count"]
    assert sha(f.get_plate_displacement()) == m["W_sha256"]


def test_f64_oracle_tracks_f32():
    """The FP64 instantiation runs the same scheme; on a short run it agrees with FP32 closely."""
    room = gaussian_room_64(0.1, n_steps=300)
    _, t32, _, _ = _room_oracle(room, True, "f32")
    _, t64, _, _ = _room_oracle(room, True, "f64")
    err = np.linalg.norm(t32.astype(np.float64) - t64) / np.linalg.norm(t64)
    assert err < 1e-5, err


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built (no reference tree)")
def test_compiled_reference_matches_fixture(golden):
    """The fixture is reproducible from the compiled reference present on this machine."""
    arrays, _ = golden
    room = seeded_room(37, 29, 23, 300, seed=7, n_rec=3, n_pml=4)
    f = RefFDTD(room.nx, room.ny, room.nz, room.dx, n_pml=room.n_pml)
    f.set_face_absorption(room.absorption)
    idx, w = f.precompute_pressure_samplers(room.receiver_xyz())
    trace = f.run(room.n_steps, room.src_flat, room.signal(), idx, w)
    assert bits_equal(trace, arrays["odd37/trace"])


@pytest.mark.parametrize("name,steps", [("large_room_prefix", 500), ("large_room_10000", 10000)])
def test_large_room_fixture_describes_the_bench_room(name, steps):
    """The reference runs of the 512x384x256 room (checked against the engine on
    the GPU) belong to the room the benchmark builds; the 500-step one is the
    prefix of the 10000-step one."""
    import json
    import os
    from spectral_analyzer_b200.rooms import large_room
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with open(os.path.join(here, name + ".json")) as fh:
        meta = json.load(fh)
    with np.load(os.path.join(here, name + ".npz")) as z:
        trace, idx8, wgt8 = z["trace"], z["idx8"], z["wgt8"]
    room = large_room(n_steps=steps)
    assert json.loads(json.dumps(room.describe())) == meta["room"]
    assert trace.shape == (steps, 8) and trace.dtype == np.float32
    assert idx8.size == 64 and wgt8.size == 64
    assert np.abs(trace).max() > 0 and meta["steps"] == steps
    with np.load(os.path.join(here, "large_room_prefix.npz")) as z:
        assert bits_equal(trace[:500], z["trace"])
    # the oracle's samplers are the reference's
    o = OracleFDTD(room.nx, room.ny, room.nz, room.dx, n_pml=room.n_pml)
    idx, w = o.precompute_pressure_samplers(room.receiver_xyz())
    assert np.array_equal(idx, idx8) and bits_equal(w, wgt8)
