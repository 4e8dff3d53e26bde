"""fdtd_b200_substep equals the co-evolver's four calls (inject_bridge_drive,
inject_plate_force, step(1), sample_plate_displacement_batch) bit for bit,
including the step where the plate guard fires and the state it leaves."""
import math

import numpy as np
import pytest

from conftest import bits_equal, first_mismatch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch


def make(sc, receivers=True):
    from spectral_analyzer_b200 import AcousticFDTD
    f = AcousticFDTD(**sc.kwargs())
    f.set_face_fractions(*sc.fracs)
    f.set_bridge_sources(sc.bridge_idx, sc.bridge_wgt)
    if receivers:
        idx, w = f.precompute_pressure_samplers(sc.rec_xyz)
        f.set_receivers(idx, w, 1000)
    return f


def drives(sc, n, amp):
    return (amp * math.sin(2 * math.pi * n / 37.0) * np.linspace(0.5, 1.5, sc.bridge_idx.size)).astype(np.float32)


def sequence(f, sc, n, amp):
    f.inject_bridge_drive(drives(sc, n, amp), 1.0)
    if n % 5 == 0:
        f.inject_plate_force(sc.force_idx, sc.force_wgt, 0.05 * math.cos(n / 11.0))
    if n < 30:
        f.add_pressure(sc.point_cells[0], 0.5 * math.exp(-0.5 * ((n - 12) / 4.0) ** 2))
    f.step(1)
    return f.sample_plate_displacement_batch(sc.plate_idx4, sc.plate_wgt4)


def combined(f, sc, n, amp):
    if n < 30:
        f.add_pressure(sc.point_cells[0], 0.5 * math.exp(-0.5 * ((n - 12) / 4.0) ** 2))
    force = 0.05 * math.cos(n / 11.0) if n % 5 == 0 else 0.0
    return f.substep(drives(sc, n, amp), 1.0, sc.force_idx, sc.force_wgt, force, sc.plate_idx4, sc.plate_wgt4)


def same_state(a, b):
    assert a.step_count == b.step_count
    for name in ("get_pressure_field", "get_velocity_x", "get_velocity_y", "get_velocity_z",
                 "get_plate_displacement", "get_traces"):
        x, y = getattr(a, name)(), getattr(b, name)()
        assert bits_equal(x, y), (name, first_mismatch(x, y))


def same_fields(a, b):
    assert a.step_count == b.step_count
    for name in ("get_pressure_field", "get_velocity_x", "get_velocity_y", "get_velocity_z",
                 "get_plate_displacement"):
        x, y = getattr(a, name)(), getattr(b, name)()
        assert bits_equal(x, y), (name, first_mismatch(x, y))


@pytest.mark.parametrize("dims", [(24, 20, 16), (60, 50, 30)])
def test_substep_equals_call_sequence(cuda, dims):
    from scenes import body_scene
    sc = body_scene(*dims, seed=4)
    a, b = make(sc), make(sc)
    for n in range(300):                       # crosses the 256-step check
        wa = sequence(a, sc, n, 0.2)
        wb = combined(b, sc, n, 0.2)
        assert bits_equal(wa, wb), (n, first_mismatch(wa, wb))
    same_state(a, b)
    assert b.launch_count > 0


@pytest.mark.parametrize("dims", [(24, 20, 16), (60, 50, 30)])
def test_substep_graph_replay_equals_call_sequence(cuda, dims):
    """Without device-recorded receivers (the co-evolver samples its
    microphones separately) the substep replays cached CUDA graphs: the same
    results, through the 256-step check (issued directly) and the plate's
    three buffer rotations, with and without pending plate forces."""
    from scenes import body_scene
    sc = body_scene(*dims, seed=5)
    a, b = make(sc, receivers=False), make(sc, receivers=False)
    for n in range(300):
        wa = sequence(a, sc, n, 0.2)
        wb = combined(b, sc, n, 0.2)
        assert bits_equal(wa, wb), (n, first_mismatch(wa, wb))
    assert a.step_count == b.step_count == 300
    same_fields(a, b)


@pytest.mark.parametrize("receivers", [True, False])
def test_substep_plate_guard(cuda, receivers):
    """A drive that throws the plate past 2 cm: both paths fail at the same
    step and leave the same state (no rotation, forces still pending), also
    when the failing substep is a graph replay (no device receivers)."""
    from scenes import body_scene
    sc = body_scene(24, 20, 16, seed=5)
    a, b = make(sc, receivers), make(sc, receivers)
    fail = []
    for f, fn in ((a, sequence), (b, combined)):
        for n in range(400):
            try:
                fn(f, sc, n, 2e4)
            except RuntimeError:
                fail.append(n)
                break
    assert len(fail) == 2 and fail[0] == fail[1], fail
    check = same_state if receivers else same_fields
    check(a, b)
    # both retry the failed step the same way
    ra, rb = a.step_rc(1), b.step_rc(1)
    assert ra == rb == -3
    check(a, b)


def test_substep_open_room(cuda):
    """Without an active plate the call is inject + step + sample with no extra wait."""
    from spectral_analyzer_b200 import AcousticFDTD
    from spectral_analyzer_b200.rooms import seeded_room
    room = seeded_room(40, 36, 44, 0, seed=3, n_rec=2, n_pml=6)
    mk = lambda: AcousticFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, cell_type=room.cell_type(),
                              plate_iz=-1, plate_active=room.plate_active(), n_pml=room.n_pml)
    a, b = mk(), mk()
    idx4 = np.array([0, 1, room.ny, room.ny + 1], np.int32)
    w4 = np.full(4, 0.25, np.float32)
    for n in range(270):
        amp = float(np.exp(-0.5 * ((n - 20) / 6.0) ** 2))
        a.add_pressure(room.src_flat, amp)
        a.step(1)
        wa = a.sample_plate_displacement_batch(idx4, w4)
        b.add_pressure(room.src_flat, amp)
        wb = b.substep(saddle_idx4=idx4, saddle_wgt4=w4)
        assert bits_equal(wa, wb)
    assert bits_equal(a.get_pressure_field(), b.get_pressure_field())


def test_substep_rejects_bad_saddle_index(cuda):
    from scenes import body_scene
    sc = body_scene(24, 20, 16, seed=6)
    f = make(sc)
    with pytest.raises(ValueError):
        f.substep(drives(sc, 0, 0.2), 1.0, saddle_idx4=np.array([0, 1, 2, 10 ** 6], np.int32),
                  saddle_wgt4=np.full(4, 0.25, np.float32))
    assert f.step_count == 0
