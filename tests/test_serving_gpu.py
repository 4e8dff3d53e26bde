"""Batched stepping on the GPU: each room is the same alone and in the mix."""
import numpy as np
import pytest

from conftest import bits_equal, first_mismatch
from spectral_analyzer_b200.rooms import seeded_room

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch


MIX = [(40, 36, 48, 150, 1), (64, 64, 64, 220, 2), (33, 90, 17, 95, 3), (100, 40, 130, 180, 4),
       (16, 16, 16, 300, 5), (72, 48, 256, 120, 6)]


def rooms():
    out = []
    for nx, ny, nz, steps, seed in MIX:
        r = seeded_room(nx, ny, nz, steps, seed=seed, n_rec=3, n_pml=4,
                        source_kind="gaussian" if seed % 2 else "ricker")
        out.append(r)
    return out


def alone(room):
    from spectral_analyzer_b200.serving import make_solver
    f = make_solver(room)
    f.set_kernel("fused")
    f.step(room.n_steps)
    return f.get_traces(), f.get_pressure_field(), f.get_velocity_z()


@pytest.mark.parametrize("use_graph,tile_k", [(True, 128), (False, 128), (True, 64), (False, 64)])
def test_batch_equals_alone(cuda, use_graph, tile_k):
    from spectral_analyzer_b200.serving import EngineBatch, make_solver
    rs = rooms()
    ref = [alone(r) for r in rs]
    solvers = [make_solver(r) for r in rs]
    b = EngineBatch()
    b.set_tile(tile_k)
    b.set(solvers, [r.n_steps for r in rs])
    steps = np.zeros(len(rs))
    while np.any(steps < [r.n_steps for r in rs]):
        b.step(37, use_graph)            # chunks that do not divide the step counts
        steps, status = b.sync()
        assert not status.any()
    b.set([], [])
    for r, f, (tr, P, Vz) in zip(rs, solvers, ref):
        assert f.step_count == r.n_steps
        got = f.get_traces()
        assert bits_equal(got, tr), (r.describe(), first_mismatch(got, tr))
        assert bits_equal(f.get_pressure_field(), P)
        assert bits_equal(f.get_velocity_z(), Vz)


def test_batch_matches_the_oracle(cuda):
    """Each room of the mixed batch against the oracle directly (not only
    against the single-room engine): traces and final fields bit for bit."""
    from oracle import OracleFDTD
    from spectral_analyzer_b200.serving import EngineBatch, make_solver
    rs = rooms()
    solvers = [make_solver(r) for r in rs]
    b = EngineBatch()
    b.set(solvers, [r.n_steps for r in rs])
    while any(f.step_count < r.n_steps for f, r in zip(solvers, rs)):
        b.step(41, True)
        _, status = b.sync()
        assert not status.any()
    b.set([], [])
    for r, f in zip(rs, solvers):
        o = OracleFDTD(r.nx, r.ny, r.nz, r.dx, r.c, r.rho, n_pml=r.n_pml)
        o.set_face_absorption(r.absorption)
        idx, w = o.precompute_pressure_samplers(r.receiver_xyz())
        tro = o.run(r.n_steps, r.src_flat, r.signal(), idx, w)
        got = f.get_traces()
        assert bits_equal(got, tro), (r.describe(), first_mismatch(got, tro))
        assert bits_equal(f.get_pressure_field(), o.get_pressure_field()), r.describe()
        assert bits_equal(f.get_velocity_x(), o.get_velocity_x()), r.describe()
        del o


def test_members_join_and_leave(cuda):
    """Rooms enter mid-run and continue on the single-room path after leaving."""
    from spectral_analyzer_b200.serving import EngineBatch, make_solver
    rs = rooms()[:4]
    ref = [alone(r) for r in rs]
    s = [make_solver(r) for r in rs]
    s[3].step(40)                        # some steps on the plain path first
    b = EngineBatch()
    b.set([s[0], s[1]], [rs[0].n_steps, rs[1].n_steps])
    b.step(50)
    b.sync()
    b.set([s[0], s[1], s[2], s[3]], [r.n_steps for r in rs])     # 2 and 3 join
    b.step(64)
    b.sync()
    b.set([s[1], s[2]], [rs[1].n_steps, rs[2].n_steps])          # 0 and 3 leave
    s[0].step(rs[0].n_steps - s[0].step_count)                   # finish alone
    s[3].step(rs[3].n_steps - s[3].step_count)
    while s[1].step_count < rs[1].n_steps or s[2].step_count < rs[2].n_steps:
        b.step(64)
        b.sync()
    b.set([], [])
    for r, f, (tr, P, _) in zip(rs, s, ref):
        assert f.step_count == r.n_steps
        assert bits_equal(f.get_traces(), tr), r.describe()
        assert bits_equal(f.get_pressure_field(), P)


def test_batch_latches_instability(cuda):
    from spectral_analyzer_b200.serving import EngineBatch, make_solver
    rs = rooms()[:2]
    s = [make_solver(r) for r in rs]
    s[1].add_pressure(rs[1].src_flat, 1e9)
    b = EngineBatch()
    b.set(s, [300, 300])
    b.step(300)
    steps, status = b.sync()
    assert list(steps) == [300, 256]          # the diverged member stopped at its check step
    assert status[0] == 0 and status[1] == -3


def test_batch_server_matches_sequential(cuda):
    from spectral_analyzer_b200.serving import (BatchServer, SequentialServer, mixed_room_requests,
                                                poisson_arrivals)
    reqs = mixed_room_requests(10, seed=9, steps=(60, 260), axes=(32, 48, 64, 80))
    for r, t in zip(reqs, poisson_arrivals(10, rate=400.0, seed=9)):
        r.arrival = float(t)
    seq = SequentialServer().run(reqs)
    bat = BatchServer(max_slots=6, chunk=32, tile_k=64).run(reqs)
    for a, b in zip(seq, bat):
        assert a.rid == b.rid
        assert bits_equal(a.traces, b.traces), a.rid


def nan_signal(room, at):
    sig = np.array(room.signal(), np.float32)
    sig[at] = np.nan
    return sig


def test_unstable_member_stops_like_a_single_room(cuda):
    """A NaN planted in one room's source: in the batch that room stops at the
    first 256-step check after it, in exactly the state the single-room step
    leaves when it returns UNSTABLE; the other rooms finish as if alone."""
    from spectral_analyzer_b200.serving import EngineBatch, make_solver
    rs = [seeded_room(40, 36, 48, 700, seed=11, n_rec=2, n_pml=4),
          seeded_room(64, 48, 40, 600, seed=12, n_rec=3, n_pml=4, source_kind="ricker"),
          seeded_room(33, 50, 27, 650, seed=13, n_rec=2, n_pml=4)]
    bad = 1
    sig = nan_signal(rs[bad], 30)
    f = make_solver(rs[bad])
    f.set_point_source(rs[bad].src_flat, sig)
    f.set_kernel("fused")
    assert f.step_rc(rs[bad].n_steps) == -3
    assert f.step_count == 256
    ref_bad = (f.get_traces(), f.get_pressure_field(), f.get_velocity_x())
    ref = [alone(r) if q != bad else None for q, r in enumerate(rs)]

    solvers = [make_solver(r) for r in rs]
    solvers[bad].set_point_source(rs[bad].src_flat, sig)
    b = EngineBatch()
    b.set(solvers, [r.n_steps for r in rs])
    b.step(300, True)
    steps, status = b.sync()
    assert list(status) == [0, -3, 0] and steps[bad] == 256
    b.step(100, True)                       # the stopped member does not move
    steps, status = b.sync()
    assert steps[bad] == 256 and status[bad] == -3
    t, P, Vx = ref_bad
    assert bits_equal(solvers[bad].get_traces(), t)
    assert bits_equal(solvers[bad].get_pressure_field(), P)
    assert bits_equal(solvers[bad].get_velocity_x(), Vx)
    keep = [s for q, s in enumerate(solvers) if q != bad]
    b.set(keep, [r.n_steps for q, r in enumerate(rs) if q != bad])
    while True:
        b.step(128, True)
        steps, status = b.sync()
        if np.all(steps >= [r.n_steps for q, r in enumerate(rs) if q != bad]):
            break
    b.set([], [])
    for q in (0, 2):
        tr, P, Vz = ref[q]
        assert bits_equal(solvers[q].get_traces(), tr)
        assert bits_equal(solvers[q].get_pressure_field(), P)


def test_server_isolates_a_diverging_request(cuda):
    """BatchServer on the engine: the NaN request leaves with an error, the rest
    return the traces they have alone."""
    from spectral_analyzer_b200.serving import BatchServer, Request, _EngineBackend
    rs = [seeded_room(40, 36, 48, 600, seed=21 + q, n_rec=2, n_pml=4) for q in range(4)]
    reqs = [Request(q, r) for q, r in enumerate(rs)]

    class Planted(_EngineBackend):
        def make(self, room):
            f = super().make(room)
            if room is rs[2]:
                f.set_point_source(room.src_flat, nan_signal(room, 10))
            return f

    res = BatchServer(max_slots=4, chunk=64, backend=Planted()).run(reqs)
    assert "UNSTABLE" in res[2].error and res[2].traces.shape[0] == 256
    for q in (0, 1, 3):
        assert res[q].ok
        assert bits_equal(res[q].traces, alone(rs[q])[0])


def test_preempted_request_resumes_bit_exact(cuda):
    """Two requests of the mix are pre-empted after their first chunk (their
    fields, step count and check phase go to host memory and their slots are
    freed), the others finish, then both resume on new solvers: every result
    equals the room run alone, bit for bit.  One of them crosses a 256-step
    check after the resume."""
    from spectral_analyzer_b200.serving import BatchServer, Request
    rs = rooms()
    ref = [alone(r) for r in rs]
    reqs = [Request(q, r, 0.0) for q, r in enumerate(rs)]
    srv = BatchServer(max_slots=8, chunk=64)
    srv.preempt(1)
    srv.preempt(4)
    first = srv.run(reqs)
    assert sorted(srv.paused) == [1, 4]
    assert sorted(r.rid for r in first) == [0, 2, 3, 5]
    srv.resume(1)
    srv.resume(4)
    second = srv.run([])
    res = {r.rid: r for r in first + second}
    for q, r in enumerate(rs):
        assert res[q].ok, res[q].error
        assert bits_equal(res[q].traces, ref[q][0]), (q, first_mismatch(res[q].traces, ref[q][0]))


def test_snapshot_restores_fields_and_progress(cuda):
    from spectral_analyzer_b200.serving import make_solver
    room = rooms()[1]
    a = make_solver(room)
    a.step(100)
    snap = a.snapshot()
    assert snap["step"] == 100
    b = make_solver(room)
    b.restore(snap)
    a.step(room.n_steps - 100)
    b.step(room.n_steps - 100)
    assert bits_equal(a.get_pressure_field(), b.get_pressure_field())
    assert bits_equal(a.get_velocity_x(), b.get_velocity_x())
    assert b.step_count == room.n_steps
