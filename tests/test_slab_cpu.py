"""Slab decomposition on CPU: plane partition, receiver ownership, and the
exchange schedule run as gloo ranks (world size 2 and 3) with a NumPy slab,
compared bit for bit with the oracle's whole-room run."""
import os
import socket
import tempfile

import numpy as np
import pytest

from spectral_analyzer_b200.rooms import Room
from spectral_analyzer_b200.slab import (LocalExchange, SlabRunner, partition, receiver_owner)


def edge_room(nx=13, steps=140):
    """Source on the last plane of the first of two slabs, receivers straddling
    the slab edges (fractional coordinates) and inside the absorbing layers."""
    return Room(nx, 11, 12, steps, (6, 5, 6),
                [(6.5, 4.25, 5.5), (7.0, 6.0, 2.0), (1.0, 1.5, 10.75), (11.6, 9.0, 3.0)],
                (0.3, 0.9, 0.5, 1.0, 0.2, 0.7), "gaussian", n_pml=3, sigma_steps=3.0)


def oracle_run(room):
    from oracle import OracleFDTD
    from spectral_analyzer_b200.precision import pressure_taps
    o = OracleFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, n_pml=room.n_pml)
    o.set_face_absorption(room.absorption)
    idx, w = pressure_taps(room.nx, room.ny, room.nz, room.receiver_xyz())
    tr = o.run(room.n_steps, room.src_flat, room.signal(), idx, w)
    return tr, o.get_pressure_field()


def test_partition():
    assert partition(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert partition(512, 8)[-1] == (448, 512)
    with pytest.raises(ValueError):
        partition(8, 3)
    for nx, w in [(13, 2), (64, 5), (12, 4)]:
        r = partition(nx, w)
        assert r[0][0] == 0 and r[-1][1] == nx
        assert all(b - a >= 3 for a, b in r) and all(r[q][1] == r[q + 1][0] for q in range(w - 1))


def test_receiver_owner():
    room = edge_room()
    ranges = partition(room.nx, 2)                 # (0, 7), (7, 13)
    assert receiver_owner(room, ranges) == [0, 1, 0, 1]


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("n_slabs", [1, 2, 4])
def test_local_slabs_equal_oracle(n_slabs, fused):
    from slab_numpy import NumpySlab
    room = edge_room()
    ranges = partition(room.nx, n_slabs)
    owners = receiver_owner(room, ranges)
    slabs = [NumpySlab(room, a, b, [q for q, o in enumerate(owners) if o == r], fused)
             for r, (a, b) in enumerate(ranges)]
    assert SlabRunner(slabs, LocalExchange(slabs)).fused == fused
    run = SlabRunner(slabs, LocalExchange(slabs))
    run.step(room.n_steps)
    tr, P = oracle_run(room)
    got = run.traces(len(room.receivers))
    assert np.array_equal(got.view(np.uint32), tr.view(np.uint32))
    assert np.array_equal(run.pressure_field().view(np.uint32), P.view(np.uint32))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path, nx, steps, fused):
    import torch.distributed as dist
    from datetime import timedelta
    from slab_numpy import NumpySlab
    from spectral_analyzer_b200.slab import DistExchange
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        room = edge_room(nx, steps)
        ranges = partition(room.nx, world)
        owners = receiver_owner(room, ranges)
        a, b = ranges[rank]
        slab = NumpySlab(room, a, b, [q for q, o in enumerate(owners) if o == rank], fused)
        run = SlabRunner([slab], DistExchange(slab, rank, world))
        run.step(room.n_steps)
        tr = run.traces(len(room.receivers))
        P = run.pressure_field()
        if rank == 0:
            np.savez(out_path, traces=tr, P=P)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,fused", [(2, True), (3, True), (2, False)])
def test_gloo_ranks_equal_oracle(world, fused):
    import torch.multiprocessing as mp
    room = edge_room(nx=13, steps=140)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "r.npz")
        mp.start_processes(_rank_main, args=(world, _free_port(), out, room.nx, room.n_steps, fused),
                           nprocs=world, join=True, start_method="spawn")
        with np.load(out) as z:
            got_tr, got_P = z["traces"], z["P"]
    tr, P = oracle_run(room)
    assert np.array_equal(got_tr.view(np.uint32), tr.view(np.uint32))
    assert np.array_equal(got_P.view(np.uint32), P.view(np.uint32))


def test_instability_is_reported_on_every_slab():
    from slab_numpy import NumpySlab
    room = edge_room(steps=300)
    room.amp = 1e9                                  # diverges: |p| > 2e3 at the 256-step check
    ranges = partition(room.nx, 2)
    slabs = [NumpySlab(room, a, b, []) for a, b in ranges]
    run = SlabRunner(slabs, LocalExchange(slabs))
    with pytest.raises(RuntimeError, match="FDTD_ERR_UNSTABLE"):
        run.step(300)
    assert run.step_count == 256


def _leaving_rank_main(rank, world, port, out_path, leave_at):
    """Rank 1 leaves between steps (after ``leave_at`` steps, nothing in flight);
    rank 0 learns of it from its next halo exchange, which ends with an error
    within the process group's short timeout instead of waiting for good."""
    import time
    import torch.distributed as dist
    from datetime import timedelta
    from slab_numpy import NumpySlab
    from spectral_analyzer_b200.slab import DistExchange
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    room = edge_room(13, 60)
    ranges = partition(room.nx, world)
    a, b = ranges[rank]
    slab = NumpySlab(room, a, b, [])
    run = SlabRunner([slab], DistExchange(slab, rank, world))
    if rank == 1:
        run.step(leave_at)
        dist.destroy_process_group()
        return
    t0 = time.monotonic()
    err = ""
    try:
        run.step(room.n_steps)
    except Exception as e:           # the collective's error (peer gone or timeout)
        err = f"{type(e).__name__}: {e}"
    with open(out_path, "w") as fh:
        fh.write(f"{run.step_count}\n{time.monotonic() - t0:.3f}\n{err}\n")


def test_rank_that_leaves_is_detected_by_the_others():
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "r0.txt")
        mp.start_processes(_leaving_rank_main, args=(2, _free_port(), out, 7), nprocs=2, join=True,
                           start_method="spawn")
        steps, secs, err = open(out).read().split("\n", 2)
    assert err.strip(), "rank 0 finished although its neighbour left"
    assert int(steps) == 7                       # it stopped at the step its neighbour did not take
    assert float(secs) < 30.0
