"""CUDA slab kernels: a room split into slabs (stepped in one process with
plane-copy exchanges), with the fused single-pass kernel or the two passes,
equals the whole-room engine bit for bit."""
import pytest

from conftest import bits_equal, first_mismatch
from spectral_analyzer_b200.rooms import Room, seeded_room

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch


def whole(room):
    from spectral_analyzer_b200.serving import make_solver
    f = make_solver(room)
    f.step(room.n_steps)
    return f.get_traces(), f.get_pressure_field()


def edge_room():
    return Room(41, 36, 44, 260, (20, 17, 21),
                [(20.5, 10.25, 15.5), (21.0, 16.0, 30.0), (3.0, 1.5, 40.75), (38.6, 30.0, 3.0),
                 (13.5, 20.0, 20.0)],
                (0.3, 0.9, 0.5, 1.0, 0.2, 0.7), "ricker", n_pml=6)


@pytest.mark.parametrize("fused,peer", [(True, False), (False, False), (True, True)])
@pytest.mark.parametrize("n_slabs", [1, 2, 3, 5])
def test_slabs_equal_whole_room(cuda, n_slabs, fused, peer):
    """peer: the fused steps write each other's ghost planes, no exchange."""
    from spectral_analyzer_b200.slab import local_room
    room = edge_room()
    tr, P = whole(room)
    run = local_room(room, n_slabs, fused=fused, peer_stores=peer)
    assert run.fused == fused
    run.step(room.n_steps)
    got = run.traces(len(room.receivers))
    assert bits_equal(got, tr), first_mismatch(got, tr)
    assert bits_equal(run.pressure_field(), P)
    assert all(s.launch_count > 0 for s in run.slabs)


@pytest.mark.parametrize("n_slabs", [1, 2, 5, 7])
def test_overlapped_exchange_equals_whole_room(cuda, n_slabs):
    """The step in two parts (ghost planes first, then the interior beside the
    exchange on a side stream) equals the whole room bit for bit; with 7 slabs
    of 41 planes every slab has six planes or fewer (part 1 covers it all)."""
    from spectral_analyzer_b200.slab import local_room
    room = edge_room()
    tr, P = whole(room)
    run = local_room(room, n_slabs, overlap=True)
    assert run.overlap
    run.step(room.n_steps)
    got = run.traces(len(room.receivers))
    assert bits_equal(got, tr), first_mismatch(got, tr)
    assert bits_equal(run.pressure_field(), P)


@pytest.mark.parametrize("fused", [True, False])
def test_seeded_room_over_four_slabs(cuda, fused):
    from spectral_analyzer_b200.slab import local_room
    room = seeded_room(96, 64, 80, 300, seed=21, n_rec=6, n_pml=8)
    tr, P = whole(room)
    for overlap in ((False, True) if fused else (False,)):
        run = local_room(room, 4, fused=fused, overlap=overlap)
        run.step(room.n_steps)
        assert bits_equal(run.traces(6), tr), overlap
        assert bits_equal(run.pressure_field(), P), overlap


def test_slab_instability(cuda):
    from spectral_analyzer_b200.slab import local_room
    room = edge_room()
    room.amp = 1e9
    run = local_room(room, 2)
    with pytest.raises(RuntimeError, match="FDTD_ERR_UNSTABLE"):
        run.step(room.n_steps)
    assert run.step_count == 256
