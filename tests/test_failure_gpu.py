"""Failure paths on the GPU, none of which faults, traps or hangs the device.

A fused step whose load never lands: the P-plane load of one plane is armed on
its mbarrier but not issued (``debug_hold_load``), so every CTA that needs it
gives up after a short bounded wait (a few milliseconds of wall time), records
a timeout status and exits.  The host reads the status, reports FDTD_ERR_CUDA
until ``reset``, and the same handle and CUDA context then run on bit-exactly
(checked against the two-pass kernel, which shares no code with the fused one).
"""
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


def open_room(room, kernel="fused"):
    from spectral_analyzer_b200 import AcousticFDTD
    f = AcousticFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, cell_type=room.cell_type(),
                     plate_iz=-1, plate_active=room.plate_active(), n_pml=room.n_pml)
    f.set_kernel(kernel)
    return f


@pytest.mark.parametrize("dims,plane", [((64, 48, 40), 12), ((40, 100, 70), 0), ((48, 32, 96), 47)])
def test_timed_out_load_is_reported_and_recovered(cuda, dims, plane):
    from spectral_analyzer_b200 import _native
    from spectral_analyzer_b200.rooms import seeded_room
    room = seeded_room(*dims, 0, seed=8, n_rec=2, n_pml=6)
    f, g = open_room(room), open_room(room, "two_pass")

    def drive(h, n):
        for s in range(n):
            h.add_pressure(room.src_flat, float(np.exp(-0.5 * ((s - 10) / 3.0) ** 2)))
            h.step(1)

    drive(f, 5)
    assert f.synchronize() == 0                 # no hold: no timeout
    f.debug_hold_load(plane, wait_us=3000)
    f.step(1)
    with pytest.raises(RuntimeError, match="timed out"):
        f.synchronize()
    assert "timed out" in _native.last_error()
    f.step(2)                                   # the latch holds until reset
    with pytest.raises(RuntimeError, match="timed out"):
        f.synchronize()
    cuda.cuda.synchronize()                     # the context is fine
    f.debug_hold_load(-1)
    f.reset()
    assert f.synchronize() == 0
    drive(f, 40)
    drive(g, 40)
    assert f.synchronize() == 0 and g.synchronize() == 0
    a, b = f.get_pressure_field(), g.get_pressure_field()
    assert np.abs(a).max() > 0
    assert bits_equal(a, b), first_mismatch(a, b)
    assert bits_equal(f.get_velocity_y(), g.get_velocity_y())


def test_hold_hook_rejects_bad_arguments(cuda):
    from spectral_analyzer_b200.rooms import seeded_room
    room = seeded_room(32, 32, 32, 0, seed=9, n_rec=1, n_pml=4)
    f = open_room(room)
    for plane, wait_us in ((-2, 0), (32, 0), (3, -1), (3, 1 << 30)):
        with pytest.raises(ValueError):
            f.debug_hold_load(plane, wait_us)
    f.debug_hold_load(-1)
    f.step(3)
    assert f.synchronize() == 0
