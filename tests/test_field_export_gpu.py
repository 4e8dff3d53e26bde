"""Headless field export: the bridge's get_volume_slice (acoustic_fdtd_bridge.py:
737-757) taken on the device equals slicing the full pressure copy."""
import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch


def bridge_slice(P, axis, idx):
    """The bridge's own rule on a full (Nx, Ny, Nz) copy."""
    if idx < 0:
        idx = P.shape[axis] // 2
    idx = max(0, min(P.shape[axis] - 1, idx))
    if axis == 0:
        return P[idx, :, :]
    if axis == 1:
        return P[:, idx, :]
    return P[:, :, idx]


@pytest.mark.parametrize("scene", ["open", "body"])
def test_volume_slice_equals_full_copy(cuda, scene):
    from spectral_analyzer_b200 import AcousticFDTD
    if scene == "open":
        from spectral_analyzer_b200.rooms import seeded_room
        room = seeded_room(37, 29, 45, 0, seed=2, n_rec=1, n_pml=5)
        f = AcousticFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, cell_type=room.cell_type(),
                         plate_iz=-1, plate_active=room.plate_active(), n_pml=room.n_pml)
        src = room.src_flat
    else:
        from scenes import body_scene
        sc = body_scene(30, 26, 20, seed=3)
        f = AcousticFDTD(**sc.kwargs())
        src = sc.point_cells[0]
    for n in range(25):
        f.add_pressure(src, float(np.exp(-0.5 * ((n - 8) / 3.0) ** 2)))
        f.step(1)
    P = f.get_pressure_field()
    for axis in range(3):
        for idx in (-1, 0, 3, P.shape[axis] - 1, P.shape[axis] + 7):
            got = f.get_volume_slice(axis, idx)
            want = bridge_slice(P, axis, idx)
            assert got.shape == want.shape
            assert bits_equal(got, want), (axis, idx)


def test_volume_slice_rejects_bad_arguments(cuda):
    from spectral_analyzer_b200 import AcousticFDTD, _native
    from spectral_analyzer_b200.fdtd import _pf
    f = AcousticFDTD(16, 12, 20, 0.01, cell_type=np.zeros(16 * 12 * 20, np.uint8), plate_iz=-1,
                     plate_active=np.zeros(16 * 12, np.uint8), n_pml=3)
    with pytest.raises(ValueError):
        f.get_volume_slice(3, 0)
    small = np.empty(5, np.float32)
    assert f._lib.fdtd_b200_get_volume_slice(f._h, 2, 0, _pf(small), small.size) == _native.FDTD_ERR_DIM
