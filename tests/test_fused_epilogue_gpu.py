"""The fused step's own epilogues at their edge cases, bit for bit against the
two-pass kernels (which deposit and record with kernels of their own).

The point-source deposit is applied by every CTA whose shared-memory P box
holds the source cell (its own tile or its halo rows/columns, and the
neighbouring i segments), so sources are placed on tile edges in j and k, in
the first and last planes, and on both tile shapes.  Receivers are recorded by
the next step's kernel or, for the last step of a call, by a kernel of their
own, so runs are split into calls of different lengths.
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


def run(room, kernel, calls):
    from spectral_analyzer_b200 import AcousticFDTD
    f = AcousticFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, cell_type=room.cell_type(),
                     plate_iz=-1, plate_active=room.plate_active(), n_pml=room.n_pml)
    f.set_face_absorption(room.absorption)
    f.set_kernel(kernel)
    idx, w = f.precompute_pressure_samplers(room.receiver_xyz())
    f.set_point_source(room.src_flat, room.signal())
    f.set_receivers(idx, w, sum(calls))
    for n in calls:
        f.step(n)
    return f.get_traces(), f.get_pressure_field(), f.get_velocity_x(), f.get_velocity_z()


# (grid, tile rows x cols the fused step picks for it, source cells)
CASES = [
    ((24, 20, 256), (8, 128), [(12, 7, 127), (12, 8, 128), (12, 15, 129), (12, 16, 0),
                              (0, 0, 0), (23, 19, 255), (5, 9, 124), (6, 10, 131)]),
    ((20, 36, 160), (16, 64), [(10, 15, 63), (10, 16, 64), (10, 31, 127), (10, 32, 128),
                              (0, 35, 159), (19, 0, 60), (9, 13, 67), (11, 19, 3)]),
]


@pytest.mark.parametrize("dims,tile,sources", CASES)
def test_source_on_tile_edges(cuda, dims, tile, sources):
    from spectral_analyzer_b200.rooms import seeded_room
    for q, src in enumerate(sources):
        room = seeded_room(*dims, 30, seed=40 + q, n_rec=3, n_pml=3, source_kind="gaussian")
        room.src = src
        room.receivers[0] = tuple(min(max(c + 2, 0), d - 1) for c, d in zip(src, dims))
        calls = (1, 7, 1, 21)                       # records both in-kernel and flushed
        got = run(room, "fused", calls)
        ref = run(room, "two_pass", calls)
        assert np.abs(got[0][:, 0]).max() > 0, src
        for name, a, b in zip(("traces", "P", "Vx", "Vz"), got, ref):
            assert bits_equal(a, b), (src, name, first_mismatch(a, b))
