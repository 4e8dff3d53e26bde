"""The allocation-free sampler agrees with the allocating one and the oracle.

fdtd_b200_sample_pressure_noalloc serves callers that must not allocate — a
real-time audio callback reading the microphones, where a cudaMalloc may
block on driver locks.  It stages its inputs and results in one fixed device
array instead of per-handle scratch; this test calls it through the C ABI and
checks it against fdtd_sample_pressure_precomputed and against the CPU
oracle's sampler on the same room, twice in a row and again after more steps,
and checks its size limit and its index check.  The file is named to be
collected last.
"""
import ctypes as C

import numpy as np
import pytest

from spectral_analyzer_b200.rooms import rel_l2, seeded_room

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5   # the relative L2 bound used by the parity tests (results are also bit-equal)
MAX_RECEIVERS = 4096


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def test_noalloc_sampler_matches_precomputed_sampler():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    from spectral_analyzer_b200 import AcousticFDTD, _native

    room = seeded_room(48, 40, 36, 80, seed=11, n_rec=4, n_pml=4)
    f = AcousticFDTD(room.nx, room.ny, room.nz, room.dx, cell_type=room.cell_type(), plate_iz=-1,
                     plate_active=room.plate_active(), n_pml=room.n_pml)
    f.set_face_absorption(room.absorption)
    f.set_point_source(room.src_flat, room.signal())
    lib = _native.load()
    from oracle import OracleFDTD
    orc = OracleFDTD(room.nx, room.ny, room.nz, room.dx, cell_type=room.cell_type(), plate_iz=-1,
                     plate_active=room.plate_active(), n_pml=room.n_pml)
    orc.set_face_absorption(room.absorption)
    sig = room.signal()

    # two receiver sets of different sizes, with fractional (trilinear) positions
    sets = [np.array([[s[0] + 0.25, s[1] - 0.5, s[2] + 0.75] for s in room.receivers], np.float32),
            np.array([[10.5, 12.25, 8.0], [30.0, 20.0, 17.5], [47.0, 39.0, 35.0]], np.float32)]
    samplers = [f.precompute_pressure_samplers(x) for x in sets]

    for block in range(2):
        f.step(30)
        for _ in range(30):   # the oracle: deposit before each step, as the engine's point source
            orc.add_pressure(room.src_flat, float(sig[orc.step_count]))
            orc.step(1)
        for idx, w in samplers:               # two calls in a row, different sizes
            n = idx.size // 8
            ref = f.sample_pressure_precomputed(idx, w)
            out = np.full(n, np.nan, np.float32)
            rc = lib.fdtd_b200_sample_pressure_noalloc(f._h, n, _ptr(idx, C.c_int), _ptr(w, C.c_float),
                                                       _ptr(out, C.c_float))
            assert rc == 0, _native.last_error()
            assert rel_l2(out, ref) <= TRACE_TOL
            assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))
            want = orc.sample_pressure_precomputed(idx, w)
            assert rel_l2(out, want) <= TRACE_TOL
            assert np.array_equal(out.view(np.uint32), np.asarray(want, np.float32).view(np.uint32))
        if block == 1:
            assert np.abs(ref).max() > 0.0

    # beyond the fixed array: rejected with a reason, nothing launched
    big = MAX_RECEIVERS + 1
    idx = np.zeros(8 * big, np.int32)
    w = np.zeros(8 * big, np.float32)
    out = np.zeros(big, np.float32)
    launches = f.launch_count
    rc = lib.fdtd_b200_sample_pressure_noalloc(f._h, big, _ptr(idx, C.c_int), _ptr(w, C.c_float),
                                               _ptr(out, C.c_float))
    assert rc == _native.FDTD_ERR_ARG
    assert "maximum" in _native.last_error()
    assert f.launch_count == launches

    # a tap index outside [0, N): rejected with the tap named, nothing launched
    idx0, w0 = samplers[1]
    n = idx0.size // 8
    for bad in (room.nx * room.ny * room.nz, -1):
        idx = idx0.copy()
        idx[5] = bad
        out = np.zeros(n, np.float32)
        launches = f.launch_count
        rc = lib.fdtd_b200_sample_pressure_noalloc(f._h, n, _ptr(idx, C.c_int), _ptr(w0, C.c_float),
                                                   _ptr(out, C.c_float))
        assert rc == _native.FDTD_ERR_ARG
        msg = _native.last_error()
        assert "tap 5" in msg and str(bad) in msg
        assert f.launch_count == launches
