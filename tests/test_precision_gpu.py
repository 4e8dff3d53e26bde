"""Storage-precision study on the GPU: the FP64 mode is the double oracle bit
for bit, the FP32 mode is the engine bit for bit, the energy audit matches a
host sum over the oracle's fields, and the 16-bit modes rank as expected."""
import numpy as np
import pytest

from conftest import bits_equal, first_mismatch
from spectral_analyzer_b200.rooms import rel_l2, seeded_room

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch


def small_room(steps=300, seed=11, kind="ricker"):
    return seeded_room(40, 36, 44, steps, seed=seed, n_rec=3, n_pml=6, source_kind=kind)


def oracle_for(room, precision):
    from oracle import OracleFDTD
    o = OracleFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, n_pml=room.n_pml,
                   precision=precision)
    o.set_face_absorption(room.absorption)
    return o


def test_fp64_mode_is_the_double_oracle(cuda):
    from spectral_analyzer_b200.precision import PrecisionRoom
    room = small_room()
    pr = PrecisionRoom(room, "fp64")
    pr.step(room.n_steps)
    idx, w = pr.taps
    o = oracle_for(room, "f64")
    assert pr.dt == o.dt
    tr = o.run(room.n_steps, room.src_flat, room.signal().astype(np.float64), idx, w)
    got_p, ref_p = pr.pressure(), o.get_pressure_field()
    assert np.array_equal(got_p.view(np.uint64), ref_p.view(np.uint64)), \
        np.max(np.abs(got_p - ref_p))
    assert np.array_equal(pr.traces().view(np.uint64), tr.view(np.uint64))


def test_fp32_mode_is_the_engine(cuda):
    from spectral_analyzer_b200.precision import PrecisionRoom
    from spectral_analyzer_b200.serving import make_solver
    room = small_room(seed=12)
    pr = PrecisionRoom(room, "fp32")
    pr.step(room.n_steps)
    f = make_solver(room)
    f.step(room.n_steps)
    got = pr.pressure().astype(np.float32)
    ref = f.get_pressure_field()
    assert bits_equal(got, ref), first_mismatch(got, ref)
    # receivers: the engine sums its 8 taps in float, this mode in double
    t_eng, t_pr = f.get_traces().astype(np.float64), pr.traces()
    assert np.max(np.abs(t_pr - t_eng)) <= 1e-6 * np.max(np.abs(t_eng))
    # and the float oracle agrees on the field
    o = oracle_for(room, "f32")
    idx, w = pr.taps
    o.run(room.n_steps, room.src_flat, room.signal(), idx, w.astype(np.float32))
    assert bits_equal(got, o.get_pressure_field())


def host_energy(o, room, p, vx_old, vy_old, vz_old):
    vx, vy, vz = o.get_velocity_x(), o.get_velocity_y(), o.get_velocity_z()
    s_p = float(np.sum(p.astype(np.float64) ** 2))
    s_v = float(np.dot(vx_old, vx) + np.dot(vy_old, vy) + np.dot(vz_old, vz))
    rc2 = room.rho * room.c * room.c
    return 0.5 * room.dx ** 3 * (s_p / rc2 + room.rho * s_v)


def test_energy_audit_matches_host_sum(cuda):
    from spectral_analyzer_b200.precision import PrecisionRoom
    room = small_room(steps=160, seed=13, kind="gaussian")
    every = 50
    pr = PrecisionRoom(room, "fp64", audit_capacity=8)
    pr.step(room.n_steps, every)
    log = pr.energy()
    assert list(log[:, 0]) == [0, 50, 100, 150]
    o = oracle_for(room, "f64")
    idx, w = pr.taps
    sig = room.signal().astype(np.float64)
    for row in log:
        n = int(row[0])
        o.run(n - o.step_count, room.src_flat, sig, idx, w)
        if n < len(sig):
            o.add_pressure(room.src_flat, float(sig[n]))
        p = o.get_pressure_field().ravel().copy()
        v_old = (o.get_velocity_x().copy(), o.get_velocity_y().copy(), o.get_velocity_z().copy())
        o.step(1)
        e = host_energy(o, room, p, *v_old)
        assert abs(row[2] - e) <= 1e-11 * abs(e), (n, row[2], e)
        assert abs(row[1] - float(np.sum(p ** 2)) / (room.rho * room.c ** 2)) <= 1e-11 * row[1]


def test_storage_modes_rank_against_fp64(cuda):
    from spectral_analyzer_b200.precision import study
    room = seeded_room(64, 64, 64, 1500, seed=14, n_rec=4, n_pml=8, source_kind="ricker")
    res = study(room, audit_every=500)
    err = {r["mode"]: r["trace_rel_l2"] for r in res["modes"]}
    e_dev = {r["mode"]: r["energy_max_rel_dev"] for r in res["modes"]}
    assert err["fp32"] <= 1e-5, err
    assert err["bf16c"] < err["bf16"] and err["fp16c"] < err["fp16"], err
    assert err["fp16c"] <= 1e-4 and err["bf16c"] <= 1e-2, err
    assert e_dev["fp32"] <= 1e-5, e_dev
    assert len(res["fp64"]["energy"]) == 3


def test_invalid_arguments(cuda):
    from spectral_analyzer_b200 import _native
    lib = _native.load()
    assert not lib.fdtd_b200_prec_create(8, 8, 8, 0.01, 343.0, 1.21, 2, None, 7, 0.0, 0.0, 0)
    assert not lib.fdtd_b200_prec_create(0, 8, 8, 0.01, 343.0, 1.21, 2, None, 0, 0.0, 0.0, 0)
    h = lib.fdtd_b200_prec_create(8, 8, 8, 0.01, 343.0, 1.21, 2, None, 0, 0.0, 0.0, 0)
    assert h
    try:
        import ctypes as C
        bad = (C.c_int * 8)(*([512] * 8))
        w = (C.c_double * 8)(*([0.125] * 8))
        assert lib.fdtd_b200_prec_set_receivers(h, 1, bad, w, 4, 0) == _native.FDTD_ERR_ARG
        assert lib.fdtd_b200_prec_set_source(h, -1, None, 0) == _native.FDTD_ERR_ARG
        assert lib.fdtd_b200_prec_step(h, 4, 1) == _native.FDTD_ERR_DIM   # audit log of size 0
    finally:
        lib.fdtd_b200_prec_destroy(h)


SIXTEEN = ("bf16", "fp16", "bf16c", "fp16c")
# room shapes: full and partial 128-column k tiles, rows beyond the last 8-row
# tile, rooms thinner than the 4-plane stencil, more planes than one segment
SHAPES = [(40, 36, 44), (37, 29, 23), (20, 24, 250), (33, 19, 129), (9, 5, 6), (150, 16, 128)]


def _pair(room, mode):
    from spectral_analyzer_b200.precision import PrecisionRoom
    a = PrecisionRoom(room, mode, kernel="fused")
    b = PrecisionRoom(room, mode, kernel="two_pass")
    assert a.kernel == "fused" and b.kernel == "two_pass"
    return a, b


@pytest.mark.parametrize("mode", SIXTEEN)
@pytest.mark.parametrize("dims", SHAPES)
def test_single_pass_16bit_step_equals_two_pass(cuda, mode, dims):
    """The single-pass 16-bit step stores the two-pass update's bits: pressure
    field and receiver traces equal after steps taken in uneven calls."""
    room = seeded_room(*dims, 90, seed=sum(dims), n_rec=3, n_pml=3, source_kind="ricker")
    a, b = _pair(room, mode)
    for n in (1, 40, 49):
        a.step(n)
    b.step(room.n_steps)
    pa, pb = a.pressure(), b.pressure()
    assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64)), \
        (mode, dims, int(np.sum(pa != pb)), float(np.max(np.abs(pa - pb))))
    assert np.array_equal(a.traces().view(np.uint64), b.traces().view(np.uint64))
    assert np.any(pa != 0.0)
    # one launch per step, plus one receiver record at the end of each call
    assert a.launch_count == room.n_steps + 3
    a.close()
    b.close()


@pytest.mark.parametrize("mode", ("bf16c", "fp16"))
def test_single_pass_mixes_with_audit_steps(cuda, mode):
    """Steps that take the energy audit run the two-pass update on the current
    velocity set; the result is unchanged and the energy log equals the
    two-pass run's."""
    from spectral_analyzer_b200.precision import PrecisionRoom
    room = seeded_room(40, 36, 44, 120, seed=21, n_rec=3, n_pml=4, source_kind="ricker")
    a = PrecisionRoom(room, mode, kernel="fused", audit_capacity=16)
    b = PrecisionRoom(room, mode, kernel="two_pass", audit_capacity=16)
    a.step(55, 25)
    a.step(65, 25)
    b.step(120, 25)
    assert np.array_equal(a.pressure().view(np.uint64), b.pressure().view(np.uint64))
    assert np.array_equal(a.traces().view(np.uint64), b.traces().view(np.uint64))
    ea, eb = a.energy(), b.energy()
    assert ea.shape == eb.shape and np.array_equal(ea[:, 0], eb[:, 0])
    np.testing.assert_allclose(ea[:, 1:], eb[:, 1:], rtol=1e-12, atol=0)


def test_single_pass_kernel_choice(cuda):
    from spectral_analyzer_b200.precision import PrecisionRoom
    room = seeded_room(16, 16, 16, 4, seed=3, n_rec=1, n_pml=2)
    assert PrecisionRoom(room, "bf16").kernel == "fused"
    assert PrecisionRoom(room, "fp32").kernel == "two_pass"
    with pytest.raises(RuntimeError):
        PrecisionRoom(room, "fp64", kernel="fused")
