"""GPU parity of the AMR pressure backend against the compiled reference.

tests/golden/amr_guitar.* holds a guitar-body AMR grid built by the reference's
own Python (acoustic_amr.build_guitar_amr_grid and
build_amr_coevolver_descriptor: 42,983 cells on two refinement levels, walls,
plate, PML cells, 128,758 faces, a 47x67 plate with 1,985 active nodes) and the
records of the reference's own AMR stepper (csrc/kernels/acoustic_amr.cpp)
driven by tests/amr_script.py for 200 steps: microphone pressure and velocity,
saddle and neck displacements, return codes, and hashes of the final
pressure, velocity and plate fields.  The engine, built from the same
descriptor through AcousticAMR.from_descriptor (the reference backend's set-up
order), must reproduce every record bit for bit, for gradient orders 2 and 8
and the three border modes; the stated tolerance (1e-5 relative L2 on the
microphone traces) is asserted as well.
"""
import numpy as np
import pytest

import amr_script as S

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5


@pytest.fixture(scope="module")
def fixture():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return S.load()


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


@pytest.mark.parametrize("name,order,border", S.CASES)
def test_amr_backend_matches_reference(fixture, name, order, border):
    from spectral_analyzer_b200.amr import AcousticAMR
    meta, arrays, desc, sc, mics = fixture
    case = meta["cases"][name]
    s = AcousticAMR.from_descriptor(desc, gradient_order=order, border=border)
    assert s.dt == case["dt"]
    l0 = s.launch_count
    out = S.run(s, desc, sc, mics, meta["steps"])
    assert s.launch_count - l0 >= 3 * meta["steps"]          # the step kernels ran on the GPU
    for k in S.RECORDS:
        want = arrays[f"{name}/{k}"]
        assert np.array_equal(bits(out[k]), bits(want)), k
    p, want = out["mic_p"], arrays[f"{name}/mic_p"]
    assert np.linalg.norm(p - want) <= TRACE_TOL * np.linalg.norm(want)
    assert np.abs(want).max() > 0
    for k in ("P", "V", "W"):
        assert S.sha(out[k]) == case["sha256"][k], k
    assert s.step_count == case["step_count"]
    s.close()


def test_amr_divergence_stops_like_reference(fixture):
    from spectral_analyzer_b200.amr import AcousticAMR, SK_ERR_DIVERGED
    meta, arrays, desc, sc, mics = fixture
    dv = meta["diverge"]
    s = AcousticAMR.from_descriptor(desc, gradient_order=2, border=S.CASES[0][2])
    s.inject_pressure_nearest(np.array(dv["xyz"]), dv["value"])
    rc = [s.step_rc(1), s.step_rc(1)]
    assert rc == dv["rc"] == [SK_ERR_DIVERGED, SK_ERR_DIVERGED]
    assert s.step_count == dv["step_count"]
    assert S.sha(s.get_pressure()) == dv["P_sha256"]
    assert S.sha(s.get_plate_displacement()) == dv["W_sha256"]
    with pytest.raises(RuntimeError, match="rc=-3"):
        s.step(1)
    # a reset makes the handle usable again, and an async window behaves like amr_step
    s.reset()
    assert s.step_count == 0
    s.step_async(5)
    assert s.synchronize() == 0 and s.step_count == 5
    s.close()


def test_amr_async_window_equals_stepwise(fixture):
    """Steps queued in one window give the fields of one-at-a-time stepping."""
    from spectral_analyzer_b200.amr import AcousticAMR
    meta, arrays, desc, sc, mics = fixture
    outs = []
    for mode in ("window", "single"):
        s = AcousticAMR.from_descriptor(desc, gradient_order=2, border=S.CASES[0][2])
        s.inject_pressure_nearest(np.array([0.0, -0.02, 0.03]), 1.0)
        if mode == "window":
            s.step_async(120)
            assert s.synchronize() == 0
        else:
            for _ in range(120):
                s.step(1)
        outs.append((s.get_pressure(), s.get_velocity(), s.get_plate_displacement()))
        s.close()
    for a, b in zip(*outs):
        assert np.array_equal(bits(a), bits(b))
    assert np.abs(outs[0][0]).max() > 0


def test_shim_exports_amr():
    import importlib
    import os
    import sys
    shim = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "spectral_analyzer_b200", "shim")
    sys.path.insert(0, shim)
    try:
        sk = importlib.import_module("_spectral_kernels")
        from spectral_analyzer_b200.amr import AcousticAMR
        assert sk.AcousticAMR is AcousticAMR
    finally:
        sys.path.remove(shim)
