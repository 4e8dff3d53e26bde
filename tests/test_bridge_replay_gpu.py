"""The reference's Python bridge on the GPU engine.

The call log in tests/golden/bridge_replay.* was recorded from the reference's
own acoustic_fdtd_bridge.py over the compiled reference: FDTDCoEvolver.
from_body_scene on the string_plate body scene (voxelise_guitar_body,
_apply_soundhole_cutout, compute_cut_cell_fractions, build_bridge_kernel;
acoustic_fdtd_bridge.py:647-699), a seeded pluck driven through coev.fdtd as the
co-evolver's substep drives it (bridge-cell forces, a neck force on plate
cells, step, saddle read-out), the microphones through sample_at_receivers
(:761-779) once per audio sample, and the field accessors (:737-757).  Here
the same calls go, in the same order and with the same keyword arguments, to
the engine class the bridge imports (``from _spectral_kernels import
AcousticFDTD`` resolved through spectral_analyzer_b200/shim), and every result
— microphone samples, saddle displacements, return codes, the plate
displacement, the bridge's slices and the four fields — must equal the
reference's bit for bit (the 1e-5 relative L2 bound on the microphone trace is
asserted as well).
"""
import importlib
import os
import sys

import numpy as np
import pytest

import bridge_replay as br

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5
SHIM = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                    "spectral_analyzer_b200", "shim")


@pytest.fixture(scope="module")
def engine_cls():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    if SHIM not in sys.path:
        sys.path.insert(0, SHIM)
    mod = importlib.import_module("_spectral_kernels")
    from spectral_analyzer_b200 import AcousticFDTD
    assert mod.AcousticFDTD is AcousticFDTD
    return mod.AcousticFDTD


@pytest.mark.parametrize("kernel", ["auto", "two_pass"])
def test_bridge_calls_on_engine_match_reference(engine_cls, kernel):
    meta, arrays = br.load()
    mics = []

    class Engine(engine_cls):
        def __init__(self, *a, **kw):
            super().__init__(*a, **kw)
            self.set_kernel(kernel)

    f, bad = br.replay(Engine, meta, arrays,
                       on_result=lambda c, out: mics.append(out) if c["m"] == "sample_pressure" else None)
    assert not bad, bad[:5]
    # the microphone trace, against the stated tolerance
    ref = np.stack([br.decode(c["result"], arrays) for c in meta["calls"] if c["m"] == "sample_pressure"])
    got = np.stack(mics)
    assert got.shape == (meta["mic_samples"], 3)
    assert np.linalg.norm(got - ref) <= TRACE_TOL * np.linalg.norm(ref)
    assert np.abs(ref).max() > 0
    # the bridge's own outputs after the run: slices of the field and the plate
    P = f.get_pressure_field()
    assert br.sha(P) == meta["fields_sha256"]["P"]
    for q, s in enumerate(br.bridge_slices(P, meta)):
        assert br.bits_equal(s, arrays[f"bridge_slice{q}"]), q
    # the engine's on-device slice gather follows the bridge's slicing rule
    for q, (axis, idx) in enumerate([(2, -1), (0, 10), (1, meta["grid"][1] // 3), (2, meta["plate_iz"])]):
        assert br.bits_equal(f.get_volume_slice(axis, idx), arrays[f"bridge_slice{q}"]), (axis, idx)
    w = f.get_plate_displacement()
    assert br.bits_equal(w, arrays["bridge_plate_w"])
    assert np.abs(w).max() > 0
    assert f.step_count == meta["steps"]
    f.close()
