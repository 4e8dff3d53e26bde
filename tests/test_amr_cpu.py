"""AMR fixture against the compiled reference (CPU), and the AMR C-ABI header.

tests/golden/amr_guitar.* holds a guitar-body AMR grid made by the reference's
own Python builder and the records of the reference's own AMR stepper driven
by tests/amr_script.py.  Re-running the script on the compiled reference
(oracle/_ref/libamr_ref.so) must reproduce every record bit for bit; the GPU
engine is held to the same records in test_amr_gpu.py.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import amr_script as S
from conftest import ROOT

REFERENCE_AMR_ABI = [
    "amr_create", "amr_get_last_create_error_stage", "amr_get_last_create_error_message",
    "amr_get_create_progress_active", "amr_get_create_progress_done_faces",
    "amr_get_create_progress_total_faces", "amr_destroy", "amr_step", "amr_reset",
    "amr_inject_pressure_nearest", "amr_get_pressure", "amr_get_cell_centers", "amr_get_velocity",
    "amr_get_dt", "amr_get_step_count", "amr_scatter_pressure_uniform", "amr_set_border_condition",
    "amr_setup_plate", "amr_set_bridge_plate_sources", "amr_set_neck_plate_sources",
    "amr_inject_bridge_drive", "amr_inject_plate_force", "amr_sample_plate_displacement_batch",
    "amr_sample_plate_weighted", "amr_get_plate_displacement", "amr_setup_mic_samplers", "amr_sample_mics",
]


def declared():
    txt = open(os.path.join(ROOT, "include", "acoustic_amr_b200.h")).read()
    txt = "\n".join(l for l in txt.splitlines() if not l.lstrip().startswith("#"))
    return re.findall(r"AMR_B200_API\s+[\w\s\*]*?\b(\w+)\s*\(", txt)


def test_header_and_library_cover_reference_abi():
    names = declared()
    assert len(names) == len(set(names))
    assert set(REFERENCE_AMR_ABI) <= set(names)
    lib = C.CDLL(os.path.join(ROOT, "spectral_analyzer_b200", "libacoustic_fdtd_b200.so"))
    for n in names:
        assert hasattr(lib, n), n
    from spectral_analyzer_b200 import amr
    assert set(names) == set(amr.AMR_SIGNATURES)


def test_null_and_bad_arguments_without_gpu():
    """Handle and argument checks return the reference's codes before any CUDA call."""
    from spectral_analyzer_b200 import amr
    L = amr.load()
    assert L.amr_step(None, 1) == amr.SK_ERR_NULL_STATE
    assert L.amr_reset(None) == amr.SK_ERR_NULL_STATE
    assert L.amr_get_dt(None) == 0.0 and L.amr_get_step_count(None) == 0
    assert L.amr_inject_pressure_nearest(None, None, 1.0) == amr.SK_ERR_NULL_STATE
    L.amr_destroy(None)
    # invalid topology: a face joining a cell to itself
    cc = np.zeros((2, 3))
    one = np.ones(2)
    ct = np.zeros(2, np.uint8)
    fn = np.array([0], np.int32)
    fa = np.ones(1)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert not L.amr_create(2, p(cc), p(one), p(one), p(ct), 1, p(fn), p(fn), p(fa), p(fa), p(fa),
                            343.0, 1.21, 0.01, 2)
    assert L.amr_get_last_create_error_message().decode() == "input validation failed"
    assert not L.amr_create(2, p(cc), p(one), p(one), p(ct), 1, p(fn), p(fn + 1), p(fa), p(fa), p(fa),
                            343.0, 1.21, 0.01, 4)
    assert "gradient_order" in L.amr_get_last_create_error_message().decode()


@pytest.mark.parametrize("name,order,border", S.CASES)
def test_reference_reproduces_fixture(name, order, border):
    from amr_oracle import AMRRef
    meta, arrays, desc, sc, mics = S.load()
    steps = 60                                  # a prefix keeps the CPU suite short
    r = AMRRef(desc, gradient_order=order, border=border)
    out = S.run(r, desc, sc, mics, steps)
    for k in S.RECORDS:
        want = arrays[f"{name}/{k}"][:steps]
        assert np.array_equal(np.asarray(out[k]).view(np.uint32) if out[k].dtype == np.float32 else out[k],
                              want.view(np.uint32) if want.dtype == np.float32 else want), k
    assert r.dt == meta["cases"][name]["dt"]
