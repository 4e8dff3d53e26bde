"""C-ABI checks that need no GPU: the library loads and exports every declared symbol."""
import ctypes as C
import glob
import os
import re

import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "spectral_analyzer_b200", "libacoustic_fdtd_b200.so")

# The reference's acoustic_fdtd.h declares exactly these 26 entry points.
REFERENCE_ABI = [
    "fdtd_create", "fdtd_destroy", "fdtd_set_bridge_sources", "fdtd_inject_bridge",
    "fdtd_inject_bridge_drive", "fdtd_inject_plate_force", "fdtd_set_face_fractions",
    "fdtd_sample_plate_weighted", "fdtd_precompute_pressure_samplers",
    "fdtd_precompute_velocity_samplers", "fdtd_sample_pressure_precomputed",
    "fdtd_sample_velocity_precomputed", "fdtd_step", "fdtd_get_step_count", "fdtd_get_dt",
    "fdtd_reset", "fdtd_get_pressure_field", "fdtd_get_plate_displacement",
    "fdtd_sample_plate_displacement_batch", "fdtd_sample_pressure", "fdtd_get_velocity_dims",
    "fdtd_get_velocity_x", "fdtd_get_velocity_y", "fdtd_get_velocity_z", "fdtd_sample_velocity",
    "fdtd_get_surface_emission",
]


def declared_symbols():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = "\n".join(l for l in open(h).read().splitlines() if not l.lstrip().startswith("#"))
        names += re.findall(r"FDTD_B200_API\s+[\w\s\*]*?\b(\w+)\s*\(", txt)
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        pytest.fail(f"engine library not built: {LIB} (run `python -m spectral_analyzer_b200.build`)")
    return C.CDLL(LIB)


def test_header_declares_reference_abi():
    names = declared_symbols()
    assert len(names) == len(set(names))
    for n in REFERENCE_ABI:
        assert n in names, n


def test_library_exports_every_declared_symbol(lib):
    for n in declared_symbols():
        assert hasattr(lib, n), n


def test_native_binding_covers_header():
    from spectral_analyzer_b200 import _native
    assert set(declared_symbols()) == set(_native.SIGNATURES)
    _native.load()


def test_field_layout_without_gpu(lib):
    from spectral_analyzer_b200 import _native
    L = _native.load()
    sz, nb = C.c_int(), C.c_size_t()
    assert L.fdtd_b200_field_layout(512, 384, 256, C.byref(sz), C.byref(nb)) == 0
    assert sz.value == 256 and nb.value == 512 * 384 * 256 * 4
    assert L.fdtd_b200_field_layout(7, 5, 6, C.byref(sz), C.byref(nb)) == 0
    assert sz.value == 8 and nb.value == 7 * 5 * 8 * 4
    assert L.fdtd_b200_field_layout(0, 5, 6, C.byref(sz), C.byref(nb)) == _native.FDTD_ERR_ARG


def test_null_handle_contract(lib):
    """Calls with a NULL handle return the reference's codes and never touch a device."""
    from spectral_analyzer_b200 import _native
    L = _native.load()
    assert L.fdtd_step(None, 1) == _native.FDTD_ERR_NULL
    assert L.fdtd_reset(None) == _native.FDTD_ERR_NULL
    assert L.fdtd_get_step_count(None) == 0
    assert L.fdtd_get_dt(None) == 0.0
    assert L.fdtd_inject_bridge(None, 1.0, 0.0, 1.0) == _native.FDTD_ERR_UNSTABLE
    a, b, c = C.c_int(7), C.c_int(7), C.c_int(7)
    L.fdtd_get_velocity_dims(None, C.byref(a), C.byref(b), C.byref(c))
    assert (a.value, b.value, c.value) == (0, 0, 0)
    L.fdtd_destroy(None)


def test_create_rejects_bad_arguments(lib):
    """Argument checks of acoustic_fdtd.cpp:342-344 happen before any CUDA call."""
    from spectral_analyzer_b200 import _native
    L = _native.load()
    ct = (C.c_uint8 * 8)()
    pa = (C.c_uint8 * 4)()
    P8 = C.cast(ct, _native.P_u8)
    P4 = C.cast(pa, _native.P_u8)
    assert not L.fdtd_create(0, 2, 2, 0.01, 343.0, 1.21, P8, 1, P4, 7.0, 0.45, 2.0, 1e-5, 1)
    assert not L.fdtd_create(2, 2, 2, -0.01, 343.0, 1.21, P8, 1, P4, 7.0, 0.45, 2.0, 1e-5, 1)
    assert not L.fdtd_create(2, 2, 2, 0.01, 0.0, 1.21, P8, 1, P4, 7.0, 0.45, 2.0, 1e-5, 1)
    assert not L.fdtd_create(2, 2, 2, 0.01, 343.0, 1.21, None, 1, P4, 7.0, 0.45, 2.0, 1e-5, 1)


def test_dropin_signature_matches_reference():
    """Constructor keywords, defaults and method names of the pybind class."""
    import inspect
    from spectral_analyzer_b200.fdtd import AcousticFDTD
    sig = inspect.signature(AcousticFDTD.__init__)
    want = {"c": 343.0, "rho_air": 1.21, "plate_mass_density": 7.0, "plate_stiffness_D": 0.45,
            "plate_alpha_M": 2.0, "plate_beta_K": 1e-5, "n_pml": 10}
    for k, v in want.items():
        assert sig.parameters[k].default == v, k
    for m in ("set_bridge_sources", "set_face_fractions", "inject_bridge", "step", "reset",
              "get_pressure_field", "get_plate_displacement", "sample_pressure", "sample_velocity",
              "get_surface_emission", "get_velocity_dims", "get_velocity_x", "get_velocity_y",
              "get_velocity_z"):
        assert callable(getattr(AcousticFDTD, m)), m
    for p in ("dt", "step_count"):
        assert isinstance(getattr(AcousticFDTD, p), property), p


def test_shim_module_exports_dropin():
    import importlib
    import sys
    shim_dir = os.path.join(ROOT, "spectral_analyzer_b200", "shim")
    sys.path.insert(0, shim_dir)
    try:
        sk = importlib.import_module("_spectral_kernels")
        from spectral_analyzer_b200.fdtd import AcousticFDTD
        assert sk.AcousticFDTD is AcousticFDTD
    finally:
        sys.path.remove(shim_dir)
