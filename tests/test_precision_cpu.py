"""Host logic of the storage-precision study, no GPU."""
import numpy as np
import pytest

from spectral_analyzer_b200.precision import BYTES_PER_VALUE, MODES, fp16_scales, pressure_taps


@pytest.mark.parametrize("dims", [(40, 36, 44), (7, 5, 3), (1, 9, 4)])
def test_pressure_taps_match_oracle(dims):
    from oracle import OracleFDTD
    nx, ny, nz = dims
    rng = np.random.default_rng(4)
    xyz = np.concatenate([rng.uniform(-2, max(dims) + 2, (12, 3)),
                          [[nx - 1, ny - 1, nz - 1], [0, 0, 0], [nx - 1.5, 0.25, nz - 0.75]]])
    xyz = xyz.astype(np.float32)
    o = OracleFDTD(nx, ny, nz, 0.01, n_pml=0)
    ref_i, ref_w = o.precompute_pressure_samplers(xyz)
    idx, w = pressure_taps(nx, ny, nz, xyz)
    assert np.array_equal(idx, ref_i)
    assert np.array_equal(w.view(np.uint32), ref_w.view(np.uint32))


def test_fp16_scales_are_powers_of_two():
    for amp in (1.0, 0.3, 5.0, 1e-3):
        ps, vs = fp16_scales(amp)
        assert np.log2(ps) == int(np.log2(ps)) and vs / ps == 512.0
        assert ps * amp * 40 < 65504          # a 40x-amplitude pressure still fits half
    assert fp16_scales(1.0) == (1024.0, 524288.0)


def test_mode_table():
    assert sorted(MODES.values()) == list(range(6))
    assert set(BYTES_PER_VALUE) == set(MODES)
    assert BYTES_PER_VALUE["bf16c"] == BYTES_PER_VALUE["fp32"] == 4
