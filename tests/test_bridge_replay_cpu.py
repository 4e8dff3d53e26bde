"""The bridge call log against the C restatement (CPU).

The log (tests/golden/bridge_replay.*) was recorded from the reference's own
acoustic_fdtd_bridge.py over the compiled reference; replaying it on the
oracle's restatement pins the restatement on the bridge's real voxelised
guitar body (walls, plate, soundhole, cut-cell fractions, bridge kernel) with
every result equal bit for bit.  The same log drives the GPU engine in
test_bridge_replay_gpu.py.
"""
import numpy as np

import bridge_replay as br


def test_fixture_shape():
    meta, arrays = br.load()
    ini = meta["calls"][0]
    assert ini["m"] == "__init__"
    kw = ini["kwargs"]
    # the bridge passes every constructor argument by keyword
    assert set(kw) >= {"Nx", "Ny", "Nz", "dx", "c", "rho_air", "cell_type", "plate_iz",
                       "plate_active", "plate_mass_density", "plate_stiffness_D", "plate_alpha_M",
                       "plate_beta_K", "n_pml"}
    nx, ny, nz = (kw[k] for k in ("Nx", "Ny", "Nz"))
    assert [nx, ny, nz] == meta["grid"]
    ct = br.decode(kw["cell_type"], arrays)
    assert ct.size == nx * ny * nz and set(np.unique(ct)) <= {0, 1, 2}
    assert (ct == 1).any() and (ct == 2).any()              # walls and the soundboard
    methods = [c["m"] for c in meta["calls"]]
    assert methods[1:3] == ["set_face_fractions", "set_bridge_sources"]
    assert methods.count("step") == meta["steps"]
    assert methods.count("sample_pressure") == meta["mic_samples"]


def test_bridge_calls_on_oracle_match_reference():
    from oracle import OracleFDTD
    meta, arrays = br.load()
    f, bad = br.replay(OracleFDTD, meta, arrays)
    assert not bad, bad[:5]
    P = f.get_pressure_field()
    for q, s in enumerate(br.bridge_slices(P, meta)):
        assert br.bits_equal(s, arrays[f"bridge_slice{q}"]), q
    assert br.bits_equal(f.get_plate_displacement(), arrays["bridge_plate_w"])
