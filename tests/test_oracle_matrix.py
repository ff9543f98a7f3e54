"""The reference's end-to-end integration test (test/t_validation_matrix.mjs):
11 seeded scenarios through the FP64 oracle pipeline, checked against the
reference's pass criteria AND the outputs it publishes (README.md section 6),
plus the G5 exposure gate."""
import pytest

import oracle as O


@pytest.mark.parametrize("sc", O.SCENARIOS, ids=[s["name"] for s in O.SCENARIOS])
def test_scenario(sc, golden):
    res, _, _ = O.run_scenario(sc)
    assert O.check_scenario(sc, res) == []
    pub = golden["matrix"][sc["name"]]
    assert res["verdict"] == pub["verdict"]
    # published values are printed to 2-3 significant digits
    if "alpha" in pub:
        assert abs(res["alpha"] - pub["alpha"]) <= 0.006
    if "vbar" in pub:
        assert abs(res["vbar"] - pub["vbar"]) <= 0.06
    assert abs(res["driftMag"] - pub["V"]) <= 0.006
    if "angle" in pub:
        d = abs(res["driftAngleDeg"] - pub["angle"]) % 360
        assert min(d, 360 - d) <= 0.6


def test_exposure_gate():
    """t_validation_matrix.mjs:97-101."""
    res, _, _ = O.run_scenario(O.SCENARIOS[0], exposureLocked=False)
    assert res["verdict"] == "UNLOCKED_EXPOSURE" and res["physicsVerdict"] == "MOTILE"


def test_bins_reference_geometry():
    """makeBins at the reference geometry: 15,676 binned modes over 32 bins
    (the count the reference documents for N=256, KMIN=4, KMAX=100)."""
    b = O.make_bins(256, 32, 4, 100)
    assert b["binOffsets"][-1] == 15676
    assert int(b["nModes"].sum()) == 15676
    # no mode on the skipped half-line or the Nyquist lines
    kx, ky = b["binModes"][:, 1], b["binModes"][:, 2]
    assert not ((kx == 0) & (ky <= 0)).any()
    assert not ((kx == 128) | (ky == -128)).any()
