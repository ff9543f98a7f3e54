"""The host half of the library's analysis (csrc/analysis.cu) against the
oracle on the oracle pipeline's Radial records of the reference's validation
scenarios, without a GPU: the bins the analysis keeps (prepare,
motility_fit.js:383-401), the temporal structure index (:735-749), the
phase-drift least squares with and without a swimmer lag mask (:672-725), and
the q-scaling exponent (:771-804). These are independent implementations
(the oracle is a line-by-line FP64 restatement of the reference; the library's
host code is its own), compared to 1e-12 relative. The device fits are
compared with the oracle in tests/test_gpu_global_fit.py."""
import numpy as np
import pytest

import oracle as O

SCEN = [O.SCENARIOS[i] for i in (0, 3, 6, 9)]  # motile_3d, killed_brownian, flow_0deg_10ums, motile_in_flow


@pytest.fixture(scope="module", params=SCEN, ids=[s["name"] for s in SCEN])
def case(request):
    sc = request.param
    ref, radial, _ = O.run_scenario(sc)
    return sc, ref, radial


def _close(a, b, rel=1e-12):
    if np.isnan(a) or np.isnan(b):
        return np.isnan(a) and np.isnan(b)
    return abs(a - b) <= rel * max(abs(a), abs(b), 1e-300)


def test_prepared_bins_and_tsi(case):
    from hackathon_b200 import motility as M
    sc, ref, radial = case
    bins, nlags = M.prepared_bins(radial, sc["sim"]["dxUm"], sc["sim"]["fps"])
    assert len(bins) == ref["nbins"] and nlags == ref["nlags"] == len(O.lag_grid(radial.L))
    assert _close(M.temporal_structure_index(radial), O.temporal_structure_index(radial))
    assert _close(M.temporal_structure_index(radial), ref["TSI"])


def test_drift_without_and_with_swimmer_mask(case):
    from hackathon_b200 import motility as M
    sc, ref, radial = case
    dx, fps = sc["sim"]["dxUm"], sc["sim"]["fps"]
    keys = ("Vx", "Vy", "mag", "sigma", "angleDeg", "samples")
    a, b = M.estimate_drift(radial, dx, fps), O.estimate_drift(radial, dx, fps, swimmer=None)
    assert a["pairs"] == b["pairs"] and a["significant"] == b["significant"]
    assert all(_close(a[k], b[k]) for k in keys), (a, b)
    # a swimmer at the oracle's fitted (vbar, Z): lags where |g| < 0.2
    v, Z = max(ref["vbar"], 1.0), ref["Z"] if ref["Z"] > 0 else 4.0
    bins, _ = M.prepared_bins(radial, dx, fps)
    L, dt = radial.L, 1.0 / fps
    q = 2 * np.pi * np.asarray(radial.kCenter)[bins] / (radial.N * dx)
    mask = np.zeros((len(bins), L), np.uint8)
    for i in range(len(bins)):
        for t in range(1, L - 1):
            mask[i, t] = abs(O.isf3d(q[i] * v * t * dt, Z)) < 0.2
    a = M.estimate_drift(radial, dx, fps, lag_mask=mask)
    b = O.estimate_drift(radial, dx, fps, swimmer=(v, Z))
    assert a["pairs"] == b["pairs"] and a["significant"] == b["significant"]
    assert all(_close(a[k], b[k]) for k in keys), (a, b)


def test_scaling_exponent(case):
    from hackathon_b200 import motility as M
    sc, ref, radial = case
    dx, fps = sc["sim"]["dxUm"], sc["sim"]["fps"]
    if ref.get("insufficient") or "dBIC" not in ref:
        pytest.skip("no fits")
    best, swim = (ref["swim"], True) if ref["dBIC"] > 0 else (ref["brown"], False)
    _, amps = O.eval_model(radial, best, dx, fps, sc["geometry"], swim=swim)
    nb = ref["nbins"]
    mu = M.scaling_exponent(radial, amps[:2 * nb].reshape(nb, 2), dx, fps)
    assert _close(mu, ref["mu"], 1e-10), (mu, ref["mu"])


def test_rejects_malformed_radial():
    from hackathon_b200.engine import DdmArgError
    from hackathon_b200.motility import analyze_motility, estimate_drift
    from hackathon_b200.radial import Radial
    r = Radial(N=256, NB=0, L=128, kCenter=np.zeros(0), kNodes=np.zeros(0), nModes=np.zeros(0, np.uint32),
               D=np.zeros(0), P=np.zeros(0), drift=np.zeros(0))
    with pytest.raises(DdmArgError):
        analyze_motility(r)
    with pytest.raises(DdmArgError):
        estimate_drift(r)
