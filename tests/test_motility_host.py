"""The library's decision layer (ddm_analyze_motility, host FP64) reproduces
the oracle's analyzeMotility exactly on the oracle pipeline's Radial records
of the reference's validation scenarios, and rejects malformed records
(no GPU)."""
import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("sc", O.SCENARIOS[:4], ids=[s["name"] for s in O.SCENARIOS[:4]])
def test_decision_layer_equals_oracle(sc):
    from hackathon_b200.motility import analyze_motility
    ref, radial, _ = O.run_scenario(sc)
    got = analyze_motility(radial, dxUm=sc["sim"]["dxUm"], fps=sc["sim"]["fps"], geometry=sc["geometry"])
    assert got["verdict"] == ref["verdict"] and got["physicsVerdict"] == ref["physicsVerdict"]
    for k in ("TSI", "alpha", "vbar", "Ddiff", "dBIC", "driftMag", "driftAngleDeg", "mu", "nEff", "rho"):
        a, b = got[k], ref[k]
        assert (np.isnan(a) and np.isnan(b)) or a == b, (k, a, b)


def test_rejects_malformed_radial():
    from hackathon_b200.engine import DdmArgError
    from hackathon_b200.motility import analyze_motility
    from hackathon_b200.radial import Radial
    r = Radial(N=256, NB=0, L=128, kCenter=np.zeros(0), kNodes=np.zeros(0), nModes=np.zeros(0, np.uint32),
               D=np.zeros(0), P=np.zeros(0), drift=np.zeros(0))
    with pytest.raises(DdmArgError):
        analyze_motility(r)
