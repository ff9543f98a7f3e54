"""The fit-worker protocol (motility_fit.js:996-1004, main.ts:325-353):
{id, radial, opt} -> {id, result} | {id, error}, served off the caller's
thread; runFit futures; fallback to the calling thread after a worker
failure. No GPU: the worker is given a host stand-in for the analysis (the
library's analysis needs the device; tests/test_gpu_verdicts.py serves the
same protocol with it)."""
import threading

import numpy as np
import pytest

import oracle as O


def _stand_in(radial, dxUm=1.0, fps=1.0, geometry="3d", exposureLocked=True, swimMin=2.0):
    """A deterministic host function of the record and options, shaped like
    the analysis result; raises on an empty record like the analysis."""
    if radial.NB < 1:
        raise ValueError("analyze_motility: invalid Radial record or options")
    tsi = float(O.temporal_structure_index(radial))
    verdict = "MOTILE" if tsi >= 0.15 else "NO_DYNAMICS"
    return {"verdict": verdict if exposureLocked else "UNLOCKED_EXPOSURE", "physicsVerdict": verdict,
            "TSI": tsi, "geometry": geometry, "fps": fps}


@pytest.fixture(scope="module")
def scenario_radial():
    sc = O.SCENARIOS[0]
    ref, radial, _ = O.run_scenario(sc)
    return sc, ref, radial


def _opt(sc, **kw):
    return dict(dxUm=sc["sim"]["dxUm"], fps=sc["sim"]["fps"], geometry=sc["geometry"], **kw)


def test_messages_and_replies(scenario_radial):
    from hackathon_b200.fit_worker import FitWorker
    from hackathon_b200.radial import Radial
    sc, ref, radial = scenario_radial
    replies, done = [], threading.Event()

    def on_message(rep):
        replies.append(rep)
        if len(replies) == 3:
            done.set()

    bad = Radial(N=256, NB=0, L=128, kCenter=np.zeros(0), kNodes=np.zeros(0), nModes=np.zeros(0, np.uint32),
                 D=np.zeros(0), P=np.zeros(0), drift=np.zeros(0))
    with FitWorker(on_message=on_message, analyze=_stand_in) as w:
        w.post_message({"id": 7, "radial": radial, "opt": _opt(sc)})
        w.post_message({"id": 8, "radial": bad, "opt": _opt(sc)})
        w.post_message({"id": 9, "radial": radial, "opt": _opt(sc, exposureLocked=False)})
        assert done.wait(120)
    assert [r["id"] for r in replies] == [7, 8, 9]
    assert replies[0]["result"] == _stand_in(radial, **_opt(sc))
    assert replies[0]["result"]["verdict"] == ref["verdict"] == "MOTILE"
    assert "error" in replies[1] and "analyze_motility" in replies[1]["error"]
    assert replies[2]["result"]["verdict"] == "UNLOCKED_EXPOSURE"


def test_run_fit_futures_and_failure_fallback(scenario_radial):
    from hackathon_b200.fit_worker import FitWorker
    sc, ref, radial = scenario_radial
    w = FitWorker(analyze=_stand_in)
    futs = [w.run_fit(radial, _opt(sc)) for _ in range(3)]
    assert all(f.result(120)["verdict"] == ref["verdict"] for f in futs)
    # a failed worker: pending and later fits run on the calling thread
    w._fail()
    assert w.failed
    assert w.fit(radial, _opt(sc))["verdict"] == ref["verdict"]
    assert w.run_fit(radial, _opt(sc)).result(0)["verdict"] == ref["verdict"]
    w.close()


def test_bin_fits_mode_is_validated(scenario_radial):
    from hackathon_b200.fit_worker import FitWorker
    sc, _, radial = scenario_radial
    with FitWorker(analyze=_stand_in) as w:
        with pytest.raises(RuntimeError, match="binFits"):
            w.run_fit(radial, _opt(sc, binFits="newton")).result(120)
