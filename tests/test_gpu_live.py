"""Live ring-buffer mode on the GPU: a live computeTemporal (analysis stream)
with frames ingested into the ring while it runs gives exactly the result of
a synchronous analysis of the same snapshot, because the slots those frames
overwrite lie inside the snapshot's guard; and the dashboard's loop
(FrameClock + LiveAnalyzer + FitWorker) reaches the reference's verdict on a
validation scenario streamed frame by frame, widening its guard after a
stale analysis (main.ts:366-398)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

H = pytest.importorskip("hackathon_b200")
from hackathon_b200.live import FrameClock, LiveAnalyzer  # noqa: E402


def test_live_equals_synchronous_under_concurrent_ingest():
    N, T, L = 64, 128, 32
    sim = dict(O.BASE, N=N, T=T + 24, seed=31, swimmers=dict(n=12, vbar=20.0, sigma=8.0, geometry="3d"),
               passive=dict(n=12))
    frames, _, _ = O.simulate(sim)
    clock = FrameClock(fps=30.0, T=T)
    live = H.DdmEngine.create(N=N, T=T, L=L, NB=8, kmin=2, kmax=28)
    sync = H.DdmEngine.create(N=N, T=T, L=L, NB=8, kmin=2, kmax=28)
    for n in range(T):
        p = clock.place(1000.0 * n / 30.0)
        live.ingest_frames(frames[n:n + 1], [p["slot"]])
        sync.ingest_frames(frames[n:n + 1], [p["slot"]])
    snap = clock.snapshot(guard=16)
    live.compute_temporal(snap.order, snap.mask, live=True)
    for n in range(T, T + 12):  # overwrite the slots of time indices 0..11 (inside the guard)
        p = clock.place(1000.0 * n / 30.0)
        live.ingest_frames(frames[n:n + 1], [p["slot"]])
    live.wait_analysis()
    assert live.analysis_done
    rl = live.read_radial()
    sync.compute_temporal(snap.order, snap.mask)
    rs = sync.read_radial()
    assert np.array_equal(rl.D, rs.D) and np.array_equal(rl.P, rs.P) and np.array_equal(rl.drift, rs.drift)
    # the live record stays readable after more ingests
    p = clock.place(1000.0 * (T + 12) / 30.0)
    live.ingest_frames(frames[T + 12:T + 13], [p["slot"]])
    assert np.array_equal(live.read_radial().D, rs.D)
    # a second live analysis replaces it; a synchronous one after that works
    live.compute_temporal(snap.order, snap.mask, live=True)
    live.compute_temporal(snap.order, snap.mask)
    live.destroy()
    sync.destroy()


def test_dashboard_loop_reaches_the_verdict():
    from hackathon_b200.fit_worker import FitWorker
    sc = O.SCENARIOS[0]
    T = sc["sim"]["T"]
    frames, valid, _ = O.simulate(dict(sc["sim"], T=T + 32))  # the scenario's statistics, 32 frames longer
    N = frames.shape[1]
    fps = sc["sim"]["fps"]
    opt = dict(dxUm=sc["sim"]["dxUm"], fps=fps, geometry=sc["geometry"])
    eng = H.DdmEngine.create(N=N, T=T, L=128, NB=32, kmin=4, kmax=100)
    clock = FrameClock(fps=fps, T=T)
    with FitWorker() as worker:
        la = LiveAnalyzer(eng, clock, opt=opt, worker=worker, guard=8)
        n = 0

        def feed(k):
            nonlocal n
            for _ in range(k):
                if valid[n]:  # the scenario's dropped frames never arrive
                    la.on_frame(frames[n], 1000.0 * n / fps)
                n += 1

        feed(T)
        assert la.start() == "started"
        feed(20)                          # 20 frames arrive during the analysis: >= guard
        r = la.finish()
        assert r["status"] == "stale" and r["elapsed"] >= 8
        assert la.guard == min(128, int(np.ceil(1.5 * r["elapsed"])) + 4)
        assert la.start() == "started"
        feed(4)
        r = la.finish()
        assert r["status"] == "ok" and r["used"] <= T - la.guard
        res = r["result"].result(600)
    assert res["verdict"] == "MOTILE"
    eng.destroy()
