"""The small plain-DDM configuration end to end on the GPU: 64 frames of
128^2 u8 (200 Brownian blobs, D = 0.3 px^2/frame, Poisson noise, seeded),
unmasked Wiener-Khinchin over all lags 1..63 (TPAD 128), 64 radial q-bins,
and the Brownian model A(q)(1 - exp(-D q^2 tau)) + B(q) fitted per bin by
the batched GPU fit (ddm_fit_lm mode 3). Against the FP64 oracle on the same
frames: radial D within 1e-4 of each bin's scale, P to 1e-5; per bin, the
fit error (cost) within 1e-3 of the oracle's fit of the same curve, and D
within 1e-3 relative (the north star's fit tolerance) wherever the decay is
resolved within the 63 lags (D q^2 tau_max >= 2; below that only A*D is
determined); and the joint Brownian fit estimates the generator's 0.3
px^2/frame within its sampling spread, with the verdict NOT_MOTILE."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

H = pytest.importorskip("hackathon_b200")
from hackathon_b200 import fit as F  # noqa: E402
from hackathon_b200 import synth  # noqa: E402

N, T, L, NB, KMIN, KMAX = 128, 64, 64, 64, 2.0, 58.0


def test_small_configuration_end_to_end():
    import torch
    spec = synth.config1(seed=1)
    f16, valid, _ = synth.generate(spec)
    frames = f16.view(torch.int16).clamp(0, 255).to(torch.uint8)
    assert valid.all()
    eng = H.DdmEngine.create(N=N, T=T, TPAD=128, L=L, NB=NB, kmin=KMIN, kmax=KMAX)
    order = np.arange(T, dtype=np.uint32)
    mask = np.ones(T, np.float32)
    eng.ingest_frames(frames, np.arange(T, dtype=np.int32))
    eng.compute_temporal(order, mask)
    rg = eng.read_radial()
    eng.destroy()

    fr = frames.cpu().numpy()
    hist = O.history_ingest(O.luma_of(fr), np.arange(T, dtype=np.int32), T)
    ro = O.analyze_radial(hist, order, mask, O.make_bins(N, NB, KMIN, KMAX), L)
    D = rg.D2()
    for b in range(NB):
        sc = ro["D"][b].max()
        if sc > 0:
            assert np.abs(D[b] - ro["D"][b]).max() <= 1e-4 * sc, b
    assert np.allclose(rg.P, ro["P"], rtol=1e-5, atol=0)

    # per-bin Brownian fits over all lags 1..63
    pr = F.prepare(rg)
    lags = np.arange(1, L)
    d = D[pr.bins][:, lags]
    w = 1.0 / d.max(1)
    b6 = F.bounds(pr, swim_min=0.0)
    res = F.fit_lm(d, lags.astype(np.float64), pr.qn, w, b6, mode="brownian")
    assert (res.status & 1).all()
    Dg = res.D
    interior = []
    for i in range(len(pr.bins)):
        th, cost = O.lm_fit_brownian(d[i], lags.astype(np.float64), pr.qn[i], w[i], b6)
        Do = np.exp(th[5])
        if not (b6[4] * 1.01 < Do < b6[5] / 1.01):
            continue  # at a bound: D not determined by this bin
        interior.append(i)
        # equal fit error everywhere; D itself where the curve's decay is
        # resolved within the lags (else only A*D is determined: a flat valley)
        assert res.cost[i] <= cost * (1 + 1e-3) + 1e-12, (i, res.cost[i], cost)
        if Do * pr.q[i] ** 2 * lags[-1] >= 2:
            assert abs(Dg[i] / Do - 1) <= 1e-3, (i, Dg[i], Do)
    assert len(interior) >= len(pr.bins) // 2
    # the generator's diffusion coefficient: 64 frames leave each bin's D
    # noisy, so the reference's joint Brownian fit (one D over all bins,
    # fitBrownian) on the GPU radial record, through the library's decision
    # layer, is the estimate; over 15 seeds of this configuration it spreads
    # over 0.19-0.36 px^2/frame (FP64 oracle pipeline), hence the 40 % band.
    # The verdict is NOT_MOTILE.
    from hackathon_b200.motility import analyze_motility
    res = analyze_motility(rg)
    assert res["verdict"] == "NOT_MOTILE"
    assert abs(res["brown"]["Dd"] / 0.3 - 1) < 0.4, res["brown"]["Dd"]
