"""The benchmark's own geometry against the FP64 oracle: 512^2 x 1024 u16
frames with a circular ROI (r = 230 px) and 2 % dropped frames, TPAD 2048,
L = 512 lags, 256 q-bins (kmin 4, kmax 200) -- the instances the headline
number runs -- and TPAD 4096.

Every temporal kernel that serves these TPADs runs on the same analysis:
the sparse-mask kernel (0/1 mask with at most 64 zeros), the one-group
radix-8 transform kernel and the two-group radix-16 transform kernel (the
autotuner's variants 0 and 1). The oracle (ddm_ref.js:196-206, 229-288,
360-437; the spatial mask is its labelled extension) runs on a sample of
the bins so that it finishes in seconds:
  - end to end: the oracle's history from the raw frames, its radial record
    on every 16th bin, against the engine's fused radial record:
    D within 1e-4 of each bin's scale, P within 1e-5 relative;
  - temporal stage alone: the oracle's per-mode D, C, P from the engine's own
    history on every 5th mode of those bins: |dD|/2P, |dC|/P, |dP|/P at
    p99 <= 1e-4 (the reference harness's metrics, harness.ts:115-151), for
    the two kernels that write full per-mode outputs;
  - D(q, 0) = 0 and the fused record equals the record of the full outputs.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

H = pytest.importorskip("hackathon_b200")
torch = pytest.importorskip("torch")

N, T, TPAD, L, NB, KMIN, KMAX = 512, 1024, 2048, 512, 256, 4.0, 200.0
VARIANTS = [("sparse", "temporal_sparse_kernel"), ("radix8", "temporal_kernel"), ("radix16", "temporal16_kernel")]


def _sub_bins(bins, sel):
    off = bins["binOffsets"]
    rows = [bins["binModes"][off[b]:off[b + 1]] for b in sel]
    sub = dict(bins)
    sub.update(NB=len(sel), binModes=np.ascontiguousarray(np.concatenate(rows)),
               binOffsets=np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint32),
               nModes=np.ascontiguousarray(bins["nModes"][sel]).astype(np.uint32))
    return sub


def _use(eng, variant):
    if variant == "sparse":
        eng.set_sparse(True)
        eng.set_tuning(0, 0, 0)
    else:
        eng.set_sparse(False)
        eng.set_tuning(0, 0, 0 if variant == "radix8" else 1)


@pytest.fixture(scope="module")
def headline():
    from hackathon_b200 import synth
    spec = synth.config2(seed=3)
    frames, valid, _ = synth.generate(spec)
    roi = synth.roi_mask(spec)
    fr = frames.view(torch.int16).cpu().numpy().view(np.uint16)
    del frames
    torch.cuda.empty_cache()
    eng = H.DdmEngine.create(N=N, T=T, TPAD=TPAD, L=L, NB=NB, kmin=KMIN, kmax=KMAX)
    eng.set_spatial_mask(roi)
    slots = np.arange(T, dtype=np.int32)
    idx = np.nonzero(valid)[0]
    eng.ingest_frames(fr[idx], slots[idx], 1.0 / 65535)
    ghist = eng.read_history()
    # the oracle's history from the raw frames (FP64, spatial-mask extension)
    hist = np.zeros((eng.modes, T), np.complex128)
    for c in range(0, idx.size, 64):
        k = idx[c:c + 64]
        O.history_ingest(fr[k].astype(np.float64) / 65535, k.astype(np.int32), T, hist=hist, smask=roi)
    order, mask = O.linear_order(valid)
    bins = O.make_bins(N, NB, KMIN, KMAX)
    sel = np.arange(0, NB, 16)
    sub = _sub_bins(bins, sel)
    ro = O.analyze_radial(hist, order, mask, sub, L, TPAD=TPAD)
    assert int((mask == 0).sum()) >= 10  # about 2 % of the frames dropped
    yield dict(eng=eng, ghist=ghist, order=order, mask=mask, bins=bins, sel=sel, sub=sub, ro=ro)
    eng.destroy()


@pytest.mark.parametrize("variant,kernel", VARIANTS, ids=[v for v, _ in VARIANTS])
def test_headline_radial_vs_oracle(headline, variant, kernel):
    eng, ro, sel = headline["eng"], headline["ro"], headline["sel"]
    _use(eng, variant)
    try:
        eng.compute_temporal(headline["order"], headline["mask"])
        assert eng.last_temporal_kernel == kernel
        rg = eng.read_radial()
    finally:
        _use(eng, "sparse")
    D = rg.D2()
    worst = 0.0
    for i, b in enumerate(sel):
        sc = ro["D"][i].max()
        assert sc > 0
        worst = max(worst, float(np.abs(D[b] - ro["D"][i]).max() / sc))
        assert abs(D[b, 0]) <= 1e-5 * sc  # D(q, 0) = 0
    assert worst <= 1e-4, worst
    assert np.allclose(rg.P[sel], ro["P"], rtol=1e-5, atol=0)


@pytest.mark.parametrize("variant,kernel", VARIANTS[:2], ids=[v for v, _ in VARIANTS[:2]])
def test_headline_modes_vs_oracle(headline, variant, kernel):
    """Per-mode outputs (readTemporalFull). The radix-16 kernel writes only
    the fused radial record, so full outputs come from the other two."""
    eng = headline["eng"]
    order, mask = headline["order"], headline["mask"]
    _use(eng, variant)
    try:
        eng.compute_temporal(order, mask, full=True)
        assert eng.last_temporal_kernel == kernel
        g = eng.read_temporal_full()
        rf = eng.read_radial()
        eng.compute_temporal(order, mask, full=False)
        rs = eng.read_radial()
    finally:
        _use(eng, "sparse")
    modes = headline["sub"]["binModes"][::5, 0].astype(np.int32)
    Do, Co, Po = O.analyze_modes(headline["ghist"].astype(np.complex128), order, mask, L, modes, TPAD=TPAD)
    ok = Po > 0
    assert ok.sum() > 0.9 * modes.size
    eP = np.abs(g["P"][modes][ok] - Po[ok]) / Po[ok]
    eD = np.abs(g["D"][modes][ok] - Do[ok]) / (2 * Po[ok, None])
    eC = np.abs(g["C"][modes][ok] - Co[ok]) / Po[ok, None]
    for e in (eP, eD.ravel(), eC.ravel()):
        assert float(np.quantile(e, 0.99)) <= 1e-4
    # fused radial record == radial record of the full outputs
    Ds, Df = rs.D2(), rf.D2()
    sc = np.abs(Ds).max(axis=1)
    use = sc > 0
    assert (np.abs(Ds - Df)[use].max(axis=1) / sc[use]).max() <= 1e-6
    assert np.allclose(rf.P, rs.P, rtol=1e-6, atol=0)


@pytest.mark.parametrize("variant,kernel", VARIANTS, ids=[v for v, _ in VARIANTS])
def test_tpad4096_radial_vs_oracle(variant, kernel):
    """TPAD 4096 (T = 2048, the batched-video configuration's longest videos):
    41 dropped frames, 256 lags, each kernel variant against the oracle."""
    n, t, lags = 64, 2048, 256
    sim = dict(O.BASE, N=n, T=t, seed=29, swimmers=dict(n=12, vbar=20.0, sigma=8.0, geometry="3d"),
               passive=dict(n=12), dropExact=41)
    frames, valid, _ = O.simulate(sim)
    idx = np.nonzero(valid)[0]
    eng = H.DdmEngine.create(N=n, T=t, L=lags, NB=12, kmin=2, kmax=28)
    try:
        assert eng.TPAD == 4096
        eng.ingest_frames(frames[idx], idx)
        order, mask = O.linear_order(valid)
        _use(eng, variant)
        eng.compute_temporal(order, mask)
        assert eng.last_temporal_kernel == kernel
        rg = eng.read_radial()
    finally:
        eng.destroy()
    hist = O.history_ingest(O.luma_of(frames[idx]), idx.astype(np.int32), t)
    ro = O.analyze_radial(hist, order, mask, O.make_bins(n, 12, 2, 28), lags, TPAD=4096)
    D = rg.D2()
    for b in range(12):
        sc = ro["D"][b].max()
        if sc > 0:
            assert np.abs(D[b] - ro["D"][b]).max() <= 1e-4 * sc, b
    assert np.allclose(rg.P, ro["P"], rtol=1e-5, atol=0)
