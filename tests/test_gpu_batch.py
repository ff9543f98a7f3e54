"""Batched videos of uneven size and frame count (ddm_batch_*): one temporal
launch over every video's units at the batch's largest TPAD gives each video
the radial record its own engine computes (zero padding beyond T + L - 1 is
exact for lags < L; the FFT lengths differ, so agreement is to FP32 rounding:
D within 1e-5 of each bin's scale, drift sums within 1e-4 of their scale);
a CUDA-graph replay reproduces the batch bit for bit; all bins of all videos
fit in one LM launch; and one small video is checked against the FP64
oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
H = pytest.importorskip("hackathon_b200")
from hackathon_b200 import synth  # noqa: E402
from hackathon_b200.batch import DdmBatch  # noqa: E402

VIDEOS = [  # (N, T, L, NB, kmin, kmax) -- uneven sizes and frame counts
    (256, 300, 128, 24, 3.0, 60.0),
    (128, 1000, 400, 16, 2.0, 40.0),
    (512, 512, 200, 32, 4.0, 120.0),
    (256, 2000, 512, 24, 3.0, 60.0),
    (384, 400, 160, 24, 4.0, 90.0),  # mixed-radix size
]


def _make(seed):
    vids = []
    for i, (N, T, L, NB, kmin, kmax) in enumerate(VIDEOS):
        spec = synth.VideoSpec(N=N, T=T, n_blobs=int(2000 * (N / 512) ** 2), roi_radius=-1, drop_frac=0.03,
                               seed=seed + i)
        frames, valid, _ = synth.generate(spec)
        vids.append(dict(frames=frames.contiguous(), valid=valid, geo=(N, T, L, NB, kmin, kmax)))
    return vids


def _engine(geo):
    N, T, L, NB, kmin, kmax = geo
    return H.DdmEngine.create(N=N, T=T, L=L, NB=NB, kmin=kmin, kmax=kmax)


def _close(ra, rb):
    D1, D2 = ra.D2(), rb.D2()
    for b in range(ra.NB):
        sc = np.abs(D2[b]).max()
        if sc > 0:
            assert np.abs(D1[b] - D2[b]).max() <= 1e-5 * sc, b
    d1, d2 = ra.drift3(), rb.drift3()
    for c in range(8):
        sc = np.abs(d2[..., c]).max()
        if sc > 0:
            assert np.abs(d1[..., c] - d2[..., c]).max() <= 1e-4 * sc, c
    assert np.allclose(ra.P, rb.P, rtol=1e-5, atol=0)


def test_batch_matches_individual_engines_and_graph_replay():
    vids = _make(seed=21)
    orders = [np.arange(v["geo"][1], dtype=np.uint32) for v in vids]
    masks = [v["valid"].astype(np.float32) for v in vids]
    slots = [np.arange(v["geo"][1], dtype=np.int32) for v in vids]
    scales = [1.0 / 65535] * len(vids)
    # reference: each video on its own engine
    solo = []
    for v, o, m, s in zip(vids, orders, masks, slots):
        e = _engine(v["geo"])
        e.ingest_frames(v["frames"], s, scales[0])
        e.compute_temporal(o, m)
        solo.append(e.read_radial())
        e.destroy()
    engines = [_engine(v["geo"]) for v in vids]
    batch = DdmBatch(engines)
    batch.ingest([v["frames"] for v in vids], slots, scales)
    batch.compute_temporal(orders, masks)
    got = batch.read_radials()
    for a, b in zip(got, solo):
        _close(a, b)
    # graph: capture the whole step, replay twice, bit-identical to the batch
    batch.capture([v["frames"] for v in vids], slots, scales)
    for _ in range(2):
        batch.launch_graph()
        rep = batch.read_radials()
        for a, b in zip(rep, got):
            assert np.array_equal(a.D, b.D) and np.array_equal(a.drift, b.drift) and np.array_equal(a.P, b.P)
    # all q-bins of all videos in one LM launch
    fits = batch.fit_all(rep, swim_min=0.0)
    assert sum(len(p.bins) for p, _ in fits) > 50
    for p, r in fits:
        assert np.isfinite(r.cost).all() and (r.iters > 0).all()
    batch.destroy()
    for e in engines:
        e.destroy()


def test_batch_small_video_against_oracle():
    N, T, L = 64, 128, 40  # the FP64 oracle transforms powers of two (TPAD = 2T)
    sim = dict(O.BASE, N=N, T=T, seed=9, swimmers=dict(n=20, vbar=20.0, sigma=8.0, geometry="3d"),
               passive=dict(n=20), dropExact=6)
    frames, valid, _ = O.simulate(sim)
    idx = np.nonzero(valid)[0]
    big = synth.generate(synth.VideoSpec(N=128, T=300, n_blobs=120, roi_radius=-1, seed=3))[0].contiguous()
    e1 = H.DdmEngine.create(N=N, T=T, L=L, NB=12, kmin=2, kmax=28)
    e2 = H.DdmEngine.create(N=128, T=300, L=100, NB=16, kmin=2, kmax=40)  # forces TPAD 1024 > e1's 256
    batch = DdmBatch([e1, e2])
    f1 = torch.from_numpy(frames[idx]).cuda().contiguous()
    batch.ingest([f1, big], [idx.astype(np.int32), np.arange(300, dtype=np.int32)], [1 / 255, 1 / 65535])
    order, mask = O.linear_order(valid)
    batch.compute_temporal([order, np.arange(300, dtype=np.uint32)], [mask, np.ones(300, np.float32)])
    rg = batch.read_radials()[0]
    hist = O.history_ingest(O.luma_of(frames[idx]), idx.astype(np.int32), T)
    ro = O.analyze_radial(hist, order, mask, O.make_bins(N, 12, 2, 28), L)
    D = rg.D2()
    for b in range(12):
        sc = ro["D"][b].max()
        if sc > 0:
            assert np.abs(D[b] - ro["D"][b]).max() <= 1e-4 * sc, b
    batch.destroy()
    e1.destroy()
    e2.destroy()


def test_batch_sparse_kernel_and_replay_guard():
    """Every video's mask within 64 zeros: the batched launch takes the
    sparse-mask kernel (per-video zero lists), equal to the transform path;
    a recorded launch replayed after a mask grew past 64 zeros reports the
    error instead of a wrong record."""
    vids = _make(seed=31)
    rng = np.random.default_rng(5)
    orders = [np.arange(v["geo"][1], dtype=np.uint32) for v in vids]
    masks = []
    for v in vids:
        m = np.ones(v["geo"][1], np.float32)
        m[rng.choice(v["geo"][1], 25, replace=False)] = 0
        masks.append(m)
    slots = [np.arange(v["geo"][1], dtype=np.int32) for v in vids]
    scales = [1.0 / 65535] * len(vids)
    engines = [_engine(v["geo"]) for v in vids]
    batch = DdmBatch(engines)
    batch.ingest([v["frames"] for v in vids], slots, scales)
    batch.compute_temporal(orders, masks)
    sparse = batch.read_radials()
    assert all(e.last_temporal_kernel == "temporal_sparse_kernel" for e in engines)
    engines[0].set_sparse(False)  # the batch follows its first engine's setting
    batch.compute_temporal(orders, masks)
    dense = batch.read_radials()
    assert all(e.last_temporal_kernel in ("temporal_kernel", "temporal16_kernel") for e in engines)
    engines[0].set_sparse(True)
    for a, b in zip(sparse, dense):
        _close(a, b)
    # record the step with the sparse kernel, then refresh the tables with a
    # mask of 100 zeros (the direct launch takes the transform path) and replay
    batch.compute_temporal(orders, masks)
    batch.capture([v["frames"] for v in vids], slots, scales)
    batch.launch_graph()
    rep = batch.read_radials()
    for a, b in zip(rep, sparse):
        _close(a, b)
    many = [m.copy() for m in masks]
    many[0][:100] = 0
    batch.compute_temporal(orders, many)
    batch.sync()
    assert engines[0].last_temporal_kernel != "temporal_sparse_kernel"
    batch.launch_graph()
    with pytest.raises(H.DdmError, match="sparse-mask kernel"):
        batch.sync()
    batch.compute_temporal(orders, masks)  # usable again
    for a, b in zip(batch.read_radials(), sparse):
        _close(a, b)
    batch.destroy()
    for e in engines:
        e.destroy()
