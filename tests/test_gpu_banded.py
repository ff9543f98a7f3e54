"""Banded analysis (ddm_create_banded / ddm_analyze_banded): the history held
one band of spectrum columns at a time, the frames streamed through the
spatial pass once per band. Its radial record equals the ordinary engine's on
the same frames up to FP32 rounding: the temporal kernels transform two modes
together, and which modes share a transform depends on the band's work units
(measured: ~1e-9 of a bin's scale). D within 1e-6 of each bin's scale, P and
the drift sums within 1e-6 relative -- for host and device
frames, with and without a spatial mask, through the column kernel of
N < 1024 and the wide column kernel of N >= 1024, and with the sparse-mask
and the transform temporal kernels. A banded engine refuses the calls that
need the whole history."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

H = pytest.importorskip("hackathon_b200")
torch = pytest.importorskip("torch")


def _compare(a, b):
    Da, Db = a.D2(), b.D2()
    sc = np.abs(Da).max(axis=1)
    use = sc > 0
    assert (np.abs(Da - Db)[use].max(axis=1) / sc[use]).max() <= 1e-6
    assert np.allclose(a.P, b.P, rtol=1e-6, atol=0)
    da, db = a.drift3(), b.drift3()
    assert np.allclose(da, db, rtol=1e-6, atol=1e-6 * np.abs(db).max())


@pytest.mark.parametrize("where,smask,sparse", [("host", False, True), ("device", True, True),
                                                ("host", True, False)])
def test_banded_equals_ordinary_engine(where, smask, sparse):
    N, T, L, NB = 256, 128, 48, 16
    sim = dict(O.BASE, N=N, T=T, seed=37, swimmers=dict(n=40, vbar=20.0, sigma=8.0, geometry="3d"),
               passive=dict(n=40), dropExact=5)
    frames, valid, _ = O.simulate(sim)
    idx = np.nonzero(valid)[0]
    order, mask = O.linear_order(valid)
    geo = dict(N=N, T=T, L=L, NB=NB, kmin=4, kmax=100)
    yy, xx = np.mgrid[:N, :N]
    roi = ((xx - N / 2) ** 2 + (yy - N / 2) ** 2 <= (0.45 * N) ** 2).astype(np.uint8)
    ref = H.DdmEngine.create(**geo)
    per_col = N * T * 8
    ban = H.DdmEngine.create_banded(40 * per_col, **geo)
    try:
        assert ban.bands == (4, 40)  # 129 columns in bands of 40
        for e in (ref, ban):
            if smask:
                e.set_spatial_mask(roi)
            e.set_sparse(sparse)
        ref.ingest_frames(frames[idx], idx)
        ref.compute_temporal(order, mask)
        r = ref.read_radial()
        fr = torch.from_numpy(frames[idx]).cuda() if where == "device" else frames[idx]
        ban.analyze_banded(fr, idx, order, mask)
        b = ban.read_radial()
        assert ban.last_temporal_kernel == ref.last_temporal_kernel
        _compare(b, r)
        # analysing again gives the same record (the first band overwrites it)
        ban.analyze_banded(fr, idx, order, mask)
        b2 = ban.read_radial()
        assert np.array_equal(b2.D, b.D) and np.array_equal(b2.P, b.P)
    finally:
        ref.destroy()
        ban.destroy()


def test_banded_wide_column_kernel():
    """N = 1024 (the wide column kernel, four frames per tile): three bands."""
    N, T, L, NB = 1024, 64, 16, 12
    rng = np.random.default_rng(5)
    frames = rng.integers(0, 4096, (T, N, N)).astype(np.uint16)
    slots = np.arange(T, dtype=np.int32)
    order = np.arange(T, dtype=np.uint32)
    mask = np.ones(T, np.float32)
    mask[[3, 40]] = 0
    geo = dict(N=N, T=T, L=L, NB=NB, kmin=4, kmax=300)
    ref = H.DdmEngine.create(**geo)
    ban = H.DdmEngine.create_banded(200 * N * T * 8, **geo)
    try:
        assert ban.bands == (3, 200)
        ref.ingest_frames(frames, slots, 1 / 4095)
        ref.compute_temporal(order, mask)
        ban.analyze_banded(frames, slots, order, mask, 1 / 4095)
        _compare(ban.read_radial(), ref.read_radial())
    finally:
        ref.destroy()
        ban.destroy()


def test_banded_engine_refuses_whole_history_calls():
    N, T = 64, 32
    e = H.DdmEngine.create_banded(8 * N * T * 8, N=N, T=T, L=16, NB=8, kmin=2, kmax=30)
    try:
        assert e.bands == (5, 8)
        frames = np.zeros((2, N, N), np.uint8)
        with pytest.raises(H.DdmError):
            e.ingest_frames(frames, [0, 1])
        with pytest.raises(H.DdmError):
            e.compute_temporal(np.arange(T), np.ones(T))
        with pytest.raises(H.DdmError):
            e.read_history()
    finally:
        e.destroy()
    with pytest.raises(H.DdmArgError):
        H.DdmEngine.create_banded(N * T * 8, N=N, T=T, L=16, NB=8, kmin=2, kmax=30)  # under two columns
