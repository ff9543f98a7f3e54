"""Pins the FP64 oracle's FFT / Wiener-Khinchin restatement to the reference's
own known-answer tests (motility-ddm/test/t_fft.mjs) and to numpy.fft."""
import numpy as np
import pytest

import oracle as O


def _rand(seed, n):
    return O.mulberry32(seed, n)


@pytest.mark.parametrize("n", [2 ** k for k in range(1, 10)])
def test_fft_vs_dft(n, golden):
    """t_fft.mjs:24-40: Stockham vs direct DFT, forward and inverse, + round trip."""
    tol = golden["known"]["fft_vs_dft_rel"]
    r = _rand(1234 + n, 2 * n) * 2 - 1
    x = r[0::2] + 1j * r[1::2]
    for inv in (False, True):
        ref = O.dft(x, inv)
        got = O.fft(x, inv)
        err = np.max(np.abs(np.c_[got.real - ref.real, got.imag - ref.imag]))
        mag = np.max(np.abs(np.c_[ref.real, ref.imag]))
        assert err / mag < tol["tol"]
        # independent check: numpy's FP64 FFT
        npref = np.fft.ifft(x) * n if inv else np.fft.fft(x)
        assert np.max(np.abs(got - npref)) / np.max(np.abs(npref)) < 1e-13
    y = O.fft(O.fft(x), True)
    assert np.max(np.abs(np.c_[(y / n - x).real, (y / n - x).imag])) < tol["round_trip"]


def test_spectrum2d_vs_direct_dft(golden):
    """t_fft.mjs:43-69: windowed half-plane 2D spectrum vs a direct 2D DFT, N=16."""
    N = 16
    NH = N // 2 + 1
    img = _rand(7, N * N).reshape(N, N)
    win = O.blackman_harris(N)
    got = O.spectrum2d_half(img)
    v = (img - img.mean()) * win[None, :] * win[:, None]
    y = np.arange(N)[:, None, None, None]
    x = np.arange(N)[None, :, None, None]
    ky = np.arange(N)[None, None, :, None]
    kx = np.arange(NH)[None, None, None, :]
    e = np.exp(-2j * np.pi * (kx * x + ky * y) / N)
    ref = (v[:, :, None, None] * e).sum(axis=(0, 1)) / N
    err = np.max(np.abs(got - ref))
    mag = np.max(np.abs(ref))
    assert err / mag < golden["known"]["spectrum2d_vs_dft"]["tol"]


def test_window_values(golden):
    """t_fft.mjs:72-77."""
    w = O.blackman_harris(256)
    k = golden["known"]["window"]
    assert abs(w[0] - k["w0"]) < k["tol"]
    assert abs(w[128] - k["w_half"]) < k["tol"]
    assert abs(w[10] - w[246]) < 1e-14


@pytest.mark.parametrize("label,drop,shuffle", [("full", 0.0, False),
                                                ("20% dropped", 0.2, False),
                                                ("shuffled + 15% dropped", 0.15, True)])
def test_wiener_khinchin_vs_direct(label, drop, shuffle, golden):
    """t_fft.mjs:80-117: masked, reordered WK (FFT) vs direct O(T*L) sums."""
    T, L = 256, 128
    r = _rand(99 + int(drop * 100) + shuffle, 3 * T * 2 + 2 * T) * 2 - 1
    hist = (r[:3 * T * 2:2] + 1j * r[1:3 * T * 2:2]).reshape(3, T)
    t = np.arange(T)
    hist[1] += 3 * np.exp(1j * 0.07 * t)
    order = np.arange(T, dtype=np.uint32)
    rs = _rand(5 + int(shuffle), 2 * T)
    if shuffle:
        for i in range(T - 1, 0, -1):
            j = int(np.floor(rs[i] * (i + 1)))
            order[i], order[j] = order[j], order[i]
    mask = (rs[T:] >= drop).astype(np.float64)
    mask[0] = 1
    k = golden["known"]["wk_vs_direct"]
    for m in range(3):
        D1, C1, P1 = O.temporal_mode(hist, m, order, mask, L)
        D2, C2, P2 = O.temporal_mode_direct(hist, m, order, mask, L)
        assert abs(P1 - P2) / P2 < k["P"]
        assert abs(D1[0]) / P2 < k["D0"]
        assert np.max(np.abs(D1 - D2)) / P2 < k["D"]
        dc = np.r_[C1.real - C2.real, C1.imag - C2.imag]
        assert np.max(np.abs(dc)) / P2 < k["C"]


def test_phase_rotation(golden):
    """t_fft.mjs:120-137: x = exp(-i w t) gives C = exp(-i w tau), D = 2-2cos."""
    T, L, w = 256, 128, 0.05
    t = np.arange(T)
    hist = np.exp(-1j * w * t)[None, :]
    order = np.arange(T, dtype=np.uint32)
    mask = np.ones(T)
    D, Cc, _ = O.temporal_mode(hist, 0, order, mask, L)
    tau = np.arange(L)
    e = max(np.max(np.abs(D - (2 - 2 * np.cos(w * tau)))),
            np.max(np.abs(Cc.real - np.cos(w * tau))),
            np.max(np.abs(Cc.imag + np.sin(w * tau))))
    assert e < golden["known"]["phase_rotation"]["tol"]


def test_padded_length_extension():
    """Extension: TPAD > 2T gives the same linear correlation as 2T."""
    T, L = 64, 40
    r = _rand(3, 4 * T) * 2 - 1
    hist = (r[:2 * T:2] + 1j * r[1:2 * T:2])[None, :]
    order = np.arange(T, dtype=np.uint32)
    mask = (r[2 * T:3 * T] > -0.6).astype(float)
    mask[0] = 1
    D1, C1, P1 = O.temporal_mode(hist, 0, order, mask, L, TPAD=2 * T)
    D2, C2, P2 = O.temporal_mode(hist, 0, order, mask, L, TPAD=8 * T)
    assert np.allclose(D1, D2, atol=1e-12) and np.allclose(C1, C2, atol=1e-12)
    assert abs(P1 - P2) < 1e-12


def test_temporal_meta_counts():
    """temporalMeta (ddm_ref.js:538-560): N(tau) are exact pair counts and
    mspec is the FFT of the zero-padded mask."""
    T, TPAD, L = 256, 512, 128
    r = _rand(11, T)
    mask = (r > 0.2).astype(float)
    order = np.arange(T, dtype=np.uint32)
    npairs, ms = O.temporal_meta(order, mask, T, TPAD, L)
    for tau in (0, 1, 7, 127):
        assert npairs[tau] == np.sum(mask[:T - tau] * mask[tau:])
    z = np.zeros(TPAD)
    z[:T] = mask
    assert np.max(np.abs(ms - np.fft.fft(z))) < 1e-10


def test_spatial_mask_extension_vs_numpy():
    """The oracle's spatial-mask extension (the reference has none): mean over
    the used pixels, masked pixels left out, against numpy's FP64 FFT; with no
    mask it is the reference's spectrum2dHalf unchanged."""
    N, T = 64, 3
    rng = np.random.default_rng(5)
    luma = rng.random((T, N, N))
    yy, xx = np.mgrid[:N, :N]
    S = ((xx - N / 2) ** 2 + (yy - N / 2) ** 2 <= (0.4 * N) ** 2).astype(np.uint8)
    h = O.history_ingest(luma, np.arange(T, dtype=np.int32), T, smask=S)
    h0 = O.history_ingest(luma, np.arange(T, dtype=np.int32), T)
    w = O.blackman_harris(N)
    NH = N // 2 + 1
    for t in range(T):
        mu = (luma[t] * S).sum() / S.sum()
        F = np.fft.fft2((luma[t] - mu) * w[None, :] * w[:, None] * S)[:, :NH] / N
        assert np.abs(h[:, t] - F.reshape(-1)).max() < 1e-12 * np.abs(F).max()
        assert np.array_equal(h0[:, t], O.spectrum2d_half(luma[t]).reshape(-1))
