"""Pins the oracle's fit restatement to the reference's known-answer tests
(motility-ddm/test/t_kernels.mjs, test/t_drift_phase.mjs)."""
import math

import numpy as np
import pytest

import oracle as O


def test_bessel_j0(golden):
    k = golden["known"]["bessel_j0"]
    for x, ref in k["pairs"]:
        assert abs(O.bessel_j0(x) - ref) < k["tol"]


def test_ln_gamma(golden):
    k = golden["known"]["ln_gamma"]
    closed = {"ln(24)": math.log(24), "ln(sqrt(pi))": math.log(math.sqrt(math.pi))}
    for x, ref in k["pairs"]:
        ref = closed.get(ref, ref)
        assert abs(O.ln_gamma(x) - ref) < k["tol"]


@pytest.mark.parametrize("c", [1, 0.9, 0.5, 0.1])
def test_legendre(c):
    """t_kernels.mjs:46-51."""
    p2 = (3 * c * c - 1) / 2
    p5 = (63 * c ** 5 - 70 * c ** 3 + 15 * c) / 8
    assert abs(O.legendre_p(2, c) - p2) < 1e-12
    assert abs(O.legendre_p(5, c) - p5) < 1e-12


def _schulz_average(f, vbar, Z):
    """Simpson quadrature of the Schulz average (t_kernels.mjs:16-27)."""
    vmax = vbar * 30
    n = 60000
    h = vmax / n
    v = np.arange(n + 1) * h
    w = np.where((np.arange(n + 1) % 2) == 1, 4.0, 2.0)
    w[0] = w[-1] = 1
    pdf = np.array([O.schulz_pdf(x, vbar, Z) for x in v])
    return float(np.sum(w * pdf * f(v)) * h / 3)


@pytest.mark.parametrize("Z", [0.8, 3, 40])
def test_schulz_norm_mean(Z):
    """t_kernels.mjs:53-58."""
    assert abs(_schulz_average(lambda v: np.ones_like(v), 10, Z) - 1) < 1e-4
    assert abs(_schulz_average(lambda v: v, 10, Z) - 10) < 1e-3


@pytest.mark.parametrize("Z", [0.8, 2, 10, 60])
def test_isf_closed_forms_vs_quadrature(Z, golden):
    """t_kernels.mjs:61-72."""
    from scipy.special import j0
    tol = golden["known"]["isf_quadrature"]["tol"]
    e3 = e2 = 0
    for x in (0.01, 0.3, 1, 2.5, 5, 12, 30):
        q3 = _schulz_average(lambda v: np.where(v > 0, np.sin(x * v) / np.maximum(x * v, 1e-300), 1.0), 1, Z)
        q2 = _schulz_average(lambda v: j0(x * v), 1, Z)
        e3 = max(e3, abs(O.isf3d(x, Z) - q3))
        e2 = max(e2, abs(O.isf2d(x, Z) - q2))
    assert e3 < tol and e2 < tol


@pytest.mark.parametrize("Z", [1, 20])
def test_isf_series_branch(Z):
    """t_kernels.mjs:74-84."""
    L = 1.0001e-4
    x = L * (Z + 1)
    exact3 = math.sin(Z * math.atan(L)) / (Z * L * math.pow(1 + L * L, Z / 2))
    exact2 = O.legendre_p(Z, 1 / math.sqrt(1 + L * L)) * math.pow(1 + L * L, -(Z + 1) / 2)
    s3 = 1 - (x * x * (Z + 2)) / (6 * (Z + 1))
    s2 = 1 - (x * x * (Z + 2)) / (4 * (Z + 1))
    assert abs(s3 - exact3) < 1e-10 and abs(s2 - exact2) < 1e-10
    assert abs(O.isf3d(x * 0.9999, Z) - O.isf3d(x, Z)) < 1e-9
    assert abs(O.isf2d(x * 0.9999, Z) - O.isf2d(x, Z)) < 1e-9


def test_isf2d_table(golden):
    """t_kernels.mjs:86-102 (grid thinned 4x in each direction for time)."""
    worst = 0
    for lz in np.arange(math.log(0.5), math.log(100) + 1e-9, 0.0371 * 4):
        Z = math.exp(lz)
        for lx in np.arange(-3, 3.5, 0.0137 * 4):
            x = 10 ** lx
            worst = max(worst, abs(O.isf2d_fast(x, Z) - O.isf2d(x, Z)))
    assert worst < golden["known"]["isf2d_table"]["tol"]


def test_narrow_limit():
    """t_kernels.mjs:104-105."""
    assert abs(O.isf3d(1, 100) - math.sin(1)) < 0.005
    assert abs(O.isf2d(1, 100) - O.bessel_j0(1)) < 0.005


def test_nnls_kkt(golden):
    """t_kernels.mjs:108-134: KKT conditions over 300 random problems."""
    rand = O.mulberry32(99, 300 * 48)
    pos = 0
    for _ in range(golden["known"]["nnls_kkt"]["trials"]):
        n = 12
        Cm = (rand[pos:pos + 36].reshape(3, n) * 2 - 1)
        d = rand[pos + 36:pos + 48] * 2 - 1
        pos += 48
        G = Cm @ Cm.T
        h = Cm @ d
        a, rss = O.nnls3(G, h, float(d @ d))
        r = d - a @ Cm
        assert abs(r @ r - rss) <= 1e-9
        g = G @ a - h
        for i in range(3):
            assert a[i] >= 0
            if a[i] > 1e-12:
                assert abs(g[i]) <= 1e-9
            else:
                assert g[i] >= -1e-9


@pytest.mark.parametrize("geometry", ["3d", "2d"])
def test_varpro_recovery(geometry, golden):
    """t_kernels.mjs:137-163: noise-free model data, VarPro recovers truth."""
    truth = dict(vbar=30.0, Z=4.0, Dd=0.3, alpha=0.6)
    NB, L, N, dxUm, fps = 32, 128, 256, 1.0, 30.0
    kernel = O.isf2d_fast if geometry == "2d" else O.isf3d
    kCenter = np.array([4 + 3 * (b + 0.5) for b in range(NB)])
    D = np.zeros((NB, L))
    for b in range(NB):
        q = 2 * math.pi * kCenter[b] / (N * dxUm)
        A, B = 1000 * math.exp(-q * q), 2.0
        for t in range(L):
            tau = t / fps
            E = math.exp(-truth["Dd"] * q * q * tau)
            f = E * (1 - truth["alpha"] + truth["alpha"] * kernel(q * truth["vbar"] * tau, truth["Z"]))
            D[b, t] = A * (1 - f) + (B if t else 0)
    # no kNodes in the reference test: the model uses q = kCenter (knodes=1)
    radial = O.Radial(N, NB, L, kCenter, kCenter.copy(), np.full(NB, 50), D,
                      np.zeros(NB), np.zeros(NB * L * 8), knodes=1)
    brown, fit = O.fit_brownian_swimmer(radial, dxUm, fps, geometry)
    k = golden["known"]["varpro_recovery"]
    assert abs(fit["vbar"] / truth["vbar"] - 1) < k["vbar_rel"]
    assert abs(fit["Z"] / truth["Z"] - 1) < k["Z_rel"]
    assert abs(fit["Dd"] / truth["Dd"] - 1) < k["D_rel"]
    assert abs(fit["alpha"] - truth["alpha"]) < k["alpha_abs"]
    assert fit["rss"] < 1e-3 * brown["rss"]


def test_lag_grid():
    """lagGrid (motility_fit.js:358-369): 43 lags at L = 128."""
    g = O.lag_grid(128)
    assert len(g) == 43 and list(g[:10]) == list(range(1, 11)) and g[-1] <= 127
    assert np.all(np.diff(g) > 0)


# ------------------------------------------------------------ t_drift_phase.mjs

_DN, _DNB, _DL, _fps = 64, 16, 64, 30.0


def _synth_full(gen):
    """t_drift_phase.mjs:193-208: per-mode C from a generator, D = 2(1 - Re C)."""
    bins = O.make_bins(_DN, _DNB, 2, 30)
    M = _DN * (_DN // 2 + 1)
    D = np.zeros((M, _DL))
    Cm = np.zeros((M, _DL), np.complex128)
    P = np.ones(M)
    for m, kx, ky, _ in bins["binModes"]:
        for t in range(_DL):
            re, im = gen(kx, ky, t)
            Cm[m, t] = re + 1j * im
            D[m, t] = 2 * (1 - re)
    rad = O.radial_from_full(D, Cm, P, bins, _DL)
    return O.Radial.from_bins(bins, _DL, rad)


def _q(k):
    return 2 * math.pi * k / _DN


@pytest.mark.parametrize("speed,deg", [(6, -34), (2.5, 90), (12, 180), (4, 225)])
def test_drift_recovery(speed, deg):
    """t_drift_phase.mjs:224-239 (noise from the oracle's normal stream)."""
    z = iter(O.rng_normals(int(speed * 100 + deg) & 0xFFFFFFFF, 200000))
    Vx = speed * math.cos(deg * math.pi / 180)
    Vy = speed * math.sin(deg * math.pi / 180)
    dt = 1 / _fps

    def gen(kx, ky, t):
        ph = -(_q(kx) * Vx + _q(ky) * Vy) * t * dt
        amp = math.exp(-0.2 * (_q(kx) ** 2 + _q(ky) ** 2) * t * dt)
        return amp * math.cos(ph) + 0.02 * next(z), amp * math.sin(ph) + 0.02 * next(z)

    r = _synth_full(gen)
    d = O.estimate_drift(r, 1.0, _fps)
    dang = abs(d["angleDeg"] - deg) % 360
    dang = 360 - dang if dang > 180 else dang
    assert abs(d["mag"] - speed) / speed < 0.01
    assert dang < 0.5
    assert d["significant"] and d["sigma"] < 0.1 * speed


def test_drift_gating():
    """t_drift_phase.mjs:251-273: exactly the lag pairs with g < 0.2 are used."""
    vbar, Z = 40.0, 4.0
    V, U = (5.0, 0.0), (-25.0, 0.0)
    dt = 1 / _fps

    def gen(kx, ky, t):
        qx, qy = _q(kx), _q(ky)
        g = O.isf3d(math.hypot(qx, qy) * vbar * t * dt, Z)
        pv = -(qx * V[0] + qy * V[1]) * t * dt
        pu = -(qx * U[0] + qy * U[1]) * t * dt
        return math.cos(pv) + 2 * g * math.cos(pu), math.sin(pv) + 2 * g * math.sin(pu)

    r = _synth_full(gen)
    gated = O.estimate_drift(r, 1.0, _fps, swimmer=(vbar, Z))
    opened = O.estimate_drift(r, 1.0, _fps)
    qs = 2 * math.pi / _DN
    expect = 0
    for b in range(_DNB):
        if r.nModes[b] < 3:
            continue
        q = qs * r.kCenter[b]
        for t in range(1, _DL - 1):
            if abs(O.isf3d(q * vbar * t * dt, Z)) < 0.2:
                expect += 1
    assert gated["pairs"] == expect
    eg = math.hypot(gated["Vx"] - V[0], gated["Vy"] - V[1])
    eo = math.hypot(opened["Vx"] - V[0], opened["Vy"] - V[1])
    assert eg < 0.15 * math.hypot(*V) and eg < 0.5 * eo


@pytest.mark.parametrize("sx,sy", [(1, 0), (0, 1), (-1, 1)])
def test_translation_sign_convention(sx, sy):
    """t_drift_phase.mjs:276-303: a translating image through the full FP64
    pipeline (History -> analyzeRadial -> drift) returns +V."""
    N, T = _DN, 64
    base = O.mulberry32(5, N * N).reshape(N, N)
    sm = sum(np.roll(np.roll(base, -j, 0), -i, 1) for j in (-1, 0, 1) for i in (-1, 0, 1)) / 9
    frames = np.stack([np.roll(np.roll(sm, sy * t, 0), sx * t, 1) for t in range(T)])
    hist = O.history_ingest(frames, np.arange(T, dtype=np.int32), T)
    order, mask = O.linear_order(np.ones(T, bool))
    bins = O.make_bins(N, _DNB, 2, 30)
    rad = O.analyze_radial(hist, order, mask, bins, 32)
    r = O.Radial.from_bins(bins, 32, rad)
    d = O.estimate_drift(r, 1.0, _fps)
    Vx, Vy = sx * _fps, sy * _fps
    assert math.hypot(d["Vx"] - Vx, d["Vy"] - Vy) / math.hypot(Vx, Vy) < 0.1


def test_brownian_per_bin_recovers_d():
    """The oracle's per-bin Brownian fit (fitBrownian's scan + golden
    section) on noise-free Brownian curves returns the generating D and
    amplitudes."""
    tau = np.arange(1, 64, dtype=np.float64)
    for k, D in ((6.0, 0.3), (15.0, 0.05), (30.0, 0.8)):
        q = 2 * np.pi * k / 128
        qn = q * np.array([0.99, 0.997, 1.003, 1.01])
        th = np.array([1.7, 0.05, 0.0, 0.0, 0.0, np.log(D)])
        d = O.lm_model(tau, qn, th)
        b6 = np.array([0.01, 10.0, 0.5, 100.0, 1e-4, 100.0])
        got, cost = O.lm_fit_brownian(d, tau, qn, 1.0 / d.max(), b6)
        # golden section stops at a 1e-6 bracket of a flat valley: D to 1e-4
        assert abs(got[5] - np.log(D)) < 1e-4 and cost < 1e-12
        assert abs(got[0] / 1.7 - 1) < 1e-3 and abs(got[1] - 0.05) < 2e-4
