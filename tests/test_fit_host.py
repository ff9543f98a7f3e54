"""Host side of the fit (no GPU): the lag grid and preparation restate the
reference (motility_fit.js:358-401), the FP64 LM oracle recovers the model's
parameters to the tolerances of the reference's own noise-free recovery test
(t_kernels.mjs:137-163: vbar 1e-3, Z and D 1e-2 relative, alpha 1e-3
absolute), and the C ABI rejects bad fit arguments before touching a device."""
import numpy as np
import pytest

import oracle as O
from tests.lm_cases import bounds6, make_cases


def test_lag_grid_matches_reference_restatement():
    from hackathon_b200 import fit
    for L in (2, 3, 11, 12, 64, 128, 512, 1024):
        assert np.array_equal(fit.lag_grid(L), np.array(O.lag_grid(L)))
    assert len(fit.lag_grid(128)) == 43  # the reference's count for L = 128


def test_prepare_and_bounds_follow_reference():
    from hackathon_b200 import fit
    from hackathon_b200.radial import Radial
    NB, L, N = 8, 64, 256
    rng = np.random.default_rng(1)
    D = rng.uniform(0.1, 1.0, (NB, L))
    D[3] = 0  # no positive maximum: dropped
    nm = np.array([5, 2, 9, 9, 9, 9, 9, 9], np.uint32)  # bin 1 has < 3 modes: dropped
    kc = np.linspace(5, 40, NB)
    kn = np.repeat(kc, 4) * (1 + 0.01 * np.tile([-1, -0.3, 0.3, 1], NB))
    r = Radial(N=N, NB=NB, L=L, kCenter=kc, kNodes=kn, nModes=nm, D=D.ravel(), P=np.ones(NB),
               drift=np.zeros(NB * L * 8))
    pr = fit.prepare(r, dxUm=0.5, fps=20.0)
    assert list(pr.bins) == [0, 2, 4, 5, 6, 7]
    lags = fit.lag_grid(L)
    qs = 2 * np.pi / (N * 0.5)
    assert np.allclose(pr.d[0], D[0, lags])
    assert np.allclose(pr.w, 1 / D[pr.bins][:, lags].max(1))
    assert np.allclose(pr.qn[1], kn[8:12] * qs)
    assert np.allclose(pr.tau, lags / 20.0)
    b = fit.bounds(pr)
    qmin, qmax, dt, tmax = pr.q.min(), pr.q.max(), 1 / 20.0, (L - 1) / 20.0
    assert np.allclose(b, [max(2.0, 0.3 / (qmax * tmax)), 3 / (qmin * dt), 0.5, 100,
                           0.01 / (qmax ** 2 * tmax), 10 / (qmin ** 2 * dt)])


def test_oracle_lm_recovers_noise_free_parameters():
    cases = make_cases(16, seed=3)
    b6 = bounds6(cases)
    good = 0
    for c in cases:
        th, cost, it, ev = O.lm_fit_plain(c["d"], c["tau"], c["qn"], c["w"], b6)
        t = c["theta"]
        ok = (abs(th[2] - t[2]) < 1e-3 and abs(np.exp(th[3] - t[3]) - 1) < 1e-3
              and abs(np.exp(th[4] - t[4]) - 1) < 1e-2 and abs(np.exp(th[5] - t[5]) - 1) < 1e-2)
        good += ok
        assert cost < 1e-12 or not ok
    # the multi-start must find the global optimum of nearly every noise-free bin
    assert good == len(cases), good


def test_oracle_lm_seeded_from_truth_is_stationary():
    for c in make_cases(4, seed=4):
        t = c["theta"]
        th, cost, it = O.lm_fit_start(c["d"], c["tau"], c["qn"], c["w"], bounds6([c]) * [0.1, 10, 1, 1, 0.1, 10],
                                      [t[2], np.exp(t[3]), np.exp(t[4]), np.exp(t[5])])
        assert np.allclose(th, t, rtol=1e-6, atol=1e-8)
        assert cost < 1e-20


def test_fit_abi_rejects_bad_arguments():
    from hackathon_b200 import fit
    from hackathon_b200.engine import DdmArgError
    d = np.ones((2, 200))
    with pytest.raises(DdmArgError):  # nt_max > 128
        fit.fit_lm(d, np.arange(200.0), np.ones((2, 4)), 1.0, np.ones(6))
    with pytest.raises(DdmArgError):  # K > 8
        fit.fit_lm(np.ones((2, 10)), np.arange(10.0), np.ones((2, 9)), 1.0, np.ones(6))
    with pytest.raises(DdmArgError):  # nrefine out of range
        fit.fit_lm(np.ones((2, 10)), np.arange(10.0), np.ones((2, 4)), 1.0, np.ones(6), nrefine=0)
