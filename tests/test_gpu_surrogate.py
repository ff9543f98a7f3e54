"""The learned seed end to end on the GPU: the model-curve generator against
the FP64 model (oracle/lm.c), the seeded-with-fallback LM mode, and what a
trained surrogate gains over the method without it (the reference's start
strategy) on held-out curves at equal fit error."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
F = pytest.importorskip("hackathon_b200.fit")
ST = pytest.importorskip("hackathon_b200.surrogate_train")


def test_model_curves_match_fp64_model():
    th, qn = ST.sample_params(64, seed=1)
    tau = ST.lm_tau()
    y = F.model_curves(th, qn, tau).cpu().numpy()
    for i in range(64):
        t = th[i].astype(np.float64)
        ref = O.lm_model(tau.astype(np.float64), qn[i].astype(np.float64),
                         [t[0], t[1], t[2], np.log(t[3]), np.log(t[4]), np.log(t[5])])
        assert np.abs(y[i] - ref).max() <= 2e-5 * np.abs(ref).max()


def test_model_curve_noise_and_tau_e():
    th, qn = ST.sample_params(2048, seed=2)
    tau = ST.lm_tau()
    clean = F.model_curves(th, qn, tau).cpu().numpy()
    noisy, te = F.model_curves(th, qn, tau, noise=0.01, seed=7, want_tau_e=True)
    r = noisy.cpu().numpy() / clean - 1
    assert abs(r.mean()) < 2e-4 and abs(r.std() - 0.01) < 3e-4
    te = te.cpu().numpy()
    for i in range(0, 2048, 97):  # c(tau_e) = 1 - 1/e on the FP64 model (A = 1, B = 0)
        t = th[i].astype(np.float64)
        c = O.lm_model(np.array([te[i]], np.float64), qn[i].astype(np.float64),
                       [1.0, 0.0, t[2], np.log(t[3]), np.log(t[4]), np.log(t[5])])[0]
        assert abs(c - (1 - np.exp(-1))) < 1e-4


def test_seeded_fallback_recovers_from_bad_seeds():
    data = ST.analytic_set(256, seed=3)
    bnds = ST.swim_bounds(data["qn"])
    d = data["d"].cpu().numpy()
    tau = ST.lm_tau()
    w = 1 / d.max(1)
    plain = F.fit_lm(d, tau, data["qn"], w, bnds, mode="plain")
    bad = np.tile([0.5, bnds[1] * 0.99, 90.0, bnds[4] * 1.01], (256, 1))  # far from every truth
    fb = F.fit_lm(d, tau, data["qn"], w, bnds, mode="seeded_fallback", start=bad)
    assert ((fb.status >> 1) & 1).mean() > 0.05  # seeds whose LM hit the cap fell back
    assert (fb.cost <= plain.cost * (1 + 1e-3) + 1e-30).mean() >= 0.95


def test_seeded_cost_fallback_rule():
    """Mode 4: a seeded fit above the bin's Brownian optimum (mode 3 on the
    same curve) falls back to the plain strategy and keeps the lower cost, so
    it ends at or below the plain fit's cost; every kept seeded fit is at or
    below the Brownian optimum."""
    data = ST.analytic_set(256, seed=3)
    bnds = ST.swim_bounds(data["qn"])
    d = data["d"].cpu().numpy()
    tau = ST.lm_tau()
    w = 1 / d.max(1)
    plain = F.fit_lm(d, tau, data["qn"], w, bnds, mode="plain")
    brown = F.fit_lm(d, tau, data["qn"], w, bnds, mode="brownian")
    bad = np.tile([0.5, bnds[1] * 0.99, 90.0, bnds[4] * 1.01], (256, 1))  # far from every truth
    good = np.stack([data["theta"][:, 2], data["theta"][:, 3], data["theta"][:, 4], data["theta"][:, 5]], 1)
    for start in (bad, good):
        r = F.fit_lm(d, tau, data["qn"], w, bnds, mode="seeded_cost", start=start.astype(np.float32))
        fell = ((r.status >> 1) & 1).astype(bool)
        assert np.all(r.cost[fell] <= plain.cost[fell] * (1 + 1e-12) + 1e-30)
        assert np.all(r.cost[~fell] <= brown.cost[~fell] * (1 + 1e-9) + 1e-30)
    assert fell.mean() < 0.2  # from the generator's own parameters few fits fall back


def test_trained_surrogate_gains_over_plain_lm():
    """Equal fit error = final cost within 1e-3 of the plain LM's (or lower)."""
    net = ST.build_and_train(n_analytic=1 << 18, epochs=16, seed=0, batch_max=4096)
    held = ST.analytic_set(8192, seed=99)
    s, _ = ST.compare_fits(net, held, ST.swim_bounds(held["qn"]))
    print(s)
    # seeded alone: far fewer model evaluations and a large q-fits/s gain
    assert s["seeded_frac_equal_or_better"] >= 0.98, s
    assert s["seeded_mean_evals"] < 0.2 * s["plain_mean_evals"], s
    assert s["seeded_speedup"] >= 4.0, s
    # with the reference's starts as fallback: equal fit error on >= 99.5 %
    assert s["fallback_frac_equal_or_better"] >= 0.995, s
    assert s["fallback_speedup"] >= 1.5, s
    net.close()
