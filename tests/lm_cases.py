"""Seeded per-bin fit problems shared by the LM tests (CPU and GPU).

Each case is one q-bin of a 512^2 geometry (|k| 4..40, where the swimmer decay
spans several lags and the parameters are identifiable per bin,
4 effective-|k| nodes per bin spread like makeBins' leakage quantiles), the
reference's lag grid for L = 512 (61 lags), and D(q, tau) = A c(tau) + B from
the motility model at parameters drawn from the batched-video ranges
(alpha 0.2..0.9, vbar 2..6 px/frame, Z 2..10, D 0.05..0.5 px^2/frame),
optionally with multiplicative Gaussian noise."""
import numpy as np

import oracle as O


def lag_tau(L=512):
    return np.array(O.lag_grid(L), np.float64)


def make_cases(n, seed=0, noise=0.0, L=512, N=512):
    rng = np.random.default_rng(seed)
    tau = lag_tau(L)
    out = []
    for _ in range(n):
        k = rng.uniform(4, 40)
        qc = 2 * np.pi * k / N
        qn = qc * (1 + np.array([-0.012, -0.004, 0.004, 0.012]))
        al, v, Z, D = rng.uniform(0.2, 0.9), rng.uniform(2, 6), rng.uniform(2, 10), rng.uniform(0.05, 0.5)
        A, B = rng.uniform(0.5, 2.0), rng.uniform(0.0, 0.1)
        th = np.array([A, B, al, np.log(v), np.log(Z), np.log(D)])
        y = O.lm_model(tau, qn, th)
        if noise:
            y = y * (1 + noise * rng.standard_normal(y.size))
        out.append(dict(d=y, tau=tau, qn=qn, w=1 / y.max(), theta=th))
    return out


def bounds6(cases, L=512):
    """bounds() (motility_fit.js:480-491) over the cases' q range, dt = 1."""
    q = np.array([c["qn"].mean() for c in cases])
    tmax = L - 1
    return np.array([max(2.0, 0.3 / (q.max() * tmax)), 3 / q.min(), 0.5, 100.0,
                     0.01 / (q.max() ** 2 * tmax), 10 / q.min() ** 2])
