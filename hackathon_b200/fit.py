"""Per-bin motility fit on the GPU: batched Levenberg-Marquardt over q-bins.

Host side of the fit stage (motility-ddm/src/motility_fit.js). ``prepare``,
``lag_grid`` and ``bounds`` restate the reference's data preparation
(lagGrid :358-369, prepare :383-401, bounds :480-491); ``fit_bins`` runs the
batched LM kernel through the C ABI (ddm_fit_lm, include/ddm_b200.h), one
warp per bin, either from the reference's start strategy (``mode="plain"``:
Brownian scan, 64-start grid, best 3 refined; fitBrownian :500-536 and
fitSwimmer :577-611 with LM in place of Nelder-Mead) or from given starting
parameters (``mode="seeded"``, e.g. the surrogate network's prediction).

Units follow the reference: q = 2 pi k / (N dxUm), tau = lag / fps. With
dxUm = fps = 1 they are px^-1 and frames.
"""
import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib

SWIM_MIN_UM_S = 2.0  # GATES.SWIM_MIN_UM_S, motility_fit.js:28-38
MODES = {"plain": 0, "seeded": 1, "seeded_fallback": 2, "brownian": 3, "seeded_cost": 4}
MAX_LAGS = 128
MAX_NODES = 8


def lag_grid(L):
    """lagGrid (motility_fit.js:358-369): lags 1..10, then ~8 % steps to L-1."""
    lags = list(range(1, min(10, L - 1) + 1))
    x = 10.0
    while True:
        x *= 1.08
        t = int(math.floor(x + 0.5))  # Math.round: ties toward +inf
        if t > L - 1:
            break
        if t > lags[-1]:
            lags.append(t)
    return np.array(lags, np.int32)


@dataclass
class Prepared:
    """prepare()'s output for the bins a fit uses (motility_fit.js:383-401)."""
    bins: np.ndarray    # [nb] bin index b
    q: np.ndarray       # [nb] q of the bin centre
    qn: np.ndarray      # [nb, K] q of the effective-|k| nodes
    d: np.ndarray       # [nb, nt] D(q_b, tau_j) at the lag grid
    w: np.ndarray       # [nb] 1 / max_j d
    lags: np.ndarray    # [nt]
    tau: np.ndarray     # [nt]
    dt: float
    tauMax: float


def prepare(radial, dxUm=1.0, fps=1.0):
    """prepare (motility_fit.js:383-401): bins with >= 3 modes and a finite,
    positive maximum; lags from lag_grid; weight 1 / max d; q-nodes from the
    bin's kNodes."""
    N, NB, L = radial.N, radial.NB, radial.L
    dt = 1.0 / fps
    lags = lag_grid(L)
    tau = lags * dt
    D = np.asarray(radial.D, np.float64).reshape(NB, L)
    K = len(radial.kNodes) // NB if radial.kNodes is not None and len(radial.kNodes) else 0
    qs = 2 * math.pi / (N * dxUm)
    keep, qv, qn, dv, wv = [], [], [], [], []
    for b in range(NB):
        if radial.nModes[b] < 3:
            continue
        d = D[b, lags]
        sc = d.max()
        if not (sc > 0) or not np.isfinite(sc):
            continue
        keep.append(b)
        qv.append(qs * radial.kCenter[b])
        qn.append(np.asarray(radial.kNodes[b * K:(b + 1) * K]) * qs if K else [qs * radial.kCenter[b]])
        dv.append(d)
        wv.append(1.0 / sc)
    nb = len(keep)
    return Prepared(np.array(keep, np.int32), np.array(qv), np.array(qn, np.float64).reshape(nb, -1),
                    np.array(dv, np.float64).reshape(nb, len(lags)), np.array(wv), lags, tau, dt,
                    (L - 1) * dt)


def bounds(pr, swim_min=SWIM_MIN_UM_S):
    """bounds (motility_fit.js:480-491) -> (vmin, vmax, Zmin, Zmax, Dmin, Dmax)."""
    qmin, qmax = pr.q.min(), pr.q.max()
    return np.array([max(swim_min, 0.3 / (qmax * pr.tauMax)), 3 / (qmin * pr.dt), 0.5, 100.0,
                     0.01 / (qmax * qmax * pr.tauMax), 10 / (qmin * qmin * pr.dt)])


@dataclass
class FitResult:
    theta: np.ndarray   # [nfit, 6] A, B, alpha, ln vbar, ln Z, ln D
    cost: np.ndarray    # [nfit] weighted RSS
    iters: np.ndarray   # [nfit] LM iterations
    evals: np.ndarray   # [nfit] model evaluations
    status: np.ndarray = None  # [nfit] bit 0 converged, bit 1 fell back to the reference's starts

    @property
    def alpha(self):
        return self.theta[:, 2]

    @property
    def vbar(self):
        return np.exp(self.theta[:, 3])

    @property
    def Z(self):
        return np.exp(self.theta[:, 4])

    @property
    def D(self):
        return np.exp(self.theta[:, 5])


def _check(rc):
    if rc != _lib.DDM_OK:
        from .engine import DdmArgError, DdmError
        msg = _lib.load().ddm_create_error().decode()
        raise (DdmArgError if rc == _lib.DDM_ERR_ARG else DdmError)(rc, msg)


def fit_lm(d, tau, qn, w, bnds, mode="plain", start=None, nt=None, max_iter=200, tol=1e-10,
           nrefine=3, geometry="3d", vmag=None):
    """Batched LM over independent bins (host arrays in, host arrays out).

    d, tau [nfit, nt_max]; qn [nfit, K]; w [nfit]; bnds [6] or [nfit, 6];
    start [nfit, 4] = (alpha, vbar, Z, D) for mode "seeded"; nt [nfit] lags
    used per fit (default nt_max). mode "brownian" fits the Brownian model
    alone, A (1 - <exp(-D q^2 tau)>) + B per bin (fitBrownian's search,
    motility_fit.js:500-536, one D per bin). geometry "2d" uses the in-plane
    swimmer kernel (swimmerKernel, motility_fit.js:227-229); vmag [nfit] (or
    a scalar) multiplies the model by J0(q |V| tau) for a known drift speed
    (modelColumn :426)."""
    lib = _lib.load()
    d = np.ascontiguousarray(d, np.float32)
    nfit, nt_max = d.shape
    tau = np.ascontiguousarray(np.broadcast_to(tau, (nfit, nt_max)), np.float32)
    qn = np.ascontiguousarray(qn, np.float32)
    qn = qn if qn.ndim == 2 else qn.reshape(nfit, -1)
    K = qn.shape[1]
    w = np.ascontiguousarray(np.broadcast_to(w, (nfit,)), np.float32)
    bnds = np.ascontiguousarray(np.broadcast_to(bnds, (nfit, 6)), np.float32)
    ntv = np.ascontiguousarray(np.full(nfit, nt_max) if nt is None else nt, np.int32)
    m = MODES[mode]
    st = None
    if mode in ("seeded", "seeded_fallback", "seeded_cost"):
        st = np.ascontiguousarray(start, np.float32).reshape(nfit, 4)
    theta = np.zeros((nfit, 6))
    cost = np.zeros(nfit)
    iters = np.zeros(nfit, np.int32)
    evals = np.zeros(nfit, np.int32)
    status = np.zeros(nfit, np.int32)
    vm = None if vmag is None else np.ascontiguousarray(np.broadcast_to(vmag, (nfit,)), np.float32)
    if geometry not in ("3d", "2d"):
        raise ValueError(f"geometry must be '3d' or '2d', not {geometry!r}")
    p = lambda a: C.c_void_p(a.ctypes.data) if a is not None else None  # noqa: E731
    _check(lib.ddm_fit_lm_model(nfit, nt_max, K, p(ntv), p(d), p(tau), p(qn), p(w), p(bnds), p(st), m,
                                max_iter, tol, nrefine, 1 if geometry == "2d" else 0, p(vm), p(theta), p(cost),
                                p(iters), p(evals), p(status), 0, None))
    return FitResult(theta, cost, iters, evals, status)


def fit_lm_device(d, tau, qn, w, bnds, nt, theta, cost, iters=None, evals=None, status=None, mode="plain",
                  start=None, max_iter=200, tol=1e-10, nrefine=3, stream=None):
    """Same on device tensors (torch, contiguous): queued on `stream`."""
    lib = _lib.load()
    nfit, nt_max = d.shape
    K = qn.shape[1]
    a = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    s = C.c_void_p(stream) if stream else None
    _check(lib.ddm_fit_lm(nfit, nt_max, K, a(nt), a(d), a(tau), a(qn), a(w), a(bnds), a(start),
                          MODES[mode], max_iter, tol, nrefine, a(theta), a(cost), a(iters), a(evals),
                          a(status), 1, s))


def model_curves(theta, qn, tau, noise=0.0, seed=0, want_tau_e=False, stream=None):
    """Model curves on the GPU (ddm_model_curves): theta [n, 6] = (A, B,
    alpha, vbar, Z, D), qn [n, K], tau [nt] -> torch CUDA y [n, nt] (and
    tau_e [n])."""
    import torch
    lib = _lib.load()
    th = torch.as_tensor(np.ascontiguousarray(theta, np.float32)).cuda()
    q = torch.as_tensor(np.ascontiguousarray(qn, np.float32)).cuda()
    t = torch.as_tensor(np.ascontiguousarray(tau, np.float32)).cuda()
    n, K = q.shape
    y = torch.empty((n, t.numel()), dtype=torch.float32, device="cuda")
    te = torch.empty(n, dtype=torch.float32, device="cuda") if want_tau_e else None
    a = lambda x: C.c_void_p(x.data_ptr()) if x is not None else None  # noqa: E731
    s = torch.cuda.current_stream().cuda_stream if stream is None else stream
    _check(lib.ddm_model_curves(n, K, a(q), a(th), t.numel(), a(t), float(noise), int(seed), a(y), a(te),
                                C.c_void_p(s) if s else None))
    return (y, te) if want_tau_e else y


def fit_bins(radial, dxUm=1.0, fps=1.0, mode="plain", start=None, swim_min=SWIM_MIN_UM_S, **kw):
    """prepare + bounds + batched LM for every fitted bin of one Radial."""
    pr = prepare(radial, dxUm, fps)
    b = bounds(pr, swim_min)
    res = fit_lm(pr.d, pr.tau, pr.qn, pr.w, b, mode=mode, start=start, **kw)
    return pr, b, res
