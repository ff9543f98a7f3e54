"""Training data, training loop and the seeded-fit comparison for the
surrogate (hackathon_b200/surrogate.py).

Data (all generated on the GPU):
  analytic   model curves (ddm_model_curves) at parameters drawn uniformly
             from the batched-video ranges -- swimmer share alpha in [0, 0.9],
             mean speed vbar in [0.3, 3] px/frame, Schulz Z in [1.5, 10],
             D in [0.05, 0.5] px^2/frame, amplitude A in [0.5, 2],
             baseline B/A in [0, 0.2] -- at q = 2 pi k / 512 with |k| in
             [4, 60] (4 effective-|k| nodes of 0.2-1 % spread), with 1 %
             multiplicative Gaussian noise;
  pipeline   the radial D(q, tau) the engine itself produces from seeded
             synthetic videos (hackathon_b200/synth.py) with per-video
             parameters drawn from the same ranges, labelled with the
             generator's parameters.
Features: surrogate.features*; targets: surrogate.encode (alpha, ln vbar,
ln Z, ln D, ln tau_e).

The comparison fits held-out curves twice with the batched LM: from the
reference's start strategy (mode 0, "plain") and from the surrogate's
prediction with the plain strategy as the fallback (mode 2), and reports
q-fits/s (device time, CUDA events), iterations and the fit error of each.
"""
import math
import time

import numpy as np

from . import fit as F
from . import surrogate as S

L_LAGS = 512       # lags 0..511 (the 512^2 x 1024 workload's L)
N_REF = 512        # q = 2 pi k / N_REF
K_NODES = 4
RANGES = dict(alpha=(0.0, 0.9), vbar=(0.3, 3.0), Z=(1.5, 10.0), D=(0.05, 0.5), A=(0.5, 2.0), BA=(0.0, 0.2),
              k=(4.0, 60.0))


def lm_tau():
    return F.lag_grid(L_LAGS).astype(np.float32)


def feat_tau():
    return S.feature_lags(L_LAGS).astype(np.float32)


def sample_params(n, seed):
    """theta [n, 6] = (A, B, alpha, vbar, Z, D) and qn [n, 4]."""
    rng = np.random.default_rng(seed)
    u = lambda key: rng.uniform(*RANGES[key], n)  # noqa: E731
    A = u("A")
    th = np.stack([A, A * u("BA"), u("alpha"), u("vbar"), u("Z"), u("D")], 1)
    q = 2 * np.pi * u("k") / N_REF
    spread = rng.uniform(0.002, 0.01, n)
    qn = q[:, None] * (1 + spread[:, None] * np.array([-1.5, -0.5, 0.5, 1.5])[None])
    return th.astype(np.float32), qn.astype(np.float32)


def swim_bounds(qn):
    """bounds() over the q range of the data set, without the reference's
    2 um/s swim floor (the workload's speeds go down to 0.3 px/frame)."""
    q = qn.mean(1)
    tmax = L_LAGS - 1
    return np.array([0.3 / (q.max() * tmax), 3 / q.min(), 0.5, 100.0, 0.01 / (q.max() ** 2 * tmax),
                     10 / q.min() ** 2], np.float32)


def analytic_set(n, seed, noise=0.01):
    """GPU tensors: LM data d [n, nt], features x [n, 65], targets y [n, 5],
    plus host theta/qn."""
    import torch
    th, qn = sample_params(n, seed)
    d = F.model_curves(th, qn, lm_tau(), noise=noise, seed=2 * seed + 1)
    s, te = F.model_curves(th, qn, feat_tau(), noise=noise, seed=2 * seed + 2, want_tau_e=True)
    q = torch.from_numpy(qn.mean(1)).cuda()
    x = features_t(s, q)
    y = torch.from_numpy(S.encode(th[:, 2], th[:, 3], th[:, 4], th[:, 5], te.cpu().numpy().astype(np.float64))).cuda()
    return dict(d=d, x=x, y=y, theta=th, qn=qn)


def features_t(samples, q):
    """Device samples [n, 64] at feature_lags, q [n] -> features [n, 65]."""
    import torch
    m = samples.max(1, keepdim=True).values
    m = torch.where(m > 0, m, torch.ones_like(m))
    return torch.cat([samples / m, (torch.log(q) / 4.0)[:, None]], 1).float().contiguous()


def pipeline_set(n_videos, seed, N=256, T=1024, NB=28, kmin=2.0, kmax=30.0, max_curves=None, log=None,
                 label="truth"):
    """Radial curves from the engine on seeded synthetic videos (up to
    n_videos, stopping once max_curves curves are collected). Returns the
    same dict as analytic_set (d at the LM lags, features, targets).

    label "truth": the generator's parameters of the curve's video; "fit":
    the batched plain LM's fit of each curve (the reference's start strategy).
    On held-out pipeline curves both give the same seeded gain (3.1-3.4x at
    63 % equal-or-better fit error, 2^20-curve training); "fit" costs the
    analytic curves some accuracy, so "truth" is the default. The returned
    "theta" is the label's (A, B, alpha, vbar, Z, D)."""
    import torch

    from . import synth
    from .engine import DdmEngine
    rng = np.random.default_rng(seed)
    eng = DdmEngine.create(N=N, T=T, L=L_LAGS, NB=NB, kmin=kmin, kmax=kmax)
    lags = F.lag_grid(L_LAGS)
    ft = S.feature_lags(L_LAGS)
    i0 = np.floor(ft).astype(int)
    i1 = np.minimum(i0 + 1, L_LAGS - 1)
    fr = ft - i0
    ds, xs, ths, qns = [], [], [], []
    order = np.arange(T, dtype=np.uint32)
    t0 = time.time()
    got = 0
    for v in range(n_videos):
        if max_curves is not None and got >= max_curves:
            break
        if log and v and v % 100 == 0:
            log(f"pipeline videos: {v}, curves {got}, {time.time() - t0:.0f} s")
        al, vb, Z, D = (rng.uniform(*RANGES[k]) for k in ("alpha", "vbar", "Z", "D"))
        spec = synth.VideoSpec(N=N, T=T, n_blobs=int(2000 * (N / 512) ** 2), frac_brownian=1 - al, D=D, vbar=vb,
                               Z=Z, roi_radius=-1, drop_frac=0.02, seed=int(seed * 100003 + v))
        frames, valid, truth = synth.generate(spec)
        eng.ingest_frames(frames, np.arange(T, dtype=np.int32), 1.0 / 65535)
        eng.compute_temporal(order, valid.astype(np.float32))
        rad = eng.read_radial()
        pr = F.prepare(rad)
        Dm = np.asarray(rad.D).reshape(NB, L_LAGS)[pr.bins]
        ds.append(Dm[:, lags])
        xs.append(S.features_from_samples(Dm[:, i0] * (1 - fr) + Dm[:, i1] * fr, pr.q))
        a_eff = truth["n_swim"] / spec.n_blobs
        ths.append(np.tile([1.0, 0.0, a_eff, vb, Z, D], (len(pr.bins), 1)))
        qns.append(pr.qn)
        got += len(pr.bins)
    eng.destroy()
    th = np.concatenate(ths).astype(np.float32)
    qn = np.concatenate(qns).astype(np.float32)
    if max_curves is not None and len(th) > max_curves:  # exactly max_curves
        ds, xs = [np.concatenate(ds)[:max_curves]], [np.concatenate(xs)[:max_curves]]
        th, qn = th[:max_curves], qn[:max_curves]
    if label == "fit":
        d = np.concatenate(ds)
        res = F.fit_lm(d, lm_tau(), qn, 1.0 / d.max(1), swim_bounds(qn), mode="plain")
        th = np.stack([res.theta[:, 0], res.theta[:, 1], res.alpha, res.vbar, res.Z, res.D], 1).astype(np.float32)
    te = F.model_curves(th, qn, np.ones(1, np.float32), want_tau_e=True)[1].cpu().numpy().astype(np.float64)
    y = S.encode(th[:, 2], th[:, 3], th[:, 4], th[:, 5], te)
    return dict(d=torch.from_numpy(np.concatenate(ds).astype(np.float32)).cuda(),
                x=torch.from_numpy(np.concatenate(xs)).cuda(), y=torch.from_numpy(y).cuda(), theta=th, qn=qn,
                videos=len(ths))


def train(net, x, y, epochs=8, batch=8192, lr=2e-3, lr_min=2e-5, seed=0, log=None):
    """Adam with a cosine learning-rate schedule over shuffled mini-batches
    (the last partial batch is dropped). Returns the final training loss."""
    import torch
    n = x.shape[0]
    batch = min(batch, net.batch_max, n // 8 * 8)
    steps_per = n // batch
    total = epochs * steps_per
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    step = 0
    loss = None
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g, device="cuda")
        for b in range(steps_per):
            idx = perm[b * batch:(b + 1) * batch]
            xb, yb = x[idx].contiguous(), y[idx].contiguous()
            cur = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * step / max(total - 1, 1)))
            want = b == steps_per - 1
            out = net.train_step(xb, yb, cur, want_loss=want)
            if want:
                loss = out
                if log:
                    log(f"epoch {ep}: loss {loss:.4f}")
            step += 1
    net.sync()
    return loss


def predict_starts(net, x, bnds):
    """Surrogate prediction -> LM seeds [n, 4] = (alpha, vbar, Z, D) on the
    device, clipped into the fit's bounds."""
    import torch
    n = x.shape[0]
    m = (n + 7) // 8 * 8
    if m != n:
        x = torch.cat([x, torch.zeros((m - n, x.shape[1]), device=x.device)], 0)
    out = torch.empty((m, S.NOUT), dtype=torch.float32, device=x.device)
    for a in range(0, m, net.batch_max):
        b = min(m, a + net.batch_max)
        net.forward(x[a:b], out=out[a:b])
    sc = torch.from_numpy(S.SCALE.astype(np.float32)).cuda()
    off = torch.from_numpy(S.OFFSET.astype(np.float32)).cuda()
    raw = out[:n] * sc + off
    al = raw[:, 0].clamp(0.02, 0.98)
    vb = torch.exp(raw[:, 1]).clamp(float(bnds[0]), float(bnds[1]))
    Z = torch.exp(raw[:, 2]).clamp(float(bnds[2]), float(bnds[3]))
    D = torch.exp(raw[:, 3]).clamp(float(bnds[4]), float(bnds[5]))
    return torch.stack([al, vb, Z, D], 1).contiguous()


def compare_fits(net, data, bnds, max_iter=200, tol=1e-10, nrefine=3):
    """Plain LM (reference starts), surrogate-seeded LM, and surrogate-seeded
    LM with the plain strategy as fallback -- on non-convergence or a cost
    above a coarse Brownian scan ("fallback", mode 2), or on a cost above the
    bin's Brownian optimum alone ("costfb", mode 4) -- on the same curves; each
    device-timed with CUDA events on one stream (the seeded timings include
    the surrogate's inference)."""
    import torch
    d = data["d"].contiguous()
    n, nt = d.shape
    tau = torch.from_numpy(np.tile(lm_tau(), (n, 1))).cuda()
    qn = torch.from_numpy(data["qn"]).cuda()
    w = (1.0 / d.max(1).values).contiguous()
    b6 = torch.from_numpy(np.tile(bnds, (n, 1))).cuda()
    ntv = torch.full((n,), nt, dtype=torch.int32, device="cuda")
    predict_starts(net, data["x"][:8], bnds)  # first-call set-up outside the timed region
    res = {}
    for name, mode in (("plain", "plain"), ("seeded", "seeded"), ("fallback", "seeded_fallback"),
                       ("costfb", "seeded_cost")):
        theta = torch.empty((n, 6), dtype=torch.float64, device="cuda")
        cost = torch.empty(n, dtype=torch.float64, device="cuda")
        iters = torch.empty(n, dtype=torch.int32, device="cuda")
        evals = torch.empty(n, dtype=torch.int32, device="cuda")
        status = torch.empty(n, dtype=torch.int32, device="cuda")
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        start = None if mode == "plain" else predict_starts(net, data["x"], bnds)
        F.fit_lm_device(d, tau, qn, w, b6, ntv, theta, cost, iters, evals, status, mode=mode, start=start,
                        max_iter=max_iter, tol=tol, nrefine=nrefine, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res[name] = dict(ms=ms, qfits_per_s=n / (ms / 1e3), theta=theta.cpu().numpy(), cost=cost.cpu().numpy(),
                         iters=iters.cpu().numpy(), evals=evals.cpu().numpy(), status=status.cpu().numpy())
    p = res["plain"]
    summary = dict(n=n, plain_qfits_per_s=p["qfits_per_s"], plain_mean_iters=float(p["iters"].mean()),
                   plain_mean_evals=float(p["evals"].mean()))
    for name in ("seeded", "fallback", "costfb"):
        r = res[name]
        equal = r["cost"] <= p["cost"] * (1 + 1e-3) + 1e-30
        ratio = r["cost"] / np.maximum(p["cost"], 1e-300)
        summary.update({f"{name}_qfits_per_s": r["qfits_per_s"],
                        f"{name}_speedup": r["qfits_per_s"] / p["qfits_per_s"],
                        f"{name}_mean_iters": float(r["iters"].mean()),
                        f"{name}_mean_evals": float(r["evals"].mean()),
                        f"{name}_frac_equal_or_better": float(equal.mean()),
                        f"{name}_cost_ratio_p50_p90_p99": [float(np.quantile(ratio, q)) for q in (0.5, 0.9, 0.99)],
                        f"{name}_frac_fallback": float(((r["status"] >> 1) & 1).mean())})
    # fit error against the curves' labels (the generator's parameters for
    # analytic and "truth"-labelled pipeline curves): D (every curve) and
    # vbar (curves whose label has a motile fraction >= 0.2)
    lab = np.asarray(data["theta"], np.float64)
    motile = lab[:, 2] >= 0.2
    for name in ("plain", "seeded", "fallback", "costfb"):
        th = res[name]["theta"]
        eD = np.abs(np.exp(th[:, 5]) / lab[:, 5] - 1)
        ev = np.abs(np.exp(th[:, 3]) / lab[:, 3] - 1)[motile]
        summary.update({f"{name}_D_relerr_p50": float(np.median(eD)),
                        f"{name}_frac_D_within_10pct": float((eD <= 0.1).mean()),
                        f"{name}_vbar_relerr_p50": float(np.median(ev)) if ev.size else None,
                        f"{name}_frac_vbar_within_10pct": float((ev <= 0.1).mean()) if ev.size else None})
    return summary, res


def build_and_train(n_analytic=1 << 19, n_videos=0, epochs=8, seed=0, batch_max=8192, log=None, pipeline=None):
    """Generates the training set, trains a fresh surrogate; returns it.
    `pipeline`: keyword arguments of pipeline_set (geometry, max_curves)."""
    import torch
    t0 = time.time()
    parts = [analytic_set(n_analytic, seed)]
    if n_videos:
        parts.append(pipeline_set(n_videos, seed + 1, log=log, **(pipeline or {})))
    x = torch.cat([p["x"] for p in parts], 0)
    y = torch.cat([p["y"] for p in parts], 0)
    if log:
        log(f"training set: {x.shape[0]} curves ({n_analytic} analytic) in {time.time() - t0:.1f} s")
    net = S.Surrogate(batch_max=batch_max, seed=seed)
    train(net, x, y, epochs=epochs, seed=seed, log=log)
    net.train_info = dict(analytic_curves=int(n_analytic), pipeline_curves=int(x.shape[0] - n_analytic),
                          pipeline_videos=int(parts[1]["videos"]) if n_videos else 0)
    return net
