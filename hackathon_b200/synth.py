"""Seeded synthetic DDM videos generated on the GPU (torch), for benchmarks.

Follows the semantics of the reference's simulator (motility-ddm/test/sim.mjs:
90-186): Gaussian blobs on a periodic N x N field, straight swimmers with
Schulz (Gamma) distributed speeds gamma(Z+1, vbar/(Z+1)) and 3D-isotropic
headings seen in projection, plus Brownian motion, and randomly dropped
frames. It extends it the way the benchmark workloads ask: uint16 frames with
Poisson shot noise around a mean count, a circular ROI mask or stuck ("hot")
pixels excluded by a pixel mask, and sizes up to 2048^2 x 4096.

Rendering: a separable Gaussian blob is an outer product gy (x) gx, so a frame
is Gy^T Gx over all particles -- one batched FP32 GEMM per chunk of frames.
Profiles use the periodic distance to the blob centre (the reference wraps
pixel indices, sim.mjs:147-154).
"""
from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class VideoSpec:
    N: int = 512
    T: int = 1024
    n_blobs: int = 2000
    sigma: float = 2.0          # blob sigma, px
    frac_brownian: float = 0.3  # non-motile share
    D: float = 0.2              # px^2 / frame, all particles
    vbar: float = 1.5           # mean swim speed, px / frame
    Z: float = 4.0              # Schulz width parameter
    mean_counts: float = 400.0  # mean photon count per pixel
    blob_peak: float = 300.0    # blob peak, counts
    roi_radius: float = 230.0   # circular ROI (<= 0: none)
    drop_frac: float = 0.02
    hot_frac: float = 0.0       # share of stuck pixels (excluded by hot_mask)
    hot_counts: float = 65000.0  # their value
    seed: int = 1


def config2(seed=1):
    """512^2 x 1024 uint16 mixed-motility video with a circular ROI and 2 %
    dropped frames (the benchmark's headline workload)."""
    return VideoSpec(seed=seed)


def config1(seed=1):
    """64 frames of 128^2 (u8 range): 200 blobs sigma 1.5 px, peak 120 over a
    background of 20 counts, pure Brownian motion D = 0.3 px^2/frame,
    periodic, Poisson noise, no mask and no dropped frames (the small plain
    DDM configuration)."""
    n, sig, peak, bg = 200, 1.5, 120.0, 20.0
    return VideoSpec(N=128, T=64, n_blobs=n, sigma=sig, frac_brownian=1.0, D=0.3,
                     mean_counts=bg + peak * n * 2 * np.pi * sig ** 2 / 128 ** 2, blob_peak=peak, roi_radius=0.0,
                     drop_frac=0.0, seed=seed)


def large(seed=1):
    """2048^2 x 4096 uint16 video with the mixed-motility statistics above,
    40,000 blobs and 5 % hot pixels (the large streamed configuration)."""
    return VideoSpec(N=2048, T=4096, n_blobs=40000, roi_radius=0.0, hot_frac=0.05, seed=seed)


def _hot_pixels(spec):
    rng = np.random.default_rng(spec.seed * 104729 + 3)
    return np.flatnonzero(rng.random(spec.N * spec.N) < spec.hot_frac)


def hot_mask(spec):
    """Pixel mask (1 = used) that excludes the stuck pixels, or None."""
    if spec.hot_frac <= 0:
        return None
    m = np.ones(spec.N * spec.N, np.uint8)
    m[_hot_pixels(spec)] = 0
    return m.reshape(spec.N, spec.N)


def roi_mask(spec):
    N = spec.N
    if spec.roi_radius <= 0:
        return None
    y, x = np.mgrid[:N, :N]
    c = N / 2
    return (((x - c) ** 2 + (y - c) ** 2) <= spec.roi_radius ** 2).astype(np.uint8)


def generate(spec, device="cuda", chunk=None):
    """Returns (frames u16 [T, N, N] on `device`, valid bool [T] numpy,
    truth dict). `chunk` frames are rendered at once (default: 64, fewer
    when the per-frame blob profiles would pass 2 GB)."""
    if chunk is None:
        chunk = int(max(1, min(64, 2e9 // (spec.n_blobs * 2 * spec.N * 8))))
    g = torch.Generator(device=device)
    g.manual_seed(spec.seed)
    N, T, P = spec.N, spec.T, spec.n_blobs
    dev = torch.device(device)
    n_swim = int(round(P * (1 - spec.frac_brownian)))
    # speeds gamma(Z+1, vbar/(Z+1)) via torch's Gamma sampler on a CPU generator
    cg = torch.Generator().manual_seed(spec.seed + 7919)
    conc = torch.full((n_swim,), spec.Z + 1, dtype=torch.float64)
    speed = torch._standard_gamma(conc, generator=cg) * (spec.vbar / (spec.Z + 1))
    phi = torch.rand(n_swim, generator=cg, dtype=torch.float64) * 2 * np.pi
    cz = torch.rand(n_swim, generator=cg, dtype=torch.float64) * 2 - 1
    s = torch.sqrt(1 - cz * cz)
    v = torch.zeros(P, 2, dtype=torch.float64)
    v[:n_swim, 0] = speed * s * torch.cos(phi)
    v[:n_swim, 1] = speed * s * torch.sin(phi)
    v = v.to(dev)
    x0 = torch.rand(P, 2, generator=g, device=dev, dtype=torch.float64) * N
    step = float(np.sqrt(2 * spec.D))
    bg = spec.mean_counts - spec.blob_peak * P * 2 * np.pi * spec.sigma ** 2 / (N * N)
    grid = torch.arange(N, device=dev, dtype=torch.float64)
    frames = torch.empty((T, N, N), dtype=torch.int16, device=dev)
    hot = torch.as_tensor(_hot_pixels(spec), device=dev) if spec.hot_frac > 0 else None
    pos = x0.clone()
    inv2s2 = 1.0 / (2 * spec.sigma ** 2)
    for t0 in range(0, T, chunk):
        m = min(chunk, T - t0)
        # positions of this chunk: drift + Brownian increments, periodic
        inc = v[None] + step * torch.randn(m, P, 2, generator=g, device=dev, dtype=torch.float64)
        path = pos[None] + torch.cumsum(inc, 0) - inc  # position at each frame
        pos = torch.remainder(path[-1] + inc[-1], N)
        path = torch.remainder(path, N)
        d = grid[None, None, :] - path[..., None]          # [m, P, 2, N]
        d = torch.remainder(d + N / 2, N) - N / 2           # periodic distance
        prof = torch.exp(-(d * d) * inv2s2).float()         # [m, P, 2, N]
        gx, gy = prof[:, :, 0, :], prof[:, :, 1, :]
        img = torch.bmm(gy.transpose(1, 2), gx)             # [m, N(y), N(x)]
        lam = (bg + spec.blob_peak * img).clamp_min(0)
        cnt = torch.poisson(lam, generator=g).clamp_(0, 65535)
        if hot is not None:
            cnt.view(m, N * N)[:, hot] = spec.hot_counts
        frames[t0:t0 + m] = cnt.to(torch.int32).to(torch.int16)
    rng = np.random.default_rng(spec.seed * 7919 + 13)
    valid = np.ones(T, bool)
    valid[1:] = rng.random(T - 1) >= spec.drop_frac
    truth = dict(n_swim=n_swim, mean_speed=float(speed.mean()), D=spec.D, vbar=spec.vbar, Z=spec.Z,
                 frac_brownian=spec.frac_brownian)
    # uint16 view of the same bits (torch's uint16 has limited op support)
    return frames.view(torch.uint16), valid, truth
