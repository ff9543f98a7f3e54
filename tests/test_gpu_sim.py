"""The GPU movie generator (ddm_simulate) against the oracle's restatement of
sim.mjs on the same parameters and seeds: drop masks and truth exactly equal;
frames equal up to one grey level on at most 1 pixel in 10^5 (exp/log differ
from the host's by an ulp, which moves a pixel only where it sits on a
rounding boundary). Covers swimmers (3D and 2D), passive and fixed particles,
drift, exact and random drops, a movie long enough to need several chunks of
the GPU's normal stream (the spare normal and the stream position carried
between chunks), and host or device output."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

H = pytest.importorskip("hackathon_b200")
from hackathon_b200 import sim as S  # noqa: E402

CASES = {
    "motile_3d": dict(O.SCENARIOS[0]["sim"], T=64),
    "mixed_2d_drift": dict(O.BASE, N=128, T=48, seed=77, swimmers=dict(n=30, vbar=15.0, sigma=5.0, geometry="2d"),
                           passive=dict(n=25), fixed=dict(n=10), drift=dict(speed=6.0, angleDeg=135.0),
                           dropFrac=0.1),
    "few_blobs_many_chunks": dict(O.BASE, N=2048, T=17, seed=9, passive=dict(n=40), fixed=dict(n=3), dropExact=2),
    "no_particles": dict(O.BASE, N=64, T=5, seed=3),
}


def _check(sim, frames_gpu, valid_g, truth_g):
    fo, vo, to = O.simulate(sim)
    assert np.array_equal(valid_g, vo)
    for k in ("meanSpeed", "Vx", "Vy", "D"):
        assert truth_g[k] == to[k], k
    d = np.abs(frames_gpu.astype(np.int16) - fo.astype(np.int16))
    assert d.max() <= 1
    assert np.count_nonzero(d) <= max(1, fo.size // 100000), np.count_nonzero(d)


@pytest.mark.parametrize("name", list(CASES))
def test_movie_equals_oracle(name):
    sim = CASES[name]
    f, v, t = S.simulate(sim)
    _check(sim, f.cpu().numpy(), v, t)


def test_host_output_equals_device_output():
    sim = CASES["mixed_2d_drift"]
    fd, vd, _ = S.simulate(sim)
    fh, vh, _ = S.simulate(sim, device=False)
    assert np.array_equal(fd.cpu().numpy(), fh) and np.array_equal(vd, vh)


def test_rejects_bad_parameters():
    with pytest.raises(H.DdmArgError):
        S.simulate(dict(N=100, T=4))
    with pytest.raises(H.DdmArgError):
        S.simulate(dict(N=64, T=4, dropExact=9))
