"""The autotuner (ddm_autotune) picks its spatial chunk and temporal unit
size from timed candidates, and the tuned engine computes the same radial
record as an untuned one (unit size only regroups FP64 partial sums:
agreement to 1e-10 of each bin's scale)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
H = pytest.importorskip("hackathon_b200")
from hackathon_b200 import synth  # noqa: E402


def test_autotune_report_and_results_unchanged():
    spec = synth.VideoSpec(N=256, T=512, n_blobs=500, roi_radius=100, seed=4)
    frames, valid, _ = synth.generate(spec)
    order = np.arange(512, dtype=np.uint32)
    mask = valid.astype(np.float32)
    slots = np.arange(512, dtype=np.int32)
    radials = []
    for tune in (False, True):
        e = H.DdmEngine.create(N=256, T=512, L=256, NB=32, kmin=3, kmax=100)
        e.set_spatial_mask(synth.roi_mask(spec))
        if tune:
            rep = e.autotune()
            t = e.tuning
            assert str(t["chunk"]) in rep["spatial_chunk"] and t["chunk"] == rep["best_chunk"]
            assert str(t["unit_size"]) in rep["temporal_unit"] and t["unit_size"] == rep["best_unit"]
            assert min(rep["spatial_chunk"].values()) == pytest.approx(rep["us_per_frame"], rel=1e-3)
        e.ingest_frames(frames, slots, 1 / 65535)
        e.compute_temporal(order, mask)
        radials.append(e.read_radial())
        e.destroy()
    a, b = radials
    for k in range(32):
        sc = np.abs(b.D2()[k]).max()
        if sc > 0:
            assert np.abs(a.D2()[k] - b.D2()[k]).max() <= 1e-10 * sc
