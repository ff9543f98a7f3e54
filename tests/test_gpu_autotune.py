"""The autotuner (ddm_autotune) picks its spatial chunk, temporal unit size
(on the sparse-mask kernel when that path is on) and temporal kernel variant
(on the transform kernels) from timed candidates, and the tuned engine
computes the same radial record as an untuned one (unit size regroups FP64
partial sums, the variant changes the FFT plan's FP32 rounding: agreement to
1e-5 of each bin's scale, the FP32 transforms' accuracy)."""
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
            key = ("r16:" if t["variant"] else "") + str(t["unit_size"])
            assert key in rep["temporal_unit"] and t["unit_size"] == rep["best_unit"]
            assert t["variant"] == rep["best_variant"]
            assert any(k.startswith("r16:") for k in rep["temporal_unit"])  # TPAD 1024 has both variants
            # the sparse-mask kernel's sweep picks the unit (the path this mask takes)
            su = rep["sparse_unit"]
            assert su[str(t["unit_size"])] == min(su.values())
            assert min(rep["spatial_chunk"].values()) == pytest.approx(rep["us_per_frame"], rel=1e-3)
        e.ingest_frames(frames, slots, 1 / 65535)
        e.compute_temporal(order, mask)
        radials.append(e.read_radial())
        e.destroy()
    a, b = radials
    for k in range(32):
        sc = np.abs(b.D2()[k]).max()
        if sc > 0:
            assert np.abs(a.D2()[k] - b.D2()[k]).max() <= 1e-5 * sc
