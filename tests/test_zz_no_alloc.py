"""The allocation-free spatial stage (ddm_spectra_noalloc) against the engine's
ingest path.

ddm_spectra_noalloc serves callers that may not allocate device memory (a
host framework that owns all device allocations and lends out planned
buffers, or a capture loop that must not stall in cudaMalloc): it takes
device frames and the caller's device history ring and keeps its own scratch
in a fixed file-scope device array. This test calls it through the C ABI,
with the output ring allocated by the test, twice in a row, and checks each
result against the history the engine's ddm_ingest_frames_device produces
for the same frames, within the spectrum tolerance the other GPU tests use
(max |difference| / rms < 2e-5).

The file name sorts last so that a run stopping at the first failure has run
every other test first; the test also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _rel_err(got, ref):
    rms = np.sqrt(np.mean(np.abs(ref) ** 2))
    return float(np.abs(got - ref).max() / rms)


def test_spectra_noalloc_matches_engine_twice():
    import hackathon_b200 as H
    from hackathon_b200 import _lib

    lib = _lib.load()
    N, T = 256, 48
    gen = torch.Generator(device="cuda").manual_seed(3)
    frames = [torch.randint(0, 4096, (T, N, N), device="cuda", generator=gen, dtype=torch.int32)
              .to(torch.int16) for _ in range(2)]
    slots = np.arange(T, dtype=np.int32)[::-1].copy()  # reversed ring order
    modes = N * (N // 2 + 1)
    eng = H.DdmEngine.create(N=N, T=T, L=8, NB=8, kmin=4, kmax=60)
    try:
        for call in range(2):
            fr = frames[call]
            eng.ingest_frames(fr, slots, 1.0 / 4095)
            ref = eng.read_history()
            out = torch.zeros((modes, T), dtype=torch.complex64, device="cuda")
            torch.cuda.synchronize()
            rc = lib.ddm_spectra_noalloc(C.c_void_p(fr.data_ptr()), 1, T, N, T,
                                         slots.ctypes.data_as(C.c_void_p), C.c_float(1.0 / 4095),
                                         C.c_void_p(out.data_ptr()), None)
            assert rc == 0, lib.ddm_create_error().decode()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert _rel_err(got, ref) < 2e-5, f"call {call}"
    finally:
        eng.destroy()


def test_spectra_noalloc_rejects_oversize_roi():
    from hackathon_b200 import _lib

    lib = _lib.load()
    slots = np.zeros(1, np.int32)
    dummy = torch.zeros(16, device="cuda")
    rc = lib.ddm_spectra_noalloc(C.c_void_p(dummy.data_ptr()), 1, 1, 1024, 4,
                                 slots.ctypes.data_as(C.c_void_p), C.c_float(1.0),
                                 C.c_void_p(dummy.data_ptr()), None)
    assert rc == 6  # DDM_ERR_TOO_LARGE, before any device work
    assert "512" in lib.ddm_create_error().decode()
