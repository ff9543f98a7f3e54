"""The allocation-free spatial stage (ddm_spectra_noalloc) against the engine's
ingest path.

ddm_spectra_noalloc serves callers that may not allocate device memory (a
host framework that owns all device allocations and lends out planned
buffers, or a capture loop that must not stall in cudaMalloc): it takes
device frames and the caller's device history ring and keeps its own scratch
in a fixed file-scope device array. This test calls it through the C ABI,
with the output ring allocated by the test, twice in a row, and checks each
result against the history the engine's ingest produces for the same frames,
within the spectrum tolerance the other GPU tests use (max |difference| /
rms < 2e-5). The two calls differ in N and scale, so the second call also
refills the fixed tables; each dtype (u8, u16, f32) runs, and N = 512 (the
largest ROI the fixed scratch takes, 4-frame chunks) is covered. After each
call ddm_spectra_noalloc_status reports that no bounded wait gave up.

The file name sorts last so that a run stopping at the first failure has run
every other test first; the test also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

# (dtype code, torch dtype, value range, scale): u8, u16 (stored as int16), f32
_DTYPES = {0: (torch.uint8, 256, 1.0 / 255), 1: (torch.int16, 4096, 1.0 / 4095), 2: (torch.float32, 1, 1.0)}


def _rel_err(got, ref):
    rms = np.sqrt(np.mean(np.abs(ref) ** 2))
    return float(np.abs(got - ref).max() / rms)


def _frames(dtype, n, N, seed):
    tdt, hi, _ = _DTYPES[dtype]
    gen = torch.Generator(device="cuda").manual_seed(seed)
    if dtype == 2:
        return torch.rand((n, N, N), device="cuda", generator=gen, dtype=torch.float32)
    return torch.randint(0, hi, (n, N, N), device="cuda", generator=gen, dtype=torch.int32).to(tdt)


@pytest.mark.parametrize("dtype", [0, 1, 2], ids=["u8", "u16", "f32"])
def test_spectra_noalloc_matches_engine_twice(dtype):
    import hackathon_b200 as H
    from hackathon_b200 import _lib

    lib = _lib.load()
    T = 24
    # two calls in a row with different N and scale: the second refills the tables
    calls = [(256, _DTYPES[dtype][2]), (64 if dtype != 1 else 512, 0.5 * _DTYPES[dtype][2])]
    for call, (N, scale) in enumerate(calls):
        fr = _frames(dtype, T, N, 3 + call)
        slots = np.arange(T, dtype=np.int32)[::-1].copy()  # reversed ring order
        modes = N * (N // 2 + 1)
        eng = H.DdmEngine.create(N=N, T=T, L=8, NB=8, kmin=4, kmax=min(60, N // 2 - 2))
        try:
            eng.ingest_frames(fr, slots, scale)
            ref = eng.read_history()
        finally:
            eng.destroy()
        out = torch.zeros((modes, T), dtype=torch.complex64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.ddm_spectra_noalloc(C.c_void_p(fr.data_ptr()), dtype, T, N, T,
                                     slots.ctypes.data_as(C.c_void_p), C.c_float(scale),
                                     C.c_void_p(out.data_ptr()), None)
        assert rc == 0, lib.ddm_create_error().decode()
        assert lib.ddm_spectra_noalloc_status(None) == 0, lib.ddm_create_error().decode()
        got = out.cpu().numpy()
        assert _rel_err(got, ref) < 2e-5, f"call {call}, N={N}"


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
