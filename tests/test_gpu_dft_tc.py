"""The tensor-core zero-padded 2048-point DFT (ddm_dft2048_tc, csrc/dft_tc.cu)
against numpy's FP64 FFT: a BF16 three-term split with FP32 accumulation, so
each series' spectrum within 4e-5 of its RMS; series scaled over four decades,
a count that is not a multiple of the kernel's group of four, and a stride
between series longer than the 1024 samples."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")


@pytest.mark.gpu
def test_dft2048_tc_matches_fft():
    from hackathon_b200 import _lib
    lib = _lib.load()
    n, ld = 37, 1100
    rng = np.random.default_rng(4)
    sc = 10 ** rng.uniform(-2, 2, n)
    x = ((rng.standard_normal((n, ld)) + 1j * rng.standard_normal((n, ld))) * sc[:, None]).astype(np.complex64)
    xd = torch.from_numpy(x).cuda()
    Xd = torch.zeros((n, 2048), dtype=torch.complex64, device="cuda")
    rc = lib.ddm_dft2048_tc(C.c_void_p(xd.data_ptr()), ld, n, C.c_void_p(Xd.data_ptr()), None)
    assert rc == 0, lib.ddm_create_error().decode()
    ref = np.fft.fft(x[:, :1024].astype(np.complex128), n=2048, axis=1)
    got = Xd.cpu().numpy()
    rel = np.abs(got - ref).max(axis=1) / np.sqrt(np.mean(np.abs(ref) ** 2, axis=1))
    assert rel.max() < 4e-5, rel.max()


def test_dft2048_tc_rejects_short_stride():
    from hackathon_b200 import _lib
    lib = _lib.load()
    assert lib.ddm_dft2048_tc(None, 1000, 4, None, None) == 1  # DDM_ERR_ARG before any device work
    assert "ld" in lib.ddm_create_error().decode()
    assert lib.ddm_dft2048_tc(None, 1024, 0, None, None) == 0  # nothing to do
