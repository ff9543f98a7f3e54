"""The learned seed for the fit: a BF16 tensor-core MLP over normalised ISF
curves (C ABI ddm_mlp_*, kernels in csrc/mlp.cu).

Input features per q-bin (65): D(q, tau) at 64 log-spaced lags in [1, L-1]
(linear interpolation between integer lags) divided by the largest of those
64 values, and ln(q)/4. Outputs (5), normalised: alpha (swimmer share of the
dynamic contrast = 1 - non-motile fraction), ln vbar, ln Z (Schulz width),
ln D, and ln tau_e (the lag where the model column first reaches 1 - 1/e;
an extension with no reference counterpart). The prediction seeds the
batched LM (ddm_fit_lm mode 1); the LM from the reference's start strategy
(mode 0) remains the fallback and the reference its error is measured against.
"""
import ctypes as C

import numpy as np

from . import _lib

NFEAT = 65
NLAG = 64
NOUT = 5
# output normalisation: target = (value - OFFSET) / SCALE
OFFSET = np.array([0.45, 0.0, np.log(4.0), np.log(0.15), np.log(10.0)])
SCALE = np.array([0.3, 1.0, 1.0, 1.0, 1.5])


def feature_lags(L):
    """The 64 log-spaced (real-valued) lags the features sample."""
    return np.exp(np.linspace(0.0, np.log(L - 1), NLAG))


def features(D, q, L):
    """D [n, L] (all lags 0..L-1), q [n] -> features [n, 65] (FP32)."""
    D = np.asarray(D, np.float64)
    t = feature_lags(L)
    i0 = np.floor(t).astype(int)
    i1 = np.minimum(i0 + 1, L - 1)
    f = t - i0
    s = D[:, i0] * (1 - f) + D[:, i1] * f
    m = s.max(1, keepdims=True)
    m[~(m > 0)] = 1.0
    return np.concatenate([s / m, (np.log(np.asarray(q, np.float64)) / 4.0)[:, None]], 1).astype(np.float32)


def features_from_samples(s, q):
    """Model/measured values already at feature_lags(L): s [n, 64]."""
    s = np.asarray(s, np.float64)
    m = s.max(1, keepdims=True)
    m[~(m > 0)] = 1.0
    return np.concatenate([s / m, (np.log(np.asarray(q, np.float64)) / 4.0)[:, None]], 1).astype(np.float32)


def encode(alpha, vbar, Z, D, tau_e):
    raw = np.stack([alpha, np.log(vbar), np.log(Z), np.log(D), np.log(tau_e)], 1)
    return ((raw - OFFSET) / SCALE).astype(np.float32)


def decode(y):
    raw = np.asarray(y, np.float64) * SCALE + OFFSET
    return dict(alpha=raw[:, 0], vbar=np.exp(raw[:, 1]), Z=np.exp(raw[:, 2]), D=np.exp(raw[:, 3]),
                tau_e=np.exp(raw[:, 4]))


class Surrogate:
    """One MLP on the current CUDA device (tensor-core forward/backward)."""

    def __init__(self, batch_max=8192, seed=0):
        self._lib = _lib.load()
        h = C.c_void_p()
        rc = self._lib.ddm_mlp_create(int(batch_max), int(seed), C.byref(h))
        if rc:
            from .engine import DdmArgError, DdmError
            msg = self._lib.ddm_mlp_last_error(None).decode()
            raise (DdmArgError if rc == _lib.DDM_ERR_ARG else DdmError)(rc, msg)
        self._h = h
        self.batch_max = batch_max
        self.nparams = self._lib.ddm_mlp_param_count()

    def _check(self, rc):
        if rc:
            from .engine import DdmArgError, DdmError
            msg = self._lib.ddm_mlp_last_error(self._h).decode()
            raise (DdmArgError if rc == _lib.DDM_ERR_ARG else DdmError)(rc, msg)

    def close(self):
        if self._h:
            self._lib.ddm_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        p = np.zeros(self.nparams, np.float32)
        self._check(self._lib.ddm_mlp_get_params(self._h, C.c_void_p(p.ctypes.data)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams
        self._check(self._lib.ddm_mlp_set_params(self._h, C.c_void_p(p.ctypes.data)))

    @staticmethod
    def _stream(stream):
        """The caller's stream, default torch's current one (ordered with torch work)."""
        import torch
        s = torch.cuda.current_stream().cuda_stream if stream is None else stream
        return C.c_void_p(s) if s else None

    def forward(self, x, out=None, stream=None):
        """x: torch CUDA tensor [n, 65] FP32 -> [n, 5] FP32 (device), queued
        on `stream` (default torch's current stream)."""
        import torch
        n = x.shape[0]
        if out is None:
            out = torch.empty((n, NOUT), dtype=torch.float32, device=x.device)
        self._check(self._lib.ddm_mlp_forward(self._h, C.c_void_p(x.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                              self._stream(stream)))
        return out

    def predict(self, feats, chunk=None):
        """Host features [n, 65] -> host outputs [n, 5] (pads n to a multiple of 8)."""
        import torch
        n = feats.shape[0]
        chunk = chunk or self.batch_max
        out = np.zeros((n, NOUT), np.float32)
        for a in range(0, n, chunk):
            b = min(n, a + chunk)
            m = (b - a + 7) // 8 * 8
            xt = torch.zeros((m, NFEAT), dtype=torch.float32, device="cuda")
            xt[: b - a] = torch.from_numpy(np.ascontiguousarray(feats[a:b], np.float32)).cuda()
            out[a:b] = self.forward(xt)[: b - a].cpu().numpy()
        self.sync()
        return out

    def gradients(self, x, y, stream=None):
        g = np.zeros(self.nparams, np.float32)
        loss = C.c_float()
        self._check(self._lib.ddm_mlp_gradients(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                                x.shape[0], C.c_void_p(g.ctypes.data), C.byref(loss),
                                                self._stream(stream)))
        return loss.value, g

    def train_step(self, x, y, lr, want_loss=False, stream=None):
        loss = C.c_float()
        self._check(self._lib.ddm_mlp_train_step(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                                 x.shape[0], float(lr), C.byref(loss) if want_loss else None,
                                                 self._stream(stream)))
        return loss.value if want_loss else None

    def sync(self, stream=None):
        self._check(self._lib.ddm_mlp_sync(self._h, self._stream(stream)))
