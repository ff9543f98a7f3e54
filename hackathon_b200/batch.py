"""Batches of videos of uneven size and frame count (C ABI ddm_batch_*).

A batch borrows engines (hackathon_b200.DdmEngine, any geometries on one
device): every video's spatial chunks go to the batch stream without host
synchronisation, the temporal analysis of all videos is ONE persistent
launch over all their work units (at the batch's largest TPAD, exact for
every lag < L), the whole step can be captured into a CUDA graph and
replayed, and all q-bins of all videos are fitted by one batched LM launch
(``fit_all``)."""
import ctypes as C

import numpy as np

from . import _lib
from . import fit as F


def _arr(ptrs, ctype=C.c_void_p):
    return (ctype * len(ptrs))(*ptrs)


class DdmBatch:
    def __init__(self, engines):
        self._lib = _lib.load()
        self.engines = list(engines)
        hs = _arr([e._h.value if isinstance(e._h, C.c_void_p) else e._h for e in self.engines])
        b = C.c_void_p()
        rc = self._lib.ddm_batch_create(hs, len(self.engines), C.byref(b))
        if rc:
            self._raise(rc, self._lib.ddm_batch_last_error(None))
        self._b = b

    def _raise(self, rc, msg):
        from .engine import DdmArgError, DdmError
        raise (DdmArgError if rc == _lib.DDM_ERR_ARG else DdmError)(rc, msg.decode())

    def _check(self, rc):
        if rc:
            self._raise(rc, self._lib.ddm_batch_last_error(self._b))

    def destroy(self):
        if getattr(self, "_b", None):
            self._lib.ddm_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def set_stream(self, stream):
        self._check(self._lib.ddm_batch_set_stream(self._b, C.c_void_p(stream) if stream else None))

    def _ingest_args(self, frames, slots, scales):
        ptrs, dts, ns, sl = [], [], [], []
        self._keep = []
        for e, f, s in zip(self.engines, frames, slots):
            code = {"torch.uint8": 0, "torch.uint16": 1, "torch.int16": 1, "torch.float32": 2}.get(str(f.dtype))
            if code is None or not f.is_cuda or not f.is_contiguous():
                from .engine import DdmArgError
                raise DdmArgError(_lib.DDM_ERR_ARG, "batch frames: contiguous CUDA u8/u16/f32 tensors")
            ptrs.append(f.data_ptr())
            dts.append(code)
            ns.append(int(f.shape[0]))
            s = np.ascontiguousarray(s, np.int32)
            self._keep.append(s)
            sl.append(s.ctypes.data)
        sc = (C.c_float * len(scales))(*[float(x) for x in scales])
        return _arr(ptrs), (C.c_int32 * len(dts))(*dts), (C.c_int32 * len(ns))(*ns), _arr(sl), sc

    def ingest(self, frames, slots, scales):
        """frames: list of CUDA tensors [n_i, N_i, N_i] (u8/u16/f32)."""
        self._check(self._lib.ddm_batch_ingest(self._b, *self._ingest_args(frames, slots, scales)))

    def compute_temporal(self, orders, masks):
        o = [np.ascontiguousarray(x, np.uint32) for x in orders]
        m = [np.ascontiguousarray(x, np.float32) for x in masks]
        self._keep_meta = (o, m)
        self._check(self._lib.ddm_batch_compute_temporal(self._b, _arr([x.ctypes.data for x in o]),
                                                         _arr([x.ctypes.data for x in m])))

    def enqueue_temporal(self):
        self._check(self._lib.ddm_batch_enqueue_temporal(self._b))

    def sync(self):
        self._check(self._lib.ddm_batch_sync(self._b))

    def capture(self, frames, slots, scales):
        self._graph_frames = frames  # the graph reads these buffers at every replay
        self._check(self._lib.ddm_batch_capture(self._b, *self._ingest_args(frames, slots, scales)))

    def launch_graph(self):
        self._check(self._lib.ddm_batch_launch_graph(self._b))

    def read_radials(self):
        self.sync()
        return [e.read_radial() for e in self.engines]

    def fit_all(self, radials=None, dxUm=1.0, fps=1.0, swim_min=F.SWIM_MIN_UM_S, mode="plain", start=None, **kw):
        """All q-bins of all videos in one batched LM launch. Bounds per video
        (bounds() over that video's bins). Returns [(Prepared, FitResult
        slice)] per video."""
        radials = radials or self.read_radials()
        preps = [F.prepare(r, dxUm, fps) for r in radials]
        ntmax = max(len(p.lags) for p in preps)
        K = max(p.qn.shape[1] for p in preps)
        rows = sum(len(p.bins) for p in preps)
        d = np.zeros((rows, ntmax))
        tau = np.zeros((rows, ntmax))
        qn = np.zeros((rows, K))
        w = np.zeros(rows)
        b6 = np.zeros((rows, 6))
        nt = np.zeros(rows, np.int32)
        r = 0
        for p in preps:
            nb, n = len(p.bins), len(p.lags)
            d[r:r + nb, :n] = p.d
            tau[r:r + nb, :n] = p.tau
            qn[r:r + nb] = p.qn
            w[r:r + nb] = p.w
            b6[r:r + nb] = F.bounds(p, swim_min) if nb else 0
            nt[r:r + nb] = n
            r += nb
        res = F.fit_lm(d, tau, qn, w, b6, mode=mode, start=start, nt=nt, **kw)
        out, r = [], 0
        for p in preps:
            nb = len(p.bins)
            out.append((p, F.FitResult(res.theta[r:r + nb], res.cost[r:r + nb], res.iters[r:r + nb],
                                       res.evals[r:r + nb], res.status[r:r + nb])))
            r += nb
        return out
