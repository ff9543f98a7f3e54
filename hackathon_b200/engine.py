"""DdmEngine: the reference's engine API (motility-ddm/src/ddm-engine.ts:62-426)
over the C ABI of the sm_100a library.

Same calls and data layouts as the TypeScript class, in Python naming:

    reference (TS)                         here
    DdmEngine.create(opts)                 DdmEngine.create(N=..., T=..., ...)
    ingestLuma(luma, slot) -> boolean      ingest_luma(luma, slot) -> bool
    ingestFrame(VideoFrame, slot)          ingest_frames(frames, slots, scale)
                                           (raw u8/u16/f32 pixels; the graphics
                                           import path has no equivalent here)
    computeTemporal(order, mask)           compute_temporal(order, mask, full=False)
    readRadial() -> Radial                 read_radial() -> Radial
    readHistory()                          read_history()
    readTemporalFull() -> {D, C, P}        read_temporal_full()
    readMean()                             read_mean()
    idle(), destroy()                      idle(), destroy()
    saturated, pendingSubmits, throttled   saturated, pending_submits, throttled
    waitForCapacity()                      wait_for_capacity()
    bins                                   bins

Errors raise DdmError (the reference throws Error); argument errors are also
ValueError.
"""
import ctypes as C

import numpy as np

from . import _lib
from .radial import Radial

MAX_PENDING = 2  # ddm-engine.ts:46


class DdmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class DdmArgError(DdmError, ValueError):
    pass


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class DdmEngine:
    """One DDM analysis engine on the current CUDA device."""

    def __init__(self, handle, geometry):
        self._h = handle
        self._lib = _lib.load()
        self.geometry = geometry
        self.N, self.T, self.TPAD, self.L = geometry.N, geometry.T, geometry.TPAD, geometry.L
        self.NB = geometry.NB
        self.NH = self.N // 2 + 1
        self.modes = self.N * self.NH
        self.bins = self._read_bins()
        self._destroyed = False
        self._pending_host = []  # host buffers of asynchronous ingests still being copied

    # ------------------------------------------------------------ lifetime
    @classmethod
    def create(cls, N=256, T=256, TPAD=0, L=128, NB=32, kmin=4.0, kmax=100.0, knodes=4):
        """DdmEngine.create (ddm-engine.ts:125-149). Defaults are the
        reference's frozen geometry (ddm_ref.js:18-31)."""
        lib = _lib.load()
        g = _lib.Geometry(N, T, TPAD, L, NB, float(kmin), float(kmax), knodes, 0)
        h = C.c_void_p()
        rc = lib.ddm_create(C.byref(g), C.byref(h))
        if rc != _lib.DDM_OK:
            msg = lib.ddm_create_error().decode()
            raise (DdmArgError if rc == _lib.DDM_ERR_ARG else DdmError)(rc, msg)
        out = _lib.Geometry()
        lib.ddm_get_geometry(h, C.byref(out))
        return cls(h, out)

    @classmethod
    def create_banded(cls, history_budget_bytes, N=256, T=256, TPAD=0, L=128, NB=32, kmin=4.0, kmax=100.0,
                      knodes=4):
        """An engine for videos whose history does not fit the device at once
        (ddm_create_banded): it holds a band of spectrum columns sized to
        history_budget_bytes and analyses a whole video with analyze_banded."""
        lib = _lib.load()
        g = _lib.Geometry(N, T, TPAD, L, NB, float(kmin), float(kmax), knodes, 0)
        h = C.c_void_p()
        rc = lib.ddm_create_banded(C.byref(g), int(history_budget_bytes), C.byref(h))
        if rc != _lib.DDM_OK:
            msg = lib.ddm_create_error().decode()
            raise (DdmArgError if rc == _lib.DDM_ERR_ARG else DdmError)(rc, msg)
        out = _lib.Geometry()
        lib.ddm_get_geometry(h, C.byref(out))
        return cls(h, out)

    @property
    def bands(self):
        """(number of bands, spectrum columns per band) -- (1, N/2+1) for an
        ordinary engine."""
        self._alive()
        nb, bc = C.c_int32(), C.c_int32()
        self._check(self._lib.ddm_get_bands(self._h, C.byref(nb), C.byref(bc)))
        return nb.value, bc.value

    def analyze_banded(self, frames, slots, order, mask, scale=None):
        """The whole analysis of one video on a banded engine
        (ddm_analyze_banded): per band the spatial pass of every frame (host
        frames stream through pinned staging once per band), then the band's
        temporal pass; read the record with read_radial()."""
        self._alive()
        dt, n, dev_ptr, host_ptr, keep, slots = self._frames_arg(frames, slots)
        if scale is None:
            scale = {"u8": 1 / 255, "u16": 1 / 65535, "f32": 1.0}[dt]
        o = np.ascontiguousarray(order, dtype=np.uint32).reshape(-1)
        m = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1)
        if o.size != self.T or m.size != self.T:
            raise DdmArgError(_lib.DDM_ERR_ARG, f"temporalMeta: order/mask must have length {self.T}")
        ptr = dev_ptr if dev_ptr is not None else host_ptr
        rc = self._lib.ddm_analyze_banded(self._h, C.c_void_p(ptr), _lib.DTYPES[dt], n, _ptr(slots), float(scale),
                                          _ptr(o), _ptr(m), 1 if dev_ptr is not None else 0)
        del keep
        self._check(rc)

    def destroy(self):
        """DdmEngine.destroy (ddm-engine.ts:421-425)."""
        if not self._destroyed:
            self._destroyed = True
            self._lib.ddm_destroy(self._h)  # waits for the copies in flight
            self._pending_host.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _check(self, rc):
        if rc != _lib.DDM_OK:
            msg = self._lib.ddm_last_error(self._h).decode()
            raise (DdmArgError if rc == _lib.DDM_ERR_ARG else DdmError)(rc, msg)

    def _alive(self):
        if self._destroyed:
            raise DdmError(_lib.DDM_ERR_STATE, "engine destroyed")

    def _read_bins(self):
        n = self._lib.ddm_bins_count(self._h)
        NB, K = self.geometry.NB, self.geometry.knodes
        off = np.empty(NB + 1, np.uint32)
        modes = np.empty((max(n, 1), 4), np.int32)
        kc = np.empty(NB)
        nm = np.empty(NB, np.uint32)
        kn = np.empty(NB * K)
        self._check(self._lib.ddm_get_bins(self._h, _ptr(off), _ptr(modes), _ptr(kc), _ptr(nm), _ptr(kn)))
        return dict(N=self.N, NB=NB, kmin=self.geometry.kmin, kmax=self.geometry.kmax, knodes=K,
                    binOffsets=off, binModes=modes[:n], kCenter=kc, nModes=nm, kNodes=kn)

    # ------------------------------------------------------------ ingest
    @property
    def pending_submits(self):
        return self._lib.ddm_pending(self._h)

    @property
    def saturated(self):
        return self.pending_submits > MAX_PENDING

    @property
    def throttled(self):
        return self._lib.ddm_throttled(self._h)

    def wait_for_capacity(self):
        self._check(self._lib.ddm_wait_for_capacity(self._h))

    def ingest_luma(self, luma, slot):
        """ingestLuma (ddm-engine.ts:308-324): N*N float luma, row-major.
        Returns False if the frame was dropped because the queue is saturated."""
        self._alive()
        a = np.ascontiguousarray(luma, dtype=np.float32).reshape(-1)
        if a.size != self.N * self.N:
            raise DdmArgError(_lib.DDM_ERR_ARG, f"ingestLuma expects {self.N * self.N} values")
        ok = C.c_int32(0)
        self._check(self._lib.ddm_ingest_luma(self._h, _ptr(a), int(slot), C.byref(ok)))
        return bool(ok.value)

    def _frames_arg(self, frames, slots):
        """(dtype name, n, device pointer or None, host pointer or None, the
        object keeping the data alive, slots) of a frames argument: numpy, or
        a torch CPU/CUDA tensor, [n, N, N] u8 / u16 / f32."""
        slots = np.ascontiguousarray(slots, dtype=np.int32).reshape(-1)
        dev_ptr = host_ptr = keep = None
        try:
            import torch
            if isinstance(frames, torch.Tensor):
                if not frames.is_contiguous():
                    frames = frames.contiguous()
                dt = {torch.uint8: "u8", torch.int16: "u16", torch.uint16: "u16",
                      torch.float32: "f32"}.get(frames.dtype)
                if dt is None:
                    raise DdmArgError(_lib.DDM_ERR_ARG, f"unsupported frame dtype {frames.dtype}")
                n = frames.shape[0] if frames.dim() == 3 else 1
                if frames.numel() != n * self.N * self.N:
                    raise DdmArgError(_lib.DDM_ERR_ARG, f"frames must be [n, {self.N}, {self.N}]")
                if frames.is_cuda:
                    dev_ptr = frames.data_ptr()
                else:
                    host_ptr = frames.data_ptr()
                keep = frames
        except ImportError:
            pass
        if keep is None:
            arr = np.ascontiguousarray(frames)
            dt = {np.dtype(np.uint8): "u8", np.dtype(np.uint16): "u16",
                  np.dtype(np.float32): "f32"}.get(arr.dtype)
            if dt is None:
                raise DdmArgError(_lib.DDM_ERR_ARG, f"unsupported frame dtype {arr.dtype}")
            n = arr.shape[0] if arr.ndim == 3 else 1
            if arr.size != n * self.N * self.N:
                raise DdmArgError(_lib.DDM_ERR_ARG, f"frames must be [n, {self.N}, {self.N}]")
            host_ptr = arr.ctypes.data
            keep = arr
        if slots.size != n:
            raise DdmArgError(_lib.DDM_ERR_ARG, f"{n} frames but {slots.size} slots")
        return dt, n, dev_ptr, host_ptr, keep, slots

    def ingest_frames(self, frames, slots, scale=None, wait=True):
        """Raw frames [n, N, N] (numpy, or torch CPU/CUDA tensor) into ring slots
        `slots[i] % T`. luma = value * scale; scale defaults to 1/255 for u8
        (lumaOf, test/sim.mjs:189-193), 1/65535 for u16 and 1 for f32.
        wait=False (host frames): return once the copies are queued
        (ddm_ingest_frames_async); the engine keeps a reference to the host
        buffer until ingest_wait() -- do not change it before then."""
        self._alive()
        dt, n, dev_ptr, host_ptr, keep, slots = self._frames_arg(frames, slots)
        if scale is None:
            scale = {"u8": 1 / 255, "u16": 1 / 65535, "f32": 1.0}[dt]
        code = _lib.DTYPES[dt]
        if dev_ptr is not None:
            rc = self._lib.ddm_ingest_frames_device(self._h, C.c_void_p(dev_ptr), code, n, _ptr(slots),
                                                    float(scale))
        elif not wait:
            rc = self._lib.ddm_ingest_frames_async(self._h, C.c_void_p(host_ptr), code, n, _ptr(slots),
                                                   float(scale))
            self._pending_host.append(keep)
        else:
            rc = self._lib.ddm_ingest_frames(self._h, C.c_void_p(host_ptr), code, n, _ptr(slots),
                                             float(scale))
            self._pending_host.clear()  # the synchronous ingest waited for every earlier copy
        del keep
        self._check(rc)

    def ingest_wait(self):
        """Wait until every earlier ingest's frames are off the host buffers
        (ddm_ingest_wait)."""
        self._alive()
        self._check(self._lib.ddm_ingest_wait(self._h))
        self._pending_host.clear()

    def set_spatial_mask(self, mask):
        """Extension: N x N ROI mask (nonzero = used), or None."""
        self._alive()
        if mask is None:
            self._check(self._lib.ddm_set_spatial_mask(self._h, None))
            return
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        if m.size != self.N * self.N:
            raise DdmArgError(_lib.DDM_ERR_ARG, f"mask must have {self.N * self.N} values")
        self._check(self._lib.ddm_set_spatial_mask(self._h, _ptr(m)))

    # ------------------------------------------------------------ analysis
    def compute_temporal(self, order, mask, full=False, wait=True, live=False):
        """computeTemporal (ddm-engine.ts:331-365). order[j] = slot of time
        index j, mask[j] = 1 where time index j holds a valid frame.
        live=True: start the analysis on the engine's analysis stream and
        return; later ingests run concurrently (mask out the slots they
        overwrite: FrameClock.snapshot's guard). DdmError "computeTemporal
        is already running" while the previous live analysis is in flight."""
        self._alive()
        o = np.ascontiguousarray(order, dtype=np.uint32).reshape(-1)
        m = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1)
        if o.size != self.T or m.size != self.T:
            raise DdmArgError(_lib.DDM_ERR_ARG, f"temporalMeta: order/mask must have length {self.T}")
        if live:
            f = self._lib.ddm_compute_temporal_live
        else:
            f = self._lib.ddm_compute_temporal if wait else self._lib.ddm_compute_temporal_async
        self._check(f(self._h, _ptr(o), _ptr(m), 1 if full else 0))

    @property
    def analysis_done(self):
        """True once no live analysis is in flight."""
        self._alive()
        d = C.c_int32(1)
        self._check(self._lib.ddm_analysis_poll(self._h, C.byref(d)))
        return bool(d.value)

    def wait_analysis(self):
        """Waits for the live analysis in flight, if any."""
        self._alive()
        self._check(self._lib.ddm_wait_analysis(self._h))

    def autotune(self):
        """Times chunk and unit-size candidates on this device and keeps the
        fastest (ddm_autotune; overwrites the history: call before ingest).
        Returns the timing report."""
        import json
        self._alive()
        buf = C.create_string_buffer(4096)
        self._check(self._lib.ddm_autotune(self._h, buf, 4096))
        return json.loads(buf.value.decode())

    def set_tuning(self, chunk=0, unit_size=0, variant=-1):
        self._alive()
        self._check(self._lib.ddm_set_tuning(self._h, int(chunk), int(unit_size), int(variant)))

    def set_sparse(self, enable=True):
        """Sparse-mask temporal kernel for masks with at most 64 zeros
        (ddm_set_sparse); False keeps the transform path for every mask."""
        self._alive()
        self._check(self._lib.ddm_set_sparse(self._h, 1 if enable else 0))

    def set_blocked(self, enable=True):
        """Extension: the blocked temporal kernel for L <= 128 at TPAD 8192
        (ddm_set_blocked); False keeps the TPAD 8192 transform kernels."""
        self._alive()
        self._check(self._lib.ddm_set_blocked(self._h, 1 if enable else 0))

    TEMPORAL_KERNELS = {0: "temporal_kernel", 1: "temporal16_kernel", 2: "temporal_sparse_kernel",
                        3: "temporal_big_kernel", 4: "temporal_sparse_big_kernel", 5: "temporal_blocked_kernel"}

    @property
    def last_temporal_kernel(self):
        """Name of the temporal kernel the last computeTemporal ran (None
        before the first one)."""
        self._alive()
        return self.TEMPORAL_KERNELS.get(self._lib.ddm_last_temporal_kernel(self._h))

    @property
    def tuning(self):
        c, u, v = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self._lib.ddm_get_tuning(self._h, C.byref(c), C.byref(u), C.byref(v)))
        return dict(chunk=c.value, unit_size=u.value, variant=v.value)

    def read_radial(self, out=None):
        """readRadial (ddm-engine.ts:391-395) -> Radial (ddm_ref.js:336-348).
        out: optional (D, P, drift) float64 arrays of NB*L, NB and NB*L*8
        values that receive the record (the Radial returned uses them), e.g.
        pinned host memory reused across videos: the copy back then runs at
        the link's rate instead of through the driver's pageable path."""
        self._alive()
        NB, L = self.NB, self.L
        if out is None:
            D = np.empty(NB * L)
            P = np.empty(NB)
            drift = np.empty(NB * L * 8)
        else:
            D, P, drift = out
            for a, n in ((D, NB * L), (P, NB), (drift, NB * L * 8)):
                if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.size == n
                        and a.flags.c_contiguous and a.flags.writeable):
                    raise DdmArgError(_lib.DDM_ERR_ARG, f"read_radial out: need writable contiguous float64 "
                                                        f"arrays of {NB * L}, {NB}, {NB * L * 8} values")
        self._check(self._lib.ddm_read_radial(self._h, _ptr(D), _ptr(P), _ptr(drift)))
        b = self.bins
        return Radial(N=self.N, NB=NB, L=L, kCenter=b["kCenter"].copy(), kNodes=b["kNodes"].copy(),
                      nModes=b["nModes"].copy(), D=D, P=P, drift=drift, knodes=b["knodes"])

    def read_history(self):
        """readHistory (ddm-engine.ts:398-400): complex64 [modes, T]."""
        self._alive()
        out = np.empty((self.modes, self.T), np.complex64)
        self._check(self._lib.ddm_read_history(self._h, _ptr(out)))
        return out

    def read_temporal_full(self):
        """readTemporalFull (ddm-engine.ts:403-408): D [modes, L] f32,
        C [modes, L] complex64, P [modes] f32."""
        self._alive()
        D = np.empty((self.modes, self.L), np.float32)
        Cm = np.empty((self.modes, self.L), np.complex64)
        P = np.empty(self.modes, np.float32)
        self._check(self._lib.ddm_read_temporal_full(self._h, _ptr(D), _ptr(Cm), _ptr(P)))
        return dict(D=D, C=Cm, P=P)

    def read_mean(self):
        """readMean (ddm-engine.ts:411-414)."""
        self._alive()
        v = C.c_double()
        self._check(self._lib.ddm_read_mean(self._h, C.byref(v)))
        return v.value

    def idle(self):
        """idle (ddm-engine.ts:417-419)."""
        self._check(self._lib.ddm_idle(self._h))
        self._pending_host.clear()

    # ------------------------------------------------------------ plumbing
    def set_stream(self, stream_ptr):
        """Queue the engine's work on a caller's CUDA stream (int handle) or
        back on its own stream (None)."""
        self._check(self._lib.ddm_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    @property
    def kernel_launches(self):
        return self._lib.ddm_kernel_launches(self._h)
