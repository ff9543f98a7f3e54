"""Live ring-buffer mode: the reference dashboard's frame clock and analysis
tick over this library's engine.

FrameClock restates motility-ddm/src/camera.ts:306-426: frame n (from its
capture time on a uniform fps grid) lives in ring slot n mod T; the mask of a
snapshot is built from the frame index actually stored in each slot, so
dropped, late, throttled and overwritten frames are excluded; the oldest
`guard` time indices are masked because new frames may overwrite their slots
while the analysis runs; shuffle = Control 1 (frame-order null test,
shuffleOrder ddm_ref.js:510-519).

LiveAnalyzer restates the camera loop of src/main.ts: on_frame is
onCameraFrame (:158-184: place the frame, ingest it, clock.drop it if the
engine refused it), and start/finish split analysisTick (:366-398): a
snapshot with the current guard starts a live computeTemporal on the engine's
analysis stream (ddm_compute_temporal_live) while frames keep arriving; when
it has finished, a result is discarded as stale if at least `guard` frames
arrived meanwhile (their slots may lie inside the snapshot), and the guard
widens to min(128, ceil(1.5 * elapsed) + 4); otherwise the radial record goes
to the fit (a FitWorker, or analyze_motility on this thread).
"""
import math
from dataclasses import dataclass

import numpy as np

MIN_FRAMES_FRACTION = 0.75   # main.ts:32: 192 of the 256-slot ring
GUARD_DEFAULT = 32           # main.ts:49
GUARD_MAX = 128              # main.ts:386


def shuffle_order(order, mask, rand):
    """shuffleOrder (ddm_ref.js:510-519): Fisher-Yates over (order, mask)
    pairs with rand() in [0, 1)."""
    order = np.array(order, np.uint32)
    mask = np.array(mask, np.float32)
    for i in range(len(order) - 1, 0, -1):
        j = int(math.floor(rand() * (i + 1)))
        order[i], order[j] = order[j], order[i]
        mask[i], mask[j] = mask[j], mask[i]
    return order, mask


@dataclass
class Snapshot:
    order: np.ndarray   # uint32 [T]: slot of time index j
    mask: np.ndarray    # float32 [T]: 1 where time index j is used
    used: int           # valid frames in the snapshot
    newestN: int        # newest frame index at snapshot time


class FrameClock:
    """Uniform T-slot frame clock (camera.ts:306-426)."""

    def __init__(self, fps, T=256):
        self.T = int(T)
        self.dtMs = 1000.0 / fps
        self._t0 = None
        self._lastN = -1
        self._slotN = np.full(self.T, -1, np.int64)
        self._src = None
        self.frames = 0
        self.missed = 0
        self.duplicates = 0
        self.resets = 0
        self._lastTs = math.nan
        self._dts = []

    @property
    def timeSource(self):
        return self._src

    @property
    def newestN(self):
        return self._lastN

    def reset(self):
        self._t0 = None
        self._lastN = -1
        self._slotN.fill(-1)
        self._src = None
        self._lastTs = math.nan
        self.resets += 1

    def place(self, tMs, source="captureTime"):
        """Slot for a frame captured at tMs, or None for a duplicate;
        switching to or from 'mediaTime' restarts the clock, and so does a
        gap of more than T frames."""
        if self._src is not None and (source == "mediaTime") != (self._src == "mediaTime"):
            self.reset()
        self._src = source
        if self._t0 is None:
            self._t0 = tMs
        n = _js_round((tMs - self._t0) / self.dtMs)
        if n <= self._lastN:
            self.duplicates += 1
            return None
        if self._lastN >= 0 and n - self._lastN > self.T:
            self.reset()
            self._src = source
            self._t0 = tMs
            n = 0
        if self._lastN >= 0:
            self.missed += n - self._lastN - 1
        if math.isfinite(self._lastTs):
            self._dts.append(tMs - self._lastTs)
            if len(self._dts) > 120:
                self._dts.pop(0)
        self._lastTs = tMs
        slot = n % self.T
        self._slotN[slot] = n
        self._lastN = n
        self.frames += 1
        return dict(slot=slot, n=n)

    def drop(self, n):
        """Frame n was not ingested (e.g. refused under back-pressure)."""
        slot = n % self.T
        if self._slotN[slot] == n:
            self._slotN[slot] = -1

    @property
    def medianDtMs(self):
        if not self._dts:
            return math.nan
        s = sorted(self._dts)
        return s[len(s) >> 1]

    @property
    def validCount(self):
        c = 0
        for j in range(self.T):
            n = self._lastN - self.T + 1 + j
            if n >= 0 and self._slotN[n % self.T] == n:
                c += 1
        return c

    def snapshot(self, guard=0, shuffle=False, rand=None):
        """Time-ordered (order, mask) for the temporal pass; the oldest
        `guard` time indices are masked."""
        T = self.T
        order = np.empty(T, np.uint32)
        mask = np.zeros(T, np.float32)
        used = 0
        for j in range(T):
            n = self._lastN - T + 1 + j
            slot = ((n % T) + T) % T
            order[j] = slot
            ok = n >= 0 and j >= guard and self._slotN[slot] == n
            if ok:
                mask[j] = 1.0
                used += 1
        if shuffle:
            order, mask = shuffle_order(order, mask, rand or np.random.random)
        return Snapshot(order, mask, used, self._lastN)


def _js_round(x):
    """Math.round: halves toward +infinity."""
    return int(math.floor(x + 0.5))


class LiveAnalyzer:
    """The dashboard's camera loop over a DdmEngine (main.ts:158-184,
    366-398). mode "camera" applies the guard and the stale test; "demo"
    (recorded movies, main.ts:376) uses guard 0."""

    def __init__(self, engine, clock, opt=None, worker=None, mode="camera", guard=GUARD_DEFAULT,
                 shuffle=False, rand=None, min_frames=None):
        self.engine = engine
        self.clock = clock
        self.opt = dict(opt or {})
        self.worker = worker
        self.mode = mode
        self.guard = guard
        self.shuffle = shuffle
        self.rand = rand
        self.min_frames = min_frames if min_frames is not None else int(round(MIN_FRAMES_FRACTION * clock.T))
        self.stale = 0
        self.throttled = 0
        self.last = None
        self._snap = None

    def on_frame(self, frame, tMs, source="captureTime", scale=None):
        """onCameraFrame: place the frame on the clock and ingest it; a frame
        the engine refuses under back-pressure is dropped from the clock."""
        placed = self.clock.place(tMs, source)
        if placed is None:
            return None
        ok = False
        try:
            if self.engine.saturated:  # ingestFrame's back-pressure (ddm-engine.ts:258-266)
                self.throttled += 1
            else:
                self.engine.ingest_frames(np.asarray(frame)[None], [placed["slot"]], scale)
                ok = True
        finally:
            if not ok:
                self.clock.drop(placed["n"])
        return placed

    @property
    def busy(self):
        return self._snap is not None

    def start(self):
        """First half of analysisTick: 'collecting' until min_frames valid
        frames; else snapshot and start the live analysis ('started')."""
        if self._snap is not None:
            return "busy"
        valid = self.clock.validCount
        if valid < self.min_frames:
            return "collecting"
        guard = 0 if self.mode == "demo" else self.guard
        snap = self.clock.snapshot(guard=guard, shuffle=self.shuffle, rand=self.rand)
        self.engine.compute_temporal(snap.order, snap.mask, live=True)
        self._snap = (snap, guard)
        return "started"

    def finish(self, block=True):
        """Second half: None while the analysis runs (block=False); then a
        dict with status 'stale' (result discarded, guard widened) or 'ok'
        (radial, fit result or its Future when a worker is used)."""
        if self._snap is None:
            return None
        if not block and not self.engine.analysis_done:
            return None
        snap, guard = self._snap
        radial = self.engine.read_radial()
        self._snap = None
        elapsed = self.clock.newestN - snap.newestN
        if self.mode == "camera" and elapsed >= guard:
            self.stale += 1
            self.guard = min(GUARD_MAX, int(math.ceil(elapsed * 1.5)) + 4)
            return dict(status="stale", elapsed=elapsed, guard=self.guard, used=snap.used)
        if self.worker is not None:
            result = self.worker.run_fit(radial, self.opt)
        else:
            from .motility import analyze_motility
            result = analyze_motility(radial, **self.opt)
        self.last = dict(status="ok", radial=radial, result=result, used=snap.used, elapsed=elapsed, snapshot=snap)
        return self.last

    def tick(self):
        """start + finish (blocking): one whole analysis tick."""
        st = self.start()
        if st != "started":
            return dict(status=st)
        return self.finish(block=True)
