"""The fit-worker protocol of the reference's dashboard, served by this
library.

Reference: motility-ddm/src/motility_fit.js:996-1004 (the Worker entry:
message {id, radial, opt} -> reply {id, result} or {id, error: stack}) and its
caller src/main.ts:325-353 (runFit: one waiter per id; if the worker fails,
every pending fit and every later one runs on the calling thread).

Here the worker is a thread that runs the library's decision layer
(ddm_analyze_motility: the reference's analyzeMotility with its model fits on
the GPU): the ctypes call releases the GIL, so a fit overlaps the caller's
ingest and temporal launches the way the reference's Worker keeps fits off
the frame-delivery thread. Replies keep the reference's shape; results are
the dicts hackathon_b200.motility.analyze_motility returns. The analysis
function can be replaced (FitWorker(analyze=...)), e.g. to serve the
protocol where no GPU is present.

Extension: opt["binFits"] = "plain" | "seeded" adds per-q-bin fits from the
batched GPU LM (ddm_fit_lm, one warp per bin) to the reply's result as
result["binFits"]: "plain" uses the reference's start strategy, "seeded" the
surrogate network's prediction (a trained Surrogate given to the worker) with
the plain strategy as fallback -- the GPU path answering the same message.
The surrogate was trained on the 512-lag grid in pixel/frame units, so
"seeded" needs radial.L == 512; other records are fitted "plain" (the reply
says which mode ran).
"""
import itertools
import math
import queue
import threading
import traceback
from concurrent.futures import Future

import numpy as np

from . import fit as F
from .motility import analyze_motility

_OPT_KEYS = ("dxUm", "fps", "geometry", "exposureLocked", "swimMin")


class WorkerFailed(RuntimeError):
    """The worker thread stopped; fits run on the calling thread."""


def handle(radial, opt, surrogate=None, analyze=None):
    """One request: analyzeMotility(radial, opt) (+ binFits when asked)."""
    opt = dict(opt or {})
    kw = {k: opt[k] for k in _OPT_KEYS if k in opt}
    result = (analyze or analyze_motility)(radial, **kw)
    mode = opt.get("binFits")
    if mode:
        result["binFits"] = bin_fits(radial, opt, mode, surrogate)
    return result


def _seeds(radial, pr, bnds, dxUm, fps, surrogate):
    """Surrogate starts (alpha, vbar, Z, D) in the fit's units for the
    prepared bins, clipped into the bounds."""
    import torch

    from . import surrogate as S
    from . import surrogate_train as ST
    L = radial.L
    D = np.asarray(radial.D, np.float64).reshape(radial.NB, L)[pr.bins]
    q_px = 2 * math.pi * np.asarray(radial.kCenter, np.float64)[pr.bins] / radial.N
    x = torch.from_numpy(S.features(D, q_px, L)).cuda()
    px = ST.predict_starts(surrogate, x, np.array([1e-9, 1e9, 0.5, 100.0, 1e-12, 1e12], np.float32))
    px = px.cpu().numpy().astype(np.float64)
    # pixel/frame -> the fit's units: v [um/s] = v_px dxUm fps, D [um^2/s] = D_px dxUm^2 fps
    st = np.stack([px[:, 0], px[:, 1] * dxUm * fps, px[:, 2], px[:, 3] * dxUm * dxUm * fps], 1)
    lo = np.array([0.02, bnds[0], bnds[2], bnds[4]])
    hi = np.array([0.98, bnds[1], bnds[3], bnds[5]])
    return np.clip(st, lo, hi)


def bin_fits(radial, opt, mode, surrogate=None):
    """Per-q-bin fits of one Radial by the batched GPU LM."""
    from .surrogate_train import L_LAGS
    dxUm, fps = float(opt.get("dxUm", 1.0)), float(opt.get("fps", 1.0))
    if mode not in ("plain", "seeded"):
        raise ValueError(f"binFits: unknown mode {mode!r} (plain | seeded)")
    ran = mode
    if mode == "seeded" and (surrogate is None or radial.L != L_LAGS):
        ran = "plain"
    pr = F.prepare(radial, dxUm, fps)
    if len(pr.bins) == 0:
        return dict(mode=ran, bins=[], alpha=[], vbar=[], Z=[], D=[], cost=[], iters=[], fellBack=[])
    b = F.bounds(pr, float(opt.get("swimMin", F.SWIM_MIN_UM_S)))
    if ran == "seeded":
        res = F.fit_lm(pr.d, pr.tau, pr.qn, pr.w, b, mode="seeded_fallback",
                       start=_seeds(radial, pr, b, dxUm, fps, surrogate))
    else:
        res = F.fit_lm(pr.d, pr.tau, pr.qn, pr.w, b, mode="plain")
    return dict(mode=ran, bins=pr.bins.tolist(), alpha=res.alpha.tolist(), vbar=res.vbar.tolist(),
                Z=res.Z.tolist(), D=res.D.tolist(), cost=res.cost.tolist(), iters=res.iters.tolist(),
                fellBack=((res.status >> 1) & 1).astype(bool).tolist())


class FitWorker:
    """A worker thread speaking the reference's fit protocol.

    post_message({id, radial, opt}) queues a request; replies go to
    `on_message(reply)` (the worker.onmessage of main.ts). run_fit(radial, opt)
    is main.ts runFit: it returns a Future of the result dict; an {error}
    reply becomes the Future's exception."""

    def __init__(self, on_message=None, surrogate=None, analyze=None):
        self._q = queue.Queue()
        self._on_message = on_message
        self._surrogate = surrogate
        self._analyze = analyze
        self._waiters = {}
        self._lock = threading.Lock()
        self._ids = itertools.count(1)
        self.failed = False
        self._t = threading.Thread(target=self._loop, name="ddm-fit-worker", daemon=True)
        self._t.start()

    # ------------------------------------------------------------ protocol
    def post_message(self, msg):
        """worker.postMessage({id, radial, opt})."""
        if self.failed:
            raise WorkerFailed("fit worker failed")
        self._q.put(msg)

    def _reply(self, rep):
        with self._lock:
            fut = self._waiters.pop(rep.get("id"), None)
        if fut is not None:
            if "result" in rep:
                fut.set_result(rep["result"])
            else:
                fut.set_exception(RuntimeError(rep["error"]))
        elif self._on_message is not None:
            self._on_message(rep)

    def _serve(self, msg):
        rid = msg.get("id") if isinstance(msg, dict) else None
        try:
            result = handle(msg["radial"], msg.get("opt"), self._surrogate, self._analyze)
        except Exception as e:  # the reference posts String(e.stack || e)
            self._reply({"id": rid, "error": "".join(traceback.format_exception(e)).rstrip()})
            return
        self._reply({"id": rid, "result": result})

    def _loop(self):
        try:
            while True:
                msg = self._q.get()
                if msg is None:
                    return
                self._serve(msg)
        except BaseException:  # the worker itself broke (main.ts worker.onerror)
            self._fail()

    def _fail(self):
        self.failed = True
        with self._lock:
            pending, self._waiters = self._waiters, {}
        for fut in pending.values():
            fut.set_exception(WorkerFailed("worker failed"))

    # ------------------------------------------------------------ runFit
    def run_fit(self, radial, opt=None):
        """Future of analyzeMotility(radial, opt) computed by the worker; once
        the worker has failed, computed here (main.ts:346-353)."""
        fut = Future()
        if self.failed:
            fut.set_result(handle(radial, opt, self._surrogate, self._analyze))
            return fut
        rid = next(self._ids)
        with self._lock:
            self._waiters[rid] = fut
        self._q.put({"id": rid, "radial": radial, "opt": opt})
        return fut

    def fit(self, radial, opt=None, timeout=None):
        """Blocking run_fit, falling back to this thread if the worker failed
        while the request was pending ('worker failed' replies, main.ts:349)."""
        try:
            return self.run_fit(radial, opt).result(timeout)
        except WorkerFailed:
            return handle(radial, opt, self._surrogate, self._analyze)

    def close(self):
        self._q.put(None)
        self._t.join(timeout=30)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
