"""analyzeMotility (motility-ddm/src/motility_fit.js:853-990) on a Radial
record: the reference's fits, drift, statistics and gates -> verdict
(C ABI ddm_analyze_motility, host FP64 like the reference's fit worker)."""
import ctypes as C

import numpy as np

from . import _lib

VERDICTS = ["MOTILE", "NOT_MOTILE", "DIRECTED_TRANSPORT", "NO_DYNAMICS", "UNLOCKED_EXPOSURE"]


def analyze_motility(radial, dxUm=1.0, fps=1.0, geometry="3d", exposureLocked=True, swimMin=2.0):
    """analyzeMotility(radial, {dxUm, fps, geometry, exposureLocked}) -> dict
    with the reference's result fields; verdicts as strings."""
    lib = _lib.load()
    keep = [np.ascontiguousarray(radial.kCenter, np.float64), np.ascontiguousarray(radial.kNodes, np.float64),
            np.ascontiguousarray(radial.nModes, np.uint32), np.ascontiguousarray(radial.D, np.float64),
            np.ascontiguousarray(radial.P, np.float64), np.ascontiguousarray(radial.drift, np.float64)]
    kn = len(keep[1]) // radial.NB if len(keep[1]) else 0
    r = _lib.RadialView(radial.N, radial.NB, radial.L, kn, *[C.c_void_p(a.ctypes.data) for a in keep])
    o = _lib.MotilityOptions(float(dxUm), float(fps), 1 if geometry == "2d" else 0, 1 if exposureLocked else 0,
                             float(swimMin))
    res = _lib.MotilityResult()
    rc = lib.ddm_analyze_motility(C.byref(r), C.byref(o), C.byref(res))
    if rc:
        from .engine import DdmArgError
        raise DdmArgError(rc, "analyze_motility: invalid Radial record or options")
    out = {k: getattr(res, k) for k, _ in _lib.MotilityResult._fields_ if k not in ("swim", "brown")}
    out["verdict"] = VERDICTS[res.verdict]
    out["physicsVerdict"] = VERDICTS[res.physicsVerdict]
    out["swim"] = {k: getattr(res.swim, k) for k, _ in _lib.MotilityFit._fields_}
    out["brown"] = {k: getattr(res.brown, k) for k, _ in _lib.MotilityFit._fields_}
    return out
