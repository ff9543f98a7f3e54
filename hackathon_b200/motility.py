"""analyzeMotility (motility-ddm/src/motility_fit.js:870-990) on Radial
records: the fits, drift, statistics and gates -> verdict (C ABI
ddm_analyze_motility / ddm_analyze_motility_batch; the model fits run on the
GPU, csrc/gfit.cu, the rest on the host, csrc/analysis.cu)."""
import ctypes as C

import numpy as np

from . import _lib

VERDICTS = ["MOTILE", "NOT_MOTILE", "DIRECTED_TRANSPORT", "NO_DYNAMICS", "UNLOCKED_EXPOSURE"]


def _view(radial, keep):
    arrs = [np.ascontiguousarray(radial.kCenter, np.float64), np.ascontiguousarray(radial.kNodes, np.float64),
            np.ascontiguousarray(radial.nModes, np.uint32), np.ascontiguousarray(radial.D, np.float64),
            np.ascontiguousarray(radial.P, np.float64), np.ascontiguousarray(radial.drift, np.float64)]
    keep.extend(arrs)
    kn = len(arrs[1]) // radial.NB if len(arrs[1]) else 0
    return _lib.RadialView(radial.N, radial.NB, radial.L, kn, *[C.c_void_p(a.ctypes.data) for a in arrs])


OPTIMIZERS = {"reference": 0, "lm": 1}


def _opts(dxUm, fps, geometry, exposureLocked, swimMin, optimizer="reference"):
    if optimizer not in OPTIMIZERS:
        raise ValueError(f"optimizer must be one of {sorted(OPTIMIZERS)}, not {optimizer!r}")
    return _lib.MotilityOptions(float(dxUm), float(fps), 1 if geometry == "2d" else 0, 1 if exposureLocked else 0,
                                float(swimMin), OPTIMIZERS[optimizer], 0)


def _result(res):
    out = {k: getattr(res, k) for k, _ in _lib.MotilityResult._fields_ if k not in ("swim", "brown")}
    out["verdict"] = VERDICTS[res.verdict]
    out["physicsVerdict"] = VERDICTS[res.physicsVerdict]
    out["swim"] = {k: getattr(res.swim, k) for k, _ in _lib.MotilityFit._fields_}
    out["brown"] = {k: getattr(res.brown, k) for k, _ in _lib.MotilityFit._fields_}
    return out


def _raise(rc, what):
    from .engine import DdmArgError, DdmError
    msg = _lib.load().ddm_create_error().decode()
    if rc == _lib.DDM_ERR_ARG:
        raise DdmArgError(rc, f"{what}: {msg}")
    raise DdmError(rc, f"{what}: {msg}")


def analyze_motility(radial, dxUm=1.0, fps=1.0, geometry="3d", exposureLocked=True, swimMin=2.0,
                     optimizer="reference"):
    """analyzeMotility(radial, {dxUm, fps, geometry, exposureLocked}) -> dict
    with the reference's result fields; verdicts as strings. optimizer
    "reference": the reference's golden section and Nelder-Mead searches on
    the GPU objective; "lm": bounded Levenberg-Marquardt from the same starts
    (faster; on flat, non-identifiable surfaces it may end at a lower cost
    than the reference's search)."""
    lib = _lib.load()
    keep = []
    r = _view(radial, keep)
    o = _opts(dxUm, fps, geometry, exposureLocked, swimMin, optimizer)
    res = _lib.MotilityResult()
    rc = lib.ddm_analyze_motility(C.byref(r), C.byref(o), C.byref(res))
    if rc:
        _raise(rc, "analyze_motility")
    return _result(res)


def analyze_motility_batch(radials, dxUm=1.0, fps=1.0, geometry="3d", exposureLocked=True, swimMin=2.0,
                           optimizer="reference"):
    """analyze_motility of many records at once (one device launch per stage
    for all of them); per-record options may be given as sequences."""
    lib = _lib.load()
    n = len(radials)
    if n == 0:
        return []

    def per(v):
        return list(v) if isinstance(v, (list, tuple, np.ndarray)) else [v] * n
    dx, fp, geo, ex, sm = per(dxUm), per(fps), per(geometry), per(exposureLocked), per(swimMin)
    opt = per(optimizer)
    keep = []
    views = (_lib.RadialView * n)(*[_view(r, keep) for r in radials])
    opts = (_lib.MotilityOptions * n)(*[_opts(dx[i], fp[i], geo[i], ex[i], sm[i], opt[i]) for i in range(n)])
    res = (_lib.MotilityResult * n)()
    rc = lib.ddm_analyze_motility_batch(n, views, opts, res)
    if rc:
        _raise(rc, "analyze_motility_batch")
    return [_result(res[i]) for i in range(n)]


def prepared_bins(radial, dxUm=1.0, fps=1.0):
    """Radial bin indices the analysis fits (prepare), and the fit lag count."""
    lib = _lib.load()
    keep = []
    r = _view(radial, keep)
    o = _opts(dxUm, fps, "3d", True, 2.0)
    bins = np.zeros(radial.NB, np.int32)
    nb, nl = C.c_int32(), C.c_int32()
    rc = lib.ddm_prepared_bins(C.byref(r), C.byref(o), C.c_void_p(bins.ctypes.data), C.byref(nb), C.byref(nl))
    if rc:
        _raise(rc, "prepared_bins")
    return bins[:nb.value], nl.value


def temporal_structure_index(radial):
    """temporalStructureIndex (motility_fit.js:735-749) on the host."""
    keep = []
    return _lib.load().ddm_temporal_structure_index(C.byref(_view(radial, keep)))


def estimate_drift(radial, dxUm=1.0, fps=1.0, lag_mask=None):
    """estimateDrift (motility_fit.js:672-725) on the host; lag_mask
    [prepared bins, L] of 0/1 (lags to use), or None for every lag."""
    lib = _lib.load()
    keep = []
    r = _view(radial, keep)
    o = _opts(dxUm, fps, "3d", True, 2.0)
    m = None
    if lag_mask is not None:
        m = np.ascontiguousarray(lag_mask, np.uint8)
        keep.append(m)
    out = np.zeros(8)
    rc = lib.ddm_estimate_drift(C.byref(r), C.byref(o), C.c_void_p(m.ctypes.data) if m is not None else None,
                                C.c_void_p(out.ctypes.data))
    if rc:
        _raise(rc, "estimate_drift")
    return dict(Vx=out[0], Vy=out[1], mag=out[2], sigma=out[3], angleDeg=out[4], significant=bool(out[5]),
                pairs=int(out[6]), samples=out[7])


def scaling_exponent(radial, amps, dxUm=1.0, fps=1.0):
    """scalingExponent's mu (motility_fit.js:771-804) from per-prepared-bin
    amplitudes [nbins, 2] = (A, B)."""
    lib = _lib.load()
    keep = []
    r = _view(radial, keep)
    o = _opts(dxUm, fps, "3d", True, 2.0)
    a = np.ascontiguousarray(amps, np.float64).reshape(-1)
    mu = C.c_double()
    rc = lib.ddm_scaling_exponent(C.byref(r), C.byref(o), C.c_void_p(a.ctypes.data), C.byref(mu))
    if rc:
        _raise(rc, "scaling_exponent")
    return mu.value
