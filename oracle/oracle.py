"""ctypes layer over the FP64 oracle library (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY. Every function names the reference function it
stands for; the C sources cite the reference lines.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")

VERDICTS = ["MOTILE", "NOT_MOTILE", "DIRECTED_TRANSPORT", "NO_DYNAMICS",
            "UNLOCKED_EXPOSURE"]


def build():
    """Compile the oracle with its Makefile (system gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


class _Radial(C.Structure):
    _fields_ = [("N", C.c_int), ("NB", C.c_int), ("L", C.c_int),
                ("knodes", C.c_int), ("kCenter", C.c_void_p),
                ("kNodes", C.c_void_p), ("nModes", C.c_void_p),
                ("D", C.c_void_p), ("P", C.c_void_p), ("drift", C.c_void_p)]


class _Options(C.Structure):
    _fields_ = [("dxUm", C.c_double), ("fps", C.c_double),
                ("geometry2d", C.c_int), ("exposureLocked", C.c_int),
                ("swimMin", C.c_double)]


class _Fit(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("vbar", "Z", "Dd", "Vmag", "alpha", "rss")]


class _Result(C.Structure):
    _fields_ = [("verdict", C.c_int), ("physicsVerdict", C.c_int),
                ("insufficient", C.c_int), ("TSI", C.c_double),
                ("alpha", C.c_double), ("alphaResolved", C.c_int),
                ("resolvedBins", C.c_int), ("vbar", C.c_double),
                ("sigmaV", C.c_double), ("Z", C.c_double),
                ("Ddiff", C.c_double), ("DdiffBrownian", C.c_double),
                ("dBIC", C.c_double), ("driftVx", C.c_double),
                ("driftVy", C.c_double), ("driftMag", C.c_double),
                ("driftSigma", C.c_double), ("driftAngleDeg", C.c_double),
                ("driftSignificant", C.c_int), ("driftPairs", C.c_int),
                ("driftSamples", C.c_double), ("mu", C.c_double),
                ("nData", C.c_int), ("nEff", C.c_double), ("rho", C.c_double),
                ("nbins", C.c_int), ("nlags", C.c_int),
                ("swim", _Fit), ("brown", _Fit)]


class _SimParams(C.Structure):
    _fields_ = [("N", C.c_int), ("T", C.c_int), ("fps", C.c_double),
                ("dxUm", C.c_double), ("seed", C.c_uint32), ("nSwim", C.c_int),
                ("swimVbar", C.c_double), ("swimSigma", C.c_double),
                ("swim2d", C.c_int), ("nPassive", C.c_int),
                ("Dum2s", C.c_double), ("nFixed", C.c_int),
                ("hasDrift", C.c_int), ("driftSpeed", C.c_double),
                ("driftAngleDeg", C.c_double), ("dropFrac", C.c_double),
                ("dropExact", C.c_int), ("blobSigmaPx", C.c_double),
                ("amp", C.c_double), ("background", C.c_double),
                ("noise", C.c_double)]


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    sig = {
        "or_fft": (None, [_dp, C.c_int, C.c_int]),
        "or_dft": (None, [_dp, _dp, C.c_int, C.c_int]),
        "or_blackman_harris": (None, [_dp, C.c_int]),
        "or_spectrum2d_half": (None, [_dp, C.c_int, _dp, _dp]),
        "or_window_leakage": (C.c_int, [C.c_int, C.c_double, _dp, _dp]),
        "or_make_bins_count": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double]),
        "or_make_bins": (None, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                _u32p, _i32p, _dp, _u32p, _dp]),
        "or_history_ingest": (None, [_dp, C.c_int, C.c_int, _dp, _i32p, C.c_int]),
        "or_history_ingest_masked": (None, [_dp, C.c_int, C.c_int, _dp, C.c_void_p, _i32p, C.c_int]),
        "or_temporal_mode": (C.c_double, [_dp, C.c_int, C.c_int, C.c_int, _u32p, _dp,
                                          C.c_int, _dp, _dp]),
        "or_temporal_mode_direct": (C.c_double, [_dp, C.c_int, C.c_int, _u32p, _dp,
                                                 C.c_int, _dp, _dp]),
        "or_analyze_radial": (None, [_dp, C.c_int, C.c_int, C.c_int, _u32p, _dp, C.c_int,
                                     _u32p, _i32p, _u32p, C.c_int, _dp, _dp, _dp, C.c_int]),
        "or_analyze_modes": (None, [_dp, C.c_int, C.c_int, _u32p, _dp, C.c_int, _i32p,
                                    C.c_int, _dp, _dp, _dp, C.c_int]),
        "or_radial_from_full": (None, [_dp, _dp, _dp, C.c_int, _u32p, _i32p, _u32p,
                                       C.c_int, _dp, _dp, _dp]),
        "or_temporal_meta": (None, [_u32p, _dp, C.c_int, C.c_int, C.c_int, _dp, _dp]),
        "or_bessel_j0": (C.c_double, [C.c_double]),
        "or_ln_gamma": (C.c_double, [C.c_double]),
        "or_schulz_pdf": (C.c_double, [C.c_double, C.c_double, C.c_double]),
        "or_legendre_p": (C.c_double, [C.c_double, C.c_double]),
        "or_isf3d": (C.c_double, [C.c_double, C.c_double]),
        "or_isf2d": (C.c_double, [C.c_double, C.c_double]),
        "or_isf2d_fast": (C.c_double, [C.c_double, C.c_double]),
        "or_nnls3": (C.c_double, [_dp, _dp, C.c_double, _dp]),
        "or_lag_grid": (C.c_int, [C.c_int, _i32p]),
        "or_analyze_motility": (None, [C.POINTER(_Radial), C.POINTER(_Options),
                                       C.POINTER(_Result)]),
        "or_fit_brownian_swimmer": (None, [C.POINTER(_Radial), C.POINTER(_Options),
                                           C.POINTER(_Fit), C.POINTER(_Fit)]),
        "or_estimate_drift": (None, [C.POINTER(_Radial), C.POINTER(_Options), C.c_int,
                                     C.c_double, C.c_double, _dp]),
        "or_temporal_structure_index": (C.c_double, [C.POINTER(_Radial)]),
        "or_model_column": (C.c_int, [C.POINTER(_Radial), C.POINTER(_Options), C.c_int,
                                      C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_int, _dp]),
        "or_eval_model": (C.c_double, [C.POINTER(_Radial), C.POINTER(_Options),
                                       C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_int, _dp]),
        "or_lm_fit": (C.c_int, [C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, _dp, _dp, C.c_int,
                                C.c_double, C.POINTER(C.c_double)]),
        "or_lm_model": (None, [C.c_int, C.c_int, _dp, _dp, _dp, _dp]),
        "or_lm_fit_start": (C.c_int, [C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, _dp, _dp,
                                      C.c_int, C.c_double, _dp, C.POINTER(C.c_double)]),
        "or_lm_fit_brownian": (C.c_double, [C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, _dp, _dp]),
        "or_lm_fit_plain": (C.c_int, [C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, _dp, C.c_int,
                                      C.c_double, C.c_int, _dp, C.POINTER(C.c_double),
                                      C.POINTER(C.c_int)]),
        "or_simulate": (None, [C.POINTER(_SimParams), _u8p, _u8p, _dp]),
        "or_mulberry32": (None, [C.c_uint32, _dp, C.c_int]),
        "or_rng_normals": (None, [C.c_uint32, _dp, C.c_int]),
        "or_rng_gammas": (None, [C.c_uint32, C.c_double, C.c_double, _dp, C.c_int]),
        "or_shuffle_order": (None, [_u32p, _dp, C.c_int, C.c_uint32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _c128_to_f64(x):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    return x.view(np.float64).reshape(-1)


# ------------------------------------------------------------------ fft.js

def fft(x, inverse=False):
    """fft.js:59-93 (unnormalised both ways)."""
    d = _c128_to_f64(np.array(x, dtype=np.complex128, copy=True))
    lib().or_fft(d, d.size // 2, int(inverse))
    return d.view(np.complex128)


def dft(x, inverse=False):
    """fft.js:101-119."""
    d = _c128_to_f64(x)
    out = np.empty_like(d)
    lib().or_dft(d, out, d.size // 2, int(inverse))
    return out.view(np.complex128)


def blackman_harris(n):
    """fft.js:126-133."""
    w = np.empty(n)
    lib().or_blackman_harris(w, n)
    return w


def spectrum2d_half(img):
    """fft.js:149-183 -> complex [N, N/2+1] indexed [ky, kx]."""
    img = np.ascontiguousarray(img, dtype=np.float64)
    N = img.shape[0]
    out = np.empty(2 * N * (N // 2 + 1))
    lib().or_spectrum2d_half(img.reshape(-1), N, blackman_harris(N), out)
    return out.view(np.complex128).reshape(N, N // 2 + 1)


# ------------------------------------------------------------------ ddm_ref.js

def window_leakage(N, step=0.5):
    """ddm_ref.js:40-55."""
    d = np.empty(64)
    p = np.empty(64)
    n = lib().or_window_leakage(N, step, d, p)
    return d[:n].copy(), p[:n].copy()


def make_bins(N, NB, kmin, kmax, knodes=4):
    """ddm_ref.js:84-170."""
    total = lib().or_make_bins_count(N, NB, kmin, kmax)
    off = np.empty(NB + 1, np.uint32)
    modes = np.empty(4 * max(total, 1), np.int32)
    kc = np.empty(NB)
    nm = np.empty(NB, np.uint32)
    kn = np.empty(NB * knodes)
    lib().or_make_bins(N, NB, float(kmin), float(kmax), knodes, off, modes, kc, nm, kn)
    return dict(N=N, NB=NB, kmin=kmin, kmax=kmax, knodes=knodes, binOffsets=off,
                binModes=modes[:4 * total].reshape(total, 4), kCenter=kc,
                nModes=nm, kNodes=kn)


def history_ingest(luma, slots, T, hist=None, smask=None):
    """History.ingest (ddm_ref.js:196-206) for a stack of frames [F, N, N].
    Returns the history as complex128 [modes, T] (the reference layout).
    smask: the spatial-mask extension (N x N, nonzero = used; the reference
    has none): mean over the used pixels, the others left out."""
    luma = np.ascontiguousarray(luma, dtype=np.float64)
    F, N, _ = luma.shape
    M = N * (N // 2 + 1)
    if hist is None:
        hist = np.zeros((M, T), np.complex128)
    h = hist.view(np.float64).reshape(-1)
    if smask is None:
        lib().or_history_ingest(h, N, T, luma.reshape(-1),
                                np.ascontiguousarray(slots, dtype=np.int32), F)
    else:
        sm = np.ascontiguousarray(smask, dtype=np.uint8).reshape(-1)
        assert sm.size == N * N
        lib().or_history_ingest_masked(h, N, T, luma.reshape(-1), sm.ctypes.data,
                                       np.ascontiguousarray(slots, dtype=np.int32), F)
    return hist


def _hist_f64(hist):
    h = np.ascontiguousarray(hist, dtype=np.complex128)
    return h.view(np.float64).reshape(-1), h.shape[1]


def temporal_mode(hist, mode, order, mask, L, TPAD=None):
    """ddm_ref.js:229-288 -> (D[L], C[L] complex, P)."""
    h, T = _hist_f64(hist)
    TPAD = TPAD or 2 * T
    D = np.empty(L)
    Cc = np.empty(2 * L)
    P = lib().or_temporal_mode(h, mode, T, TPAD, np.ascontiguousarray(order, np.uint32),
                               np.ascontiguousarray(mask, np.float64), L, D, Cc)
    return D, Cc.view(np.complex128), P


def temporal_mode_direct(hist, mode, order, mask, L):
    """ddm_ref.js:306-333."""
    h, T = _hist_f64(hist)
    D = np.empty(L)
    Cc = np.empty(2 * L)
    P = lib().or_temporal_mode_direct(h, mode, T, np.ascontiguousarray(order, np.uint32),
                                      np.ascontiguousarray(mask, np.float64), L, D, Cc)
    return D, Cc.view(np.complex128), P


def analyze_radial(hist, order, mask, bins, L, TPAD=None, threads=None):
    """ddm_ref.js:425-437 -> dict(D[NB, L], P[NB], drift[NB, L, 8])."""
    h, T = _hist_f64(hist)
    TPAD = TPAD or 2 * T
    NB = bins["NB"]
    D = np.empty(NB * L)
    P = np.empty(NB)
    dr = np.empty(NB * L * 8)
    lib().or_analyze_radial(h, bins["N"], T, TPAD, np.ascontiguousarray(order, np.uint32),
                            np.ascontiguousarray(mask, np.float64), NB, bins["binOffsets"],
                            np.ascontiguousarray(bins["binModes"]).reshape(-1), bins["nModes"],
                            L, D, P, dr, threads or os.cpu_count())
    return dict(D=D.reshape(NB, L), P=P, drift=dr.reshape(NB, L, 8))


def analyze_modes(hist, order, mask, L, modes, TPAD=None, threads=None):
    """analyzeFull (ddm_ref.js:450-463) for a list of modes."""
    h, T = _hist_f64(hist)
    TPAD = TPAD or 2 * T
    modes = np.ascontiguousarray(modes, np.int32)
    n = modes.size
    D = np.empty(n * L)
    Cc = np.empty(n * 2 * L)
    P = np.empty(n)
    lib().or_analyze_modes(h, T, TPAD, np.ascontiguousarray(order, np.uint32),
                           np.ascontiguousarray(mask, np.float64), L, modes, n, D, Cc, P,
                           threads or os.cpu_count())
    return D.reshape(n, L), Cc.view(np.complex128).reshape(n, L), P


def radial_from_full(D, Cm, P, bins, L):
    """ddm_ref.js:474-487. D[modes, L], C[modes, L] complex, P[modes]."""
    NB = bins["NB"]
    oD = np.empty(NB * L)
    oP = np.empty(NB)
    dr = np.empty(NB * L * 8)
    lib().or_radial_from_full(np.ascontiguousarray(D, np.float64).reshape(-1),
                              _c128_to_f64(Cm), np.ascontiguousarray(P, np.float64), NB,
                              bins["binOffsets"], np.ascontiguousarray(bins["binModes"]).reshape(-1),
                              bins["nModes"], L, oD, oP, dr)
    return dict(D=oD.reshape(NB, L), P=oP, drift=dr.reshape(NB, L, 8))


def temporal_meta(order, mask, T, TPAD, L):
    """temporalMeta (ddm_ref.js:538-560) before the f32 rounding."""
    npairs = np.empty(L)
    ms = np.empty(2 * TPAD)
    lib().or_temporal_meta(np.ascontiguousarray(order, np.uint32),
                           np.ascontiguousarray(mask, np.float64), T, TPAD, L, npairs, ms)
    return npairs, ms.view(np.complex128)


def linear_order(valid):
    """ddm_ref.js:493-502."""
    valid = np.asarray(valid)
    return np.arange(valid.size, dtype=np.uint32), valid.astype(np.float64)


def shuffle_order(order, mask, seed):
    """ddm_ref.js:510-519 with rand = mulberry32(seed)."""
    o = np.array(order, np.uint32)
    m = np.array(mask, np.float64)
    lib().or_shuffle_order(o, m, o.size, seed)
    return o, m


# ------------------------------------------------------------------ motility_fit.js

def bessel_j0(x): return lib().or_bessel_j0(x)
def ln_gamma(x): return lib().or_ln_gamma(x)
def schulz_pdf(v, vbar, Z): return lib().or_schulz_pdf(v, vbar, Z)
def legendre_p(nu, c): return lib().or_legendre_p(nu, c)
def isf3d(x, Z): return lib().or_isf3d(x, Z)
def isf2d(x, Z): return lib().or_isf2d(x, Z)
def isf2d_fast(x, Z): return lib().or_isf2d_fast(x, Z)


def nnls3(G, h, dd):
    """motility_fit.js:243-263 -> (a[3], rss)."""
    a = np.empty(3)
    rss = lib().or_nnls3(np.ascontiguousarray(G, np.float64).reshape(-1),
                         np.ascontiguousarray(h, np.float64), dd, a)
    return a, rss


def lag_grid(L):
    """motility_fit.js:358-369."""
    out = np.empty(L + 16, np.int32)
    n = lib().or_lag_grid(L, out)
    return out[:n].copy()


class Radial:
    """The Radial record (ddm_ref.js:336-348) as numpy arrays."""

    def __init__(self, N, NB, L, kCenter, kNodes, nModes, D, P, drift, knodes=4):
        self.N, self.NB, self.L, self.knodes = N, NB, L, knodes
        self.kCenter = np.ascontiguousarray(kCenter, np.float64)
        self.kNodes = np.ascontiguousarray(kNodes, np.float64).reshape(-1)
        self.nModes = np.ascontiguousarray(nModes, np.uint32)
        self.D = np.ascontiguousarray(D, np.float64).reshape(-1)
        self.P = np.ascontiguousarray(P, np.float64).reshape(-1)
        self.drift = np.ascontiguousarray(drift, np.float64).reshape(-1)

    @classmethod
    def from_bins(cls, bins, L, rad):
        return cls(bins["N"], bins["NB"], L, bins["kCenter"], bins["kNodes"],
                   bins["nModes"], rad["D"], rad["P"], rad["drift"], bins["knodes"])

    def _c(self):
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        s = _Radial(self.N, self.NB, self.L, self.knodes, p(self.kCenter), p(self.kNodes),
                    p(self.nModes), p(self.D), p(self.P), p(self.drift))
        return s


def _opts(dxUm=1.0, fps=1.0, geometry="3d", exposureLocked=True, swimMin=2.0):
    return _Options(dxUm, fps, 1 if geometry == "2d" else 0, 1 if exposureLocked else 0, swimMin)


def analyze_motility(radial, dxUm=1.0, fps=1.0, geometry="3d", exposureLocked=True,
                     swimMin=2.0):
    """analyzeMotility (motility_fit.js:870-912) -> dict."""
    res = _Result()
    r = radial._c()
    o = _opts(dxUm, fps, geometry, exposureLocked, swimMin)
    lib().or_analyze_motility(C.byref(r), C.byref(o), C.byref(res))
    out = {k: getattr(res, k) for k, _ in _Result._fields_ if k not in ("swim", "brown")}
    out["verdict"] = VERDICTS[res.verdict]
    out["physicsVerdict"] = VERDICTS[res.physicsVerdict]
    out["swim"] = {k: getattr(res.swim, k) for k, _ in _Fit._fields_}
    out["brown"] = {k: getattr(res.brown, k) for k, _ in _Fit._fields_}
    return out


def fit_brownian_swimmer(radial, dxUm=1.0, fps=1.0, geometry="3d"):
    b, s = _Fit(), _Fit()
    r = radial._c()
    o = _opts(dxUm, fps, geometry)
    lib().or_fit_brownian_swimmer(C.byref(r), C.byref(o), C.byref(b), C.byref(s))
    return ({k: getattr(b, k) for k, _ in _Fit._fields_},
            {k: getattr(s, k) for k, _ in _Fit._fields_})


def estimate_drift(radial, dxUm=1.0, fps=1.0, geometry="3d", swimmer=None):
    """estimateDrift (motility_fit.js:672-725)."""
    out = np.empty(8)
    r = radial._c()
    o = _opts(dxUm, fps, geometry)
    sv, sz = (swimmer if swimmer else (0.0, 1.0))
    lib().or_estimate_drift(C.byref(r), C.byref(o), 1 if swimmer else 0, sv, sz, out)
    return dict(Vx=out[0], Vy=out[1], mag=out[2], sigma=out[3], angleDeg=out[4],
                significant=bool(out[5]), pairs=int(out[6]), samples=out[7])


def temporal_structure_index(radial):
    r = radial._c()
    return lib().or_temporal_structure_index(C.byref(r))


def eval_model(radial, p, dxUm=1.0, fps=1.0, geometry="3d", swim=True):
    """evalModel (motility_fit.js:450-474) -> (rss, amps[nbins, 2])."""
    amps = np.zeros(2 * radial.NB + 2)
    r = radial._c()
    o = _opts(dxUm, fps, geometry)
    rss = lib().or_eval_model(C.byref(r), C.byref(o), p["vbar"], p["Z"], p["Dd"],
                              p.get("Vmag", 0.0), p["alpha"], 1 if swim else 0, amps)
    return rss, amps


# ------------------------------------------------------------------ sim.mjs

def simulate(sim):
    """simulate (sim.mjs:90-186) -> (frames u8[T, N, N], valid bool[T], truth)."""
    p = _SimParams()
    p.N, p.T = sim.get("N", 256), sim.get("T", 256)
    p.fps, p.dxUm = sim.get("fps", 30.0), sim.get("dxUm", 1.0)
    p.seed = sim.get("seed", 1)
    sw = sim.get("swimmers")
    if sw and sw["n"] > 0:
        p.nSwim, p.swimVbar, p.swimSigma = sw["n"], sw["vbar"], sw["sigma"]
        p.swim2d = 1 if sw.get("geometry") == "2d" else 0
    p.nPassive = (sim.get("passive") or {}).get("n", 0)
    p.Dum2s = sim.get("Dum2s", 0.0)
    p.nFixed = (sim.get("fixed") or {}).get("n", 0)
    dr = sim.get("drift")
    if dr:
        p.hasDrift, p.driftSpeed, p.driftAngleDeg = 1, dr["speed"], dr["angleDeg"]
    p.dropFrac = sim.get("dropFrac", 0.0)
    p.dropExact = sim.get("dropExact", 0)
    p.blobSigmaPx = sim.get("blobSigmaPx", 1.5)
    p.amp = sim.get("amp", 0.15)
    p.background = sim.get("background", 0.25)
    p.noise = sim.get("noise", 0.01)
    frames = np.empty(p.T * p.N * p.N, np.uint8)
    valid = np.empty(p.T, np.uint8)
    truth = np.empty(4)
    lib().or_simulate(C.byref(p), frames, valid, truth)
    return (frames.reshape(p.T, p.N, p.N), valid.astype(bool),
            dict(meanSpeed=truth[0], Vx=truth[1], Vy=truth[2], D=truth[3]))


def mulberry32(seed, n):
    out = np.empty(n)
    lib().or_mulberry32(seed, out, n)
    return out


def rng_normals(seed, n):
    out = np.empty(n)
    lib().or_rng_normals(seed, out, n)
    return out


def rng_gammas(seed, k, theta, n):
    out = np.empty(n)
    lib().or_rng_gammas(seed, k, theta, out, n)
    return out


def luma_of(frames):
    """sim.mjs:189-193: u8 / 255 in FP64."""
    return np.asarray(frames, np.float64) / 255.0


def run_scenario(sc, exposureLocked=True, threads=None):
    """runScenario (t_validation_matrix.mjs:20-40) through the oracle."""
    frames, valid, truth = simulate(sc["sim"])
    N, T = frames.shape[1], frames.shape[0]
    idx = np.nonzero(valid)[0]
    hist = history_ingest(luma_of(frames[idx]), idx.astype(np.int32), T)
    order, mask = linear_order(valid)
    if sc.get("shuffle"):
        order, mask = shuffle_order(order, mask, 4242)
    bins = make_bins(N, 32, 4, 100)
    L = 128
    rad = analyze_radial(hist, order, mask, bins, L, threads=threads)
    radial = Radial.from_bins(bins, L, rad)
    res = analyze_motility(radial, dxUm=sc["sim"]["dxUm"], fps=sc["sim"]["fps"],
                           geometry=sc["geometry"], exposureLocked=exposureLocked)
    return res, radial, hist


def check_scenario(sc, res):
    """checkScenario (t_validation_matrix.mjs:47-67) -> list of failures."""
    fails = []
    if res["verdict"] != sc["expect"]:
        fails.append(f"verdict {res['verdict']}, expected {sc['expect']}")
    c = sc["checks"]
    if "vbar" in c:
        v, tol = c["vbar"]
        if not abs(res["vbar"] - v) / v <= tol:
            fails.append(f"vbar {res['vbar']:.2f}")
    if "alpha" in c:
        v, tol = c["alpha"]
        if not abs(res["alpha"] - v) <= tol:
            fails.append(f"alpha {res['alpha']:.3f}")
    if "drift" in c:
        sp, ang, rel, deg = c["drift"]
        err = abs(res["driftMag"] - sp) / sp
        d = abs(res["driftAngleDeg"] - ang) % 360
        if d > 180:
            d = 360 - d
        if not err <= rel:
            fails.append(f"|V| {res['driftMag']:.2f}")
        if not d <= deg:
            fails.append(f"angle {res['driftAngleDeg']:.1f}")
    return fails


# ------------------------------------------------------------------ per-bin LM (new)

def lm_fit(d, tau, qn, w, bounds6, theta0, max_iter=200, tol=1e-10):
    """FP64 LM on one bin (oracle/lm.c) -> (theta, cost, iterations)."""
    th = np.array(theta0, np.float64)
    cost = C.c_double()
    it = lib().or_lm_fit(len(d), len(qn), np.ascontiguousarray(d, np.float64),
                         np.ascontiguousarray(tau, np.float64), np.ascontiguousarray(qn, np.float64),
                         float(w), np.ascontiguousarray(bounds6, np.float64), th, max_iter, tol,
                         C.byref(cost))
    return th, cost.value, it


def lm_model(tau, qn, theta):
    y = np.empty(len(tau))
    lib().or_lm_model(len(tau), len(qn), np.ascontiguousarray(tau, np.float64),
                      np.ascontiguousarray(qn, np.float64), np.ascontiguousarray(theta, np.float64), y)
    return y


def _f64(a):
    return np.ascontiguousarray(a, np.float64)


def lm_fit_start(d, tau, qn, w, bounds6, start4, max_iter=200, tol=1e-10):
    """FP64 LM from (alpha, vbar, Z, D) with VarPro amplitudes -> (theta, cost, iters)."""
    th = np.zeros(6)
    cost = C.c_double()
    it = lib().or_lm_fit_start(len(d), len(qn), _f64(d), _f64(tau), _f64(qn), float(w),
                               _f64(bounds6), _f64(start4), max_iter, tol, th, C.byref(cost))
    return th, cost.value, it


def lm_fit_brownian(d, tau, qn, w, bounds6):
    """FP64 Brownian model per bin (fitBrownian's scan + golden section) -> (theta, cost)."""
    th = np.zeros(6)
    cost = lib().or_lm_fit_brownian(len(d), len(qn), _f64(d), _f64(tau), _f64(qn), float(w), _f64(bounds6), th)
    return th, cost


def lm_fit_plain(d, tau, qn, w, bounds6, max_iter=200, tol=1e-10, nrefine=3):
    """FP64 LM from the reference's start strategy -> (theta, cost, iters, evals)."""
    th = np.zeros(6)
    cost = C.c_double()
    ev = C.c_int()
    it = lib().or_lm_fit_plain(len(d), len(qn), _f64(d), _f64(tau), _f64(qn), float(w),
                               _f64(bounds6), max_iter, tol, nrefine, th, C.byref(cost),
                               C.byref(ev))
    return th, cost.value, it, ev.value
