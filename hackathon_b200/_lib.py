"""Loads the in-tree CUDA library and declares the C ABI (include/ddm_b200.h).

There is no fallback: if the library is missing or cannot load, importing the
engine fails with the reason.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libddm_b200.so")

DDM_OK, DDM_ERR_ARG, DDM_ERR_CUDA, DDM_ERR_STATE, DDM_ERR_NOMEM, DDM_ERR_NODEV = range(6)
DTYPES = {"u8": 0, "u16": 1, "f32": 2}


class RadialView(C.Structure):
    _fields_ = [("N", C.c_int32), ("NB", C.c_int32), ("L", C.c_int32), ("knodes", C.c_int32),
                ("kCenter", C.c_void_p), ("kNodes", C.c_void_p), ("nModes", C.c_void_p), ("D", C.c_void_p),
                ("P", C.c_void_p), ("drift", C.c_void_p)]


class MotilityOptions(C.Structure):
    _fields_ = [("dxUm", C.c_double), ("fps", C.c_double), ("geometry2d", C.c_int32),
                ("exposureLocked", C.c_int32), ("swimMin", C.c_double), ("optimizer", C.c_int32),
                ("reserved", C.c_int32)]


class MotilityFit(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("vbar", "Z", "Dd", "Vmag", "alpha", "rss")]


class MotilityResult(C.Structure):
    _fields_ = [("verdict", C.c_int32), ("physicsVerdict", C.c_int32), ("insufficient", C.c_int32),
                ("TSI", C.c_double), ("alpha", C.c_double), ("alphaResolved", C.c_int32),
                ("resolvedBins", C.c_int32), ("vbar", C.c_double), ("sigmaV", C.c_double), ("Z", C.c_double),
                ("Ddiff", C.c_double), ("DdiffBrownian", C.c_double), ("dBIC", C.c_double),
                ("driftVx", C.c_double), ("driftVy", C.c_double), ("driftMag", C.c_double),
                ("driftSigma", C.c_double), ("driftAngleDeg", C.c_double), ("driftSignificant", C.c_int32),
                ("driftPairs", C.c_int32), ("driftSamples", C.c_double), ("mu", C.c_double),
                ("nData", C.c_int32), ("nEff", C.c_double), ("rho", C.c_double), ("nbins", C.c_int32),
                ("nlags", C.c_int32), ("swim", MotilityFit), ("brown", MotilityFit)]


class SimParams(C.Structure):
    """ddm_sim_params (include/ddm_b200.h)."""
    _fields_ = [("N", C.c_int32), ("T", C.c_int32), ("fps", C.c_double), ("dxUm", C.c_double),
                ("seed", C.c_uint32), ("nSwim", C.c_int32), ("swimVbar", C.c_double), ("swimSigma", C.c_double),
                ("swim2d", C.c_int32), ("nPassive", C.c_int32), ("Dum2s", C.c_double), ("nFixed", C.c_int32),
                ("hasDrift", C.c_int32), ("driftSpeed", C.c_double), ("driftAngleDeg", C.c_double),
                ("dropFrac", C.c_double), ("dropExact", C.c_int32), ("blobSigmaPx", C.c_double),
                ("amp", C.c_double), ("background", C.c_double), ("noise", C.c_double)]


class Geometry(C.Structure):
    _fields_ = [("N", C.c_int32), ("T", C.c_int32), ("TPAD", C.c_int32), ("L", C.c_int32),
                ("NB", C.c_int32), ("kmin", C.c_double), ("kmax", C.c_double),
                ("knodes", C.c_int32), ("reserved", C.c_int32)]


_vp = C.c_void_p
_i32 = C.c_int32
_SIGS = {
    "ddm_create": (C.c_int, [C.POINTER(Geometry), C.POINTER(_vp)]),
    "ddm_destroy": (None, [_vp]),
    "ddm_last_error": (C.c_char_p, [_vp]),
    "ddm_create_error": (C.c_char_p, []),
    "ddm_get_geometry": (C.c_int, [_vp, C.POINTER(Geometry)]),
    "ddm_bins_count": (C.c_int, [_vp]),
    "ddm_get_bins": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "ddm_ingest_luma": (C.c_int, [_vp, _vp, _i32, C.POINTER(_i32)]),
    "ddm_ingest_frames": (C.c_int, [_vp, _vp, _i32, _i32, _vp, C.c_float]),
    "ddm_ingest_frames_device": (C.c_int, [_vp, _vp, _i32, _i32, _vp, C.c_float]),
    "ddm_ingest_frames_async": (C.c_int, [_vp, _vp, _i32, _i32, _vp, C.c_float]),
    "ddm_ingest_wait": (C.c_int, [_vp]),
    "ddm_set_spatial_mask": (C.c_int, [_vp, _vp]),
    "ddm_compute_temporal": (C.c_int, [_vp, _vp, _vp, _i32]),
    "ddm_compute_temporal_async": (C.c_int, [_vp, _vp, _vp, _i32]),
    "ddm_compute_temporal_live": (C.c_int, [_vp, _vp, _vp, _i32]),
    "ddm_set_sparse": (C.c_int, [_vp, _i32]),
    "ddm_set_blocked": (C.c_int, [_vp, _i32]),
    "ddm_last_temporal_kernel": (C.c_int, [_vp]),
    "ddm_analysis_poll": (C.c_int, [_vp, _vp]),
    "ddm_wait_analysis": (C.c_int, [_vp]),
    "ddm_read_radial": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ddm_read_history": (C.c_int, [_vp, _vp]),
    "ddm_read_temporal_full": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ddm_read_mean": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "ddm_idle": (C.c_int, [_vp]),
    "ddm_pending": (C.c_int, [_vp]),
    "ddm_wait_for_capacity": (C.c_int, [_vp]),
    "ddm_throttled": (C.c_int64, [_vp]),
    "ddm_set_stream": (C.c_int, [_vp, _vp]),
    "ddm_kernel_launches": (C.c_int64, [_vp]),
    "ddm_fit_lm": (C.c_int, [_i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _i32,
                             C.c_double, _i32, _vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "ddm_fit_lm_model": (C.c_int, [_i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _i32,
                                   C.c_double, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "ddm_model_curves": (C.c_int, [_i32, _i32, _vp, _vp, _i32, _vp, C.c_float, C.c_uint64, _vp, _vp, _vp]),
    "ddm_autotune": (C.c_int, [_vp, C.c_char_p, _i32]),
    "ddm_get_tuning": (C.c_int, [_vp, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32)]),
    "ddm_set_tuning": (C.c_int, [_vp, _i32, _i32, _i32]),
    "ddm_simulate": (C.c_int, [C.POINTER(SimParams), _vp, _i32, _vp, _vp, _vp]),
    "ddm_simulate_error": (C.c_char_p, []),
    "ddm_analyze_motility": (C.c_int, [C.POINTER(RadialView), C.POINTER(MotilityOptions),
                                       C.POINTER(MotilityResult)]),
    "ddm_analyze_motility_batch": (C.c_int, [_i32, C.POINTER(RadialView), C.POINTER(MotilityOptions),
                                             C.POINTER(MotilityResult)]),
    "ddm_isf_eval": (C.c_int, [_i32, _i32, _vp, _vp, _vp, _vp, _vp]),
    "ddm_dft2048_tc": (C.c_int, [_vp, C.c_int64, _i32, _vp, _vp]),
    "ddm_create_banded": (C.c_int, [C.POINTER(Geometry), C.c_uint64, C.POINTER(_vp)]),
    "ddm_get_bands": (C.c_int, [_vp, C.POINTER(_i32), C.POINTER(_i32)]),
    "ddm_analyze_banded": (C.c_int, [_vp, _vp, _i32, _i32, _vp, C.c_float, _vp, _vp, _i32]),
    "ddm_prepared_bins": (C.c_int, [C.POINTER(RadialView), C.POINTER(MotilityOptions), _vp, C.POINTER(_i32),
                                    C.POINTER(_i32)]),
    "ddm_temporal_structure_index": (C.c_double, [C.POINTER(RadialView)]),
    "ddm_estimate_drift": (C.c_int, [C.POINTER(RadialView), C.POINTER(MotilityOptions), _vp, _vp]),
    "ddm_scaling_exponent": (C.c_int, [C.POINTER(RadialView), C.POINTER(MotilityOptions), _vp,
                                       C.POINTER(C.c_double)]),
    "ddm_batch_create": (C.c_int, [_vp, _i32, C.POINTER(_vp)]),
    "ddm_batch_destroy": (None, [_vp]),
    "ddm_batch_last_error": (C.c_char_p, [_vp]),
    "ddm_batch_set_stream": (C.c_int, [_vp, _vp]),
    "ddm_batch_ingest": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "ddm_batch_compute_temporal": (C.c_int, [_vp, _vp, _vp]),
    "ddm_batch_enqueue_temporal": (C.c_int, [_vp]),
    "ddm_batch_sync": (C.c_int, [_vp]),
    "ddm_batch_capture": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "ddm_batch_launch_graph": (C.c_int, [_vp]),
    "ddm_mlp_create": (C.c_int, [_i32, C.c_uint64, C.POINTER(_vp)]),
    "ddm_mlp_destroy": (None, [_vp]),
    "ddm_mlp_last_error": (C.c_char_p, [_vp]),
    "ddm_mlp_param_count": (_i32, []),
    "ddm_mlp_get_params": (C.c_int, [_vp, _vp]),
    "ddm_mlp_set_params": (C.c_int, [_vp, _vp]),
    "ddm_mlp_forward": (C.c_int, [_vp, _vp, _i32, _vp, _vp]),
    "ddm_mlp_gradients": (C.c_int, [_vp, _vp, _vp, _i32, _vp, _vp, _vp]),
    "ddm_mlp_train_step": (C.c_int, [_vp, _vp, _vp, _i32, C.c_float, _vp, _vp]),
    "ddm_mlp_sync": (C.c_int, [_vp, _vp]),
    "ddm_spectra_noalloc": (C.c_int, [_vp, _i32, _i32, _i32, _i32, _vp, C.c_float, _vp, _vp]),
    "ddm_spectra_noalloc_status": (C.c_int, [_vp]),
}

_lib = None


def load():
    """The loaded library with every C-ABI signature declared."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m hackathon_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def exported_symbols():
    return list(_SIGS)
