"""ctypes bindings of libxts_cuda.so (include/xtsrcmaps_b200.h).

The library is built in-tree by ``xtsrcmaps_b200/build.py``.  There is no CPU
fallback: if the shared object is missing or no sm_100 device is visible, the
calls raise.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxts_cuda.so")

XTS_OK = 0
XTS_ERR_ARG = -1
XTS_ERR_CUDA = -2
XTS_ERR_OOM = -3
XTS_ERR_TIMEOUT = -4
XTS_ERR_NODEV = -5
XTS_ERR_IO = -6

XTS_DEVICE_PTRS = 1 << 0
XTS_OUT_F64 = 1 << 1
XTS_CUDA_CORES = 1 << 3
XTS_TCGEN05 = 1 << 4
XTS_FITS_F32 = 1 << 5

ND = 401
NOALLOC_SCRATCH_DOUBLES = 1 << 20  # XTS_NOALLOC_SCRATCH_DOUBLES

# xts_cutout: one source's window of the map and its first pixel in the ragged output
CUTOUT_DTYPE = np.dtype([("h0", "<i4"), ("w0", "<i4"), ("nh", "<i4"), ("nw", "<i4"), ("offset", "<i8")])

_vp = C.c_void_p


class XtsWcs(C.Structure):
    _fields_ = [
        ("naxis1", C.c_long), ("naxis2", C.c_long),
        ("crpix1", C.c_double), ("crpix2", C.c_double),
        ("crval1", C.c_double), ("crval2", C.c_double),
        ("cdelt1", C.c_double), ("cdelt2", C.c_double),
        ("crota2", C.c_double), ("proj", C.c_int), ("galactic", C.c_int),
    ]


class XtsGrid(C.Structure):
    _fields_ = [
        ("cosths", _vp), ("n_cos", C.c_int),
        ("logEs", _vp), ("n_e", C.c_int),
        ("params", _vp), ("n_par", C.c_int),
        ("min_cos_theta", C.c_double),
    ]


class XtsExpcube(C.Structure):
    _fields_ = [
        ("cosbins", _vp), ("nside", C.c_long), ("nbrbins", C.c_int),
        ("cosmin", C.c_double), ("thetabin", C.c_int),
    ]


class XtsExposureOut(C.Structure):
    _fields_ = [
        ("exp_costhetas", _vp), ("front_aeff", _vp), ("back_aeff", _vp),
        ("src_exposure_cosbins", _vp), ("src_weighted_exposure_cosbins", _vp),
        ("exposure", _vp),
    ]


class XtsSrcmapInfo(C.Structure):
    _fields_ = [
        ("inv_map_integral", _vp), ("correction", _vp), ("psf_radius", _vp), ("in_fov", _vp),
    ]


MLP_IN = 5
MLP_HID = 128
MLP_W1 = 0
MLP_B1 = MLP_W1 + MLP_HID * MLP_IN
MLP_W2 = MLP_B1 + MLP_HID
MLP_B2 = MLP_W2 + MLP_HID * MLP_HID
MLP_W3 = MLP_B2 + MLP_HID
MLP_B3 = MLP_W3 + MLP_HID * MLP_HID
MLP_W4 = MLP_B3 + MLP_HID
MLP_B4 = MLP_W4 + MLP_HID
MLP_NPARAM = MLP_B4 + 1
MLP_CELL_NR = 32  # XTS_MLP_CELL_NR
MLP_CELL_NS = 16  # XTS_MLP_CELL_NS


class XtsMlp(C.Structure):
    _fields_ = [
        ("params", _vp), ("wbf16", _vp),
        ("in_mu", C.c_float * MLP_IN), ("in_sd", C.c_float * MLP_IN),
        ("out_mu", C.c_float), ("out_sd", C.c_float),
        ("lo", C.c_float * MLP_IN), ("hi", C.c_float * MLP_IN),
        ("rho_min", C.c_float),
        ("cell_lo", C.c_float * 2), ("cell_hi", C.c_float * 2),
        ("cell_ok", _vp),
    ]


class XtsTuning(C.Structure):
    _fields_ = [("window_blocks_per_sm", C.c_int), ("write_blocks_per_sm", C.c_int), ("queue_blocks_per_sm", C.c_int),
                ("mlp_blocks_per_sm", C.c_int), ("chunk_sources", C.c_int)]


class XtsSurrogateStats(C.Structure):
    _fields_ = [
        ("values", C.c_longlong), ("accepted", C.c_longlong), ("checked", C.c_longlong),
        ("maps_fallback", C.c_int), ("max_check_err", C.c_float), ("evaluated", C.c_longlong),
    ]


# Every symbol the header declares, with its signature.
SIGNATURES = {
    "xts_init": (C.c_int, [C.c_int]),
    "xts_release": (None, []),
    "xts_last_error": (C.c_char_p, []),
    "xts_version": (C.c_int, []),
    "xts_profile_enable": (C.c_int, [C.c_int]),
    "xts_profile_read": (C.c_int, [C.c_char_p, C.c_int]),
    "xts_livetime_efficiency_factors": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_uint, _vp]),
    "xts_normalize_rpsf": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_float, C.c_float, C.c_float,
                                     C.c_uint, _vp]),
    "xts_compute_exposure": (C.c_int, [C.POINTER(XtsExpcube), C.POINTER(XtsExpcube), _vp, C.c_int,
                                       _vp, C.c_int, C.POINTER(XtsGrid), C.POINTER(XtsGrid), _vp,
                                       C.POINTER(XtsExposureOut), C.c_uint, _vp]),
    "xts_exposure_contract": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _vp, _vp, _vp, C.c_int, _vp,
                                        C.c_uint, _vp]),
    "xts_compute_psf_data": (C.c_int, [C.POINTER(XtsGrid), C.POINTER(XtsGrid), _vp, C.c_int, _vp,
                                       C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp, _vp, _vp,
                                       C.c_uint, _vp]),
    "xts_compute_psf_data_noalloc": (C.c_int, [C.POINTER(XtsGrid), C.POINTER(XtsGrid), _vp, C.c_int,
                                               _vp, C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp,
                                               _vp, _vp, _vp]),
    "xts_point_source_maps": (C.c_int, [C.POINTER(XtsExpcube), C.POINTER(XtsExpcube), _vp, C.c_int, _vp,
                                        C.c_int, C.POINTER(XtsGrid), C.POINTER(XtsGrid), C.POINTER(XtsGrid),
                                        C.POINTER(XtsGrid), _vp, C.POINTER(XtsWcs), _vp,
                                        C.POINTER(XtsSrcmapInfo), C.c_uint, _vp]),
    "xts_exposure_map": (C.c_int, [C.POINTER(XtsExpcube), C.POINTER(XtsExpcube), _vp, C.c_int,
                                   C.POINTER(XtsGrid), C.POINTER(XtsGrid), _vp, _vp, C.c_uint, _vp]),
    "xts_point_src_model_map_wcs_adaptive": (C.c_int, [C.POINTER(XtsWcs), _vp, C.c_int, _vp, _vp, _vp,
                                                       C.c_int, C.c_double, C.c_int, _vp,
                                                       C.POINTER(XtsSrcmapInfo), C.c_uint, _vp]),
    "xts_point_src_model_map_wcs": (C.c_int, [C.POINTER(XtsWcs), _vp, C.c_int, _vp, _vp, _vp,
                                              C.c_int, _vp, C.POINTER(XtsSrcmapInfo), C.c_uint, _vp]),
    "xts_write_src_model": (C.c_int, [C.c_char_p, _vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.POINTER(C.c_char_p), C.c_uint, _vp]),
    "xts_make_psf_kernel": (C.c_int, [C.POINTER(XtsWcs), C.c_int, _vp, C.c_int, _vp, C.c_uint, _vp]),
    "xts_convolve_map_psf": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_uint, _vp]),
    "xts_gemm_bf16": (C.c_int, [_vp, C.c_int, _vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_int, _vp]),
    "xts_mlp_forward": (C.c_int, [C.POINTER(XtsMlp), _vp, C.c_longlong, _vp, _vp]),
    "xts_mlp_grads": (C.c_int, [C.POINTER(XtsMlp), _vp, _vp, C.c_longlong, _vp, _vp, _vp]),
    "xts_mlp_train_step": (C.c_int, [C.POINTER(XtsMlp), _vp, _vp, C.c_longlong, _vp, _vp, _vp, C.c_int,
                                     C.c_float, _vp, _vp]),
    "xts_surrogate_samples": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_longlong, C.c_ulonglong, C.c_double,
                                        _vp, _vp, _vp]),
    "xts_point_src_model_map_wcs_surrogate": (C.c_int, [C.POINTER(XtsWcs), _vp, C.c_int, _vp, _vp, _vp, _vp,
                                                        C.c_int, C.POINTER(XtsMlp), C.c_double, _vp,
                                                        C.POINTER(XtsSrcmapInfo),
                                                        C.POINTER(XtsSurrogateStats), _vp]),
    "xts_surrogate_last_stats": (C.c_int, [C.POINTER(XtsSurrogateStats), _vp]),
    "xts_point_source_maps_surrogate": (C.c_int, [C.POINTER(XtsExpcube), C.POINTER(XtsExpcube), _vp, C.c_int, _vp,
                                                  C.c_int, C.POINTER(XtsGrid), C.POINTER(XtsGrid),
                                                  C.POINTER(XtsGrid), C.POINTER(XtsGrid), _vp, C.POINTER(XtsWcs),
                                                  C.POINTER(XtsMlp), C.c_double, _vp, C.POINTER(XtsSrcmapInfo),
                                                  C.POINTER(XtsSurrogateStats), C.c_uint, _vp]),
    "xts_cutout_windows": (C.c_int, [C.POINTER(XtsWcs), _vp, _vp, C.c_int, _vp, C.POINTER(C.c_longlong)]),
    "xts_point_src_model_map_cutouts": (C.c_int, [C.POINTER(XtsWcs), _vp, C.c_int, _vp, _vp, _vp, _vp, C.c_int,
                                                  _vp, C.POINTER(XtsSrcmapInfo), C.c_uint, _vp]),
    "xts_set_tuning": (C.c_int, [C.POINTER(XtsTuning)]),
    "xts_get_tuning": (C.c_int, [C.POINTER(XtsTuning)]),
    "xts_rebin_wcs": (C.c_int, [C.POINTER(XtsWcs), C.c_double, C.POINTER(XtsWcs)]),
    "xts_allsky_crop_range": (C.c_int, [C.POINTER(XtsWcs), C.POINTER(XtsWcs), C.POINTER(C.c_long)]),
    "xts_crop_allsky": (C.c_int, [_vp, C.c_int, C.c_long, C.c_long, C.POINTER(C.c_long), _vp, C.c_uint, _vp]),
    "xts_trilerp_ehw": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_int, C.c_int, C.c_uint, _vp]),
    "xts_scale_model_map": (C.c_int, [C.POINTER(XtsWcs), _vp, C.c_int, _vp, _vp, _vp, C.c_int, _vp,
                                      C.POINTER(XtsSrcmapInfo), C.c_uint, _vp]),
}


class XtsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"xtsrcmaps_b200 error {code}: {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m xtsrcmaps_b200.build` "
                "(there is no CPU fallback)")
        l = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def check(rc: int) -> None:
    if rc != XTS_OK:
        msg = lib().xts_last_error()
        raise XtsError(rc, msg.decode() if msg else "")
