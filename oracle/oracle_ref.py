"""ctypes front end of oracle/_ref/libxts_ref.so: the reference's own hot-path
translation units compiled in place (recipe: oracle/build_ref.sh, entry points:
oracle/ref_driver.cxx).

TEST INFRASTRUCTURE ONLY.  Used by the tests as a second checker (it pins the
oracle's restatement of the model-map step to the reference's code) and by
``bench.py --impl reference`` as the timed CPU reference.  The library is built
where the reference tree is present and travels with the repository; where it
is absent, ``available()`` is False.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libxts_ref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB_PATH)
    return _lib


def set_threads(n: int) -> int:
    """OpenMP threads of the reference code; returns the count in effect."""
    return int(lib().xr_set_threads(C.c_int(int(n))))


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def exposure(cube, wcube, nside, cosmin, thetabin, src_sph, aeff_f, aeff_b, ltf):
    """Exposure::costhetas, map, src_cosbins, exposure (exposure/exposure.cxx:16-160).
    Returns (costh [C], ecb [S,C], wecb [S,C], exposure [S,E])."""
    c, cp = _f(cube)
    w, wp = _f(wcube)
    C_ = c.shape[1]
    s, sp = O._d(src_sph)
    S = s.shape[0]
    af, afp = O._d(aeff_f)
    ab, abp = O._d(aeff_b)
    lt, ltp = O._d(ltf)
    E = af.shape[1]
    ct, ctp = O._out((C_,))
    x, xp = O._out((S, C_))
    wx, wxp = O._out((S, C_))
    e, ep = O._out((S, E))
    lib().xr_exposure(cp, wp, C.c_long(int(nside)), C.c_int(C_), C.c_double(cosmin), C.c_int(int(bool(thetabin))),
                      sp, C.c_int(S), afp, abp, ltp, C.c_int(E), ctp, xp, wxp, ep)
    return ct, x, wx, e


def psf(rpsf_front, rpsf_back, costh, logEs, aeff_f, aeff_b, ecb, wecb, ltf, expo):
    """Psf::psf_lookup_table_and_partial_integrals
    (psf/psf.psf_lookup_table_and_partial_integrals.cxx:8-57) on normalised King
    grids.  Returns (uPsf, partial) [S, 401, E]."""
    gf, gb = O._GridHold(rpsf_front, 6), O._GridHold(rpsf_back, 6)
    ct, ctp = O._d(costh)
    le, lep = O._d(logEs)
    af, afp = O._d(aeff_f)
    ab, abp = O._d(aeff_b)
    x, xp = O._d(ecb)
    w, wp = O._d(wecb)
    lt, ltp = O._d(ltf)
    ex, exp_ = O._d(expo)
    S, E = ex.shape
    u, up = O._out((S, O.ND, E))
    p, pp = O._out((S, O.ND, E))
    lib().xr_psf(C.byref(gf.s), C.byref(gb.s), ctp, C.c_int(len(ct)), lep, C.c_int(E), afp, abp, xp, wp,
                 C.c_int(S), ltp, exp_, up, pp)
    return u, p


def point_src_model_map_wcs(wcs, src_sph, expo, upsf, partial) -> np.ndarray:
    """ModelMap::point_src_model_map_wcs (model_map/model_map.point_src_model_map_wcs.cxx:6-45)
    with the keys-fixed logsep cubature.  Returns the FP64 map [S, H, W, E]."""
    w = O._wcs(wcs)
    s, sp = O._d(src_sph)
    ex, exp_ = O._d(expo)
    u, up = O._d(upsf)
    p, pp = O._d(partial)
    S, E = ex.shape
    m, mp = O._out((S, int(wcs.naxis1), int(wcs.naxis2), E))
    lib().xr_point_src_model_map_wcs(C.byref(w), sp, C.c_int(S), exp_, up, pp, C.c_int(E), mp)
    return m
