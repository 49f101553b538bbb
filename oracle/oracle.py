"""ctypes front end of the FP64 CPU oracle (oracle/xts_oracle.c).

TEST INFRASTRUCTURE ONLY.  The product package never imports this module.  It is
used by the tests, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of
``bench.py`` as the checker.  Each wrapper names the reference routine it
restates (paths relative to the xtsrcmaps source tree).

Objects passed as ``wcs`` only need the attributes naxis1, naxis2, crpix1,
crpix2, crval1, crval2, cdelt1, cdelt2, crota2, proj ('CAR' | 'AIT') and galactic.
Objects passed as IRF grids need cosths, logEs, params and min_cos_theta.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libxts_oracle.so")
ND = 401

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class _Wcs(C.Structure):
    _fields_ = [
        ("naxis1", C.c_long), ("naxis2", C.c_long),
        ("crpix1", C.c_double), ("crpix2", C.c_double),
        ("crval1", C.c_double), ("crval2", C.c_double),
        ("cdelt1", C.c_double), ("cdelt2", C.c_double),
        ("crota2", C.c_double), ("proj", C.c_int), ("galactic", C.c_int),
    ]


class _Grid(C.Structure):
    _fields_ = [
        ("cosths", _dp), ("n_cos", C.c_int),
        ("logEs", _dp), ("n_e", C.c_int),
        ("params", _dp), ("n_par", C.c_int),
        ("min_cos_theta", C.c_double),
    ]


def build() -> str:
    """Compile the oracle shared library with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "xts_oracle.c"))
        ):
            build()
        _lib = C.CDLL(_LIB_PATH)
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _out(shape):
    a = np.zeros(shape, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _wcs(w) -> _Wcs:
    proj = {"CAR": 0, "AIT": 1}[str(w.proj).upper()] if not isinstance(w.proj, int) else w.proj
    return _Wcs(int(w.naxis1), int(w.naxis2), float(w.crpix1), float(w.crpix2),
                float(w.crval1), float(w.crval2), float(w.cdelt1), float(w.cdelt2),
                float(getattr(w, "crota2", 0.0)), int(proj), int(bool(getattr(w, "galactic", False))))


class _GridHold:
    """Keeps the numpy buffers of a _Grid alive."""

    def __init__(self, g, n_par):
        self.c, cp = _d(g.cosths)
        self.e, ep = _d(g.logEs)
        self.p, pp = _d(g.params)
        self.s = _Grid(cp, len(self.c), ep, len(self.e), pp, n_par, float(g.min_cos_theta))


# --------------------------------------------------------------------------- a
def separations() -> np.ndarray:
    """psf/psf.hxx:24-31."""
    o, op = _out(ND)
    lib().xo_separations(op)
    return o


def costhetas(nbins: int, cosmin: float, thetabin: bool) -> np.ndarray:
    """exposure/exposure.cxx:29-40."""
    o, op = _out(nbins)
    lib().xo_costhetas(C.c_int(nbins), C.c_double(cosmin), C.c_int(int(thetabin)), op)
    return o


def ang2pix_nest(theta: float, phi: float, nside: int) -> int:
    """healpix/healpix.cxx:181-229."""
    f = lib().xo_ang2pix_nest
    f.restype = C.c_longlong
    return int(f(C.c_double(theta), C.c_double(phi), C.c_longlong(nside)))


def pix2ang_nest(pix: int, nside: int):
    """healpix/healpix.cxx:136-179."""
    t, p = C.c_double(), C.c_double()
    lib().xo_pix2ang_nest(C.c_longlong(pix), C.c_longlong(nside), C.byref(t), C.byref(p))
    return t.value, p.value


def src_cosbins(src_sph, cube, nside) -> np.ndarray:
    """exposure/exposure.cxx:42-63; cube is float32 [12 nside^2, C]."""
    s, sp = _d(src_sph)
    cube = np.ascontiguousarray(cube, dtype=np.float32)
    S, Cb = s.shape[0], cube.shape[1]
    o, op = _out((S, Cb))
    lib().xo_src_cosbins(sp, C.c_int(S), cube.ctypes.data_as(_fp), C.c_longlong(nside), C.c_int(Cb), op)
    return o


def aeff_value(costh, logEs, grid) -> np.ndarray:
    """irf/irf.aeff_value.cxx:11-55 -> [C, E] in cm^2."""
    c, cp = _d(costh)
    e, ep = _d(logEs)
    g = _GridHold(grid, 1)
    o, op = _out((len(c), len(e)))
    lib().xo_aeff_value(cp, C.c_int(len(c)), ep, C.c_int(len(e)), C.byref(g.s), op)
    return o


def livetime_efficiency_factors(logEs, p0, p1) -> np.ndarray:
    """irf/irf.cxx:70-109 -> [2, E]."""
    e, ep = _d(logEs)
    a0 = np.ascontiguousarray(p0, dtype=np.float32)
    a1 = np.ascontiguousarray(p1, dtype=np.float32)
    o, op = _out((2, len(e)))
    lib().xo_livetime_efficiency_factors(ep, C.c_int(len(e)), a0.ctypes.data_as(_fp),
                                         a1.ctypes.data_as(_fp), op)
    return o


def exposure(ecb, wecb, aeff_f, aeff_b, ltf) -> np.ndarray:
    """exposure/exposure.cxx:159-263 -> [S, E]."""
    x, xp = _d(ecb)
    w, wp = _d(wecb)
    af, afp = _d(aeff_f)
    ab, abp = _d(aeff_b)
    l, lp = _d(ltf)
    S, Cb = x.shape
    E = af.shape[1]
    o, op = _out((S, E))
    lib().xo_exposure(xp, wp, C.c_int(S), C.c_int(Cb), afp, abp, lp, C.c_int(E), op)
    return o


# --------------------------------------------------------------------------- b
def gauss_legendre_64():
    n, npp = _out(64)
    w, wp = _out(64)
    lib().xo_gauss_legendre_64(npp, wp)
    return n, w


def evaluate_king(sep: float, sf: float, pars) -> float:
    f = lib().xo_evaluate_king
    f.restype = C.c_double
    p, pp = _d(pars)
    return float(f(C.c_double(sep), C.c_double(sf), pp))


def normalize_rpsf(params, grid_logEs, scale0, scale1, scale_index) -> np.ndarray:
    """irf/irf.normalize_rpsf.cpp:11-61; returns a normalised copy of params [Mc, Me, 6]."""
    p = np.array(params, dtype=np.float64, copy=True, order="C")
    g, gp = _d(grid_logEs)
    Mc, Me = p.shape[0], p.shape[1]
    lib().xo_normalize_rpsf(p.ctypes.data_as(_dp), C.c_int(Mc), C.c_int(Me), gp,
                            C.c_float(scale0), C.c_float(scale1), C.c_float(scale_index))
    return p


def king(grid) -> np.ndarray:
    """psf/psf.king.cxx:9-43 -> [D, Mc, Me]."""
    g = _GridHold(grid, 6)
    o, op = _out((ND, len(g.c), len(g.e)))
    lib().xo_king(C.byref(g.s), op)
    return o


def compute_psf_data(psf_front, psf_back, costh, logEs, aeff_f, aeff_b, ecb, wecb, ltf, expo):
    """psf/psf.psf_lookup_table_and_partial_integrals.cxx:8-57 -> (uPsf, partial) [S, D, E]."""
    gf, gb = _GridHold(psf_front, 6), _GridHold(psf_back, 6)
    c, cp = _d(costh)
    e, ep = _d(logEs)
    af, afp = _d(aeff_f)
    ab, abp = _d(aeff_b)
    x, xp = _d(ecb)
    w, wp = _d(wecb)
    l, lp = _d(ltf)
    ex, exp_ = _d(expo)
    S, E = ex.shape
    u, up = _out((S, ND, E))
    pa, pap = _out((S, ND, E))
    lib().xo_compute_psf_data(C.byref(gf.s), C.byref(gb.s), cp, C.c_int(len(c)), ep, C.c_int(E),
                              afp, abp, xp, wp, C.c_int(S), lp, exp_, up, pap)
    return u, pa


# --------------------------------------------------------------------------- c, d
def pix2sph(wcs, p1: float, p2: float):
    ra, dec = C.c_double(), C.c_double()
    w = _wcs(wcs)
    lib().xo_wcs_pix2sph(C.byref(w), C.c_double(p1), C.c_double(p2), C.byref(ra), C.byref(dec))
    return ra.value, dec.value


def sph2pix(wcs, ra: float, dec: float):
    p1, p2 = C.c_double(), C.c_double()
    w = _wcs(wcs)
    lib().xo_wcs_sph2pix(C.byref(w), C.c_double(ra), C.c_double(dec), C.byref(p1), C.byref(p2))
    return p1.value, p2.value


def square_ptswts(wcs) -> np.ndarray:
    """model_map/mm_cubature/points_weights.hpp:5-56 -> [H, W, 48]."""
    w = _wcs(wcs)
    o, op = _out((w.naxis1, w.naxis2, 48))
    lib().xo_square_ptswts(C.byref(w), C.c_long(w.naxis1), C.c_long(w.naxis2), op)
    return o


def cubature_map(wcs, src_sph, upsf) -> np.ndarray:
    """model_map/mm_cubature/cubature.implementation.cxx:21-55 (keys-fixed logsep)."""
    w = _wcs(wcs)
    s, sp = _d(src_sph)
    u, up = _d(upsf)
    S, E = s.shape[0], u.shape[2]
    o, op = _out((S, w.naxis1, w.naxis2, E))
    lib().xo_cubature_map(C.byref(w), C.c_long(w.naxis1), C.c_long(w.naxis2), sp, C.c_int(S), up,
                          C.c_int(E), op)
    return o


def solid_angle(wcs) -> np.ndarray:
    """math/solid_angle.hpp:42-79 -> [H, W]."""
    w = _wcs(wcs)
    o, op = _out((w.naxis1, w.naxis2))
    lib().xo_solid_angle(C.byref(w), C.c_long(w.naxis1), C.c_long(w.naxis2), op)
    return o


def psf_boundary_radius(wcs, src_sph):
    """model_map/model_map.psf_boundary_radius.cxx:9-62 -> (radius_deg [S], in_fov [S])."""
    w = _wcs(wcs)
    s, sp = _d(src_sph)
    S = s.shape[0]
    r, rp = _out(S)
    f = np.zeros(S, dtype=np.int32)
    lib().xo_psf_boundary_radius(C.byref(w), C.c_long(w.naxis1), C.c_long(w.naxis2), sp, C.c_int(S),
                                 rp, f.ctypes.data_as(_ip))
    return r, f.astype(bool)


def point_src_model_map_wcs(wcs, src_sph, expo, upsf, partial):
    """model_map/model_map.point_src_model_map_wcs.cxx:6-45.

    Returns a dict with the map [S, H, W, E] (FP64) and the per-map quantities
    inv_integ [S, E] (1 / map integral), factor [S, E], radius [S], in_fov [S].
    """
    w = _wcs(wcs)
    s, sp = _d(src_sph)
    ex, exp_ = _d(expo)
    u, up = _d(upsf)
    pa, pap = _d(partial)
    S, E = ex.shape
    o, op = _out((S, w.naxis1, w.naxis2, E))
    inv, invp = _out((S, E))
    fac, facp = _out((S, E))
    r, rp = _out(S)
    f = np.zeros(S, dtype=np.int32)
    lib().xo_point_src_model_map_wcs(C.byref(w), sp, C.c_int(S), exp_, up, pap, C.c_int(E), op,
                                     invp, facp, rp, f.ctypes.data_as(_ip))
    return {"map": o, "inv_integ": inv, "factor": fac, "radius": r, "in_fov": f.astype(bool)}


def convolve_pixel_logsep(pw48, lut, src3) -> np.ndarray:
    """One pixel of the keys-fixed logsep kernel (convolve_pixel_psf_logsep.hpp:23-96)."""
    p, pp = _d(pw48)
    l, lp = _d(lut)
    s3, s3p = _d(src3)
    E = l.shape[1]
    o, op = _out(E)
    lib().xo_convolve_pixel_logsep(op, C.c_int(E), pp, lp, s3p)
    return o


def adaptive_cubature_map(wcs, src_sph, upsf, rtol: float, max_depth: int = 6):
    """Pixel-mean PSF [S, H, W, E] by adaptive Genz-Malik cubature (the reference's
    math/genz_malik.hxx:18-85 design, published rule with rectangular sub-regions)
    and the number of regions evaluated per (source, pixel)."""
    w = _wcs(wcs)
    s, sp = _d(src_sph)
    u, up = _d(upsf)
    S, E = s.shape[0], u.shape[2]
    H, W = int(wcs.naxis1), int(wcs.naxis2)
    out, op = _out((S, H, W, E))
    n = np.zeros((S, H, W), dtype=np.int32)
    lib().xo_adaptive_cubature_map(C.byref(w), sp, C.c_int(S), up, C.c_int(E), C.c_double(rtol),
                                   C.c_int(max_depth), op, n.ctypes.data_as(_ip))
    return out, n


def point_src_model_map_wcs_adaptive(wcs, src_sph, expo, upsf, partial, rtol: float, max_depth: int = 6):
    """ModelMap::point_src_model_map_wcs with the adaptive cubature in place of the
    12-point rule; returns the same dict as point_src_model_map_wcs plus 'nregions'."""
    w = _wcs(wcs)
    s, sp = _d(src_sph)
    ex, exp_ = _d(expo)
    u, up = _d(upsf)
    p, pp = _d(partial)
    S, E = ex.shape
    H, W = int(wcs.naxis1), int(wcs.naxis2)
    m, mp = _out((S, H, W, E))
    inv, ip = _out((S, E))
    fac, fp = _out((S, E))
    rad, rp = _out((S,))
    fov = np.zeros(S, dtype=np.int32)
    n = np.zeros((S, H, W), dtype=np.int32)
    lib().xo_point_src_model_map_wcs_adaptive(C.byref(w), sp, C.c_int(S), exp_, up, pp, C.c_int(E),
                                              C.c_double(rtol), C.c_int(max_depth), mp, ip, fp, rp,
                                              fov.ctypes.data_as(_ip), n.ctypes.data_as(_ip))
    return dict(map=m, inv_integ=inv, factor=fac, radius=rad, in_fov=fov.astype(bool), nregions=n)


def cutout_windows(wcs, src_sph, radius_deg):
    """Per-source cutout windows (the library's xts_cutout_windows, restated): the
    source's pixel (p1, p2) = sph2pix (1-based), n = ceil(radius / |CDELT|), rows
    round(p1) - 1 - n .. round(p1) - 1 + n and columns likewise, clipped to the map.
    Returns a list of (h0, w0, nh, nw, offset)."""
    out, off = [], 0
    H, W = int(wcs.naxis1), int(wcs.naxis2)
    for (ra, dec), r in zip(np.asarray(src_sph, dtype=np.float64), np.asarray(radius_deg, dtype=np.float64)):
        ra = ra - 360.0 if ra > 180.0 else (ra + 360.0 if ra < -180.0 else ra)
        p1, p2 = sph2pix(wcs, ra, dec)
        c = (0, 0, 0, 0)
        if np.isfinite(p1) and np.isfinite(p2) and abs(p1) < 1e9 and abs(p2) < 1e9:
            n1 = int(math.ceil(r / abs(wcs.cdelt1)))
            n2 = int(math.ceil(r / abs(wcs.cdelt2)))
            i = int(math.floor(abs(p1) + 0.5)) * (1 if p1 >= 0 else -1) - 1  # lround
            j = int(math.floor(abs(p2) + 0.5)) * (1 if p2 >= 0 else -1) - 1
            h0, h1 = max(0, i - n1), min(H, i + n1 + 1)
            w0, w1 = max(0, j - n2), min(W, j + n2 + 1)
            if h1 > h0 and w1 > w0:
                c = (h0, w0, h1 - h0, w1 - w0)
        out.append(c + (off,))
        off += c[2] * c[3]
    return out


def point_src_model_map_cutouts(wcs, src_sph, cut, expo, upsf, partial):
    """point_src_model_map_wcs of every source on its own window's sub-map (the WCS
    with CRPIX shifted by the window's origin): the ragged map [sum nh nw, E] and
    the per-source inv_integ, factor [S, E], radius, in_fov [S]."""
    import copy

    src = np.asarray(src_sph, dtype=np.float64)
    E = np.asarray(expo).shape[1]
    cut = [tuple(int(v) for v in c) for c in cut]
    total = sum(c[2] * c[3] for c in cut)
    m = np.zeros((total, E))
    S = len(cut)
    inv, fac = np.zeros((S, E)), np.ones((S, E))
    rad, fov = np.zeros(S), np.zeros(S, dtype=bool)
    for s, (h0, w0, nh, nw, off) in enumerate(cut):
        if nh == 0 or nw == 0:
            continue
        sub = copy.copy(wcs)
        sub.naxis1, sub.naxis2 = nh, nw
        sub.crpix1, sub.crpix2 = wcs.crpix1 - h0, wcs.crpix2 - w0
        r = point_src_model_map_wcs(sub, src[s:s + 1], np.asarray(expo)[s:s + 1], np.asarray(upsf)[s:s + 1],
                                    np.asarray(partial)[s:s + 1])
        m[off:off + nh * nw] = r["map"][0].reshape(nh * nw, E)
        inv[s], fac[s], rad[s], fov[s] = r["inv_integ"][0], r["factor"][0], r["radius"][0], r["in_fov"][0]
    return {"map": m, "inv_integ": inv, "factor": fac, "radius": rad, "in_fov": fov}
