"""Oracle for the diffuse-map steps -- TEST INFRASTRUCTURE ONLY.

Only tests/ may import this module, as the checker.  FP64 numpy restatements of
the two numeric steps of the reference's work-in-progress diffuse-source map
(model_map/model_map.diffuse_src_model_map_wcs.cxx:8-97):

  * make_kernel -- Psf::make_kernel (psf/psf.make_kernel.cpp:8-90): for each pixel
    centre (h + 1, w + 1) of an Nk x Nk grid, the separation from the grid's
    reference point (SkyGeom::refdir, the CRVAL direction) in degrees, the logsep
    row i (j = 1 below 1e-4 deg, else 1 + recipstep (ln 1e4 + ln s); i = 1 + floor(j)
    capped at 400) and weight t = redm1 (s 1e4 e^{step (2 - i)} - 1), the value
    (1 - t) uPsf[i - 1] + t uPsf[i] per energy (the reference writes t uPsf[i - 1] +
    (1 - t) uPsf[i] at :43-45, the reverse of its own cubature; the cubature's order is
    used here), and each energy plane scaled to unit sum (:57-88);
  * convolve_full -- FFT::convolve_map_psf (model_map/mm_fft/fft.convolve_map_psf.cpp:7-43):
    per energy plane the full linear convolution [E, H + K - 1, W + K - 1], here by
    direct summation over the kernel offsets (the reference's fftw_convolve_3d,
    math/convolve/fft/fft.fftw_convolve_CHW.cpp:7-90, transforms over all three axes
    and misparenthesises its scale; the per-plane linear convolution is what it is
    written for).
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

SEP_STEP = math.log(70.0 / 1e-4) / 399.0
RECIPSTEP = 1.0 / SEP_STEP
REDM1 = 1.0 / (math.exp(SEP_STEP) - 1.0)
LN_1E4 = math.log(1e4)


def _dir(ra, dec):
    r, d = np.radians(ra), np.radians(dec)
    return np.array([np.cos(d) * np.cos(r), np.cos(d) * np.sin(r), np.sin(d)])


def make_kernel(wcs, Nk: int, upsf: np.ndarray) -> np.ndarray:
    upsf = np.asarray(upsf, dtype=np.float64)
    E = upsf.shape[1]
    ref = _dir(wcs.crval1, wcs.crval2)
    k = np.empty((E, Nk, Nk))
    for h in range(Nk):
        for w in range(Nk):
            ra, dec = O.pix2sph(wcs, h + 1.0, w + 1.0)
            d = _dir(ra, dec) - ref
            s = math.degrees(2.0 * math.asin(0.5 * math.sqrt(float(d @ d))))
            j = 1.0 if s < 1e-4 else 1.0 + RECIPSTEP * (LN_1E4 + math.log(s))
            i = min(1 + int(j), 400)
            t = REDM1 * (s * 1e4 * math.exp(SEP_STEP * (2.0 - i)) - 1.0)
            k[:, h, w] = (1.0 - t) * upsf[i - 1] + t * upsf[i]
    return k / k.sum(axis=(1, 2), keepdims=True)


def convolve_full(image: np.ndarray, kernel: np.ndarray) -> np.ndarray:
    image = np.asarray(image, dtype=np.float64)
    kernel = np.asarray(kernel, dtype=np.float64)
    E, H, W = image.shape
    K = kernel.shape[1]
    out = np.zeros((E, H + K - 1, W + K - 1))
    for a in range(K):
        for b in range(K):
            out[:, a:a + H, b:b + W] += kernel[:, a, b][:, None, None] * image
    return out


def rebin_wcs(wcs, target: float):
    """rebin_wcs_config (sky_geom/sky_geom.hxx:352-371), with the rebinned CDELT2
    where the reference stores CRPIX2 (:367)."""
    import copy

    out = copy.copy(wcs)
    c1 = -target if wcs.cdelt1 < 0 else target
    c2 = -target if wcs.cdelt2 < 0 else target
    s1, s2 = abs(wcs.cdelt1 / c1), abs(wcs.cdelt2 / c2)
    out.cdelt1, out.cdelt2 = c1, c2
    out.naxis1 = int(math.floor(wcs.naxis1 * s1 + 0.5))  # std::round (halves away from zero)
    out.naxis2 = int(math.floor(wcs.naxis2 * s2 + 0.5))
    out.crpix1, out.crpix2 = wcs.crpix1 * s1, wcs.crpix2 * s2
    return out


def allsky_crop_range(sky_wcs, roi_wcs):
    """fits/fits.read_allsky_cropped.cpp:155-194: the ROI's pixels (1, 1) and
    (NAXIS1, NAXIS2) to the sky (longitude wrapped into [0, 360), latitude clamped),
    to all-sky pixels, rounded and bounded to [1, NAXISn]; (min, max) per axis."""
    px, py = [], []
    for p1, p2 in ((1.0, 1.0), (float(roi_wcs.naxis1), float(roi_wcs.naxis2))):
        lon, lat = O.pix2sph(roi_wcs, p1, p2)
        lon = math.fmod(lon + 360.0, 360.0)
        lat = min(90.0, max(-90.0, lat))
        x, y = O.sph2pix(sky_wcs, lon, lat)
        px.append(x)
        py.append(y)

    def bound(v, mx):
        r = int(math.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)  # std::round
        return max(1, min(r, mx))

    return (bound(min(px), sky_wcs.naxis1), bound(max(px), sky_wcs.naxis1),
            bound(min(py), sky_wcs.naxis2), bound(max(py), sky_wcs.naxis2))


def crop_allsky(sky: np.ndarray, rng) -> np.ndarray:
    """The block [E0, ny, nx] of sky [E0, NY, NX] inside rng = (x0, x1, y0, y1),
    1-based inclusive; x0 > x1 wraps across the longitude seam (the two segments of
    readSegmentsAcrossBoundary, fits.read_allsky_cropped.cpp:119-147, side by side)."""
    x0, x1, y0, y1 = rng
    rows = sky[:, y0 - 1:y1, :]
    if x1 >= x0:
        return np.ascontiguousarray(rows[:, :, x0 - 1:x1])
    return np.ascontiguousarray(np.concatenate([rows[:, :, x0 - 1:], rows[:, :, :x1]], axis=2))


def trilerp_ehw(src: np.ndarray, shape) -> np.ndarray:
    """Fermi::math::trilerpEHW (math/trilerp.hpp:7-59) in float32, step by step:
    scale = (n0 - 1) / (n1 - 1) (0 where n1 = 1), lower index int(k * scale),
    upper min(lower + 1, n0 - 1); C00..C11 over h, then w, then e."""
    src = np.asarray(src, dtype=np.float32)
    E0, H0, W0 = src.shape
    E1, H1, W1 = shape
    f = np.float32

    def axis(n0, n1):
        sc = f(n0 - 1) / f(n1 - 1) if n1 > 1 else f(0.0)
        x = np.arange(n1, dtype=np.float32) * sc
        i0 = x.astype(np.int64)
        i1 = np.minimum(i0 + 1, n0 - 1)
        fr = (x - i0.astype(np.float32)).astype(np.float32)
        return i0, i1, fr, (f(1.0) - fr).astype(np.float32)

    e0, e1, fe, ce = axis(E0, E1)
    h0, h1, fh, ch = axis(H0, H1)
    w0, w1, fw, cw = axis(W0, W1)
    E_, H_, W_ = np.ix_(np.arange(E1), np.arange(H1), np.arange(W1))

    def at(a, b, c):
        return src[a[E_], b[H_], c[W_]]

    chh, fhh = ch[H_], fh[H_]
    c00 = chh * at(e0, h0, w0) + fhh * at(e0, h1, w0)
    c01 = chh * at(e1, h0, w0) + fhh * at(e1, h1, w0)
    c10 = chh * at(e0, h0, w1) + fhh * at(e0, h1, w1)
    c11 = chh * at(e1, h0, w1) + fhh * at(e1, h1, w1)
    c0 = cw[W_] * c00 + fw[W_] * c10
    c1 = cw[W_] * c01 + fw[W_] * c11
    return (ce[E_] * c0 + fe[E_] * c1).astype(np.float32)


def scale_model_map(wcs, src_sph, expo, upsf, partial, means):
    """The scalings of model_map.diffuse_src_model_map_wcs.cxx:76-95 (those of
    point_src_model_map_wcs.cxx:24-42) applied to a map of pixel means [S, H, W, E]
    in FP64: solid angle, boundary radius and in-FOV flag, 1 / map integral,
    exposure, containment correction.  Returns (map, inv_integ, factor, radius, in_fov)."""
    import ctypes as C

    m = np.array(means, dtype=np.float64, copy=True, order="C")
    S, H, W, E = m.shape
    om = O.solid_angle(wcs)
    m *= om[None, :, :, None]
    radius, fov = O.psf_boundary_radius(wcs, src_sph)
    w = O._wcs(wcs)
    s, sp = O._d(src_sph)
    mm, mp = O._d(m)
    r, rp = O._d(radius)
    fi = np.ascontiguousarray(fov.astype(np.int32))
    inv, invp = O._out((S, E))
    O.lib().xo_map_integral(mp, C.byref(w), C.c_long(H), C.c_long(W), sp, C.c_int(S), C.c_int(E), rp,
                            fi.ctypes.data_as(C.POINTER(C.c_int)), invp)
    mm = mm * np.asarray(expo, dtype=np.float64)[:, None, None, :]
    u, up = O._d(upsf)
    pa, pap = O._d(partial)
    fac, facp = O._out((S, E))
    O.lib().xo_map_correction_factor(invp, rp, fi.ctypes.data_as(C.POINTER(C.c_int)), up, pap, C.c_int(S),
                                     C.c_int(E), facp)
    return mm * fac[:, None, None, :], inv, fac, radius, fov
