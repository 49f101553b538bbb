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
