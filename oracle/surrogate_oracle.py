"""CPU oracle of the surrogate's training samples and pixel features (test
infrastructure only: the product path never imports this file).

Restates, in Python FP64, the sample generator of the library (a hash of seed
and sample index drives every draw; a synthetic pixel is placed on the sphere
around a source at the pole) and the per-pixel quantities of the surrogate
model map: the 12 rule points of the pixel as the bilinear blend of its corner
unit vectors (square_ptswts, model_map/mm_cubature/points_weights.hpp:5-56, rule
square_deg7 of model_map/mm_cubature/cubature.hpp:209-225), their separations,
the logsep row and weight (convolve_pixel_psf_logsep.hpp:39-55, keys fixed), the
rule mean of the mean PSF, the centre value and the features.
"""
from __future__ import annotations

import math

import numpy as np

M64 = (1 << 64) - 1
SEP_STEP = math.log(7e5) / 399.0
RECIPSTEP = 1.0 / SEP_STEP
REDM1 = 1.0 / (math.exp(SEP_STEP) - 1.0)
LN_1E4 = math.log(1e4)
R2D = 180.0 / math.pi
D2R = math.pi / 180.0

# Sommariva & Festa degree-7 12-point rule on [-1, 1]^2: (u, v, weight), weights sum to 4
RULE = np.array([
    [3.9383136101878902e-01, -3.6699793434042738e-01, 5.2092862230230441e-01],
    [8.0196847620659251e-01, 8.0992592975809186e-01, 2.3740240561379911e-01],
    [-1.8327327664247231e-02, 9.2596092593108370e-01, 2.4166897208389651e-01],
    [3.6699793434042738e-01, 3.9383136101878902e-01, 5.2092862230230441e-01],
    [-8.0992592975809186e-01, 8.0196847620659251e-01, 2.3740240561379911e-01],
    [-9.2596092593108370e-01, -1.8327327664247231e-02, 2.4166897208389651e-01],
    [-3.9383136101878902e-01, 3.6699793434042738e-01, 5.2092862230230441e-01],
    [-8.0196847620659251e-01, -8.0992592975809186e-01, 2.3740240561379911e-01],
    [1.8327327664247231e-02, -9.2596092593108370e-01, 2.4166897208389651e-01],
    [-3.6699793434042738e-01, -3.9383136101878902e-01, 5.2092862230230441e-01],
    [8.0992592975809186e-01, -8.0196847620659251e-01, 2.3740240561379911e-01],
    [9.2596092593108370e-01, 1.8327327664247231e-02, 2.4166897208389651e-01],
])


def _splitmix(state):
    state = (state + 0x9E3779B97F4A7C15) & M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return state, z ^ (z >> 31)


def sep_row(sdeg):
    """Row idx in [2, 400] and weight t of the keys-fixed logsep rule."""
    j = 1.0 if sdeg < 1e-4 else 1.0 + RECIPSTEP * (LN_1E4 + math.log(sdeg))
    idx = min(max(1 + int(j), 2), 400)
    return idx, REDM1 * (sdeg * 1e4 * math.exp(SEP_STEP * (2.0 - idx)) - 1.0)


def pixel_quantities(corners, src, U, e):
    """corners: LL, LR, UR, UL unit vectors; src unit vector; U [401, E].
    Returns (features f0, f1, f2, slope; u_c; rule mean m; rho)."""
    a, b, c, d = (np.asarray(v, np.float64) for v in corners)
    s = np.asarray(src, np.float64)
    A = 0.25 * ((a + b) + (c + d)) - s
    B = 0.25 * ((b + c) - (a + d))
    Cv = 0.25 * ((c + d) - (a + b))
    D = 0.25 * ((a + c) - (b + d))
    m = 0.0
    for u, v, w in RULE:
        p = A + B * u + Cv * v + D * (u * v)
        sd = 2.0 * R2D * math.asin(0.5 * math.sqrt(float(p @ p)))
        i, t = sep_row(sd)
        m += 0.25 * w * ((1.0 - t) * U[i - 1, e] + t * U[i, e])
    alen = math.sqrt(float(A @ A))
    thc = 2.0 * math.asin(0.5 * alen)
    om = 4.0 * float(np.linalg.norm(np.cross(B, Cv)))
    rho = thc / math.sqrt(om)
    ic, tc = sep_row(R2D * thc)
    lo, hi = U[ic - 1, e], U[ic, e]
    slope = math.log(hi / lo) / SEP_STEP if lo > 0 and hi > 0 else 0.0
    uc = (1.0 - tc) * lo + tc * hi
    return (math.log10(rho), tc, math.log10(om * R2D * R2D), slope), uc, m, rho


def sample(upsf, logEs, i, seed, rho_min):
    """Features [5] and target of sample i (as the library's generator)."""
    S, _, E = upsf.shape
    st = (seed ^ ((i * 0xD1B54A32D192ED03) & M64)) & M64
    st, _ = _splitmix(st)
    draws = []
    for _ in range(6):
        st, z = _splitmix(st)
        draws.append((z >> 11) * 2.0 ** -53)
    s = min(int(draws[0] * S), S - 1)
    e = min(int(draws[1] * E), E - 1)
    size = 0.025 + 0.175 * draws[2]
    asp = math.exp(math.log(1.25) * (2.0 * draws[3] - 1.0))
    lo = max(0.001, rho_min * size)
    th = lo * math.exp(draws[4] * math.log(30.0 / lo)) * D2R
    al = draws[5] * (math.pi / 2)
    ha, hb = 0.5 * size * math.sqrt(asp) * D2R, 0.5 * size / math.sqrt(asp) * D2R
    c = np.array([math.sin(th), 0.0, math.cos(th)])
    e1, e2 = np.array([math.cos(th), 0.0, -math.sin(th)]), np.array([0.0, 1.0, 0.0])
    Uax = math.cos(al) * e1 + math.sin(al) * e2
    Vax = -math.sin(al) * e1 + math.cos(al) * e2
    corners = []
    for su, sv in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
        k = c + su * ha * Uax + sv * hb * Vax
        corners.append(k / math.sqrt(float(k @ k)))
    (f0, f1, f2, slope), uc, m, rho = pixel_quantities(corners, [0.0, 0.0, 1.0], upsf[s], e)
    return np.array([f0, f1, f2, logEs[e], slope]), math.log(m / uc) * rho * rho
