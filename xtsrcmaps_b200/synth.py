"""Seeded synthetic inputs for the point-source path.

No public dataset is involved: the reference's own workload is a Fermi-LAT
analysis (counts cube, livetime cube, Pass-8 IRF tables, XML source model).
These generators produce inputs with the same shapes, layouts and value ranges:

* livetime cube on HEALPix NESTED x 40 sqrt-binned cos-theta bins (cosmin 0),
  a constant times lognormal(0, 0.2) noise, weighted cube = 0.9 x the same;
* effective area as a raw FITS row of 32 cos-theta x 74 log-energy bins in m^2,
  a smooth seeded surface rising from 0 to about 0.9 m^2 (9000 cm^2);
* King PSF parameters as a raw FITS row of 8 cos-theta x 23 energy bins, core
  and tail widths log-decreasing with energy from 5 deg to 0.05 deg (after the
  PSF_SCALING factor), gammas uniform in [1.5, 4], ntail uniform in
  [0.05, 0.5], ncore renormalised by the reference rule;
* a CAR counts-map WCS centred at (193.98, -5.82) and source positions drawn
  uniformly in a square field around it.

The raw rows go through ``irf.prepare_grid`` exactly as FITS rows would.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .api import ExpCube
from .irf import IrfEffic, IrfGrid, IrfScale, prepare_grid
from .wcs import Wcs

CENTER = (193.98, -5.82)


@dataclass
class PointSourceJob:
    """Everything the reference's main.cxx collects before the three hot-path calls."""

    name: str
    wcs: Wcs
    energies: np.ndarray
    logEs: np.ndarray
    exp_cube: ExpCube
    wexp_cube: ExpCube
    aeff_front: IrfGrid
    aeff_back: IrfGrid
    effic_front: IrfEffic
    rpsf_front: IrfGrid        # raw (not yet normalised) King grids
    rpsf_back: IrfGrid
    scale_front: IrfScale
    scale_back: IrfScale
    src_sph: np.ndarray        # [S, 2] (ra, dec) degrees
    src_names: list = field(default_factory=list)
    cutout_deg: np.ndarray | None = None

    @property
    def S(self) -> int:
        return int(self.src_sph.shape[0])

    @property
    def E(self) -> int:
        return int(len(self.energies))

    @property
    def n_values(self) -> int:
        return self.S * int(self.wcs.naxis1) * int(self.wcs.naxis2) * self.E


CONFIGS = {
    # name: (S, npix, pixdeg, E, Emin, Emax, nside, field_deg)
    "c0": dict(S=1, npix=100, pix=0.2, E=20, emin=100.0, emax=1e5, nside=32, field=0.0),
    "c1": dict(S=50, npix=200, pix=0.1, E=37, emin=100.0, emax=1e6, nside=64, field=20.0),
    "c2": dict(S=500, npix=400, pix=0.05, E=37, emin=100.0, emax=1e6, nside=64, field=20.0),
    "c4": dict(S=2000, npix=800, pix=0.025, E=50, emin=30.0, emax=1e6, nside=128, field=40.0),
}
DESCRIPTIONS = {
    "c0": "1 source at the field centre, CAR 100x100 @0.2 deg, 20 energies 100 MeV-100 GeV, nside 32 x 40",
    "c1": "50 sources uniform in 20x20 deg, CAR 200x200 @0.1 deg, 37 energies 100 MeV-1 TeV, nside 64 x 40",
    "c2": "500 sources (10% within 1 deg of the edge), CAR 400x400 @0.05 deg, 37 energies, nside 64 x 40",
    "c4": "2000 sources uniform in 40x40 deg, CAR 800x800 @0.025 deg, 50 energies 30 MeV-1 TeV, nside 128 x 40",
}


def native_to_celestial(wcs: Wcs, phi_deg, theta_deg):
    """Native spherical (phi, theta) of a theta0 = 0 projection -> (ra, dec), degrees."""
    a0 = wcs.crval1 - 360.0 if wcs.crval1 > 180.0 else wcs.crval1
    d0 = wcs.crval2
    if d0 >= 0:
        pp, dp, ap = 0.0, 90.0 - d0, a0 - 180.0
    else:
        pp, dp, ap = 180.0, 90.0 + d0, a0
    ph, th = np.radians(np.asarray(phi_deg)), np.radians(np.asarray(theta_deg))
    dph = ph - np.radians(pp)
    sdp, cdp = np.sin(np.radians(dp)), np.cos(np.radians(dp))
    xr = np.sin(th) * cdp - np.cos(th) * sdp * np.cos(dph)
    yr = -np.cos(th) * np.sin(dph)
    ra = (ap + np.degrees(np.arctan2(yr, xr))) % 360.0
    dec = np.degrees(np.arcsin(np.clip(np.sin(th) * sdp + np.cos(th) * cdp * np.cos(dph), -1, 1)))
    return ra, dec


def _aeff_row(rng, front: bool):
    """Raw EFFECTIVE AREA row: ENERG_LO/HI[74], CTHETA_LO/HI[32], EFFAREA[32 x 74] (m^2)."""
    ne, nc = 74, 32
    eedges = np.linspace(0.75, 6.5, ne + 1)
    cedges = np.linspace(0.2, 1.0, nc + 1)
    le = 0.5 * (eedges[:-1] + eedges[1:])
    cc = 0.5 * (cedges[:-1] + cedges[1:])
    amax = 0.9 if front else 0.8
    rise = 1.0 / (1.0 + np.exp(-(le - (1.9 if front else 2.1)) / 0.22))
    fall = 1.0 - 0.08 * np.clip(le - 5.0, 0.0, None)
    g = ((cc - 0.2) / 0.8).clip(0.0, 1.0) ** 0.6
    ph = rng.uniform(0, 2 * np.pi, 3)
    wob = 1.0 + 0.02 * np.sin(3.1 * le[None, :] + ph[0]) * np.cos(5.3 * cc[:, None] + ph[1])
    area = amax * g[:, None] * (rise * fall)[None, :] * wob
    row = np.concatenate([10 ** eedges[:-1], 10 ** eedges[1:], cedges[:-1], cedges[1:], area.ravel()])
    ext = [ne, ne, nc, nc, nc * ne]
    off = np.cumsum([0] + ext[:-1])
    return ext, off, row.astype(np.float32)


def _king_row(rng, scale: IrfScale, front: bool):
    """Raw RPSF row: ENERG_LO/HI[23], CTHETA_LO/HI[8], NCORE, NTAIL, SCORE, STAIL, GCORE, GTAIL [8 x 23]."""
    ne, nc = 23, 8
    eedges = np.linspace(0.75, 6.5, ne + 1)
    cedges = np.linspace(0.2, 1.0, nc + 1)
    le = 0.5 * (eedges[:-1] + eedges[1:])
    cc = 0.5 * (cedges[:-1] + cedges[1:])
    energy = 10 ** le
    tt = (energy * 1e-2) ** np.float32(scale.scale_index)
    sf = np.sqrt(np.float32(scale.scale0) ** 2 * tt * tt + np.float32(scale.scale1) ** 2)
    frac = (le - le[0]) / (le[-1] - le[0])
    width_deg = np.exp(np.log(5.0) + frac * (np.log(0.05) - np.log(5.0))) * (1.0 if front else 1.6)
    inc = 1.0 + 0.25 * (1.0 - cc)
    score = np.radians(width_deg[None, :] * inc[:, None]) / sf[None, :]
    stail = score * rng.uniform(1.5, 3.0, (nc, ne))
    ncore = np.ones((nc, ne))
    ntail = rng.uniform(0.05, 0.5, (nc, ne))
    gcore = rng.uniform(1.5, 4.0, (nc, ne))
    gtail = rng.uniform(1.5, 4.0, (nc, ne))
    pars = [ncore, ntail, score, stail, gcore, gtail]
    row = np.concatenate([10 ** eedges[:-1], 10 ** eedges[1:], cedges[:-1], cedges[1:]] + [p.ravel() for p in pars])
    ext = [ne, ne, nc, nc] + [nc * ne] * 6
    off = np.cumsum([0] + ext[:-1])
    return ext, off, row.astype(np.float32)


def make_job(name: str = "c1", seed: int = 1, n_sources: int | None = None) -> PointSourceJob:
    """Build the seeded synthetic job of one configuration (c0, c1, c2, c4)."""
    cfg = CONFIGS[name]
    rng = np.random.default_rng(seed)
    n = cfg["npix"]
    wcs = Wcs(n, n, (n + 1) / 2.0, (n + 1) / 2.0, CENTER[0], CENTER[1], -cfg["pix"], cfg["pix"], proj="CAR")
    energies = np.logspace(np.log10(cfg["emin"]), np.log10(cfg["emax"]), cfg["E"])
    logEs = np.log10(energies)
    nside = cfg["nside"]
    npix = 12 * nside * nside
    base = 2.0e5 * rng.lognormal(0.0, 0.2, (npix, 40))
    cube = base.astype(np.float32)
    wcube = (0.9 * base).astype(np.float32)
    exp_cube = ExpCube(cube, nside, 40, 0.0, True)
    wexp_cube = ExpCube(wcube, nside, 40, 0.0, True)
    aeff_f = prepare_grid(*_aeff_row(rng, True))
    aeff_b = prepare_grid(*_aeff_row(rng, False))
    effic = IrfEffic(np.array([-2.2, 6.0, -0.53, 2.34, -0.073, 3.5], np.float32),
                     np.array([2.0, -4.45, 0.475, 2.34, 0.066, 3.5], np.float32))
    sc_f = IrfScale(float(np.float32(0.06)), float(np.float32(0.0012)), float(np.float32(-0.8)))
    sc_b = IrfScale(float(np.float32(0.12)), float(np.float32(0.0022)), float(np.float32(-0.8)))
    rpsf_f = prepare_grid(*_king_row(rng, sc_f, True))
    rpsf_b = prepare_grid(*_king_row(rng, sc_b, False))
    S = cfg["S"] if n_sources is None else int(n_sources)
    half = cfg["field"] / 2.0
    cut = None
    if name == "c0":
        phi = np.zeros(S)
        th = np.zeros(S)
    elif name == "c2":
        edge = n * cfg["pix"] / 2.0
        k = max(1, S // 10)
        phi = rng.uniform(-edge + 1.0, edge - 1.0, S)
        th = rng.uniform(-edge + 1.0, edge - 1.0, S)
        side = rng.integers(0, 4, k)
        off = rng.uniform(-1.0, 1.0, k) + edge
        along = rng.uniform(-edge, edge, k)
        phi[:k] = np.where(side == 0, off, np.where(side == 1, -off, along))
        th[:k] = np.where(side == 2, off, np.where(side == 3, -off, along))
        cut = rng.uniform(2.0, 15.0, S)
    else:
        phi = rng.uniform(-half, half, S)
        th = rng.uniform(-half, half, S)
    ra, dec = native_to_celestial(wcs, phi, th)
    src = np.stack([ra, dec], axis=1)
    names = ["SRC%05d" % i for i in range(S)]
    return PointSourceJob(name, wcs, energies, logEs, exp_cube, wexp_cube, aeff_f, aeff_b, effic,
                          rpsf_f, rpsf_b, sc_f, sc_b, src, names, cut)
