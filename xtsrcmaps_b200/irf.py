"""Host-side IRF table preparation (the reference's irf/ ingest, in numpy).

These are the host steps that turn the raw rows of a Pass-8 IRF FITS table into
the padded grids the kernels consume.  They run once per job, on the host, just
as in the reference (irf/irf.collect_irf_data.cpp:3-19).  The heavy per-source
work happens in the CUDA library.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class IrfGrid:
    """One padded IRF grid (irf/irf_types.hxx:11-16, ``IrfData3``).

    cosths: [Mc] cos-theta bin centres, padded with -1 and +1 at the ends.
    logEs:  [Me] log10(E/MeV) bin centres, padded with 0 and 10 at the ends.
    params: [Mc, Me, Ngrids] parameter values, edge rows/columns duplicated.
    min_cos_theta: the lowest cos-theta bin edge of the raw table.
    """

    cosths: np.ndarray
    logEs: np.ndarray
    params: np.ndarray
    min_cos_theta: float


@dataclass
class IrfScale:
    """PSF_SCALING_PARAMS row (irf/irf_types.hxx:18-22); float32 as in FITS."""

    scale0: float
    scale1: float
    scale_index: float


@dataclass
class IrfEffic:
    """EFFICIENCY_PARAMS rows p0, p1 (irf/irf_types.hxx:24-27); float32 [6] each."""

    p0: np.ndarray
    p1: np.ndarray


def prepare_grid(extents, offsets, row) -> IrfGrid:
    """Pad and reshape one raw IRF row (irf/irf.prepare_grid.cpp:26-102).

    ``row`` is the float32 FITS row: columns ENERG_LO, ENERG_HI, CTHETA_LO,
    CTHETA_HI, then one column per parameter over the (cos-theta, energy) grid
    with energy fastest.  Cos-theta centres are the float sums halved; log-energy
    centres are 0.5 * log10 of the float product, with log10 taken in float as
    the reference's ``std::log10(float)`` does.
    """
    ext = [int(x) for x in extents]
    off = [int(x) for x in offsets]
    row = np.asarray(row, dtype=np.float32)
    if len(ext) < 5 or ext[0] != ext[1] or ext[2] != ext[3] or ext[4] != ext[0] * ext[2]:
        raise ValueError("malformed IRF table extents %r" % (ext,))
    me_b, mt_b = ext[0], ext[2]
    me, mt = me_b + 2, mt_b + 2
    c0 = row[off[2]:off[2] + mt_b]
    c1 = row[off[3]:off[3] + mt_b]
    cos = np.empty(mt, dtype=np.float64)
    cos[1:mt_b + 1] = 0.5 * (c0 + c1).astype(np.float64)
    cos[0], cos[-1] = -1.0, 1.0
    e0 = row[off[0]:off[0] + me_b]
    e1 = row[off[1]:off[1] + me_b]
    loge = np.empty(me, dtype=np.float64)
    loge[1:me_b + 1] = 0.5 * np.log10((e0 * e1).astype(np.float32)).astype(np.float64)
    loge[0], loge[-1] = 0.0, 10.0
    ngrids = len(ext) - 4
    pv = row[off[4]:off[4] + ngrids * mt_b * me_b].reshape(ngrids, mt_b, me_b)
    ti = np.clip(np.arange(mt) - 1, 0, mt_b - 1)
    ei = np.clip(np.arange(me) - 1, 0, me_b - 1)
    params = pv[:, ti][:, :, ei].transpose(1, 2, 0).astype(np.float64)
    return IrfGrid(cos, loge, np.ascontiguousarray(params), float(row[off[2]]))


def prepare_scale(row) -> IrfScale:
    """irf/irf.prepare_scale.cpp:5-13."""
    r = np.asarray(row, dtype=np.float32)
    return IrfScale(float(r[0]), float(r[1]), float(r[2]))


def prepare_effic(p0, p1) -> IrfEffic:
    """irf/irf.prepare_effic.cpp:6-22."""
    return IrfEffic(np.asarray(p0, dtype=np.float32), np.asarray(p1, dtype=np.float32))


@dataclass
class IrfSide:
    """One event class side of an IRF file: the grids the reference keeps in
    ``aeff::Data`` / ``psf::Data`` (irf/irf_types.hxx)."""

    grid: IrfGrid               # EFFECTIVE AREA or RPSF (raw, not normalised)
    second: IrfGrid             # PHI_DEPENDENCE or FISHEYE_CORRECTION (loaded, unused on the path)
    effic: IrfEffic | None = None   # EFFICIENCY_PARAMS (aeff files)
    scale: IrfScale | None = None   # PSF_SCALING_PARAMS (psf files)


def _grid(path: str, table: str) -> IrfGrid:
    from .fits_io import read_irf_pars

    ext, off, rows = read_irf_pars(path, table)
    return prepare_grid(ext, off, rows[0])


def load_aeff(path: str) -> dict:
    """Fermi::Irf::load_aeff (irf/irf.cxx:24-46) and prepare_aeff_data
    (irf/irf.prepare_aeff_data.cpp:7-23): front and back EFFECTIVE AREA and
    PHI_DEPENDENCE grids and the two EFFICIENCY_PARAMS rows."""
    from .fits_io import read_irf_pars

    out = {}
    for side in ("FRONT", "BACK"):
        ext, _, rows = read_irf_pars(path, f"EFFICIENCY_PARAMS_{side}")
        if list(ext) != [6] or rows.shape != (2, 6):
            raise ValueError(f"{path}: EFFICIENCY_PARAMS_{side} must be 2 rows of 6 (irf.prepare_effic.cpp:8-10)")
        out[side.lower()] = IrfSide(_grid(path, f"EFFECTIVE AREA_{side}"), _grid(path, f"PHI_DEPENDENCE_{side}"),
                                    effic=prepare_effic(rows[0], rows[1]))
    return out


def load_psf(path: str) -> dict:
    """Fermi::Irf::load_psf (irf/irf.cxx:48-70) and prepare_psf_data
    (irf/irf.prepare_psf_data.cpp:6-25) up to the normalisation: front and back
    RPSF and FISHEYE_CORRECTION grids and the PSF_SCALING_PARAMS row.  The King
    grids are normalised by the library (``api.normalize_rpsf``, the reference's
    irf/irf.normalize_rpsf.cpp:11-61)."""
    from .fits_io import read_irf_pars

    out = {}
    for side in ("FRONT", "BACK"):
        _, _, rows = read_irf_pars(path, f"PSF_SCALING_PARAMS_{side}")
        if rows.shape != (1, 3):
            raise ValueError(f"{path}: PSF_SCALING_PARAMS_{side} must be 1 row of 3 (irf.prepare_scale.cpp:7-8)")
        out[side.lower()] = IrfSide(_grid(path, f"RPSF_{side}"), _grid(path, f"FISHEYE_CORRECTION_{side}"),
                                    scale=prepare_scale(rows[0]))
    return out
