"""Shared test helpers: the oracle pipeline over a synthetic job and error metrics."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from xtsrcmaps_b200.irf import IrfGrid


def oracle_pipeline(job, with_map: bool = True):
    """Run the FP64 oracle over a synthetic job (main.cxx:27-31 order)."""
    cube, wcube = job.exp_cube, job.wexp_cube
    cos = O.costhetas(cube.nbrbins, cube.cosmin, cube.thetabin)
    ecb = O.src_cosbins(job.src_sph, cube.cosbins, cube.nside) if job.S else np.zeros((0, cube.nbrbins))
    wecb = O.src_cosbins(job.src_sph, wcube.cosbins, wcube.nside) if job.S else np.zeros((0, cube.nbrbins))
    af = O.aeff_value(cos, job.logEs, job.aeff_front)
    ab = O.aeff_value(cos, job.logEs, job.aeff_back)
    ltf = O.livetime_efficiency_factors(job.logEs, job.effic_front.p0, job.effic_front.p1)
    expo = O.exposure(ecb, wecb, af, ab, ltf)
    nf = normalized(job.rpsf_front, job.scale_front)
    nb = normalized(job.rpsf_back, job.scale_back)
    upsf, partial = O.compute_psf_data(nf, nb, cos, job.logEs, af, ab, ecb, wecb, ltf, expo)
    out = dict(costh=cos, ecb=ecb, wecb=wecb, af=af, ab=ab, ltf=ltf, exposure=expo, nf=nf, nb=nb,
               upsf=upsf, partial=partial)
    if with_map:
        out.update(O.point_src_model_map_wcs(job.wcs, job.src_sph, expo, upsf, partial))
    return out


def irf_setup(job):
    """IRF set-up outside the timed path (Irf::collect_irf_data): livetime
    efficiency factors and normalised King grids, with the FP64 oracle."""
    ltf = O.livetime_efficiency_factors(job.logEs, job.effic_front.p0, job.effic_front.p1)
    return ltf, normalized(job.rpsf_front, job.scale_front), normalized(job.rpsf_back, job.scale_back)


def reference_pipeline(job, setup=None, with_map: bool = True, times=None):
    """The same steps through the reference's own code compiled under oracle/_ref
    (oracle/oracle_ref.py): exposure, mean PSF and the model map.  The effective
    area tables come from the oracle's restatement of Irf::aeff_value, whose
    reference translation unit needs <mdspan>.  times (a dict) accumulates the
    seconds of compute_exposure, compute_psf_data and point_src_model_map_wcs."""
    import time

    from oracle import oracle_ref as R

    ltf, nf, nb = setup if setup is not None else irf_setup(job)
    cube, wcube = job.exp_cube, job.wexp_cube
    t0 = time.perf_counter()
    cos = O.costhetas(cube.nbrbins, cube.cosmin, cube.thetabin)
    af = O.aeff_value(cos, job.logEs, job.aeff_front)
    ab = O.aeff_value(cos, job.logEs, job.aeff_back)
    cos, ecb, wecb, expo = R.exposure(cube.cosbins, wcube.cosbins, cube.nside, cube.cosmin, cube.thetabin,
                                      job.src_sph, af, ab, ltf)
    t1 = time.perf_counter()
    upsf, partial = R.psf(nf, nb, cos, job.logEs, af, ab, ecb, wecb, ltf, expo)
    t2 = time.perf_counter()
    out = dict(costh=cos, ecb=ecb, wecb=wecb, af=af, ab=ab, ltf=ltf, exposure=expo, upsf=upsf, partial=partial)
    if with_map:
        out["map"] = R.point_src_model_map_wcs(job.wcs, job.src_sph, expo, upsf, partial)
    t3 = time.perf_counter()
    if times is not None:
        for k, v in (("compute_exposure", t1 - t0), ("compute_psf_data", t2 - t1), ("point_src_model_map_wcs", t3 - t2)):
            times[k] = times.get(k, 0.0) + v
    return out


def normalized(grid: IrfGrid, scale) -> IrfGrid:
    p = O.normalize_rpsf(grid.params, grid.logEs, scale.scale0, scale.scale1, scale.scale_index)
    return IrfGrid(grid.cosths, grid.logEs, p, grid.min_cos_theta)


def max_rel(a, b, floor: float = 0.0) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(b), floor)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(den > 0, np.abs(a - b) / den, np.abs(a - b))
    return float(r.max()) if r.size else 0.0
