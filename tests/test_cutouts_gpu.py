"""Cutout maps on the GPU against the FP64 oracle of the same windows: every
source's ragged block is the reference's model map of its window's sub-map
(oracle.point_src_model_map_cutouts).  Tolerances as the dense map: 1e-5 per
value, 1e-7 on 1 / map integral and the correction; radii 1e-13 and in-FOV flags
exact.  Small job with sources by and beyond the edge, then the c2 job (500
sources, its cutout radii) on sampled sources."""
import numpy as np
import pytest

from helpers import max_rel
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from xtsrcmaps_b200 import api as A
    from xtsrcmaps_b200 import build

    build.build()
    A.init(0)
    return A


def _tables(A, job):
    ltf = A.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = A.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = A.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = A.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front, job.aeff_back, ltf)
    ps = A.compute_psf_data(nf, nb, ex, job.logEs, ltf)
    return ex.exposure, ps.uPsf, ps.partial_psf_integral


def _check(got, info, ref, cut, idx=None):
    idx = range(len(cut)) if idx is None else idx
    for s in idx:
        h0, w0, nh, nw, off = (int(v) for v in cut[s])
        if nh * nw == 0:
            continue
        assert max_rel(got[off:off + nh * nw], ref["map"][off:off + nh * nw]) < 1e-5, s
    i = np.asarray(list(idx))
    assert max_rel(info.inv_map_integral[i], ref["inv_integ"][i]) < 1e-7
    assert max_rel(info.correction[i], ref["factor"][i]) < 1e-7
    np.testing.assert_array_equal(info.in_fov[i].astype(bool), ref["in_fov"][i])
    assert max_rel(info.psf_radius[i], ref["radius"][i]) < 1e-12


def test_cutouts_small_vs_oracle(api):
    import torch

    from xtsrcmaps_b200.synth import make_job
    from xtsrcmaps_b200.wcs import Wcs

    job = make_job("c1", seed=31, n_sources=9)
    job.wcs = Wcs(70, 60, 35.5, 30.5, job.wcs.crval1, job.wcs.crval2, -0.2, 0.2, proj="CAR")
    pix = [(35.5, 30.5), (3.0, 4.0), (69.0, 58.0), (80.0, 30.0), (35.0, -6.0), (10.2, 50.7), (60.1, 12.3),
           (200.0, 200.0), (36.0, 31.0)]
    job.src_sph = np.array([O.pix2sph(job.wcs, p1, p2) for p1, p2 in pix])
    radii = np.array([3.0, 2.0, 4.0, 5.0, 1.5, 0.6, 2.5, 3.0, 8.0])
    expo, upsf, partial = _tables(api, job)
    cut, total = api.cutout_windows(job.wcs, job.src_sph, radii)
    ref = O.point_src_model_map_cutouts(job.wcs, job.src_sph, cut, expo, upsf, partial)
    got, info = api.point_src_model_map_cutouts(job.wcs, job.src_sph, cut, expo, upsf, partial)
    assert got.shape == (total, job.E)
    _check(got, info, ref, cut)
    # device pointers, twice (the work queue restarts at zero each call)
    d = torch.device("cuda")
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=d)
    for _ in range(2):
        gd, infod = api.point_src_model_map_cutouts(job.wcs, t(job.src_sph), cut, t(expo), t(upsf), t(partial))
        torch.cuda.synchronize()
        assert max_rel(gd.cpu().numpy(), got) < 1e-6
        assert max_rel(infod.inv_map_integral.cpu().numpy(), info.inv_map_integral) < 1e-12


def test_cutouts_c2_sampled_sources(api):
    import torch

    from xtsrcmaps_b200.synth import make_job

    job = make_job("c2", seed=11)
    expo, upsf, partial = _tables(api, job)
    cut, total = api.cutout_windows(job.wcs, job.src_sph, job.cutout_deg)
    d = torch.device("cuda")
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=d)
    got, info = api.point_src_model_map_cutouts(job.wcs, t(job.src_sph), cut, t(expo), t(upsf), t(partial))
    torch.cuda.synchronize()
    idx = np.unique(np.linspace(0, job.S - 1, 12).round().astype(int))
    sub_cut = cut[idx].copy()
    sub_cut["offset"] = np.concatenate([[0], np.cumsum(sub_cut["nh"].astype(np.int64) * sub_cut["nw"])[:-1]])
    ref = O.point_src_model_map_cutouts(job.wcs, job.src_sph[idx], sub_cut, expo[idx], upsf[idx], partial[idx])
    g = got.cpu().numpy()
    for k, s in enumerate(idx):
        h0, w0, nh, nw, off = (int(v) for v in cut[s])
        o2 = int(sub_cut[k]["offset"])
        if nh * nw:
            assert max_rel(g[off:off + nh * nw], ref["map"][o2:o2 + nh * nw]) < 1e-5, s
    inv = info.inv_map_integral.cpu().numpy()[idx]
    assert max_rel(inv, ref["inv_integ"]) < 1e-7
    assert max_rel(info.correction.cpu().numpy()[idx], ref["factor"]) < 1e-7
    assert np.isfinite(g).all() and (g >= 0).all()
