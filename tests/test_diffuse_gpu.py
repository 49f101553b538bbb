"""The diffuse-map steps on the GPU against the FP64 oracle: the PSF kernel image
(xts_make_psf_kernel) and the per-plane FFT convolution (xts_convolve_map_psf)."""
import numpy as np
import pytest

from helpers import max_rel
from oracle import diffuse_oracle as D

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


@pytest.fixture(scope="module")
def upsf(api):
    """A real mean-PSF table: source 0 of a c0 job through the GPU pipeline."""
    from xtsrcmaps_b200.synth import make_job

    job = make_job("c0", seed=3)
    ltf = api.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = api.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = api.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = api.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front, job.aeff_back, ltf)
    return np.ascontiguousarray(api.compute_psf_data(nf, nb, ex, job.logEs, ltf).uPsf[0])


@pytest.mark.parametrize("proj,Nk,pix", [("CAR", 41, 0.05), ("AIT", 25, 0.2)])
def test_psf_kernel_image(api, upsf, proj, Nk, pix):
    from xtsrcmaps_b200.wcs import Wcs

    w = Wcs(Nk, Nk, (Nk + 1) / 2, (Nk + 1) / 2, 193.98, -5.82, -pix, pix, proj=proj)
    k = api.make_psf_kernel(w, Nk, upsf)
    ref = D.make_kernel(w, Nk, upsf)
    assert k.shape == ref.shape == (upsf.shape[1], Nk, Nk)
    assert max_rel(k, ref) < 1e-12
    np.testing.assert_allclose(k.sum(axis=(1, 2)), 1.0, rtol=1e-13)


def test_fft_convolution(api, upsf):
    import torch

    from xtsrcmaps_b200.wcs import Wcs

    rng = np.random.default_rng(4)
    E = upsf.shape[1]
    img = rng.lognormal(0.0, 1.0, (E, 67, 45))
    w = Wcs(21, 21, 11, 11, 193.98, -5.82, -0.1, 0.1, proj="CAR")
    ker = D.make_kernel(w, 21, upsf)
    out = api.convolve_map_psf(img, ker)
    ref = D.convolve_full(img, ker)
    assert out.shape == ref.shape == (E, 87, 65)
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()
    d = torch.device("cuda")
    outd = api.convolve_map_psf(torch.as_tensor(img, device=d), torch.as_tensor(ker, device=d))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(outd.cpu().numpy(), out)
    # a second shape re-plans; a delta kernel returns the image
    delta = np.zeros((E, 5, 5))
    delta[:, 0, 0] = 1.0
    o2 = api.convolve_map_psf(img[:, :30, :20], delta)
    assert np.abs(o2[:, :30, :20] - img[:, :30, :20]).max() <= 1e-12 * img.max()
    assert np.abs(o2[:, 30:, :]).max() <= 1e-12 * img.max()


def test_diffuse_argument_errors(api, upsf):
    """Shape errors come back as XTS_ERR_ARG, before any launch."""
    from xtsrcmaps_b200 import _lib
    from xtsrcmaps_b200.wcs import Wcs

    w = Wcs(20, 20, 10.5, 10.5, 193.98, -5.82, -0.1, 0.1, proj="CAR")
    with pytest.raises(_lib.XtsError) as ei:
        api.make_psf_kernel(w, 20, upsf)  # even kernel size
    assert ei.value.code == _lib.XTS_ERR_ARG
    with pytest.raises(ValueError):
        api.convolve_map_psf(np.zeros((2, 8, 8)), np.zeros((3, 5, 5)))  # energies differ


def test_trilerp_crop_rebin_on_gpu(api):
    """trilerpEHW on the device against the float32 oracle (a few ulps: the device
    contracts a * b + c * d into FMAs); the all-sky crop (with the seam wrap) and
    the crop range and rebinned WCS bit for bit."""
    import torch

    from xtsrcmaps_b200.wcs import Wcs

    rng = np.random.default_rng(8)
    src = rng.lognormal(0.0, 1.0, (6, 31, 45)).astype(np.float32)
    for shape in ((11, 91, 133), (6, 31, 45), (1, 16, 16)):
        got = api.trilerp_ehw(src, shape)
        ref = D.trilerp_ehw(src, shape)
        assert got.shape == ref.shape
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=0)
    d = torch.device("cuda")
    gd = api.trilerp_ehw(torch.as_tensor(src, device=d), (11, 91, 133))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(gd.cpu().numpy(), api.trilerp_ehw(src, (11, 91, 133)))

    roi = Wcs(100, 80, 50.5, 40.5, 193.98, -5.82, -0.2, 0.2, proj="CAR")
    r = api.rebin_wcs(roi, 0.05)
    o = D.rebin_wcs(roi, 0.05)
    assert (r.naxis1, r.naxis2, r.crpix1, r.crpix2, r.cdelt1, r.cdelt2) == \
        (o.naxis1, o.naxis2, o.crpix1, o.crpix2, o.cdelt1, o.cdelt2)
    sky = Wcs(720, 361, 360.5, 181.0, 0.0, 0.0, -0.5, 0.5, proj="CAR")
    rng_ = api.allsky_crop_range(sky, roi)
    assert rng_ == D.allsky_crop_range(sky, roi)
    cube = rng.lognormal(0.0, 1.0, (4, 361, 720)).astype(np.float32)
    np.testing.assert_array_equal(api.crop_allsky(cube, rng_), D.crop_allsky(cube, rng_))
    wrap = (700, 15, 100, 140)  # across the longitude seam
    np.testing.assert_array_equal(api.crop_allsky(cube, wrap), D.crop_allsky(cube, wrap))
    from xtsrcmaps_b200 import _lib

    with pytest.raises(_lib.XtsError) as ei:
        api.crop_allsky(cube, (0, 5, 1, 2))  # outside the image
    assert ei.value.code == _lib.XTS_ERR_ARG


def test_scale_model_map_matches_oracle_and_point_path(api):
    """The diffuse map's final scalings on pixel means: against the FP64 oracle of
    the same scalings (1e-6 on the FP32 map, 1e-7 on 1 / map integral), and, fed the
    point-source path's own pixel means, equal to that path's model map (1e-5)."""
    import torch

    from oracle import oracle as O
    from xtsrcmaps_b200.synth import make_job
    from xtsrcmaps_b200.wcs import Wcs

    job = make_job("c1", seed=12, n_sources=4)
    job.wcs = Wcs(60, 50, 30.5, 25.5, job.wcs.crval1, job.wcs.crval2, -0.2, 0.2, proj="CAR")
    src = np.array(job.wcs.crval1 + np.array([0.0, 1.3, -2.0, 7.9]))
    job.src_sph = np.stack([src, job.wcs.crval2 + np.array([0.0, -0.8, 1.1, 0.2])], axis=1)
    ltf = api.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = api.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = api.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = api.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front,
                              job.aeff_back, ltf)
    ps = api.compute_psf_data(nf, nb, ex, job.logEs, ltf)
    means = O.cubature_map(job.wcs, job.src_sph, ps.uPsf)  # FP64 pixel means of the 12-point rule
    m, info = api.scale_model_map(job.wcs, job.src_sph, ex.exposure, ps.uPsf, ps.partial_psf_integral,
                                  means.astype(np.float32))
    ref, inv, fac, rad, fov = D.scale_model_map(job.wcs, job.src_sph, ex.exposure, ps.uPsf,
                                                ps.partial_psf_integral, means.astype(np.float32))
    assert max_rel(m, ref) < 1e-6
    assert max_rel(info.inv_map_integral, inv) < 1e-7 and max_rel(info.correction, fac) < 1e-7
    np.testing.assert_array_equal(info.in_fov.astype(bool), fov)
    point, pinfo = api.point_src_model_map_wcs(job.wcs, job.src_sph, ex.exposure, ps.uPsf, ps.partial_psf_integral)
    assert max_rel(m, point) < 1e-5
    assert max_rel(info.inv_map_integral, pinfo.inv_map_integral) < 1e-7
    # device pointers: scaled in place
    d = torch.device("cuda")
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=d)
    md = t(means.astype(np.float32))
    out, _ = api.scale_model_map(job.wcs, t(job.src_sph), t(ex.exposure), t(ps.uPsf), t(ps.partial_psf_integral),
                                 md, with_info=False)
    torch.cuda.synchronize()
    assert out.data_ptr() == md.data_ptr()
    assert max_rel(md.cpu().numpy(), m) < 1e-7
