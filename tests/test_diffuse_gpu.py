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
