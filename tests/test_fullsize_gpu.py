"""The source-map path at the configured full sizes: c2 (500 sources, CAR 400x400
@ 0.05 deg, 37 energies, 10% of the sources within 1 deg of the map edge or
just outside; 11.8 GB of maps) and c4 (2000 sources, CAR 800x800 @ 0.025 deg,
50 energies; 256 GB of maps, run in chunks of sources).

Two checks that do not need the oracle on the whole job:
  * a property of the normalisation (c7, c9): with factor = integ / sum, the
    map summed over the pixels inside the boundary radius equals
    exposure * correction / inv_map_integral for every in-FOV source and energy;
  * the full end-to-end comparison with the FP64 oracle (1e-5 per pixel) for a
    few sampled sources, edge-placed ones included.
"""
import numpy as np
import pytest

from helpers import max_rel, oracle_pipeline

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


def _centres(wcs):
    """Unit vectors of the pixel centres (h + 1, w + 1), the points the map
    integral tests against the boundary radius (model_map.map_integral.cxx:25-31)."""
    from oracle import oracle as O

    H, W = int(wcs.naxis1), int(wcs.naxis2)
    d = np.empty((H * W, 3))
    for h in range(H):
        for w in range(W):
            ra, dec = np.radians(O.pix2sph(wcs, h + 1.0, w + 1.0))
            d[h * W + w] = (np.cos(dec) * np.cos(ra), np.cos(dec) * np.sin(ra), np.sin(dec))
    return d


@pytest.mark.parametrize("name,chunk,samples", [("c2", 500, (0, 1, 57, 499)), ("c4", 100, (0, 1234))])
def test_full_size_maps(api, name, chunk, samples):
    import torch

    from xtsrcmaps_b200.synth import make_job

    job = make_job(name, seed=11)
    S, H, W, E = job.S, int(job.wcs.naxis1), int(job.wcs.naxis2), job.E
    dev = torch.device("cuda")
    ltf = api.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = api.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = api.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = api.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front, job.aeff_back, ltf)
    ps = api.compute_psf_data(nf, nb, ex, job.logEs, ltf)
    cen = torch.as_tensor(_centres(job.wcs), device=dev)
    out = torch.empty((chunk, H, W, E), dtype=torch.float32, device=dev)
    checked = 0
    for s0 in range(0, S, chunk):
        n = min(chunk, S - s0)
        sl = slice(s0, s0 + n)
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a[sl]), device=dev)
        m, info = api.point_src_model_map_wcs(job.wcs, t(job.src_sph), t(ex.exposure), t(ps.uPsf),
                                              t(ps.partial_psf_integral), out=out[:n])
        torch.cuda.synchronize()
        # normalisation property over the pixels inside each source's boundary radius
        ra, dec = np.radians(job.src_sph[sl, 0]), np.radians(job.src_sph[sl, 1])
        src = torch.as_tensor(np.stack([np.cos(dec) * np.cos(ra), np.cos(dec) * np.sin(ra), np.sin(dec)], 1),
                              device=dev)
        sep = 2.0 * torch.asin(0.5 * torch.cdist(src, cen).clamp(max=2.0))          # [n, npix]
        inside = (sep <= torch.deg2rad(info.psf_radius)[:, None]).to(torch.float64)
        sums = torch.bmm(inside[:, None, :], m[:n].view(n, H * W, E).to(torch.float64))[:, 0, :]
        inv, corr = info.inv_map_integral, info.correction
        fov = info.in_fov.bool()
        expect = torch.as_tensor(ex.exposure[sl], device=dev) * corr / torch.where(inv != 0, inv, torch.ones_like(inv))
        rel = ((sums - expect).abs() / expect.abs())[fov]
        assert rel.numel() == 0 or float(rel.max()) < 2e-5, (name, s0, float(rel.max()))
        # end to end against the FP64 oracle for the sampled sources of this chunk
        for s in [k for k in samples if s0 <= k < s0 + n]:
            sub = make_job(name, seed=11)
            sub.src_sph = job.src_sph[s:s + 1]
            ref = oracle_pipeline(sub)
            assert max_rel(m[s - s0].cpu().numpy(), ref["map"][0]) < 1e-5, (name, s)
            assert bool(info.in_fov[s - s0]) == bool(ref["in_fov"][0])
            checked += 1
    assert checked == len(samples)
