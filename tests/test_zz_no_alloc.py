"""The no-allocation mean-PSF entry point, xts_compute_psf_data_noalloc.

It serves callers that may not allocate device memory while they run: work
recorded into a stream capture, a service whose own memory pool owns the GPU, a
real-time loop.  Its King and psf*aeff scratch sit in one fixed device array
shared by every call, so this test makes two calls in a row with different
sources and checks each against xts_compute_psf_data (which allocates its
scratch) within the mean-PSF tolerance of the parity tests (1e-11 relative);
the second call would show stale scratch from the first.  It also checks that a
shape larger than the fixed scratch is refused before anything is launched, and
the exact limit: the King tables are padded to a multiple of 32 doubles before
the psf*aeff table, and the largest shape whose padded layout fits is accepted
(and matches), while the next larger one is refused.  Every scratch size is a
multiple of 401 doubles, so no shape can fit unpadded yet overflow by the
padding alone: the limit is tested where it binds.

The file is named to be collected last, so that a run stopping at its first
failure has already run every other test; it also passes alone in a fresh
process.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import max_rel

pytestmark = pytest.mark.gpu

ND = 401


def _vp(t):
    return C.c_void_p(t.data_ptr())


def test_psf_noalloc_matches_compute_psf_data_on_two_calls():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from xtsrcmaps_b200 import _lib as L
    from xtsrcmaps_b200 import api as A
    from xtsrcmaps_b200 import build
    from xtsrcmaps_b200.synth import make_job

    build.build()
    A.init(0)
    lib = L.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)

    for seed, n in ((21, 7), (22, 12)):
        job = make_job("c1", seed=seed, n_sources=n)
        ltf = A.livetime_efficiency_factors(job.logEs, job.effic_front)
        nf = A.normalize_rpsf(job.rpsf_front, job.scale_front)
        nb = A.normalize_rpsf(job.rpsf_back, job.scale_back)
        ex = A.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front,
                                job.aeff_back, ltf)
        ref = A.compute_psf_data(nf, nb, ex, job.logEs, ltf)  # the allocating entry point

        c = A._Call(True, torch.empty(0, device=dev))
        gf, gb = c.grid(nf, 6), c.grid(nb, 6)
        d = {k: torch.as_tensor(np.ascontiguousarray(v), dtype=torch.float64, device=dev)
             for k, v in dict(costh=ex.exp_costhetas, logEs=job.logEs, af=ex.front_aeff,
                              ab=ex.back_aeff, ecb=ex.src_exposure_cosbins,
                              wecb=ex.src_weighted_exposure_cosbins, ltf=ltf,
                              exposure=ex.exposure).items()}
        S, E, Cn = int(d["ecb"].shape[0]), int(d["logEs"].numel()), int(d["costh"].numel())
        upsf = torch.full((S, ND, E), float("nan"), dtype=torch.float64, device=dev)
        part = torch.full((S, ND, E), float("nan"), dtype=torch.float64, device=dev)
        stream.wait_stream(torch.cuda.current_stream(dev))
        rc = lib.xts_compute_psf_data_noalloc(
            C.byref(gf), C.byref(gb), _vp(d["costh"]), Cn, _vp(d["logEs"]), E, _vp(d["af"]),
            _vp(d["ab"]), _vp(d["ecb"]), _vp(d["wecb"]), S, _vp(d["ltf"]), _vp(d["exposure"]),
            _vp(upsf), _vp(part), C.c_void_p(stream.cuda_stream))
        L.check(rc)
        stream.synchronize()
        assert max_rel(upsf.cpu().numpy(), ref.uPsf) < 1e-11
        assert max_rel(part.cpu().numpy(), ref.partial_psf_integral, floor=1e-300) < 1e-11

    # A shape beyond the fixed scratch (C * 401 * E doubles alone > 2^20) is refused
    # on the host with XTS_ERR_ARG; nothing is launched, so the small buffers
    # passed here are never read.
    big_e = 64
    rc = lib.xts_compute_psf_data_noalloc(
        C.byref(gf), C.byref(gb), _vp(d["costh"]), 48, _vp(d["logEs"]), big_e, _vp(d["af"]),
        _vp(d["ab"]), _vp(d["ecb"]), _vp(d["wecb"]), S, _vp(d["ltf"]), _vp(d["exposure"]),
        _vp(upsf), _vp(part), C.c_void_p(stream.cuda_stream))
    assert rc == L.XTS_ERR_ARG
    assert "scratch" in lib.xts_last_error().decode()


def _resampled(grid, n_cos, n_e):
    """A King grid of the same parameter surface on n_cos x n_e nodes (bilinear)."""
    from xtsrcmaps_b200.irf import IrfGrid

    c0, e0, p0 = np.asarray(grid.cosths), np.asarray(grid.logEs), np.asarray(grid.params)
    cn = np.linspace(c0[0], c0[-1], n_cos)
    en = np.linspace(e0[0], e0[-1], n_e)
    tmp = np.stack([np.stack([np.interp(en, e0, p0[i, :, k]) for k in range(6)], axis=-1)
                    for i in range(len(c0))])                      # [Mc0, n_e, 6]
    out = np.stack([np.stack([np.interp(cn, c0, tmp[:, j, k]) for k in range(6)], axis=-1)
                    for j in range(n_e)], axis=1)                  # [n_cos, n_e, 6]
    return IrfGrid(cn, en, np.ascontiguousarray(out), grid.min_cos_theta)


def test_psf_noalloc_scratch_limit():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from xtsrcmaps_b200 import _lib as L
    from xtsrcmaps_b200 import api as A
    from xtsrcmaps_b200 import build
    from xtsrcmaps_b200.synth import make_job

    build.build()
    A.init(0)
    lib = L.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    limit = int(L.NOALLOC_SCRATCH_DOUBLES)

    job = make_job("c1", seed=23, n_sources=5)
    ltf = A.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = A.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = A.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = A.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front,
                            job.aeff_back, ltf)
    Cn, E = len(ex.exp_costhetas), len(job.logEs)
    kf = nf.params.shape[0] * nf.params.shape[1]
    pa_n = Cn * ND * E

    def padded(k):
        return (ND * k + 31) // 32 * 32 + pa_n

    # the largest King node count whose padded layout fits, and a back grid with it
    k_fit = max(k for k in range(kf + 4, limit // ND) if padded(k) <= limit)
    assert padded(k_fit + 1) > limit
    kb = k_fit - kf
    shape = next((a, kb // a) for a in range(4, 64) if kb % a == 0 and kb // a >= 4)
    assert (ND * k_fit) % 32 != 0  # the padding is non-zero at the binding shape
    nb_fit = _resampled(nb, *shape)
    ref = A.compute_psf_data(nf, nb_fit, ex, job.logEs, ltf)  # the allocating entry point

    c = A._Call(True, torch.empty(0, device=dev))
    gf, gb = c.grid(nf, 6), c.grid(nb_fit, 6)
    d = {k: torch.as_tensor(np.ascontiguousarray(v), dtype=torch.float64, device=dev)
         for k, v in dict(costh=ex.exp_costhetas, logEs=job.logEs, af=ex.front_aeff,
                          ab=ex.back_aeff, ecb=ex.src_exposure_cosbins,
                          wecb=ex.src_weighted_exposure_cosbins, ltf=ltf,
                          exposure=ex.exposure).items()}
    S = int(d["ecb"].shape[0])
    upsf = torch.full((S, ND, E), float("nan"), dtype=torch.float64, device=dev)
    part = torch.full((S, ND, E), float("nan"), dtype=torch.float64, device=dev)
    stream.wait_stream(torch.cuda.current_stream(dev))

    def call(grid_b):
        return lib.xts_compute_psf_data_noalloc(
            C.byref(gf), C.byref(grid_b), _vp(d["costh"]), Cn, _vp(d["logEs"]), E, _vp(d["af"]),
            _vp(d["ab"]), _vp(d["ecb"]), _vp(d["wecb"]), S, _vp(d["ltf"]), _vp(d["exposure"]),
            _vp(upsf), _vp(part), C.c_void_p(stream.cuda_stream))

    L.check(call(gb))
    stream.synchronize()
    assert max_rel(upsf.cpu().numpy(), ref.uPsf) < 1e-11
    assert max_rel(part.cpu().numpy(), ref.partial_psf_integral, floor=1e-300) < 1e-11

    # one King node more no longer fits: refused on the host, nothing launched
    # (only the grid's sizes are read before the refusal)
    over = (2, (kb + 2) // 2)  # 2 * ((kb + 2) // 2) = kb + 1 or kb + 2 nodes
    gb_over = L.XtsGrid(gb.cosths, over[0], gb.logEs, over[1], gb.params, 6, gb.min_cos_theta)
    assert call(gb_over) == L.XTS_ERR_ARG
    msg = lib.xts_last_error().decode()
    assert "scratch" in msg and str(padded(kf + over[0] * over[1])) in msg
