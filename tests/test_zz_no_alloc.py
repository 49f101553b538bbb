"""The no-allocation mean-PSF entry point, xts_compute_psf_data_noalloc.

It serves callers that may not allocate device memory while they run: work
recorded into a stream capture, a service whose own memory pool owns the GPU, a
real-time loop.  Its King and psf*aeff scratch sit in one fixed device array
shared by every call, so this test makes two calls in a row with different
sources and checks each against xts_compute_psf_data (which allocates its
scratch) within the mean-PSF tolerance of the parity tests (1e-11 relative);
the second call would show stale scratch from the first.  It also checks that a
shape larger than the fixed scratch is refused before anything is launched.

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
