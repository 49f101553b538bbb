"""CPU-side checks of the boundary: the C-ABI library builds for sm_100a, loads,
exports every symbol include/xtsrcmaps_b200.h declares, and fails loudly (an
error code and message, no crash, no CPU fallback) when no GPU is present.
Plus the host logic: synthetic inputs and IRF preparation."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "xtsrcmaps_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(xts_[a-z0-9_]+)\s*\(", txt)))


def test_library_builds_and_exports_every_declared_symbol():
    from xtsrcmaps_b200 import _lib, build

    build.build()
    lib = _lib.lib()
    names = _declared()
    assert len(names) >= 8
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, n


def test_no_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from xtsrcmaps_b200 import _lib, api
    from xtsrcmaps_b200.synth import make_job

    lib = _lib.lib()
    rc = lib.xts_init(0)
    assert rc == _lib.XTS_ERR_NODEV
    assert lib.xts_last_error()
    job = make_job("c0")
    with pytest.raises(_lib.XtsError) as ei:
        api.livetime_efficiency_factors(job.logEs, job.effic_front)
    assert ei.value.code == _lib.XTS_ERR_NODEV


def test_synthetic_jobs_have_reference_shapes():
    from xtsrcmaps_b200.synth import make_job

    for name, (S, n, E, nside) in {"c0": (1, 100, 20, 32), "c1": (50, 200, 37, 64)}.items():
        job = make_job(name, seed=1)
        assert job.src_sph.shape == (S, 2)
        assert (job.wcs.naxis1, job.wcs.naxis2) == (n, n)
        assert job.E == E and len(job.logEs) == E
        assert job.exp_cube.cosbins.shape == (12 * nside * nside, 40)
        assert job.exp_cube.cosbins.dtype == np.float32
        assert job.aeff_front.params.shape == (34, 76, 1)
        assert job.rpsf_front.params.shape == (10, 25, 6)
        amax = job.aeff_front.params.max() * 1e4
        assert 7000 < amax < 10000  # "rising from 0 to about 9000 cm^2"
    j2 = make_job("c1", seed=1)
    assert np.array_equal(j2.src_sph, make_job("c1", seed=1).src_sph)  # seeded
    assert not np.array_equal(j2.src_sph, make_job("c1", seed=2).src_sph)


def test_synthetic_psf_widths_follow_the_spec():
    """score*sf in radians log-decreasing from 5 deg to 0.05 deg with energy."""
    from oracle import oracle as O
    from xtsrcmaps_b200.synth import make_job

    job = make_job("c1", seed=1)
    g, sc = job.rpsf_front, job.scale_front
    n = O.normalize_rpsf(g.params, g.logEs, sc.scale0, sc.scale1, sc.scale_index)
    w = np.degrees(n[1:-1, 1:-1, 2])
    assert 3.0 < w[-1, 0] < 7.0 and 0.03 < w[-1, -1] < 0.08
    assert np.all(np.diff(w, axis=1) < 0)
    assert np.all((n[..., 4] >= 1.5) & (n[..., 4] <= 4.0))
