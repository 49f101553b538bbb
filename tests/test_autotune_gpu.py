"""GPU check of the autotuner: the write-pass choice is one of the parity-tested
kernels and the adaptive cubature's (rtol, depth) choice meets its error target
against the converged map it was measured on."""
import numpy as np
import pytest

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


def test_autotune_choices(api):
    import torch

    from xtsrcmaps_b200 import autotune as T
    from xtsrcmaps_b200.synth import make_job

    job = make_job("c1", seed=9, n_sources=4)
    ltf = api.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = api.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = api.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = api.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front,
                              job.aeff_back, ltf)
    ps = api.compute_psf_data(nf, nb, ex, job.logEs, ltf)
    d = torch.device("cuda")
    t = lambda x: torch.as_tensor(np.ascontiguousarray(x), device=d)
    src, expo, upsf, part = t(job.src_sph), t(ex.exposure), t(ps.uPsf), t(ps.partial_psf_integral)
    w = T.tune_write_pass(job.wcs, src, expo, upsf, part)
    assert w["kernel"] in ("windows", "cuda_cores", "tcgen05")
    assert all(v > 0 for v in w["ms"].values()) and w["ms"][w["kernel"]] == min(w["ms"].values())
    assert T.tune_write_pass(job.wcs, src, expo, upsf, part) is w  # cached per shape
    a = T.tune_adaptive(job.wcs, src, expo, upsf, part, target=1e-3, rtols=(1e-3, 1e-4), depths=(4, 6, 8),
                        n_sources=2)
    assert a is not None, "no adaptive setting met 1e-3"
    assert a["err"] <= 1e-3 and (a["rtol"], a["max_depth"]) in [(r, dd) for r in (1e-3, 1e-4) for dd in (4, 6, 8)]
    ok = [v["ms"] for v in a["table"].values() if v["err"] <= 1e-3]
    assert a["ms"] == min(ok)
    print(f"\nwrite pass: {w}\nadaptive: rtol {a['rtol']:g}, depth {a['max_depth']}, {a['ms']:.3f} ms, "
          f"err {a['err']:.2e}")


def test_launch_shape_tuning(api):
    """The launch-shape tuner times each candidate, sets the fastest, and the maps
    stay the same whatever the shape (the shapes change the work split, not the
    arithmetic of a value)."""
    import torch

    from xtsrcmaps_b200 import autotune as T
    from xtsrcmaps_b200.synth import make_job

    job = make_job("c1", seed=19, n_sources=6)
    ltf = api.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = api.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = api.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = api.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front,
                              job.aeff_back, ltf)
    ps = api.compute_psf_data(nf, nb, ex, job.logEs, ltf)
    d = torch.device("cuda")
    t = lambda x: torch.as_tensor(np.ascontiguousarray(x), device=d)
    src, expo, upsf, part = t(job.src_sph), t(ex.exposure), t(ps.uPsf), t(ps.partial_psf_integral)
    api.reset_tuning()
    ref, _ = api.point_src_model_map_wcs(job.wcs, src, expo, upsf, part, with_info=False)
    res = T.tune_launch_shapes(job.wcs, src, expo, upsf, part)
    assert len(res["ms"]) == 6 and all(v > 0 for v in res["ms"].values())
    assert api.get_tuning()["window_blocks_per_sm"] == res["choice"]["window_blocks_per_sm"]
    for wv, wb in ((2, 1), (4, 2)):
        api.set_tuning(window_blocks_per_sm=wv, write_blocks_per_sm=wb)
        m, _ = api.point_src_model_map_wcs(job.wcs, src, expo, upsf, part, with_info=False)
        torch.cuda.synchronize()
        rel = ((m.double() - ref.double()).abs() / ref.double().abs().clamp_min(1e-300)).max().item()
        assert rel < 1e-6, (wv, wb, rel)
    from xtsrcmaps_b200 import _lib as L

    with pytest.raises(L.XtsError):
        api.set_tuning(window_blocks_per_sm=9)
    api.reset_tuning()
    assert api.get_tuning() == {k: 0 for k in api.TUNING_FIELDS}
