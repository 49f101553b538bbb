"""GPU parity: every step of the point-source path through the C-ABI against the
FP64 CPU oracle on the same seeded inputs, and against the reference's golden
vectors where they exist.

Tolerances (the bar of the path's specification):
  * FP64 steps (exposure, mean PSF, per-map sums): relative 1e-10 or tighter;
  * FP32 source maps: 1e-5 relative per pixel, per-map totals 1e-7;
  * FP64 source maps (XTS_OUT_F64): 1e-10 relative per pixel.
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


def _job(name, seed=3, n=None):
    from xtsrcmaps_b200.synth import make_job

    return make_job(name, seed=seed, n_sources=n)


def _gpu_pipeline(A, job, out_dtype="float32"):
    ltf = A.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = A.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = A.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = A.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front,
                            job.aeff_back, ltf)
    ps = A.compute_psf_data(nf, nb, ex, job.logEs, ltf)
    mm, info = A.point_src_model_map_wcs(job.wcs, job.src_sph, ex.exposure, ps.uPsf,
                                         ps.partial_psf_integral, out_dtype=out_dtype)
    return dict(ltf=ltf, nf=nf, nb=nb, ex=ex, ps=ps, map=mm, info=info)


@pytest.fixture(scope="module")
def c1_small(api):
    job = _job("c1", seed=5, n=6)
    return job, oracle_pipeline(job), _gpu_pipeline(api, job)


def test_irf_setup_vs_oracle(api, c1_small):
    job, ref, gpu = c1_small
    assert max_rel(gpu["ltf"], ref["ltf"]) < 1e-15
    assert max_rel(gpu["nf"].params, ref["nf"].params) < 1e-12
    assert max_rel(gpu["nb"].params, ref["nb"].params) < 1e-12


def test_exposure_vs_oracle(api, c1_small):
    job, ref, gpu = c1_small
    ex = gpu["ex"]
    assert np.array_equal(ex.exp_costhetas, ref["costh"])
    assert np.array_equal(ex.src_exposure_cosbins, ref["ecb"])  # gather: bit-exact
    assert np.array_equal(ex.src_weighted_exposure_cosbins, ref["wecb"])
    assert max_rel(ex.front_aeff, ref["af"]) < 1e-14
    assert max_rel(ex.back_aeff, ref["ab"]) < 1e-14
    assert max_rel(ex.exposure, ref["exposure"]) < 1e-13


def test_exposure_host_rows_match_device(api):
    """With host buffers only the livetime rows at the sources' pixels are uploaded;
    the result equals the device-pointer call, which reads the whole cubes, also for
    a repeated source and a non-finite position (whatever row that maps to)."""
    import torch

    from xtsrcmaps_b200.api import ExpCube

    job = _job("c1", seed=8, n=5)
    src = np.vstack([job.src_sph, job.src_sph[:1], [[np.nan, 0.0]]])
    ltf = api.livetime_efficiency_factors(job.logEs, job.effic_front)
    eh = api.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, src, job.aeff_front, job.aeff_back, ltf)
    d = torch.device("cuda")
    tc = lambda c: ExpCube(torch.as_tensor(c.cosbins, device=d), c.nside, c.nbrbins, c.cosmin, c.thetabin)
    ed = api.compute_exposure(tc(job.exp_cube), tc(job.wexp_cube), torch.as_tensor(job.logEs, device=d),
                              torch.as_tensor(src, device=d), job.aeff_front, job.aeff_back,
                              torch.as_tensor(ltf, device=d))
    torch.cuda.synchronize()
    for a, b in ((eh.src_exposure_cosbins, ed.src_exposure_cosbins), (eh.exposure, ed.exposure)):
        b = b.cpu().numpy()
        np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
        np.testing.assert_array_equal(a[:-1], b[:-1])
    np.testing.assert_array_equal(eh.exposure[0], eh.exposure[5])


def test_mean_psf_vs_oracle(api, c1_small):
    job, ref, gpu = c1_small
    assert max_rel(gpu["ps"].uPsf, ref["upsf"]) < 1e-11
    assert max_rel(gpu["ps"].partial_psf_integral, ref["partial"], floor=1e-300) < 1e-11


def test_srcmap_f32_vs_oracle(api, c1_small):
    job, ref, gpu = c1_small
    m, info = gpu["map"], gpu["info"]
    assert m.dtype == np.float32 and m.shape == ref["map"].shape
    assert max_rel(m, ref["map"]) < 1e-5
    np.testing.assert_array_equal(info.in_fov.astype(bool), ref["in_fov"])
    assert max_rel(info.psf_radius, ref["radius"]) < 1e-13
    # per-map normalisation sums and their use
    assert max_rel(info.inv_map_integral, ref["inv_integ"]) < 1e-7
    assert max_rel(info.correction, ref["factor"]) < 1e-7
    # totals of the written maps
    tot_g = m.astype(np.float64).sum(axis=(1, 2))
    tot_r = ref["map"].sum(axis=(1, 2))
    assert max_rel(tot_g, tot_r) < 1e-7


@pytest.mark.parametrize("kernel", ["cuda_cores", "tcgen05"])
def test_srcmap_other_fp32_kernels_vs_oracle(api, c1_small, kernel):
    """The single-pass CUDA-core kernel (XTS_CUDA_CORES) and the tcgen05 kernel
    (XTS_TCGEN05) against the oracle and the default two-pass window path."""
    job, ref, gpu = c1_small
    m, info = api.point_src_model_map_wcs(job.wcs, job.src_sph, gpu["ex"].exposure, gpu["ps"].uPsf,
                                          gpu["ps"].partial_psf_integral, kernel=kernel)
    assert max_rel(m, ref["map"]) < 1e-5
    assert max_rel(m, gpu["map"]) < 2e-6
    assert max_rel(info.inv_map_integral, ref["inv_integ"]) < 1e-7
    tot_g = m.astype(np.float64).sum(axis=(1, 2))
    assert max_rel(tot_g, ref["map"].sum(axis=(1, 2))) < 1e-7


def test_srcmap_f64_vs_oracle(api, c1_small):
    job, ref, gpu = c1_small
    m, info = api.point_src_model_map_wcs(job.wcs, job.src_sph, gpu["ex"].exposure, gpu["ps"].uPsf,
                                          gpu["ps"].partial_psf_integral, out_dtype="float64")
    assert m.dtype == np.float64
    assert max_rel(m, ref["map"]) < 1e-10
    assert max_rel(info.inv_map_integral, ref["inv_integ"]) < 1e-10


def test_config0_full(api):
    """config 0: one source at the field centre (the point-source pixel itself)."""
    job = _job("c0", seed=1)
    ref = oracle_pipeline(job)
    gpu = _gpu_pipeline(api, job)
    assert max_rel(gpu["map"], ref["map"]) < 1e-5
    m64, _ = api.point_src_model_map_wcs(job.wcs, job.src_sph, gpu["ex"].exposure, gpu["ps"].uPsf,
                                         gpu["ps"].partial_psf_integral, out_dtype="float64")
    assert max_rel(m64, ref["map"]) < 1e-10


def test_device_pointer_mode(api, c1_small):
    """Same call with CUDA tensors: XTS_DEVICE_PTRS path, asynchronous on torch's stream."""
    import torch

    job, ref, gpu = c1_small
    d = torch.device("cuda")
    ex = gpu["ex"]
    m, info = api.point_src_model_map_wcs(job.wcs, torch.as_tensor(job.src_sph, device=d),
                                          torch.as_tensor(ex.exposure, device=d),
                                          torch.as_tensor(gpu["ps"].uPsf, device=d),
                                          torch.as_tensor(gpu["ps"].partial_psf_integral, device=d))
    torch.cuda.synchronize()
    assert m.is_cuda
    assert np.array_equal(m.cpu().numpy(), gpu["map"])


def test_edge_sources(api):
    """Sources exactly on a pixel centre, on a pixel corner, just outside the map
    (in-FOV false) and 80 deg away (LUT clamp at row 400), on a non-square AIT map."""
    from xtsrcmaps_b200.synth import make_job
    from xtsrcmaps_b200.wcs import Wcs
    from oracle import oracle as O

    job = make_job("c0", seed=7)
    job.wcs = Wcs(60, 44, 30.5, 22.5, 193.98, -5.82, -0.2, 0.2, proj="AIT")
    pts = [O.pix2sph(job.wcs, 31.0, 20.0), O.pix2sph(job.wcs, 10.5, 7.5), O.pix2sph(job.wcs, 62.0, 10.0)]
    pts.append((pts[0][0] + 85.0, pts[0][1]))
    # a source on the unit-vector direction of one rule point: that point's chord is
    # the blend's radial shrink (~1e-6 rad), below the table's first separation (1e-4 deg)
    pw = O.square_ptswts(job.wcs)[20, 15, 0:3]
    d = pw / np.linalg.norm(pw)
    pts.append((np.degrees(np.arctan2(d[1], d[0])) % 360.0, np.degrees(np.arcsin(d[2]))))
    job.src_sph = np.array(pts, dtype=np.float64)
    ref = oracle_pipeline(job)
    gpu = _gpu_pipeline(api, job)
    near = [0, 1, 2, 4]
    assert max_rel(gpu["map"][near], ref["map"][near]) < 1e-5
    # Beyond the table's last separation (70 deg) the reference extrapolates
    # linearly past row 400 (convolve_pixel_psf_logsep.hpp:45-47); the values
    # cross zero, so the error there is measured against the map's largest value.
    far_ref = ref["map"][3]
    assert (far_ref < 0).any()
    scale = np.abs(far_ref).max()
    assert np.abs(gpu["map"][3] - far_ref).max() / scale < 1e-5
    m64, _ = api.point_src_model_map_wcs(job.wcs, job.src_sph, gpu["ex"].exposure, gpu["ps"].uPsf,
                                         gpu["ps"].partial_psf_integral, out_dtype="float64")
    assert np.abs(m64[3] - far_ref).max() / scale < 1e-10
    assert max_rel(m64[near], ref["map"][near]) < 1e-10
    np.testing.assert_array_equal(gpu["info"].in_fov.astype(bool), ref["in_fov"])
    assert list(ref["in_fov"]) == [True, True, False, False, True]


def test_empty_and_single_energy(api):
    job = _job("c0", seed=2)
    gpu = _gpu_pipeline(api, job)
    m, info = api.point_src_model_map_wcs(job.wcs, np.zeros((0, 2)), np.zeros((0, job.E)),
                                          np.zeros((0, 401, job.E)), np.zeros((0, 401, job.E)))
    assert m.shape == (0, 100, 100, job.E)
    ex = gpu["ex"]
    m1, _ = api.point_src_model_map_wcs(job.wcs, job.src_sph, ex.exposure[:, :1].copy(),
                                        gpu["ps"].uPsf[:, :, :1].copy(),
                                        gpu["ps"].partial_psf_integral[:, :, :1].copy())
    assert max_rel(m1[..., 0], gpu["map"][..., 0]) < 1e-6


def test_bad_arguments_raise(api):
    from xtsrcmaps_b200._lib import XTS_ERR_ARG, XtsError
    from xtsrcmaps_b200.wcs import Wcs

    w = Wcs(10, 10, 5.5, 5.5, 0.0, 0.0, 0.0, 0.1)  # CDELT1 = 0
    with pytest.raises(XtsError) as ei:
        api.point_src_model_map_wcs(w, np.zeros((1, 2)), np.ones((1, 3)), np.ones((1, 401, 3)),
                                    np.ones((1, 401, 3)))
    assert ei.value.code == XTS_ERR_ARG


def test_golden_exposure_and_psf_on_gpu(api, golden):
    """The reference's own livetime rows and IRFs through the GPU contraction and
    mean-PSF kernels, against tests/expected/exposure.bin and uPsf_peak_SE.bin."""
    from test_oracle_golden import _exposure_inputs
    from oracle import oracle as O
    from xtsrcmaps_b200.irf import IrfGrid

    z, g, e, cos, loge, af, ab, ltf, ecb, wecb = _exposure_inputs(golden)
    ex = api.exposure(ecb, wecb, af, ab, ltf)
    assert max_rel(ex, e["exposure"]) < 5e-6
    pf, pb = g["rpsf_front"], g["rpsf_back"]
    nf = api.normalize_rpsf(pf, g["scale_front"])
    nb = api.normalize_rpsf(pb, g["scale_back"])
    from xtsrcmaps_b200.api import XtExp

    xe = XtExp(cos, af, ab, ecb, wecb, ex)
    ps = api.compute_psf_data(nf, nb, xe, loge, ltf)
    assert max_rel(ps.uPsf[:, 0, :], golden("psf")["upsf_peak"]) < 2e-6


def test_golden_inputs_model_maps(api, golden):
    """Model maps on the reference's own inputs end to end: its 3C279 counts-cube
    WCS (AIT, 100 x 100 @ 0.2 deg), its 263 point sources, livetime rows and P8R3
    IRFs (as the reference's tests hold them) through exposure, mean PSF and maps
    on the GPU; in-FOV flags as Fermitools (47), maps against the FP64 oracle."""
    from test_oracle_golden import _exposure_inputs
    from oracle import oracle as O
    from xtsrcmaps_b200.api import XtExp
    from xtsrcmaps_b200.wcs import Wcs

    z, g, e, cos, loge, af, ab, ltf, ecb, wecb = _exposure_inputs(golden)
    gm = golden("geom")
    w = Wcs(int(gm["naxis"][0]), int(gm["naxis"][1]), *gm["crpix"], *gm["crval"], *gm["cdelt"],
            crota2=float(gm["crota2"]), proj=str(gm["proj"]))
    src = gm["src_sph"]
    ex = api.exposure(ecb, wecb, af, ab, ltf)
    nf = api.normalize_rpsf(g["rpsf_front"], g["scale_front"])
    nb = api.normalize_rpsf(g["rpsf_back"], g["scale_back"])
    ps = api.compute_psf_data(nf, nb, XtExp(cos, af, ab, ecb, wecb, ex), loge, ltf)
    m, info = api.point_src_model_map_wcs(w, src, ex, ps.uPsf, ps.partial_psf_integral)
    fov = np.asarray(info.in_fov).astype(bool)
    assert fov.sum() == gm["ft_in_fov"].sum() == 47
    sample = list(np.flatnonzero(fov)[::12]) + list(np.flatnonzero(~fov)[::60])
    ref = O.point_src_model_map_wcs(w, src[sample], ex[sample], ps.uPsf[sample], ps.partial_psf_integral[sample])
    assert max_rel(m[sample], ref["map"]) < 1e-5
    np.testing.assert_allclose(info.inv_map_integral[sample], ref["inv_integ"], rtol=1e-7)


@pytest.mark.parametrize("out_dtype", ["float32", "float64"])
def test_point_source_maps_fused_call(api, c1_small, out_dtype):
    """xts_point_source_maps (the three calls of main.cxx:28-30 in one) gives the
    same maps and per-map results as the three separate calls, with host buffers
    (chunked copy-out) and with device tensors."""
    import torch

    job, ref, gpu = c1_small
    m, info = api.point_source_maps(job.wcs, job.src_sph, job.exp_cube, job.wexp_cube, job.logEs,
                                    job.aeff_front, job.aeff_back, gpu["nf"], gpu["nb"], gpu["ltf"],
                                    out_dtype=out_dtype)
    m3, info3 = api.point_src_model_map_wcs(job.wcs, job.src_sph, gpu["ex"].exposure, gpu["ps"].uPsf,
                                            gpu["ps"].partial_psf_integral, out_dtype=out_dtype)
    # the map integrals add the points of pixels next to the source with FP64
    # atomics, so two runs agree to rounding, not bit for bit
    same = 1e-6 if out_dtype == "float32" else 1e-13
    assert max_rel(m, m3) < same
    assert max_rel(info.inv_map_integral, info3.inv_map_integral) < 1e-13
    assert max_rel(info.correction, info3.correction) < 1e-13
    tol = 1e-5 if out_dtype == "float32" else 1e-10
    assert max_rel(m, ref["map"]) < tol
    d = torch.device("cuda")
    tg = lambda g: type(g)(*[torch.as_tensor(np.asarray(v), device=d) if isinstance(v, np.ndarray) else v
                             for v in (g.cosths, g.logEs, g.params, g.min_cos_theta)])
    from xtsrcmaps_b200.api import ExpCube

    tc = lambda c: ExpCube(torch.as_tensor(c.cosbins, device=d), c.nside, c.nbrbins, c.cosmin, c.thetabin)
    md, _ = api.point_source_maps(job.wcs, torch.as_tensor(job.src_sph, device=d), tc(job.exp_cube),
                                  tc(job.wexp_cube), torch.as_tensor(job.logEs, device=d), tg(job.aeff_front),
                                  tg(job.aeff_back), tg(gpu["nf"]), tg(gpu["nb"]),
                                  torch.as_tensor(gpu["ltf"], device=d), out_dtype=out_dtype)
    torch.cuda.synchronize()
    assert max_rel(md.cpu().numpy(), m) < same


def test_fused_call_graph_capture(api, c1_small):
    """The fused device-pointer call runs its map geometry on a second stream that
    forks from and joins the caller's stream: captured into a CUDA graph and
    replayed twice (on a poisoned output) it reproduces the eager maps."""
    import torch

    from xtsrcmaps_b200.api import ExpCube

    job, ref, gpu = c1_small
    d = torch.device("cuda")
    tg = lambda g: type(g)(*[torch.as_tensor(np.asarray(v), device=d) if isinstance(v, np.ndarray) else v
                             for v in (g.cosths, g.logEs, g.params, g.min_cos_theta)])
    tc = lambda c: ExpCube(torch.as_tensor(c.cosbins, device=d), c.nside, c.nbrbins, c.cosmin, c.thetabin)
    args = (job.wcs, torch.as_tensor(job.src_sph, device=d), tc(job.exp_cube), tc(job.wexp_cube),
            torch.as_tensor(job.logEs, device=d), tg(job.aeff_front), tg(job.aeff_back), tg(gpu["nf"]),
            tg(gpu["nb"]), torch.as_tensor(gpu["ltf"], device=d))
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        eager, _ = api.point_source_maps(*args, with_info=False)
        out = torch.empty_like(eager)
        api.point_source_maps(*args, out=out, with_info=False)  # warm: workspaces sized
    st.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=st):
        api.point_source_maps(*args, out=out, with_info=False)
    for _ in range(2):
        with torch.cuda.stream(st):
            out.fill_(float("nan"))
            g.replay()
        st.synchronize()
        assert max_rel(out.cpu().numpy(), eager.cpu().numpy()) < 1e-6
    assert max_rel(out.cpu().numpy(), ref["map"]) < 1e-5
    del g


def test_srcmap_vs_compiled_reference(api, c1_small):
    """GPU maps (FP32 and FP64) against ModelMap::point_src_model_map_wcs of the
    reference's own code compiled under oracle/_ref, fed the same exposure and
    mean-PSF tables."""
    from oracle import oracle_ref as R

    if not R.available():
        pytest.skip("oracle/_ref/libxts_ref.so not built")
    job, ref, gpu = c1_small
    rm = R.point_src_model_map_wcs(job.wcs, job.src_sph, ref["exposure"], ref["upsf"], ref["partial"])
    m32, _ = api.point_src_model_map_wcs(job.wcs, job.src_sph, ref["exposure"], ref["upsf"], ref["partial"])
    m64, _ = api.point_src_model_map_wcs(job.wcs, job.src_sph, ref["exposure"], ref["upsf"], ref["partial"],
                                         out_dtype="float64")
    assert max_rel(m32, rm) < 1e-5
    assert max_rel(m32.astype(np.float64).sum(axis=(1, 2)), rm.sum(axis=(1, 2))) < 1e-7
    assert max_rel(m64, rm) < 1e-10


def test_adaptive_map_vs_oracle(api, c1_small):
    """Adaptive Genz-Malik cubature on the GPU against the oracle's FP64 version
    of the same algorithm (rtol 1e-4, depth 6).  The GPU decides a region in FP64,
    with the oracle's arithmetic, whenever its FP32 estimate lies near the
    threshold or the split dimension is nearly tied, and accumulates the pixel
    means in FP64: every region is decided as in the oracle, so every value
    agrees to FP32 rounding (1e-5) and the map integrals to 1e-7."""
    from oracle import oracle as O

    job, ref, gpu = c1_small
    m, info = api.point_src_model_map_wcs_adaptive(job.wcs, job.src_sph, ref["exposure"], ref["upsf"],
                                                   ref["partial"], rtol=1e-4, max_depth=6)
    o = O.point_src_model_map_wcs_adaptive(job.wcs, job.src_sph, ref["exposure"], ref["upsf"], ref["partial"],
                                           1e-4, 6)
    assert m.dtype == np.float32
    rel = np.abs(m - o["map"]) / np.abs(o["map"])
    assert rel.max() < 1e-5, (rel.max(), (rel > 1e-5).sum())
    assert max_rel(info.inv_map_integral, o["inv_integ"]) < 1e-7
    np.testing.assert_array_equal(info.in_fov.astype(bool), o["in_fov"])


def test_adaptive_map_accuracy_gain(api):
    """Against the integral of the LUT interpolant converged by the oracle
    (rtol 1e-10, depth 16), the adaptive GPU map at rtol 1e-4 / depth 6 is
    several times closer than the fixed 12-point rule next to the source."""
    from oracle import oracle as O
    from xtsrcmaps_b200.synth import make_job
    from xtsrcmaps_b200.wcs import Wcs

    job = make_job("c1", seed=5, n_sources=1)
    job.wcs = Wcs(24, 24, 12.5, 12.5, job.wcs.crval1, job.wcs.crval2, -0.1, 0.1, proj="CAR")
    job.src_sph = np.array([O.pix2sph(job.wcs, 12.3, 12.6)])
    ref = oracle_pipeline(job, with_map=False)
    truth = O.point_src_model_map_wcs_adaptive(job.wcs, job.src_sph, ref["exposure"], ref["upsf"],
                                               ref["partial"], 1e-10, 16)["map"]
    ad, _ = api.point_src_model_map_wcs_adaptive(job.wcs, job.src_sph, ref["exposure"], ref["upsf"],
                                                 ref["partial"], rtol=1e-4, max_depth=6)
    pl, _ = api.point_src_model_map_wcs(job.wcs, job.src_sph, ref["exposure"], ref["upsf"], ref["partial"])
    e_ad, e_pl = max_rel(ad, truth), max_rel(pl, truth)
    assert e_pl > 5e-4
    assert e_ad < 0.5 * e_pl


@pytest.mark.parametrize("name,n_e", [("c0", None), ("c1", None), ("c0", 80)])
def test_exposure_map_tensor_cores(api, name, n_e):
    """The full-sky exposure contraction on tcgen05 (3xTF32, FP32 accumulation)
    against the FP64 oracle applied to every livetime-cube row, and its rows at
    the sources' NESTED pixels against the FP64 per-source exposures, for E = 20,
    37 and 80 (N = 32, 48 and 80 columns of the accumulator)."""
    from oracle import oracle as O

    job = _job(name, seed=4)
    if n_e:
        job.energies = np.logspace(2.0, 5.0, n_e)
        job.logEs = np.log10(job.energies)
    ref = oracle_pipeline(job, with_map=False)
    cube, wcube = job.exp_cube, job.wexp_cube
    m = api.exposure_map(cube, wcube, job.logEs, job.aeff_front, job.aeff_back, ref["ltf"])
    npix = 12 * cube.nside ** 2
    assert m.shape == (npix, job.E)
    want = O.exposure(cube.cosbins.astype(np.float64), wcube.cosbins.astype(np.float64), ref["af"], ref["ab"],
                      ref["ltf"])
    rel = np.abs(m - want) / np.abs(want)
    assert rel.max() < 5e-6
    assert rel.mean() < 1e-6
    pix = [O.ang2pix_nest(np.pi / 2 - np.radians(dec), np.radians(ra), cube.nside) for ra, dec in job.src_sph]
    assert max_rel(m[pix], ref["exposure"]) < 5e-6
