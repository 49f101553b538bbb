"""Pins the FP64 CPU oracle (and the host-side IRF preparation) to the
reference's own golden vectors (tests/golden/*.npz, generated from the
reference's tests/fits/*.hxx and tests/expected/*.bin by make_golden.py).

Tolerances follow the reference's NearRelative (tests/fermi_tests.hxx:22-40,
rtol = atol = 1e-5) unless stated: the .hxx goldens are printed with six
significant digits, so they cannot pin anything tighter than ~1e-6.
"""
import numpy as np
import pytest

from oracle import oracle as O
from xtsrcmaps_b200 import irf as I


def near_relative(a, b, rtol=1e-5, atol=1e-5):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.all(np.abs(a - b) <= atol + rtol * np.abs(b))


def _irf(golden):
    z = golden("irf")
    g = {}
    for side in ("front", "back"):
        g["aeff_" + side] = I.prepare_grid(z[f"aeff_{side}_extents"], z[f"aeff_{side}_offsets"], z[f"aeff_{side}_row"])
        g["rpsf_" + side] = I.prepare_grid(z[f"rpsf_{side}_extents"], z[f"rpsf_{side}_offsets"], z[f"rpsf_{side}_row"])
        g["scale_" + side] = I.prepare_scale(z[f"scaling_{side}"])
    return z, g


def test_separations(golden):
    """tests/test_psf.cxx:15-31 and separations_expected.hxx."""
    seps = O.separations()
    exp = golden("psf")["separations"]
    assert seps[0] == 0.0 and abs(seps[400] - 70.0) < 1e-9
    assert near_relative(seps, exp, rtol=1e-5, atol=1e-9)
    step = np.log(seps[2:] / seps[1:-1])
    assert np.allclose(step, np.log(7e5) / 399, rtol=1e-12)


def test_costhetas(golden):
    """exposure/exposure.cxx:29-40 vs exposure_cosbins_expected.hxx:10 (3C279 cube: 40 sqrt bins, cosmin 0)."""
    c = O.costhetas(40, 0.0, True)
    assert near_relative(c, golden("irf")["exp_costhetas"], rtol=1e-5, atol=1e-6)


def test_prepare_grid_psf(golden):
    """irf/irf.prepare_grid.cpp vs psf3_rpsf.{front,back}.bin (tests/test_irf.psf.cpp:60-75)."""
    _, g = _irf(golden)
    p = golden("psf")
    for side in ("front", "back"):
        grid = g["rpsf_" + side]
        assert grid.params.shape == (10, 25, 6)
        np.testing.assert_allclose(grid.params, p["rpsf_" + side], rtol=1e-6)
        thetas = np.array([180.0, 75.5225, 69.5127, 63.2563, 56.633, 49.4584, 41.4096, 31.7883, 18.1949, 0.0])
        np.testing.assert_allclose(grid.cosths, np.cos(np.radians(thetas)), rtol=1e-5, atol=1e-5)


def test_normalize_rpsf(golden):
    """irf/irf.normalize_rpsf.cpp vs psf3_normalized_rpsf.*.bin (tests/test_irf.psf.cpp:95-150):
    the golden's score/stail are stored before the sf scaling, as the reference test checks."""
    _, g = _irf(golden)
    p = golden("psf")
    for side in ("front", "back"):
        grid, sc = g["rpsf_" + side], g["scale_" + side]
        n = O.normalize_rpsf(grid.params, grid.logEs, sc.scale0, sc.scale1, sc.scale_index)
        exp = p["norm_rpsf_" + side]
        energy = 10.0 ** grid.logEs
        sp0 = np.float32(sc.scale0) * np.float32(sc.scale0)
        sp1 = np.float32(sc.scale1) * np.float32(sc.scale1)
        tt = (energy * 1e-2) ** np.float32(sc.scale_index)
        sf = np.sqrt(np.float64(sp0) * tt * tt + np.float64(sp1))
        for k in (0, 1, 4, 5):
            assert near_relative(n[..., k], exp[..., k], rtol=1e-5, atol=1e-12), (side, k)
        for k in (2, 3):
            assert near_relative(n[..., k], sf[None, :] * exp[..., k], rtol=1e-5, atol=1e-12), (side, k)


def test_king_table(golden):
    """psf/psf.king.cxx vs king_front.bin (tests/test_king.cxx:14-118, rtol 1e-2 there)."""
    z, g = _irf(golden)
    grid, sc = g["rpsf_front"], g["scale_front"]
    n = O.normalize_rpsf(grid.params, grid.logEs, sc.scale0, sc.scale1, sc.scale_index)
    k = O.king(I.IrfGrid(grid.cosths, grid.logEs, n, grid.min_cos_theta))
    p = golden("psf")
    rows = p["king_front_rows"]
    exp = p["king_front"]
    rel = np.abs(k[rows] - exp) / np.maximum(np.abs(exp), 1e-300)
    assert rel.max() < 1e-5, rel.max()


def test_aeff_and_ltf(golden):
    """irf/irf.aeff_value.cxx and irf/irf.cxx:70-109 vs aeff_*_c_e and livetime_factor{1,2}
    (tests/test_exposure.cxx:150-195)."""
    z, g = _irf(golden)
    cos = O.costhetas(40, 0.0, True)
    loge = np.log10(z["energies"])
    for side in ("front", "back"):
        a = O.aeff_value(cos, loge, g["aeff_" + side])
        exp = z[f"aeff_{side}_c_e"]
        assert near_relative(a, exp, rtol=2e-5, atol=1e-3), side
    ltf = O.livetime_efficiency_factors(loge, z["effic_front_p0"], z["effic_front_p1"])
    assert near_relative(ltf[0], z["livetime_factor1"], rtol=1e-5, atol=1e-5)
    assert near_relative(ltf[1], z["livetime_factor2"], rtol=1e-5, atol=1e-5)


def _exposure_inputs(golden):
    z, g = _irf(golden)
    e = golden("exposure")
    cos = O.costhetas(40, 0.0, True)
    loge = np.log10(z["energies"])
    af = O.aeff_value(cos, loge, g["aeff_front"])
    ab = O.aeff_value(cos, loge, g["aeff_back"])
    ltf = O.livetime_efficiency_factors(loge, z["effic_front_p0"], z["effic_front_p1"])
    ecb = e["ecb"].astype(np.float64)
    wecb = e["wecb"].astype(np.float64)
    return z, g, e, cos, loge, af, ab, ltf, ecb, wecb


def test_exposure_golden(golden):
    """exposure/exposure.cxx:159-263 vs tests/expected/exposure.bin [263, 38]."""
    z, g, e, cos, loge, af, ab, ltf, ecb, wecb = _exposure_inputs(golden)
    ex = O.exposure(ecb, wecb, af, ab, ltf)
    rel = np.abs(ex - e["exposure"]) / np.abs(e["exposure"])
    assert rel.max() < 5e-6, rel.max()


def test_mean_psf_peak_golden(golden):
    """psf/psf.psf_lookup_table_and_partial_integrals.cxx vs uPsf_peak_SE.bin [263, 38]."""
    z, g, e, cos, loge, af, ab, ltf, ecb, wecb = _exposure_inputs(golden)
    ex = O.exposure(ecb, wecb, af, ab, ltf)
    pf, pb = g["rpsf_front"], g["rpsf_back"]
    nf = O.normalize_rpsf(pf.params, pf.logEs, *vars(g["scale_front"]).values())
    nb = O.normalize_rpsf(pb.params, pb.logEs, *vars(g["scale_back"]).values())
    gf = I.IrfGrid(pf.cosths, pf.logEs, nf, pf.min_cos_theta)
    gb = I.IrfGrid(pb.cosths, pb.logEs, nb, pb.min_cos_theta)
    upsf, partial = O.compute_psf_data(gf, gb, cos, loge, af, ab, ecb, wecb, ltf, ex)
    peak = golden("psf")["upsf_peak"]
    rel = np.abs(upsf[:, 0, :] - peak) / np.abs(peak)
    assert rel.max() < 2e-6, rel.max()
    # partial integrals are normalised prefix sums in [0, 1]
    assert np.allclose(partial[:, -1, :], 1.0, rtol=1e-12)
    assert np.all(np.diff(partial, axis=1) >= -1e-15)


def test_boundary_radius_vs_fermitools(golden):
    """model_map.psf_boundary_radius.cxx with the restated AIT WCS vs Fermitools
    ft_mm_psf_radius.bin / ft_mm_withinBounds.bin (tests/test_model_map_v2.cxx:100-140).
    Source order differs between the two tools, so sorted lists are compared."""
    from xtsrcmaps_b200.wcs import Wcs

    gm = golden("geom")
    w = Wcs(int(gm["naxis"][0]), int(gm["naxis"][1]), *gm["crpix"], *gm["crval"], *gm["cdelt"],
            crota2=float(gm["crota2"]), proj=str(gm["proj"]))
    r, fov = O.psf_boundary_radius(w, gm["src_sph"])
    assert fov.sum() == gm["ft_in_fov"].sum() == 47
    d = np.abs(np.sort(r) - np.sort(gm["ft_psf_radius"]))
    assert d.max() < 1e-9, d.max()


def test_wcs_round_trip():
    """tests/test_sky_geom.cxx:25-64: pix -> sph -> pix round trip for CAR and AIT."""
    from xtsrcmaps_b200.wcs import Wcs

    for proj in ("CAR", "AIT"):
        for dec0 in (-5.82, 0.0, 33.0):
            w = Wcs(100, 100, 50.5, 50.5, 193.98, dec0, -0.2, 0.2, proj=proj)
            for p in [(1, 1), (50.5, 50.5), (100, 3), (17.25, 88.5)]:
                ra, dec = O.pix2sph(w, *p)
                q = O.sph2pix(w, ra, dec)
                assert np.allclose(q, p, atol=1e-9), (proj, dec0, p, q)
            ra, dec = O.pix2sph(w, 50.5, 50.5)
            assert abs(ra - 193.98) < 1e-9 and abs(dec - dec0) < 1e-9


@pytest.mark.parametrize("nside", [1, 4, 32, 64, 128])
def test_healpix_round_trip(nside):
    """tests/test_healpix.cxx:8-23: pix2ang(ang2pix) lands in the same pixel."""
    rng = np.random.default_rng(nside)
    for pix in rng.integers(0, 12 * nside * nside, 200):
        th, ph = O.pix2ang_nest(int(pix), nside)
        assert O.ang2pix_nest(th, ph, nside) == pix
    th = np.arccos(rng.uniform(-1, 1, 200))
    ph = rng.uniform(0, 2 * np.pi, 200)
    for t, p in zip(th, ph):
        pix = O.ang2pix_nest(t, p, nside)
        assert 0 <= pix < 12 * nside * nside
