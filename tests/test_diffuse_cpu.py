"""The diffuse-map oracle on the CPU: the direct convolution against numpy's 1-D
convolution for separable cases, the kernel image's normalisation and symmetry."""
import numpy as np

from oracle import diffuse_oracle as D


def test_convolution_is_linear_convolution():
    rng = np.random.default_rng(0)
    img = rng.standard_normal((3, 9, 7))
    u, v = rng.standard_normal((3, 5)), rng.standard_normal((3, 5))
    ker = u[:, :, None] * v[:, None, :]  # separable kernel
    out = D.convolve_full(img, ker)
    assert out.shape == (3, 13, 11)
    for e in range(3):
        rows = np.array([np.convolve(r, v[e]) for r in img[e]])            # along w
        ref = np.array([np.convolve(c, u[e]) for c in rows.T]).T            # along h
        np.testing.assert_allclose(out[e], ref, rtol=1e-12, atol=1e-12)
    delta = np.zeros((3, 5, 5))
    delta[:, 0, 0] = 1.0
    np.testing.assert_array_equal(D.convolve_full(img, delta)[:, :9, :7], img)


def test_kernel_image_normalised_and_centred():
    from xtsrcmaps_b200.wcs import Wcs

    Nk = 21
    w = Wcs(Nk, Nk, (Nk + 1) / 2, (Nk + 1) / 2, 193.98, -5.82, -0.05, 0.05, proj="CAR")
    sep = np.array([0.0] + [1e-4 * np.exp((k - 1) * D.SEP_STEP) for k in range(1, 401)])
    upsf = np.exp(-0.5 * (sep[:, None] / np.array([0.1, 0.3, 1.0])) ** 2)  # [401, 3], falling
    k = D.make_kernel(w, Nk, upsf)
    np.testing.assert_allclose(k.sum(axis=(1, 2)), 1.0, rtol=1e-14)
    c = Nk // 2
    assert (k[:, c, c] == k.max(axis=(1, 2))).all()          # peak at the reference pixel
    np.testing.assert_allclose(k[:, c, :], k[:, :, c], rtol=1e-3)  # nearly symmetric near the equator


def _trilerp_loops(src, shape):
    """math/trilerp.hpp:7-59 literally, as scalar float32 loops (a second oracle)."""
    f = np.float32
    E0, H0, W0 = src.shape
    E1, H1, W1 = shape
    se = f(E0 - 1) / f(E1 - 1) if E1 > 1 else f(0)
    sh = f(H0 - 1) / f(H1 - 1) if H1 > 1 else f(0)
    sw = f(W0 - 1) / f(W1 - 1) if W1 > 1 else f(0)
    out = np.zeros(shape, np.float32)
    for k in range(E1):
        e = f(k) * se
        e0 = int(e)
        e1 = min(e0 + 1, E0 - 1)
        fe = f(e - f(e0))
        ce = f(f(1) - fe)
        for i in range(H1):
            h = f(i) * sh
            h0 = int(h)
            h1 = min(h0 + 1, H0 - 1)
            fh = f(h - f(h0))
            ch = f(f(1) - fh)
            for j in range(W1):
                w = f(j) * sw
                w0 = int(w)
                w1 = min(w0 + 1, W0 - 1)
                fw = f(w - f(w0))
                cw = f(f(1) - fw)
                c00 = f(ch * src[e0, h0, w0] + fh * src[e0, h1, w0])
                c01 = f(ch * src[e1, h0, w0] + fh * src[e1, h1, w0])
                c10 = f(ch * src[e0, h0, w1] + fh * src[e0, h1, w1])
                c11 = f(ch * src[e1, h0, w1] + fh * src[e1, h1, w1])
                c0 = f(cw * c00 + fw * c10)
                c1 = f(cw * c01 + fw * c11)
                out[k, i, j] = f(ce * c0 + fe * c1)
    return out


def test_trilerp_oracle_matches_the_loops_and_interpolates():
    rng = np.random.default_rng(5)
    src = rng.lognormal(0.0, 1.0, (5, 7, 9)).astype(np.float32)
    for shape in ((9, 13, 17), (5, 7, 9), (3, 4, 30), (1, 7, 9)):
        got = D.trilerp_ehw(src, shape)
        ref = _trilerp_loops(src, shape)
        np.testing.assert_allclose(got, ref, rtol=2e-7, atol=0)
    # corner alignment: the grid's corners are the source's corners
    g = D.trilerp_ehw(src, (9, 13, 17))
    np.testing.assert_allclose(g[[0, -1]][:, [0, -1]][:, :, [0, -1]], src[[0, -1]][:, [0, -1]][:, :, [0, -1]],
                               rtol=1e-6)
    # a function linear in each index is reproduced
    e, h, w = np.meshgrid(np.arange(5), np.arange(7), np.arange(9), indexing="ij")
    lin = (1.0 + 0.5 * e + 0.25 * h + 0.125 * w).astype(np.float32)
    g = D.trilerp_ehw(lin, (9, 13, 17))
    E, H, W = np.meshgrid(np.arange(9) * 4 / 8, np.arange(13) * 6 / 12, np.arange(17) * 8 / 16, indexing="ij")
    np.testing.assert_allclose(g, 1.0 + 0.5 * E + 0.25 * H + 0.125 * W, rtol=2e-6)


def test_rebin_and_crop_range():
    from xtsrcmaps_b200.wcs import Wcs

    roi = Wcs(100, 80, 50.5, 40.5, 193.98, -5.82, -0.2, 0.2, proj="CAR")
    r = D.rebin_wcs(roi, 0.05)
    assert (r.naxis1, r.naxis2, r.cdelt1, r.cdelt2) == (400, 320, -0.05, 0.05)
    assert (r.crpix1, r.crpix2) == (50.5 * 4, 40.5 * 4)
    assert (r.crval1, r.crval2, r.proj) == (roi.crval1, roi.crval2, roi.proj)
    # an all-sky CAR cube at 0.5 deg (longitude decreasing with x, as Fermi's galdiffuse)
    sky = Wcs(720, 361, 360.5, 181.0, 0.0, 0.0, -0.5, 0.5, proj="CAR")
    x0, x1, y0, y1 = D.allsky_crop_range(sky, roi)
    assert 1 <= x0 <= x1 <= 720 and 1 <= y0 <= y1 <= 361
    # the range covers the ROI's corners in the sky image's pixel grid
    for p1, p2 in ((1.0, 1.0), (100.0, 80.0)):
        lon, lat = D.O.pix2sph(roi, p1, p2)
        x, y = D.O.sph2pix(sky, lon % 360.0, lat)
        assert x0 - 0.5 <= x <= x1 + 0.5 and y0 - 0.5 <= y <= y1 + 0.5
    cube = np.arange(2 * 5 * 8, dtype=np.float32).reshape(2, 5, 8)
    np.testing.assert_array_equal(D.crop_allsky(cube, (3, 6, 2, 4)), cube[:, 1:4, 2:6])
    wrapped = D.crop_allsky(cube, (7, 2, 1, 5))  # columns 7, 8, then 1, 2
    np.testing.assert_array_equal(wrapped, cube[:, :, [6, 7, 0, 1]])
