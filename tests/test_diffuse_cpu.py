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
