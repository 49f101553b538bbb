"""FITS output on the GPU (xts_write_src_model): the library's file is
byte-identical to the oracle's restatement of Fermi::fits::write_src_model for
the same maps, from device and host maps, float and double, BITPIX -64 and -32,
in one chunk and in many; every HDU satisfies the checksum convention."""
import os

import numpy as np
import pytest

from oracle import fits_oracle as F

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


@pytest.mark.parametrize("dtype,bitpix,device,chunk_mb", [
    (np.float32, -64, True, None), (np.float32, -32, False, None),
    (np.float64, -32, True, None), (np.float64, -64, False, "1"), (np.float32, -64, True, "1")])
def test_fits_bytes_match_oracle(api, tmp_path, monkeypatch, dtype, bitpix, device, chunk_mb):
    import torch

    if chunk_mb:
        monkeypatch.setenv("XTS_FITS_CHUNK_MB", chunk_mb)
    rng = np.random.default_rng(5)
    S, H, W, E = 9, 67, 45, 37  # ragged tiles in h and e; 9 x 0.9 MB (f64) spans several 1 MiB chunks
    m = (rng.lognormal(0.0, 3.0, (S, H, W, E)) * rng.choice([-1.0, 1.0], (S, H, W, E))).astype(dtype)
    names = ["PS J%04d" % s for s in range(S)]
    names[2] = "it's"
    ours, ref = str(tmp_path / "gpu.fits"), str(tmp_path / "ref.fits")
    arg = torch.as_tensor(m, device="cuda") if device else m
    api.write_src_model(ours, arg, names, bitpix)
    F.write_src_model(ref, m, names, bitpix)
    a, b = open(ours, "rb").read(), open(ref, "rb").read()
    assert len(a) == len(b)
    assert a == b
    for hdr, hb, db, _ in F.read_fits(ours)[1:]:
        assert F.hdu_checksum(hb, db) == 0xffffffff


def test_fits_of_computed_maps(api, tmp_path):
    """The maps of the fused call on c0, straight from device memory to a file
    whose images are the maps in SEHW order."""
    import torch

    from xtsrcmaps_b200.synth import make_job

    job = make_job("c0", seed=2)
    d = torch.device("cuda")
    ltf = api.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = api.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = api.normalize_rpsf(job.rpsf_back, job.scale_back)
    m, _ = api.point_source_maps(job.wcs, job.src_sph, job.exp_cube, job.wexp_cube, job.logEs, job.aeff_front,
                                 job.aeff_back, nf, nb, ltf, with_info=False)
    fn = str(tmp_path / "c0.fits")
    api.write_src_model(fn, torch.as_tensor(m, device=d), ["SRC A"])
    hdus = F.read_fits(fn)
    assert len(hdus) == 2 and hdus[1][0]["EXTNAME"] == "SRC A"
    np.testing.assert_array_equal(hdus[1][3], np.transpose(m[0], (2, 1, 0)).astype(np.float64))
    assert F.hdu_checksum(hdus[1][1], hdus[1][2]) == 0xffffffff


def test_fits_bad_names(api, tmp_path):
    from xtsrcmaps_b200 import _lib

    m = np.zeros((1, 2, 2, 1), np.float32)
    with pytest.raises(_lib.XtsError) as ei:
        api.write_src_model(str(tmp_path / "x.fits"), m, ["x" * 69])
    assert ei.value.code == _lib.XTS_ERR_ARG
    with pytest.raises(_lib.XtsError) as ei:
        api.write_src_model(str(tmp_path / "no_such_dir" / "x.fits"), m)
    assert ei.value.code == _lib.XTS_ERR_IO


def test_cli_end_to_end(api, tmp_path):
    """python -m xtsrcmaps_b200: the main.cxx flow with the write call, on c0."""
    from xtsrcmaps_b200.__main__ import main

    src = tmp_path / "src.npz"
    np.savez(src, src_sph=np.array([[193.98, -5.82], [194.5, -6.3]]), names=np.array(["A", "B"]))
    fn = str(tmp_path / "cli.fits")
    assert main(["--config", "c0", "--sources", str(src), "--out", fn, "--bitpix", "-32"]) == 0
    hdus = F.read_fits(fn)
    assert [h[0].get("EXTNAME") for h in hdus[1:]] == ["A", "B"]
    for hdr, hb, db, arr in hdus[1:]:
        assert hdr["BITPIX"] == -32 and arr.shape == (20, 100, 100)
        assert F.hdu_checksum(hb, db) == 0xffffffff
        assert np.isfinite(arr).all() and arr.max() > 0


def test_cli_surrogate(api, tmp_path):
    """python -m xtsrcmaps_b200 --train-surrogate, then --surrogate with the saved network."""
    from xtsrcmaps_b200.__main__ import main

    net = str(tmp_path / "net.npz")
    fn1, fn2, fn0 = (str(tmp_path / f) for f in ("s1.fits", "s2.fits", "plain.fits"))
    base = ["--config", "c0", "--bitpix", "-32"]
    assert main(base + ["--out", fn0]) == 0
    assert main(base + ["--out", fn1, "--train-surrogate", net, "--surrogate-samples", "400000",
                        "--surrogate-epochs", "4"]) == 0
    assert main(base + ["--out", fn2, "--surrogate", net]) == 0
    a0, a1, a2 = (F.read_fits(f)[1][3] for f in (fn0, fn1, fn2))
    np.testing.assert_array_equal(a1, a2)  # the saved network reproduces the maps
    assert np.isfinite(a1).all() and a1.shape == a0.shape
    assert np.max(np.abs(a1.astype(np.float64) - a0) / np.maximum(np.abs(a0), 1e-30)) < 1e-3
