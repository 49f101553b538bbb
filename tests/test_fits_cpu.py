"""The FITS source-map format on the CPU: the oracle's writer against the FITS
checksum convention and a parse-back of its own files (no GPU needed)."""
import numpy as np

from oracle import fits_oracle as F


def test_checksum_encoding_adds_its_value():
    """Replacing the 16 '0' characters of a CHECKSUM value by the encoding of v
    raises the card's ones'-complement sum by exactly v (mod 2^32 - 1): the
    defining property of the convention's char_encode."""
    rng = np.random.default_rng(3)
    zero = F._card("CHECKSUM", "0" * 16, True)
    for v in [0, 1, 0xffffffff, 0x7fffffff, 0x80000000] + [int(x) for x in rng.integers(0, 2**32, 200)]:
        enc = F.checksum_encode(v)
        assert len(enc) == 16 and all(c.isalnum() for c in enc), enc
        card = zero[:11] + enc.encode() + zero[27:]
        d = (F.ones_sum(card) - F.ones_sum(zero)) % 0xffffffff
        assert d == v % 0xffffffff, (v, enc)


def test_oracle_file_round_trip(tmp_path):
    rng = np.random.default_rng(4)
    S, H, W, E = 3, 7, 5, 4
    m = rng.standard_normal((S, H, W, E)).astype(np.float32)
    names = ["4FGL J1118.2-0415", "src'q", "X"]
    for bitpix in (-64, -32):
        fn = str(tmp_path / f"m{-bitpix}.fits")
        F.write_src_model(fn, m, names, bitpix)
        raw = open(fn, "rb").read()
        assert len(raw) % F.BLOCK == 0
        hdus = F.read_fits(fn)
        assert len(hdus) == S + 1
        h0 = hdus[0][0]
        assert h0["SIMPLE"] is True and h0["NAXIS"] == 0 and h0["HDUNAME"] == "PRIMARY"
        for s in range(S):
            hdr, hb, db, arr = hdus[s + 1]
            assert hdr["XTENSION"] == "IMAGE" and hdr["BITPIX"] == bitpix
            assert (hdr["NAXIS1"], hdr["NAXIS2"], hdr["NAXIS3"]) == (H, W, E)
            assert hdr["EXTNAME"] == names[s]
            # SHWE -> SEHW: img[e][w][h] = map[s][h][w][e]
            np.testing.assert_array_equal(arr, np.transpose(m[s], (2, 1, 0)).astype(arr.dtype))
            assert int(hdr["DATASUM"]) == F.ones_sum(db)
            assert F.hdu_checksum(hb, db) == 0xffffffff


def test_checksum_detects_a_flipped_byte(tmp_path):
    """A mistake planted in the oracle's output (one data byte changed) breaks
    the HDU checksum property the tests rely on."""
    fn = str(tmp_path / "m.fits")
    F.write_src_model(fn, np.ones((1, 4, 4, 2), np.float32))
    hdr, hb, db, _ = F.read_fits(fn)[1]
    bad = bytearray(db)
    bad[5] ^= 0x10
    assert F.hdu_checksum(hb, bytes(bad)) != 0xffffffff


def test_cli_help():
    import subprocess
    import sys

    r = subprocess.run([sys.executable, "-m", "xtsrcmaps_b200", "--help"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and "--out" in r.stdout
