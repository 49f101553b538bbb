"""IRF ingest without cfitsio (fits/fits.read_irf_pars.cxx:12-126, irf/irf.cxx:24-70):
the host FITS reader on a binary table written here, and on the reference's own
Pass-8 IRF files when the reference tree is present, against the rows its tests
expect (tests/fits/aeff_expected.hxx, psf_expected.hxx, kept in tests/golden/irf.npz)."""
import os

import numpy as np
import pytest

from xtsrcmaps_b200 import fits_io, irf

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("XTS_REFERENCE", "/root/reference")
ANALYSIS = os.path.join(REF, "analysis")


def _card(k, v):
    if isinstance(v, str):
        s = f"{k:<8}= '{v:<8}'"
    elif isinstance(v, bool):
        s = f"{k:<8}= {'T' if v else 'F':>20}"
    else:
        s = f"{k:<8}= {v:>20}"
    return s.ljust(80).encode()


def _hdr(cards):
    h = b"".join(_card(k, v) for k, v in cards) + b"END".ljust(80)
    return h + b" " * ((-len(h)) % 2880)


def _bintable(path, name, cols, nrows, data):
    """cols: [(TTYPE, TFORM)], data: bytes of nrows rows."""
    width = len(data) // nrows
    cards = [("XTENSION", "BINTABLE"), ("BITPIX", 8), ("NAXIS", 2), ("NAXIS1", width), ("NAXIS2", nrows),
             ("PCOUNT", 0), ("GCOUNT", 1), ("TFIELDS", len(cols))]
    for i, (t, f) in enumerate(cols):
        cards += [(f"TTYPE{i + 1}", t), (f"TFORM{i + 1}", f)]
    cards.append(("EXTNAME", name))
    prim = _hdr([("SIMPLE", True), ("BITPIX", 8), ("NAXIS", 0), ("EXTEND", True)])
    with open(path, "wb") as f:
        f.write(prim + _hdr(cards) + data + b"\0" * ((-len(data)) % 2880))


def test_read_irf_pars_on_a_written_table(tmp_path):
    rng = np.random.default_rng(1)
    rows = rng.standard_normal((2, 3 + 5 + 1)).astype(np.float32)
    fn = str(tmp_path / "t.fits")
    _bintable(fn, "EFFICIENCY_PARAMS_FRONT", [("A", "3E"), ("B", "5E"), ("C", "E")], 2, rows.astype(">f4").tobytes())
    ext, off, data = fits_io.read_irf_pars(fn, "efficiency_params_front")  # names match case-insensitively
    assert list(ext) == [3, 5, 1] and list(off) == [0, 3, 8]
    np.testing.assert_array_equal(data, rows)
    with pytest.raises(KeyError):
        fits_io.read_irf_pars(fn, "RPSF_FRONT")
    _bintable(fn, "X", [("A", "2D")], 1, np.ones(2, ">f8").tobytes())
    with pytest.raises(ValueError):  # the reference accepts FLOAT columns only
        fits_io.read_irf_pars(fn, "X")


@pytest.mark.skipif(not os.path.isdir(ANALYSIS), reason="reference tree not present")
def test_reference_irf_files_match_the_expected_rows():
    g = np.load(os.path.join(HERE, "golden", "irf.npz"))
    gp = np.load(os.path.join(HERE, "golden", "psf.npz"))
    aeff = os.path.join(ANALYSIS, "aeff_P8R3_SOURCE_V2_FB.fits")
    psf = os.path.join(ANALYSIS, "psf_P8R3_SOURCE_V2_FB.fits")
    for side in ("front", "back"):
        S = side.upper()
        for fn, table, key in ((aeff, f"EFFECTIVE AREA_{S}", "aeff"), (psf, f"RPSF_{S}", "rpsf")):
            ext, off, rows = fits_io.read_irf_pars(fn, table)
            np.testing.assert_array_equal(ext, g[f"{key}_{side}_extents"])
            np.testing.assert_array_equal(off, g[f"{key}_{side}_offsets"])
            np.testing.assert_array_equal(rows[0], g[f"{key}_{side}_row"])
    a, p = irf.load_aeff(aeff), irf.load_psf(psf)
    for side in ("front", "back"):
        np.testing.assert_array_equal(a[side].effic.p0, g[f"effic_{side}_p0"])
        np.testing.assert_array_equal(a[side].effic.p1, g[f"effic_{side}_p1"])
        sc = p[side].scale
        np.testing.assert_array_equal(np.float32([sc.scale0, sc.scale1, sc.scale_index]), g[f"scaling_{side}"])
        np.testing.assert_array_equal(p[side].grid.params, gp[f"rpsf_{side}"])
        assert a[side].grid.params.shape == (34, 76, 1)


@pytest.mark.skipif(not os.path.isdir(ANALYSIS), reason="reference tree not present")
def test_reference_counts_cube_energies_and_wcs():
    """fits.read_energies / read_image_meta on the reference's 3C279 counts cube
    against tests/fits/ccube_energies_expected.hxx (8 digits) and the header values
    the reference's test_fitsfuncs.cxx requires."""
    fn = os.path.join(ANALYSIS, "3C279_binned_ccube.fits")
    e = fits_io.read_energies(fn)
    g = np.load(os.path.join(HERE, "golden", "irf.npz"))["energies"]
    np.testing.assert_allclose(e, g, rtol=1e-7)
    w, n3 = fits_io.read_image_meta(fn)
    gg = np.load(os.path.join(HERE, "golden", "geom.npz"))
    assert (w.naxis1, w.naxis2, n3) == (100, 100, 37) and w.proj == "AIT" and not w.galactic
    np.testing.assert_array_equal([w.crpix1, w.crpix2], gg["crpix"])
    np.testing.assert_array_equal([w.crval1, w.crval2], gg["crval"])
    np.testing.assert_array_equal([w.cdelt1, w.cdelt2], gg["cdelt"])


def test_read_expcube_on_a_written_cube(tmp_path):
    nside, nbr = 2, 40
    npix = 12 * nside * nside
    rng = np.random.default_rng(2)
    cos = rng.lognormal(0, 0.2, (npix, nbr)).astype(np.float32)
    radec = rng.uniform(0, 90, (npix, 2)).astype(np.float32)
    rows = b"".join(cos[i].astype(">f4").tobytes() + radec[i].astype(">f4").tobytes() for i in range(npix))
    fn = str(tmp_path / "lt.fits")
    _bintable(fn, "EXPOSURE", [("COSBINS", f"{nbr}E"), ("RA", "E"), ("DEC", "E")], npix, rows)
    # the keys read_expcube needs, spliced into the table header
    raw = bytearray(open(fn, "rb").read())
    end = raw.index(b"END" + b" " * 77, 2880)
    keys = b"".join(_card(k, v) for k, v in [("NSIDE", nside), ("NBRBINS", nbr), ("COSMIN", 0.0),
                                             ("ORDERING", "NESTED"), ("COORDSYS", "EQU"), ("THETABIN", "SQRT(1-COSTHETA)")])
    assert raw[end + 80:end + 80 + len(keys)].strip() == b""  # room in the header block
    raw[end:end + 80 + len(keys)] = keys + b"END".ljust(80)
    open(fn, "wb").write(bytes(raw))
    c = fits_io.read_expcube(fn, "EXPOSURE")
    assert (c.nside, c.nbrbins, c.cosmin, c.thetabin) == (nside, nbr, 0.0, True)
    np.testing.assert_array_equal(c.cosbins, cos)


def test_point_sources_from_xml(tmp_path):
    from xtsrcmaps_b200.sources import read_point_sources

    xml = tmp_path / "m.xml"
    xml.write_text("""<source_library>
 <source name="b src" type="PointSource"><spectrum type="PowerLaw"/>
  <spatialModel type="SkyDirFunction"><parameter name="RA" value="193.123456789" free="0" scale="1" min="0" max="360"/>
   <parameter name="DEC" value="-5.5" free="0" scale="1" min="-90" max="90"/></spatialModel></source>
 <source name="galdiff" type="DiffuseSource"><spatialModel type="MapCubeFunction" file="x.fits"/></source>
 <source name="A src" type="PointSource"><spatialModel type="SkyDirFunction">
   <parameter name="DEC" value="1.25" free="0" scale="1" min="-90" max="90"/>
   <parameter name="RA" value="10" free="0" scale="1" min="0" max="360"/></spatialModel></source>
</source_library>""")
    names, sph = read_point_sources(str(xml))
    assert names == ["A src", "b src"]  # byte order, as std::sort on std::string
    np.testing.assert_array_equal(sph, [[10.0, 1.25], [float(np.float32(193.123456789)), -5.5]])


@pytest.mark.skipif(not os.path.isdir(ANALYSIS), reason="reference tree not present")
def test_reference_point_source_model():
    from xtsrcmaps_b200.sources import read_point_sources

    names, sph = read_point_sources(os.path.join(ANALYSIS, "3C279_input_model_point.xml"))
    gg = np.load(os.path.join(HERE, "golden", "geom.npz"))
    assert names == [str(n) for n in gg["src_names"]] and len(names) == 263
    np.testing.assert_allclose(sph, gg["src_sph"], atol=1e-5)  # float32 values, as std::stof
