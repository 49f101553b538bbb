"""Generate the golden fixtures in tests/golden/ from the reference's own test data.

Run in a container that has the xtsrcmaps reference checkout (default
/root/reference, override with XTS_REFERENCE):

    python tests/golden/make_golden.py

The script only reads the reference's test headers (tests/fits/*.hxx, parsed as
text), its expected-output blobs (tests/expected/*.bin, little-endian row-major
doubles), the FITS header of the counts cube and the source-model XML in
analysis/.  It writes small compressed .npz files next to itself.  The GPU box
never runs it; the committed .npz files travel instead.

Fixtures:
  irf.npz       raw Aeff / PSF / efficiency / scaling rows of the P8R3_SOURCE_V2
                IRF tables (tests/fits/aeff_expected.hxx, psf_expected.hxx),
                expected Aeff [C,E] tables, livetime-efficiency factors,
                cos-theta bin centres and counts-cube energies.
  exposure.npz  livetime rows of the 263 sources (exposure_cosbins_expected.hxx)
                and the expected exposure [263, 38] (expected/exposure.bin) plus
                the four intermediate contractions (exposure_le{f,b}, lw{f,b}).
  psf.npz       prepared and normalised King parameter grids (psf3_*.bin), a
                strided slice of king_front.bin, the normalised mean-PSF peak
                uPsf[:, 0, :] (uPsf_peak_SE.bin) and the separation grid.
  geom.npz      counts-cube WCS (AIT), source positions from the XML model (in
                the reference's name-sorted order), Fermitools boundary radii
                and in-FOV flags (ft_mm_psf_radius.bin, ft_mm_withinBounds.bin).
"""
from __future__ import annotations

import os
import re
import xml.etree.ElementTree as ET

import numpy as np

REF = os.environ.get("XTS_REFERENCE", "/root/reference")
OUT = os.path.dirname(os.path.abspath(__file__))
NUM = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?")


def _strip_comments(txt: str) -> str:
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return re.sub(r"//[^\n]*", "", txt)


def _read(path: str) -> str:
    with open(os.path.join(REF, path)) as f:
        return _strip_comments(f.read())


def _block(txt: str, start: int) -> tuple[str, int]:
    """Return the balanced {...} block that opens at or after ``start``."""
    i = txt.index("{", start)
    depth = 0
    for j in range(i, len(txt)):
        if txt[j] == "{":
            depth += 1
        elif txt[j] == "}":
            depth -= 1
            if depth == 0:
                return txt[i + 1:j], j + 1
    raise ValueError("unbalanced braces")


def _subblocks(body: str) -> list[str]:
    out, i = [], 0
    while True:
        k = body.find("{", i)
        if k < 0:
            return out
        b, i = _block(body, k)
        out.append(b)


def _nums(s: str, dtype=np.float64) -> np.ndarray:
    return np.array([float(x) for x in NUM.findall(s)], dtype=dtype)


def vector(txt: str, name: str, after: int = 0) -> np.ndarray:
    m = re.compile(r"\b" + re.escape(name) + r"\s*(?:=\s*std::vector\s*<[^>]*>\s*)?(?=\{)").search(txt, after)
    body, _ = _block(txt, m.end())
    return _nums(body)


def expected(txt: str, name: str) -> list[np.ndarray]:
    m = re.compile(r"\bconst\s+Expected\w*\s+" + re.escape(name) + r"\b").search(txt)
    body, _ = _block(txt, m.end())
    return [_nums(b) for b in _subblocks(body)]


def binfile(name: str, shape) -> np.ndarray:
    a = np.fromfile(os.path.join(REF, "tests/expected", name + ".bin"), dtype="<f8")
    return a.reshape(shape)


def fits_header(path: str) -> dict:
    raw = open(os.path.join(REF, path), "rb").read(2880 * 4).decode("ascii", "replace")
    hdr = {}
    for i in range(0, len(raw), 80):
        card = raw[i:i + 80]
        if card.startswith("END"):
            break
        if card[8:10] == "= ":
            key, val = card[:8].strip(), card[10:].split("/")[0].strip()
            hdr[key] = val.strip("'").strip()
    return hdr


def main() -> None:
    aeff = _read("tests/fits/aeff_expected.hxx")
    psf = _read("tests/fits/psf_expected.hxx")
    cos = _read("tests/fits/exposure_cosbins_expected.hxx")
    ene = _read("tests/fits/ccube_energies_expected.hxx")
    sep = _read("tests/fits/separations_expected.hxx")

    irf = {}
    for side in ("FRONT", "BACK"):
        ext, off, row = expected(aeff, "EFFECTIVE_AREA_" + side)
        irf[f"aeff_{side.lower()}_extents"] = ext.astype(np.int64)
        irf[f"aeff_{side.lower()}_offsets"] = off.astype(np.int64)
        irf[f"aeff_{side.lower()}_row"] = row.astype(np.float32)
        _, _, p0, p1 = expected(aeff, "EFFICIENCY_PARAMS_" + side)
        irf[f"effic_{side.lower()}_p0"] = p0.astype(np.float32)
        irf[f"effic_{side.lower()}_p1"] = p1.astype(np.float32)
        ext, off, row = expected(psf, "RPSF_" + side)
        irf[f"rpsf_{side.lower()}_extents"] = ext.astype(np.int64)
        irf[f"rpsf_{side.lower()}_offsets"] = off.astype(np.int64)
        irf[f"rpsf_{side.lower()}_row"] = row.astype(np.float32)
        _, _, sc = expected(psf, "PSF_SCALING_PARAMS_" + side)
        irf[f"scaling_{side.lower()}"] = sc.astype(np.float32)
    irf["livetime_factor1"] = vector(aeff, "livetime_factor1")
    irf["livetime_factor2"] = vector(aeff, "livetime_factor2")
    irf["aeff_front_c_e"] = vector(cos, "aeff_front_c_e").reshape(40, 38)
    irf["aeff_back_c_e"] = vector(cos, "aeff_back_c_e").reshape(40, 38)
    irf["exp_costhetas"] = vector(cos, "exp_costhetas")
    irf["energies"] = vector(ene, "expected")
    np.savez_compressed(os.path.join(OUT, "irf.npz"), **irf)

    front = aeff.index("namespace Front")
    back = aeff.index("namespace Back")
    expo = {
        "ecb": vector(cos, "exposure_source_cosine_bins").reshape(-1, 40).astype(np.float32),
        "wecb": vector(cos, "weighted_exposure_source_cosine_bins").reshape(-1, 40).astype(np.float32),
        "exposure": binfile("exposure", (263, 38)),
        "lef": binfile("exposure_lef", (263, 38)),
        "lwf": binfile("exposure_lwf", (263, 38)),
        "leb": binfile("exposure_leb", (263, 38)),
        "lwb": binfile("exposure_lwb", (263, 38)),
        "exp_aeff_front": vector(aeff, "exp_aeff", front).reshape(263, 38),
        "exp_aeff_back": vector(aeff, "exp_aeff", back).reshape(263, 38),
    }
    np.savez_compressed(os.path.join(OUT, "exposure.npz"), **expo)

    kf = binfile("king_front", (401, 10, 25))
    psfz = {
        "rpsf_front": binfile("psf3_rpsf.front", (10, 25, 6)),
        "rpsf_back": binfile("psf3_rpsf.back", (10, 25, 6)),
        "norm_rpsf_front": binfile("psf3_normalized_rpsf.front", (10, 25, 6)),
        "norm_rpsf_back": binfile("psf3_normalized_rpsf.back", (10, 25, 6)),
        "king_front_rows": np.arange(0, 401, 8),
        "king_front": kf[0:401:8],
        "upsf_peak": binfile("uPsf_peak_SE", (263, 38)),
        "separations": vector(sep, "expected_separations"),
    }
    np.savez_compressed(os.path.join(OUT, "psf.npz"), **psfz)

    hdr = fits_header("analysis/3C279_binned_ccube.fits")
    root = ET.parse(os.path.join(REF, "analysis/3C279_input_model_point.xml")).getroot()
    srcs = []
    for s in root.iter("source"):
        if s.get("type") != "PointSource":
            continue
        pars = {p.get("name"): float(p.get("value")) for p in s.find("spatialModel").iter("parameter")}
        srcs.append((s.get("name"), pars["RA"], pars["DEC"]))
    srcs.sort(key=lambda t: t[0])  # source/source.parse_src_mdl.cxx sorts by name
    geom = {
        "naxis": np.array([int(hdr["NAXIS1"]), int(hdr["NAXIS2"])]),
        "crpix": np.array([float(hdr["CRPIX1"]), float(hdr["CRPIX2"])]),
        "crval": np.array([float(hdr["CRVAL1"]), float(hdr["CRVAL2"])]),
        "cdelt": np.array([float(hdr["CDELT1"]), float(hdr["CDELT2"])]),
        "crota2": np.array(float(hdr.get("CROTA2", "0"))),
        "proj": np.array(hdr["CTYPE1"][-3:]),
        "src_sph": np.array([[r, d] for _, r, d in srcs]),
        "src_names": np.array([n for n, _, _ in srcs]),
        "ft_psf_radius": np.fromfile(os.path.join(REF, "tests/expected/ft_mm_psf_radius.bin"), "<f8"),
        "ft_in_fov": np.fromfile(os.path.join(REF, "tests/expected/ft_mm_withinBounds.bin"), np.uint8),
    }
    np.savez_compressed(os.path.join(OUT, "geom.npz"), **geom)
    for f in ("irf", "exposure", "psf", "geom"):
        print(f, os.path.getsize(os.path.join(OUT, f + ".npz")), "bytes")


if __name__ == "__main__":
    main()
