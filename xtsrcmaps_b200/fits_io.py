"""Minimal FITS reading on the host: the IRF tables and the counts-cube header.

The reference reads its inputs through cfitsio (fits/fits.read_irf_pars.cxx:12-126 for
the IRF parameter tables, observation/observation.cxx for the counts cube); cfitsio is
not a dependency of this package, so the few structures the path needs are parsed here
from the FITS standard 4.0: 80-byte header cards in 2880-byte blocks, IMAGE and
BINTABLE extensions, big-endian data.  Only fixed-length columns are read (the IRF
tables have no variable-length arrays).
"""
from __future__ import annotations

import numpy as np

BLOCK = 2880

# TFORM type codes of fixed-length binary-table columns -> (numpy big-endian type, bytes)
_TFORM = {"L": ("u1", 1), "X": ("u1", 1), "B": ("u1", 1), "I": (">i2", 2), "J": (">i4", 4), "K": (">i8", 8),
          "A": ("S1", 1), "E": (">f4", 4), "D": (">f8", 8), "C": (">c8", 8), "M": (">c16", 16)}


def _value(v: str):
    v = v.strip()
    if v.startswith("'"):
        end = v.find("'", 1)
        while end != -1 and end + 1 < len(v) and v[end + 1] == "'":  # doubled quote
            end = v.find("'", end + 2)
        return v[1:end].replace("''", "'").rstrip()
    v = v.split("/", 1)[0].strip()
    if v in ("T", "F"):
        return v == "T"
    try:
        return int(v)
    except ValueError:
        pass
    try:
        return float(v.replace("D", "E"))
    except ValueError:
        return v


class Hdu:
    """One header-data unit: ``header`` (keyword -> value, in order) and the
    position of its data in the file."""

    def __init__(self, header: dict, data_start: int, data_bytes: int):
        self.header = header
        self.data_start = data_start
        self.data_bytes = data_bytes

    @property
    def name(self) -> str:
        return str(self.header.get("EXTNAME", self.header.get("HDUNAME", "")))


def read_hdus(raw: bytes) -> list:
    """Split a FITS file into HDUs."""
    hdus, pos = [], 0
    while pos + BLOCK <= len(raw):
        header, start = {}, pos
        while True:
            if pos + 80 > len(raw):
                raise ValueError("FITS header without END")
            card = raw[pos:pos + 80].decode("ascii", "replace")
            pos += 80
            key = card[:8].strip()
            if key == "END":
                break
            if card[8:10] == "= " and key not in header:
                header[key] = _value(card[10:])
        pos = start + -(-(pos - start) // BLOCK) * BLOCK
        naxis = int(header.get("NAXIS", 0))
        n = 1
        for i in range(naxis):
            n *= int(header[f"NAXIS{i + 1}"])
        nbytes = abs(int(header.get("BITPIX", 8))) // 8 * int(header.get("GCOUNT", 1)) * \
            (int(header.get("PCOUNT", 0)) + (n if naxis else 0))
        hdus.append(Hdu(header, pos, nbytes))
        pos += -(-nbytes // BLOCK) * BLOCK
    return hdus


def _tform(tform: str):
    t = tform.strip()
    i = 0
    while i < len(t) and t[i].isdigit():
        i += 1
    repeat = int(t[:i]) if i else 1
    code = t[i]
    if code in "PQ":
        raise ValueError(f"variable-length column {tform!r} is not supported")
    dt, size = _TFORM[code]
    return repeat, code, dt, size


def read_bintable(path: str, extname: str):
    """Columns of the binary table ``extname`` (matched case-insensitively, as
    cfitsio's fits_movnam_hdu does): list of (TTYPE, TFORM code, repeat, array
    [nrows, repeat]) and the raw row bytes [nrows, NAXIS1]."""
    raw = open(path, "rb").read()
    for h in read_hdus(raw):
        if h.header.get("XTENSION", "").strip().upper() != "BINTABLE":
            continue
        if h.name.strip().upper() != extname.strip().upper():
            continue
        width, nrows = int(h.header["NAXIS1"]), int(h.header["NAXIS2"])
        rows = np.frombuffer(raw, dtype=np.uint8, count=width * nrows, offset=h.data_start).reshape(nrows, width)
        cols, off = [], 0
        for c in range(int(h.header["TFIELDS"])):
            repeat, code, dt, size = _tform(h.header[f"TFORM{c + 1}"])
            nb = repeat * size if code != "X" else (repeat + 7) // 8
            block = np.ascontiguousarray(rows[:, off:off + nb])
            arr = block.view(dt).reshape(nrows, -1) if code not in "X" else block
            cols.append((str(h.header.get(f"TTYPE{c + 1}", "")), code, repeat, arr))
            off += nb
        if off != width:
            raise ValueError(f"{extname}: column widths {off} != NAXIS1 {width}")
        return cols, rows
    raise KeyError(f"{path}: no binary table named {extname!r}")


def read_irf_pars(path: str, tblname: str):
    """Fermi::fits::read_irf_pars (fits/fits.read_irf_pars.cxx:12-126): every column
    must be FLOAT ('E'); returns (extents = column repeats, offsets = their exclusive
    scan, rowdata float32 [nrows, sum(extents)]) -- each row's columns back to back,
    converted from big-endian."""
    cols, rows = read_bintable(path, tblname)
    for name, code, _, _ in cols:
        if code != "E":
            raise ValueError(f"{path} {tblname}: column {name} is {code!r}, expected a FLOAT column")
    extents = np.array([c[2] for c in cols], dtype=np.int64)
    offsets = np.concatenate([[0], np.cumsum(extents)[:-1]]).astype(np.int64)
    rowdata = np.ascontiguousarray(rows).view(">f4").astype(np.float32).reshape(rows.shape[0], -1)
    return extents, offsets, rowdata


def read_image_header(path: str, hdu: int = 0) -> dict:
    """Header of HDU ``hdu`` (0 = primary), e.g. a counts cube's WCS keywords."""
    return read_hdus(open(path, "rb").read())[hdu].header


def read_energies(path: str) -> np.ndarray:
    """Fermi::fits::read_energies (fits/fits.read_energies.cxx:6-46): the second HDU's
    E_MIN column (column 2) for every row and E_MAX (column 3) of the last row, as
    doubles, divided by 1000 (keV -> MeV): NAXIS2 + 1 energies."""
    raw = open(path, "rb").read()
    h = read_hdus(raw)[1]
    cols, _ = read_bintable(path, h.name) if h.name else (None, None)
    if cols is None or len(cols) < 3:
        raise ValueError(f"{path}: second HDU is not an energy-bounds table")
    emin, emax = cols[1][3].astype(np.float64).ravel(), cols[2][3].astype(np.float64).ravel()
    return np.concatenate([emin, emax[-1:]]) / 1000.0


def read_image_meta(path: str):
    """Fermi::fits::read_image_meta (fits/fits.read_image_meta.cxx): the counts
    cube's NAXIS1..3, CRPIX, CRVAL, CDELT, CROTA2 and CTYPE1 (projection = its last
    '-'-separated token, galactic when the first is GLON), as (Wcs, NAXIS3)."""
    from .wcs import Wcs

    h = read_image_header(path, 0)
    tokens = [t for t in str(h["CTYPE1"]).split("-") if t]
    return (Wcs(int(h["NAXIS1"]), int(h["NAXIS2"]), float(h["CRPIX1"]), float(h["CRPIX2"]), float(h["CRVAL1"]),
                float(h["CRVAL2"]), float(h["CDELT1"]), float(h["CDELT2"]), float(h.get("CROTA2", 0.0)),
                tokens[-1], tokens[0] == "GLON"), int(h.get("NAXIS3", 1)))


def read_expcube(path: str, tblname: str = "EXPOSURE"):
    """Fermi::fits::read_expcube (fits/fits.read_expcube.cxx:8-130): the livetime cube
    table ``tblname`` (EXPOSURE or WEIGHTED_EXPOSURE) with keys NSIDE, NBRBINS,
    COSMIN, ORDERING (must be NESTED), COORDSYS (must be EQU) and THETABIN
    (anything but COSTHETA means sqrt binning); column 1 holds NBRBINS float
    livetimes per HEALPix pixel.  Returns an api.ExpCube."""
    from .api import ExpCube

    raw = open(path, "rb").read()
    h = next((x for x in read_hdus(raw) if x.header.get("XTENSION", "").strip().upper() == "BINTABLE"
              and x.name.strip().upper() == tblname.strip().upper()), None)
    if h is None:
        raise KeyError(f"{path}: no binary table named {tblname!r}")
    hd = h.header
    nside, nbr, cosmin = int(hd["NSIDE"]), int(hd["NBRBINS"]), float(hd["COSMIN"])
    if str(hd["ORDERING"]).strip() != "NESTED":
        raise ValueError(f"{path}: ORDERING {hd['ORDERING']!r}; only NESTED cubes are read")
    if str(hd["COORDSYS"]).strip() != "EQU":
        raise ValueError(f"{path}: COORDSYS {hd['COORDSYS']!r}; only EQU cubes are read")
    cols, _ = read_bintable(path, tblname)
    cos = cols[0][3]
    if cols[0][1] not in "ED":
        raise ValueError(f"{path}: {tblname} column 1 must be floating point")
    cube = np.ascontiguousarray(cos.astype(np.float32).reshape(-1)[: 12 * nside * nside * nbr]
                                .reshape(12 * nside * nside, nbr))
    return ExpCube(cube, nside, nbr, cosmin, str(hd["THETABIN"]).strip() != "COSTHETA")
