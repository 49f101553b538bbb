"""Oracle for the FITS source-map output -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may import this
module, as the checker.  It restates, in numpy, Fermi::fits::write_src_model
(xtsrcmaps/fits/fits.write_src_model.cxx:10-66), which writes through cfitsio:

  * a primary HDU without data, ``HDUNAME = 'PRIMARY'`` (:25-29);
  * per source an IMAGE extension with NAXIS = 3 and ``EXTNAME`` = the source
    name (:51-60), holding the map reordered SHWE -> SEHW by
    ``reorder_tensor(model_map, {0, 3, 2, 1})`` (:43;
    xtsrcmaps/tensor/reorder_tensor.hpp:10-56: new[i0][i3][i2][i1] = old[i0][i1][i2][i3]),
    written as doubles (TDOUBLE into a DOUBLE_IMG, :49, :63);
  * ``fits_write_chksum`` (:65): DATASUM and CHECKSUM.

The reference's header gives NAXIS1 = Nw and NAXIS2 = Nh although h is the
fastest axis of its data; both are equal for the square maps its cubature
fills (points_weights.hpp:21).  This restatement (and the library) declare
NAXIS1 = H, the data's fastest axis.

Card layout and the checksum follow the FITS standard 4.0 (fixed-format cards,
2880-byte blocks, big-endian IEEE data) and the FITS checksum convention
(Seaman, Pence and Rots 2002): DATASUM is the 32-bit ones'-complement sum of the
data unit; CHECKSUM is the ASCII encoding of the complement of the whole HDU's
sum, after which the HDU sums to -0 (0xffffffff).  cfitsio is not installed
here, so parity is pinned by that defining property (``hdu_checksum``) and by
round trips, not by files the reference wrote.
"""
from __future__ import annotations

import numpy as np

BLOCK = 2880
_EXCLUDE = (0x3a, 0x3b, 0x3c, 0x3d, 0x3e, 0x3f, 0x40, 0x5b, 0x5c, 0x5d, 0x5e, 0x5f, 0x60)


def ones_sum(data: bytes, start: int = 0) -> int:
    """32-bit ones'-complement sum of big-endian words (len % 4 == 0)."""
    w = np.frombuffer(data, dtype=">u4").astype(np.uint64)
    s = int(w.sum(dtype=np.uint64)) + start
    while s >> 32:
        s = (s & 0xffffffff) + (s >> 32)
    return s


def checksum_encode(value: int) -> str:
    """ASCII encoding of a 32-bit value (the checksum convention's char_encode)."""
    asc = [0] * 16
    for i in range(4):
        byte = (value >> (24 - 8 * i)) & 0xff
        quot, rem = byte // 4 + 0x30, byte % 4
        ch = [quot + rem, quot, quot, quot]
        again = True
        while again:
            again = False
            for ex in _EXCLUDE:
                for j in (0, 2):
                    if ch[j] == ex or ch[j + 1] == ex:
                        ch[j] += 1
                        ch[j + 1] -= 1
                        again = True
        for j in range(4):
            asc[4 * j + i] = ch[j]
    return "".join(chr(asc[(i + 15) % 16]) for i in range(16))


def _card(key: str, value, string: bool = False) -> bytes:
    if string:
        q = "'" + str(value).replace("'", "''")
        q = q.ljust(9) + "'"
        s = f"{key:<8.8}= {q:<70.70}"
    else:
        if isinstance(value, bool):
            value = "T" if value else "F"
        s = f"{key:<8.8}= {str(value):>20}" + " " * 50
    assert len(s) == 80
    return s.encode("ascii")


def _end(h: bytes) -> bytes:
    h += b"END".ljust(80)
    return h + b" " * ((-len(h)) % BLOCK)


def primary_header(bitpix: int) -> bytes:
    h = _card("SIMPLE", True) + _card("BITPIX", bitpix) + _card("NAXIS", 0) + _card("EXTEND", True)
    h += _card("HDUNAME", "PRIMARY", True)
    return _end(h)


def image_hdu(img: np.ndarray, name: str, bitpix: int) -> bytes:
    """One IMAGE extension (header with CHECKSUM/DATASUM, data, padding) for
    img [E, W, H] (FITS order, H fastest)."""
    E, W, H = img.shape
    data = np.ascontiguousarray(img, dtype=">f8" if bitpix == -64 else ">f4").tobytes()
    data += b"\0" * ((-len(data)) % BLOCK)
    datasum = ones_sum(data)
    h = (_card("XTENSION", "IMAGE", True) + _card("BITPIX", bitpix) + _card("NAXIS", 3) + _card("NAXIS1", H)
         + _card("NAXIS2", W) + _card("NAXIS3", E) + _card("PCOUNT", 0) + _card("GCOUNT", 1)
         + _card("EXTNAME", name, True))
    ck = len(h)
    h += _card("CHECKSUM", "0" * 16, True) + _card("DATASUM", str(datasum), True)
    h = bytearray(_end(h))
    total = ones_sum(bytes(h), datasum)
    h[ck + 11:ck + 27] = checksum_encode(~total & 0xffffffff).encode("ascii")
    return bytes(h) + data


def write_src_model(filename: str, model_map: np.ndarray, names=None, bitpix: int = -64) -> None:
    """The whole file for maps [S, H, W, E]."""
    S = model_map.shape[0]
    img = np.transpose(model_map, (0, 3, 2, 1))  # SHWE -> SEHW (reorder order {0, 3, 2, 1})
    with open(filename, "wb") as f:
        f.write(primary_header(bitpix))
        for s in range(S):
            f.write(image_hdu(img[s], names[s] if names is not None else "SRC%05d" % s, bitpix))


def read_fits(filename: str):
    """Minimal reader: list of (header dict, raw header bytes, data bytes, data array or None)."""
    raw = open(filename, "rb").read()
    out, pos = [], 0
    while pos < len(raw):
        hdr, start = {}, pos
        while True:
            card = raw[pos:pos + 80].decode("ascii")
            pos += 80
            key = card[:8].strip()
            if key == "END":
                break
            if card[8:10] == "= ":
                v = card[10:].strip()
                if v.startswith("'"):
                    v = v[1:v.rindex("'")].replace("''", "'").rstrip()
                elif v in ("T", "F"):
                    v = v == "T"
                else:
                    v = int(v)
                hdr[key] = v
        pos = start + -(-(pos - start) // BLOCK) * BLOCK
        hbytes = raw[start:pos]
        nax = [hdr.get(f"NAXIS{i + 1}") for i in range(hdr.get("NAXIS", 0))]
        nbytes = int(np.prod(nax)) * abs(hdr["BITPIX"]) // 8 if nax else 0
        dbytes = raw[pos:pos + nbytes + ((-nbytes) % BLOCK)]
        arr = None
        if nax:
            arr = np.frombuffer(raw[pos:pos + nbytes], dtype=">f8" if hdr["BITPIX"] == -64 else ">f4")
            arr = arr.reshape(nax[::-1])
        out.append((hdr, hbytes, dbytes, arr))
        pos += len(dbytes)
    return out


def hdu_checksum(hbytes: bytes, dbytes: bytes) -> int:
    """Ones'-complement sum of a whole HDU: 0xffffffff when CHECKSUM is right."""
    return ones_sum(hbytes, ones_sum(dbytes))
