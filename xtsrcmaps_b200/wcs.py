"""Host-side description of the counts-map WCS (sky_geom/sky_geom.hxx:17-25).

The projection arithmetic itself runs on the GPU (csrc/xts_geom.cuh); this is
only the parameter record that crosses the C-ABI.
"""
from __future__ import annotations

from dataclasses import dataclass

PROJ_CODES = {"CAR": 0, "AIT": 1}


@dataclass
class Wcs:
    """FITS celestial WCS of an H x W map, H = NAXIS1 (longitude axis).

    Pixel coordinates are 1-based FITS coordinates, as in the reference's
    ``SkyGeom::pix2sph`` (wcslib ``wcsp2s``).
    """

    naxis1: int
    naxis2: int
    crpix1: float
    crpix2: float
    crval1: float
    crval2: float
    cdelt1: float
    cdelt2: float
    crota2: float = 0.0
    proj: str = "CAR"
    galactic: bool = False

    def __post_init__(self):
        self.proj = str(self.proj).upper()
        if self.proj not in PROJ_CODES:
            raise ValueError("unsupported projection %r (CAR and AIT are supported)" % self.proj)

    @property
    def proj_code(self) -> int:
        return PROJ_CODES[self.proj]
