"""Point sources of a Fermi XML source model (the reference's
source/source.parse_src_mdl.cxx and Source::spherical_coords, source/source.cxx:6-40).

Only what the point-source path needs: each PointSource's name and the RA and DEC
parameters of its SkyDirFunction spatial model.  As in the reference, parameter
values are parsed as float (std::stof, parse_src_mdl.cxx:153) before they become the
double [S, 2] position table, and the sources are sorted by name
(sort_source_vector, parse_src_mdl.cxx:25-31).
"""
from __future__ import annotations

import xml.etree.ElementTree as ET

import numpy as np


def read_point_sources(path: str):
    """(names sorted, sph [S, 2] degrees as float64 of the float32 values)."""
    root = ET.parse(path).getroot()
    out = []
    for s in root.iter("source"):
        if s.get("type") != "PointSource":
            continue
        sm = s.find("spatialModel")
        if sm is None:
            raise ValueError(f"{path}: point source {s.get('name')!r} has no spatialModel")
        pars = {p.get("name"): np.float32(p.get("value")) for p in sm.iter("parameter")}
        if "RA" not in pars or "DEC" not in pars:
            raise ValueError(f"{path}: point source {s.get('name')!r} lacks RA or DEC")
        out.append((s.get("name"), float(pars["RA"]), float(pars["DEC"])))
    out.sort(key=lambda t: t[0].encode())
    names = [t[0] for t in out]
    sph = np.array([[t[1], t[2]] for t in out], dtype=np.float64).reshape(-1, 2)
    return names, sph
