"""Cutout windows on the host (no GPU): the library's xts_cutout_windows against
the oracle's restatement on the c2 job (500 sources, 10 % near or beyond the
edge), and the window rules at the map's edges."""
import numpy as np

from oracle import oracle as O


def test_windows_match_oracle_on_c2():
    from xtsrcmaps_b200 import api as A
    from xtsrcmaps_b200.synth import make_job

    job = make_job("c2", seed=11)
    cut, total = A.cutout_windows(job.wcs, job.src_sph, job.cutout_deg)
    ref = O.cutout_windows(job.wcs, job.src_sph, job.cutout_deg)
    assert [tuple(int(v) for v in c) for c in cut] == ref
    assert total == sum(r[2] * r[3] for r in ref)
    # windows lie inside the map and follow each other in the ragged output
    assert np.all(cut["h0"] >= 0) and np.all(cut["h0"] + cut["nh"] <= job.wcs.naxis1)
    assert np.all(cut["w0"] >= 0) and np.all(cut["w0"] + cut["nw"] <= job.wcs.naxis2)
    off = np.concatenate([[0], np.cumsum(cut["nh"].astype(np.int64) * cut["nw"])[:-1]])
    np.testing.assert_array_equal(cut["offset"], off)


def test_window_edges():
    from xtsrcmaps_b200 import api as A
    from xtsrcmaps_b200.wcs import Wcs

    w = Wcs(40, 30, 20.5, 15.5, 10.0, 20.0, -0.5, 0.5, proj="CAR")
    # the centre pixel, a source beyond the map (empty window), one by the edge
    pix = [(20.5, 15.5), (200.0, 15.0), (1.2, 29.7)]
    src = np.array([O.pix2sph(w, p1, p2) for p1, p2 in pix])
    cut, total = A.cutout_windows(w, src, [2.0, 3.0, 1.0])
    assert tuple(cut[0])[:4] == (20 - 1 - 4, 15 - 1 - 4, 9, 9) or tuple(cut[0])[:4] == (21 - 1 - 4, 16 - 1 - 4, 9, 9)
    assert cut[1]["nh"] * cut[1]["nw"] == 0
    assert cut[2]["h0"] == 0 and cut[2]["w0"] + cut[2]["nw"] == 30
    assert total == int(sum(int(c["nh"]) * int(c["nw"]) for c in cut))
