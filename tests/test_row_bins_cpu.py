"""The LUT-row lookup of the source-map passes (xts_point.cuh, build_septab and
point_row_bin) restated in numpy: bins of the squared chord q by FP64 exponent
and top five mantissa bits (32 per binade, 2^-39 .. 8), each holding row k0 of
its low edge and the next row's squared chord as threshold.  The row is then
k0 + (q >= threshold); this checks that it equals the bracket of a bisection over
the 401 squared chords (rows clamped to [1, 399], as the reference's logsep
convolution clamps idx to [2, 400]) for random chords and at every row boundary."""
import math

import numpy as np

ND = 401
SB_EXP0, SB_BITS = 984, 5
NSB = (1025 - SB_EXP0 + 1) << SB_BITS


def _tables():
    xstep = math.log(70 / 1e-4) / 399
    S = np.array([0.0] + [1e-4 * math.exp((k - 1) * xstep) for k in range(1, ND)])
    q = (2 * np.sin(0.5 * np.radians(S))) ** 2
    k0 = np.zeros(NSB, int)
    thr = np.zeros(NSB)
    for b in range(NSB):
        qa = math.ldexp(1.0 + (b & 31) / 32, SB_EXP0 + (b >> 5) - 1023)
        k = int(np.searchsorted(q, qa, side="right") - 1)
        k = min(max(k, 1), 399)
        k0[b], thr[b] = k, (q[k + 1] if k < 399 else np.inf)
    return q, k0, thr


def test_bins_give_the_exact_row():
    q, k0, thr = _tables()
    # a bin is narrower in ln q than any row: at most one boundary inside
    lnq = np.log(q[1:])
    assert np.diff(lnq).min() > math.log(33 / 32)
    rng = np.random.default_rng(0)
    qs = np.concatenate([10 ** rng.uniform(-14, 0.6, 500_000), q[1:], np.nextafter(q[1:], 0),
                         np.nextafter(q[1:], 9), [0.0, 4.0, 1e-300]])
    hi = (qs.view(np.int64) >> 32).astype(np.int64)
    b = np.clip((hi >> (20 - SB_BITS)) - (SB_EXP0 << SB_BITS), 0, NSB - 1)
    k = k0[b] + (qs >= thr[b])
    ref = np.clip(np.searchsorted(q, qs, side="right") - 1, 1, 399)
    assert (k == ref).all(), int((k != ref).sum())
