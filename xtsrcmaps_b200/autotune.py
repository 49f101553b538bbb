"""Autotuner of the model-map step (no counterpart in the reference).

Three choices are made by measurement on the job at hand rather than fixed:

* ``tune_write_pass``: the FP32 write pass of the 12-point rule -- the two-pass
  window path, the single-pass CUDA-core kernel or the tcgen05 window-times-table
  product (all three parity-tested against the FP64 oracle) -- timed with CUDA
  events on the job's own geometry; the fastest wins.
* ``tune_launch_shapes``: the launch shapes of the plain path (xts_set_tuning):
  the window pass's blocks per SM (one persistent wave), the write pass's
  persistent blocks per SM and, with a network given, the surrogate forward
  pass's blocks per SM -- each candidate timed on the job's own maps, the
  fastest set for the calls that follow;
* ``tune_adaptive``: the subdivision threshold (rtol) and depth limit of the
  adaptive Genz-Malik cubature.  rtol bounds the rule's own |R7 - R5| / |R7|
  estimate, not the error of the result, so the tuner measures the error against
  a converged map (rtol 1e-6, depth 12) on a sample of the sources and picks the
  fastest (rtol, depth) whose largest relative error over values above
  ``floor`` of each map's peak meets ``target``.

Results are cached per job shape for the process.  CUDA tensors in; there is no
CPU path.
"""
from __future__ import annotations

from typing import Dict, Optional, Sequence, Tuple

_CACHE: Dict[tuple, dict] = {}


def _timed(fn, reps: int) -> float:
    import torch

    fn()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for a, b in ev:
        a.record()
        fn()
        b.record()
    torch.cuda.synchronize()
    return min(a.elapsed_time(b) for a, b in ev)


def _key(kind, wcs, src, uPsf, extra=()):
    return (kind, int(wcs.naxis1), int(wcs.naxis2), float(wcs.cdelt1), float(wcs.cdelt2), int(src.shape[0]),
            int(uPsf.shape[-1])) + tuple(extra)


def tune_write_pass(wcs, src_sph, exposure, uPsf, partial_integrals,
                    candidates: Sequence[str] = ("windows", "cuda_cores", "tcgen05"), reps: int = 3) -> dict:
    """Time each FP32 write pass on this job; returns {"kernel": best, "ms": {...}}."""
    from . import api as A

    key = _key("write", wcs, src_sph, uPsf, tuple(candidates))
    if key in _CACHE:
        return _CACHE[key]
    import torch

    out = torch.empty((int(src_sph.shape[0]), int(wcs.naxis1), int(wcs.naxis2), int(uPsf.shape[-1])),
                      dtype=torch.float32, device=uPsf.device)
    ms = {}
    for k in candidates:
        ms[k] = _timed(lambda: A.point_src_model_map_wcs(wcs, src_sph, exposure, uPsf, partial_integrals,
                                                         out=out, with_info=False, kernel=k), reps)
    best = min(ms, key=ms.get)
    _CACHE[key] = {"kernel": best, "ms": ms}
    return _CACHE[key]


def _max_rel(a, b, floor: float) -> float:
    """Largest relative difference over the values above floor of each map's peak."""
    S = a.shape[0]
    a2, b2 = a.reshape(S, -1).double(), b.reshape(S, -1).double()
    peak = b2.abs().amax(dim=1, keepdim=True)
    mask = b2.abs() > floor * peak
    rel = (a2 - b2).abs() / b2.abs().clamp_min(1e-300)
    return float(rel[mask].max()) if bool(mask.any()) else 0.0


def tune_adaptive(wcs, src_sph, exposure, uPsf, partial_integrals, target: float = 1e-4,
                  rtols: Sequence[float] = (3e-3, 1e-3, 3e-4, 1e-4, 3e-5),
                  depths: Sequence[int] = (4, 6, 8), n_sources: int = 4, floor: float = 1e-6,
                  reps: int = 2) -> Optional[dict]:
    """Fastest (rtol, max_depth) of the adaptive cubature whose error against a
    converged map meets target on a sample of n_sources sources; None if no
    candidate does.  Returns {"rtol", "max_depth", "ms", "err", "table"}."""
    from . import api as A

    key = _key("adaptive", wcs, src_sph, uPsf, (float(target), tuple(rtols), tuple(depths), n_sources, floor))
    if key in _CACHE:
        return _CACHE[key]
    n = min(int(n_sources), int(src_sph.shape[0]))
    s, ex, up, pp = src_sph[:n].contiguous(), exposure[:n].contiguous(), uPsf[:n].contiguous(), \
        partial_integrals[:n].contiguous()
    ref, _ = A.point_src_model_map_wcs_adaptive(wcs, s, ex, up, pp, rtol=1e-6, max_depth=12, with_info=False)
    table: Dict[Tuple[float, int], Tuple[float, float]] = {}
    for d in depths:
        for r in rtols:
            m, _ = A.point_src_model_map_wcs_adaptive(wcs, s, ex, up, pp, rtol=r, max_depth=d, with_info=False)
            err = _max_rel(m, ref, floor)
            t = _timed(lambda: A.point_src_model_map_wcs_adaptive(wcs, s, ex, up, pp, rtol=r, max_depth=d,
                                                                  with_info=False), reps)
            table[(r, d)] = (t, err)
    ok = [(t, r, d, e) for (r, d), (t, e) in table.items() if e <= target]
    if not ok:
        _CACHE[key] = None
        return None
    t, r, d, e = min(ok)
    _CACHE[key] = {"rtol": r, "max_depth": d, "ms": t, "err": e,
                   "table": {f"{r_:g}/{d_}": {"ms": v[0], "err": v[1]} for (r_, d_), v in table.items()}}
    return _CACHE[key]


def tune_launch_shapes(wcs, src_sph, exposure, uPsf, partial_integrals, net=None,
                       window_blocks_per_sm: Sequence[int] = (1, 2, 3), write_blocks_per_sm: Sequence[int] = (1, 2),
                       mlp_blocks_per_sm: Sequence[int] = (0, 1, 2), reps: int = 3, apply: bool = True) -> dict:
    """Time the plain model map for every (window-pass blocks per SM, write-pass blocks per SM)
    pair and, with ``net``, the network's forward pass on a million rows for each
    blocks-per-SM count; set the fastest (apply) and return
    {"choice": {...}, "ms": {...}}."""
    from . import api as A

    key = _key("shapes", wcs, src_sph, uPsf, (tuple(window_blocks_per_sm), tuple(write_blocks_per_sm),
                                               tuple(mlp_blocks_per_sm), net is not None))
    if key in _CACHE:
        res = _CACHE[key]
        if apply:
            A.set_tuning(**res["choice"])
        return res
    import torch

    out = torch.empty((int(src_sph.shape[0]), int(wcs.naxis1), int(wcs.naxis2), int(uPsf.shape[-1])),
                      dtype=torch.float32, device=uPsf.device)
    before = A.get_tuning()
    ms = {}
    for wv in window_blocks_per_sm:
        for wb in write_blocks_per_sm:
            A.set_tuning(window_blocks_per_sm=wv, write_blocks_per_sm=wb)
            ms[f"window{wv}/write{wb}"] = (_timed(lambda: A.point_src_model_map_wcs(
                wcs, src_sph, exposure, uPsf, partial_integrals, out=out, with_info=False), reps), wv, wb)
    best = min(ms.values())
    choice = {"window_blocks_per_sm": best[1], "write_blocks_per_sm": best[2]}
    table = {k: v[0] for k, v in ms.items()}
    if net is not None:
        X = torch.randn((1 << 20, 5), device=uPsf.device) * torch.as_tensor(net.in_sd, device=uPsf.device) + \
            torch.as_tensor(net.in_mu, device=uPsf.device)
        mm = {}
        for mb in mlp_blocks_per_sm:
            A.set_tuning(mlp_blocks_per_sm=mb)
            mm[mb] = _timed(lambda: net.predict(X), reps)
            table[f"mlp{mb}"] = mm[mb]
        choice["mlp_blocks_per_sm"] = min(mm, key=mm.get)
    A.set_tuning(**before)
    res = {"choice": choice, "ms": table}
    _CACHE[key] = res
    if apply:
        A.set_tuning(**choice)
    return res
