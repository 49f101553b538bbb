"""Host-side mirror of the reference's point-source entry points.

The reference's seam is three C++ namespace functions called from
xtsrcmaps/main.cxx:28-30::

    auto ptexp = Exposure::compute_exposure(cfg, obs, src.point, irf);
    auto ptpsf = Psf::compute_psf_data(obs, irf, ptexp);
    maps.pt    = ModelMap::compute_srcmaps(obs, src.point, ptexp, ptpsf);

This module offers the same three calls (plus the finer routines they use) with
the same inputs, outputs and tensor layouts, executed by the sm_100a kernels of
``libxts_cuda.so`` through its C-ABI.  Arrays may be numpy arrays (host memory:
the library stages them on the device and copies results back) or CUDA torch
tensors (device memory: the call is asynchronous on torch's current stream and
returns CUDA tensors).  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any, Optional

import numpy as np

from . import _lib as L
from .irf import IrfEffic, IrfGrid, IrfScale
from .wcs import Wcs

ND = L.ND


@dataclass
class ExpCube:
    """Livetime cube (observation/obs_types.hxx:24-32): cosbins float32 [12 nside^2, nbrbins]."""

    cosbins: Any
    nside: int
    nbrbins: int
    cosmin: float = 0.0
    thetabin: bool = True


@dataclass
class XtExp:
    """exposure/exposure.hxx:19-26."""

    exp_costhetas: Any
    front_aeff: Any
    back_aeff: Any
    src_exposure_cosbins: Any
    src_weighted_exposure_cosbins: Any
    exposure: Any


@dataclass
class XtPsf:
    """psf/psf.hxx:14-17."""

    uPsf: Any
    partial_psf_integral: Any


@dataclass
class SrcmapInfo:
    inv_map_integral: Any
    correction: Any
    psf_radius: Any
    in_fov: Any


# --------------------------------------------------------------------------- plumbing
def _is_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


_PINNED = None  # torch's pinned host allocator, when CUDA is usable


def _host_empty(shape, dtype) -> np.ndarray:
    """Host output array in page-locked memory when CUDA is usable (device-to-host
    copies into pageable memory run at about a third of the speed), else numpy."""
    global _PINNED
    if _PINNED is None:
        try:
            import torch

            _PINNED = torch if torch.cuda.is_available() else False
        except ImportError:
            _PINNED = False
    if _PINNED:
        t = _PINNED
        tdt = {np.float64: t.float64, np.float32: t.float32, np.int32: t.int32}[np.dtype(dtype).type]
        shp = tuple(int(v) for v in shape) if isinstance(shape, (tuple, list)) else (int(shape),)
        return t.empty(shp, dtype=tdt, pin_memory=True).numpy()  # the array keeps the tensor alive
    return np.empty(shape, dtype=dtype)


class _Call:
    """Holds the buffers of one C-ABI call and converts arrays to pointers."""

    _NP = {"f64": np.float64, "f32": np.float32, "i32": np.int32}

    def __init__(self, device: bool, like=None):
        self.device = device
        self.keep = []
        if device:
            import torch

            self.torch = torch
            self.dev = like.device if like is not None else torch.device("cuda")
            handle = torch.cuda.current_stream(self.dev).cuda_stream
            # torch's default stream has handle 0, which the C-ABI reads as "the
            # library's own stream"; pass cudaStreamLegacy (0x1) so the work stays
            # ordered with the caller's default-stream work.
            self.stream = C.c_void_p(handle if handle else 1)
        else:
            self.stream = None
        self.flags = L.XTS_DEVICE_PTRS if device else 0

    def inp(self, x, kind="f64"):
        if self.device:
            t = self.torch
            dt = {"f64": t.float64, "f32": t.float32, "i32": t.int32}[kind]
            if not _is_cuda(x):
                x = t.as_tensor(np.asarray(x), device=self.dev)
            x = x.to(dt).contiguous()
            self.keep.append(x)
            return C.c_void_p(x.data_ptr()), x
        a = np.ascontiguousarray(np.asarray(x), dtype=self._NP[kind])
        self.keep.append(a)
        return C.c_void_p(a.ctypes.data), a

    def out(self, shape, kind="f64"):
        if self.device:
            t = self.torch
            dt = {"f64": t.float64, "f32": t.float32, "i32": t.int32}[kind]
            x = t.empty(shape, dtype=dt, device=self.dev)
            self.keep.append(x)
            return C.c_void_p(x.data_ptr()), x
        a = _host_empty(shape, self._NP[kind])
        self.keep.append(a)
        return C.c_void_p(a.ctypes.data), a

    def grid(self, g: IrfGrid, n_par: int) -> L.XtsGrid:
        params = g.params
        if n_par == 1 and getattr(params, "ndim", 3) == 3:
            params = params[..., 0]
        cp, c = self.inp(g.cosths)
        ep, e = self.inp(g.logEs)
        pp, p = self.inp(params)
        return L.XtsGrid(cp, len(c), ep, len(e), pp, n_par, float(g.min_cos_theta))


def _device_of(*xs) -> Optional[Any]:
    for x in xs:
        if _is_cuda(x):
            return x
    return None


# --------------------------------------------------------------------------- IRF set-up
def livetime_efficiency_factors(logEs, effic: IrfEffic):
    """Irf::livetime_efficiency_factors (irf/irf.cxx:70-109) -> [2, E]."""
    like = _device_of(logEs)
    c = _Call(like is not None, like)
    lp, le = c.inp(logEs)
    p0, _ = c.inp(effic.p0, "f32")
    p1, _ = c.inp(effic.p1, "f32")
    op, o = c.out((2, len(le)))
    L.check(L.lib().xts_livetime_efficiency_factors(lp, len(le), p0, p1, op, c.flags, c.stream))
    return o


def normalize_rpsf(grid: IrfGrid, scale: IrfScale) -> IrfGrid:
    """irf_private::normalize_rpsf (irf/irf.normalize_rpsf.cpp:11-61); returns a normalised copy."""
    p = np.array(grid.params, dtype=np.float64, order="C", copy=True)
    gl = np.ascontiguousarray(grid.logEs, dtype=np.float64)
    Mc, Me = p.shape[0], p.shape[1]
    L.check(L.lib().xts_normalize_rpsf(C.c_void_p(p.ctypes.data), Mc, Me, C.c_void_p(gl.ctypes.data),
                                       scale.scale0, scale.scale1, scale.scale_index, 0, None))
    return IrfGrid(np.array(grid.cosths), np.array(grid.logEs), p, grid.min_cos_theta)


# --------------------------------------------------------------------------- step (a)
def compute_exposure(exp_cube: ExpCube, wexp_cube: ExpCube, logEs, src_sph, aeff_front: IrfGrid,
                     aeff_back: IrfGrid, front_ltf) -> XtExp:
    """Exposure::compute_exposure (exposure/exposure.hxx:44-88)."""
    like = _device_of(exp_cube.cosbins, src_sph, logEs)
    c = _Call(like is not None, like)
    cb, cube = c.inp(exp_cube.cosbins, "f32")
    wb, _ = c.inp(wexp_cube.cosbins, "f32")
    C_ = int(exp_cube.nbrbins)
    cube_s = L.XtsExpcube(cb, int(exp_cube.nside), C_, float(exp_cube.cosmin), int(bool(exp_cube.thetabin)))
    wcube_s = L.XtsExpcube(wb, int(wexp_cube.nside), int(wexp_cube.nbrbins), float(wexp_cube.cosmin),
                           int(bool(wexp_cube.thetabin)))
    lp, le = c.inp(logEs)
    E = len(le)
    sp, sa = c.inp(src_sph)
    S = int(sa.shape[0]) if sa.ndim == 2 else 0
    af = c.grid(aeff_front, 1)
    ab = c.grid(aeff_back, 1)
    ltfp, _ = c.inp(front_ltf)
    o = [c.out(s) for s in ((C_,), (C_, E), (C_, E), (S, C_), (S, C_), (S, E))]
    outs = L.XtsExposureOut(*[x[0] for x in o])
    flags = c.flags
    L.check(L.lib().xts_compute_exposure(C.byref(cube_s), C.byref(wcube_s), lp, E, sp, S, C.byref(af),
                                         C.byref(ab), ltfp, C.byref(outs), flags, c.stream))
    return XtExp(*[x[1] for x in o])


def exposure_map(exp_cube: ExpCube, wexp_cube: ExpCube, logEs, aeff_front: IrfGrid, aeff_back: IrfGrid,
                 front_ltf):
    """Exposure of every HEALPix pixel [12 nside^2, E] (the contraction of
    exposure/exposure.cxx:159-263 over all livetime-cube rows) on tcgen05 tensor
    cores as 3xTF32; a source's exposure is the row at its NESTED pixel."""
    like = _device_of(exp_cube.cosbins, logEs)
    c = _Call(like is not None, like)
    cb, cube = c.inp(exp_cube.cosbins, "f32")
    wb, _ = c.inp(wexp_cube.cosbins, "f32")
    cube_s = L.XtsExpcube(cb, int(exp_cube.nside), int(exp_cube.nbrbins), float(exp_cube.cosmin),
                          int(bool(exp_cube.thetabin)))
    wcube_s = L.XtsExpcube(wb, int(wexp_cube.nside), int(wexp_cube.nbrbins), float(wexp_cube.cosmin),
                           int(bool(wexp_cube.thetabin)))
    lp, le = c.inp(logEs)
    E = len(le)
    af = c.grid(aeff_front, 1)
    ab = c.grid(aeff_back, 1)
    ltfp, _ = c.inp(front_ltf)
    op, o = c.out((12 * int(exp_cube.nside) ** 2, E))
    L.check(L.lib().xts_exposure_map(C.byref(cube_s), C.byref(wcube_s), lp, E, C.byref(af), C.byref(ab), ltfp,
                                     op, c.flags, c.stream))
    return o


def exposure(src_exposure_cosbins, src_weighted_exposure_cosbins, front_aeff, back_aeff, front_ltf):
    """Exposure::exposure (exposure/exposure.cxx:159-263): step a5 from gathered livetime rows."""
    like = _device_of(src_exposure_cosbins, front_aeff)
    c = _Call(like is not None, like)
    xp, xa = c.inp(src_exposure_cosbins)
    wp, _ = c.inp(src_weighted_exposure_cosbins)
    afp, afa = c.inp(front_aeff)
    abp, _ = c.inp(back_aeff)
    lp, _ = c.inp(front_ltf)
    S, C_ = int(xa.shape[0]), int(xa.shape[1])
    E = int(afa.shape[1])
    op, o = c.out((S, E))
    L.check(L.lib().xts_exposure_contract(xp, wp, S, C_, afp, abp, lp, E, op, c.flags, c.stream))
    return o


# --------------------------------------------------------------------------- step (b)
def compute_psf_data(psf_front: IrfGrid, psf_back: IrfGrid, exp: XtExp, logEs, front_ltf) -> XtPsf:
    """Psf::compute_psf_data (psf/psf.compute_psf_data.cxx:7-33); King grids already normalised."""
    like = _device_of(exp.exposure, logEs)
    c = _Call(like is not None, like)
    gf = c.grid(psf_front, 6)
    gb = c.grid(psf_back, 6)
    cp, ca = c.inp(exp.exp_costhetas)
    lp, le = c.inp(logEs)
    afp, _ = c.inp(exp.front_aeff)
    abp, _ = c.inp(exp.back_aeff)
    xp, xa = c.inp(exp.src_exposure_cosbins)
    wp, _ = c.inp(exp.src_weighted_exposure_cosbins)
    ltfp, _ = c.inp(front_ltf)
    ep, _ = c.inp(exp.exposure)
    S, E = int(xa.shape[0]), len(le)
    up, u = c.out((S, ND, E))
    pp, p = c.out((S, ND, E))
    L.check(L.lib().xts_compute_psf_data(C.byref(gf), C.byref(gb), cp, len(ca), lp, E, afp, abp, xp, wp,
                                         S, ltfp, ep, up, pp, c.flags, c.stream))
    return XtPsf(u, p)


# --------------------------------------------------------------------------- steps (c)+(d)
def _wcs_struct(w: Wcs) -> L.XtsWcs:
    return L.XtsWcs(int(w.naxis1), int(w.naxis2), float(w.crpix1), float(w.crpix2), float(w.crval1),
                    float(w.crval2), float(w.cdelt1), float(w.cdelt2), float(w.crota2), w.proj_code,
                    int(bool(w.galactic)))


def point_src_model_map_wcs(wcs: Wcs, src_sph, exposure, uPsf, partial_integrals,
                            out_dtype: str = "float32", out=None, with_info: bool = True,
                            kernel: str = "windows"):
    """ModelMap::point_src_model_map_wcs (model_map/model_map.point_src_model_map_wcs.cxx:6-45).

    Returns (model_map [S, H, W, E], SrcmapInfo or None).  ``out`` may supply a
    preallocated output of the right dtype and shape (16-byte aligned).
    ``kernel`` picks the FP32 write pass: "windows" (default: geometry pass +
    streaming write pass), "cuda_cores" (single-pass CUDA-core kernel) or
    "tcgen05" (window-times-table product on tensor cores).
    """
    kflag = {"windows": 0, "cuda_cores": L.XTS_CUDA_CORES, "tcgen05": L.XTS_TCGEN05}[kernel]
    like = _device_of(uPsf, exposure, src_sph)
    c = _Call(like is not None, like)
    sp, sa = c.inp(src_sph)
    S = int(sa.shape[0])
    ep, ea = c.inp(exposure)
    E = int(ea.shape[1])
    up, _ = c.inp(uPsf)
    pp, _ = c.inp(partial_integrals)
    kind = {"float32": "f32", "float64": "f64"}[out_dtype]
    shape = (S, int(wcs.naxis1), int(wcs.naxis2), E)
    if out is None:
        mp, m = c.out(shape, kind)
    else:
        m = out
        mp = C.c_void_p(m.data_ptr() if c.device else m.ctypes.data)
    info = None
    info_s = None
    if with_info:
        o = [c.out((S, E)), c.out((S, E)), c.out((S,)), c.out((S,), "i32")]
        info_s = L.XtsSrcmapInfo(*[x[0] for x in o])
        info = SrcmapInfo(*[x[1] for x in o])
    flags = c.flags | (L.XTS_OUT_F64 if kind == "f64" else 0) | kflag
    w = _wcs_struct(wcs)
    L.check(L.lib().xts_point_src_model_map_wcs(C.byref(w), sp, S, ep, up, pp, E, mp,
                                                C.byref(info_s) if info_s is not None else None,
                                                flags, c.stream))
    return m, info


def point_src_model_map_wcs_adaptive(wcs: Wcs, src_sph, exposure, uPsf, partial_integrals,
                                     rtol: float = 1e-4, max_depth: int = 6, out=None,
                                     with_info: bool = True):
    """point_src_model_map_wcs with adaptive Genz-Malik cubature of each pixel
    (the design of math/genz_malik.hxx:18-195 and
    model_map/model_map.pixel_mean_psf_genz.cxx:21-108) in place of the 12-point
    rule.  Returns (float32 model_map [S, H, W, E], SrcmapInfo or None)."""
    like = _device_of(uPsf, exposure, src_sph)
    c = _Call(like is not None, like)
    sp, sa = c.inp(src_sph)
    S = int(sa.shape[0])
    ep, ea = c.inp(exposure)
    E = int(ea.shape[1])
    up, _ = c.inp(uPsf)
    pp, _ = c.inp(partial_integrals)
    shape = (S, int(wcs.naxis1), int(wcs.naxis2), E)
    if out is None:
        mp, m = c.out(shape, "f32")
    else:
        m = out
        mp = C.c_void_p(m.data_ptr() if c.device else m.ctypes.data)
    info = info_s = None
    if with_info:
        o = [c.out((S, E)), c.out((S, E)), c.out((S,)), c.out((S,), "i32")]
        info_s = L.XtsSrcmapInfo(*[x[0] for x in o])
        info = SrcmapInfo(*[x[1] for x in o])
    w = _wcs_struct(wcs)
    L.check(L.lib().xts_point_src_model_map_wcs_adaptive(C.byref(w), sp, S, ep, up, pp, E, float(rtol),
                                                         int(max_depth), mp,
                                                         C.byref(info_s) if info_s is not None else None,
                                                         c.flags, c.stream))
    return m, info


def point_source_maps(wcs: Wcs, src_sph, exp_cube: ExpCube, wexp_cube: ExpCube, logEs, aeff_front: IrfGrid,
                      aeff_back: IrfGrid, psf_front: IrfGrid, psf_back: IrfGrid, front_ltf,
                      out_dtype: str = "float32", out=None, with_info: bool = True,
                      kernel: str = "windows"):
    """The three calls of main.cxx:28-30 (compute_exposure, compute_psf_data,
    compute_srcmaps<PointSource>) in one library call; the exposure and mean-PSF
    tables stay in device memory.  ``psf_front``/``psf_back`` are normalised King
    grids (normalize_rpsf).  Returns (model_map [S, H, W, E], SrcmapInfo or None).
    With host arrays the maps are copied to the host by chunks of sources while the
    later chunks are computed; pass a page-locked ``out`` for full copy speed."""
    like = _device_of(exp_cube.cosbins, src_sph, logEs)
    c = _Call(like is not None, like)
    cb, _ = c.inp(exp_cube.cosbins, "f32")
    wb, _ = c.inp(wexp_cube.cosbins, "f32")
    cube_s = L.XtsExpcube(cb, int(exp_cube.nside), int(exp_cube.nbrbins), float(exp_cube.cosmin),
                          int(bool(exp_cube.thetabin)))
    wcube_s = L.XtsExpcube(wb, int(wexp_cube.nside), int(wexp_cube.nbrbins), float(wexp_cube.cosmin),
                           int(bool(wexp_cube.thetabin)))
    lp, le = c.inp(logEs)
    E = len(le)
    sp, sa = c.inp(src_sph)
    S = int(sa.shape[0]) if sa.ndim == 2 else 0
    af = c.grid(aeff_front, 1)
    ab = c.grid(aeff_back, 1)
    gf = c.grid(psf_front, 6)
    gb = c.grid(psf_back, 6)
    ltfp, _ = c.inp(front_ltf)
    kind = {"float32": "f32", "float64": "f64"}[out_dtype]
    shape = (S, int(wcs.naxis1), int(wcs.naxis2), E)
    if out is None:
        mp, m = c.out(shape, kind)
    else:
        m = out
        mp = C.c_void_p(m.data_ptr() if c.device else m.ctypes.data)
    info = info_s = None
    if with_info:
        o = [c.out((S, E)), c.out((S, E)), c.out((S,)), c.out((S,), "i32")]
        info_s = L.XtsSrcmapInfo(*[x[0] for x in o])
        info = SrcmapInfo(*[x[1] for x in o])
    kflag = {"windows": 0, "cuda_cores": L.XTS_CUDA_CORES, "tcgen05": L.XTS_TCGEN05}[kernel]
    flags = c.flags | (L.XTS_OUT_F64 if kind == "f64" else 0) | kflag
    w = _wcs_struct(wcs)
    L.check(L.lib().xts_point_source_maps(C.byref(cube_s), C.byref(wcube_s), lp, E, sp, S, C.byref(af),
                                          C.byref(ab), C.byref(gf), C.byref(gb), ltfp, C.byref(w), mp,
                                          C.byref(info_s) if info_s is not None else None, flags, c.stream))
    return m, info


def point_source_maps_surrogate(wcs: Wcs, src_sph, exp_cube: ExpCube, wexp_cube: ExpCube, logEs,
                                aeff_front: IrfGrid, aeff_back: IrfGrid, psf_front: IrfGrid, psf_back: IrfGrid,
                                front_ltf, net, check_tol: float = 1e-4, out=None, with_info: bool = False,
                                stats: bool = True):
    """The three calls of main.cxx:28-30 with the model map of the learned
    surrogate (point_src_model_map_wcs_surrogate) in place of the plain cubature,
    in one library call (xts_point_source_maps_surrogate).  Inputs may be host
    arrays (numpy, or CPU torch tensors, pinned for asynchronous copies) or CUDA
    tensors on the network's device; with host arrays the maps are copied to the
    host in groups of sources while the later groups are computed (pass a
    page-locked ``out`` for full copy speed).  Returns (model_map, SrcmapInfo or
    None, stats or None)."""
    from .surrogate import _stats_dict

    like = _device_of(exp_cube.cosbins, src_sph, logEs)
    c = _Call(like is not None, like)
    cb, _ = c.inp(exp_cube.cosbins, "f32")
    wb, _ = c.inp(wexp_cube.cosbins, "f32")
    cube_s = L.XtsExpcube(cb, int(exp_cube.nside), int(exp_cube.nbrbins), float(exp_cube.cosmin),
                          int(bool(exp_cube.thetabin)))
    wcube_s = L.XtsExpcube(wb, int(wexp_cube.nside), int(wexp_cube.nbrbins), float(wexp_cube.cosmin),
                           int(bool(wexp_cube.thetabin)))
    lp, le = c.inp(logEs)
    E = len(le)
    sp, sa = c.inp(src_sph)
    S = int(sa.shape[0]) if sa.ndim == 2 else 0
    af = c.grid(aeff_front, 1)
    ab = c.grid(aeff_back, 1)
    gf = c.grid(psf_front, 6)
    gb = c.grid(psf_back, 6)
    ltfp, _ = c.inp(front_ltf)
    shape = (S, int(wcs.naxis1), int(wcs.naxis2), E)
    if out is None:
        mp, m = c.out(shape, "f32")
    else:
        m = out
        mp = C.c_void_p(m.data_ptr() if hasattr(m, "data_ptr") else m.ctypes.data)
    info = info_s = None
    if with_info:
        o = [c.out((S, E)), c.out((S, E)), c.out((S,)), c.out((S,), "i32")]
        info_s = L.XtsSrcmapInfo(*[x[0] for x in o])
        info = SrcmapInfo(*[x[1] for x in o])
    st = L.XtsSurrogateStats() if stats else None
    ns = net.struct()
    w = _wcs_struct(wcs)
    L.check(L.lib().xts_point_source_maps_surrogate(
        C.byref(cube_s), C.byref(wcube_s), lp, E, sp, S, C.byref(af), C.byref(ab), C.byref(gf), C.byref(gb), ltfp,
        C.byref(w), C.byref(ns), float(check_tol), mp, C.byref(info_s) if info_s is not None else None,
        C.byref(st) if st is not None else None, c.flags, c.stream))
    return m, info, (_stats_dict(st) if st is not None else None)


def write_src_model(filename: str, model_map, names=None, bitpix: int = -64) -> None:
    """Fermi::fits::write_src_model (fits/fits.write_src_model.cxx:10-66): the maps
    [S, H, W, E] (float32 or float64, host array or CUDA tensor) written as a FITS
    file, one IMAGE extension per source named ``names[s]`` (default SRC%05d),
    data in SEHW order (img[e][w][h] = map[s][h][w][e]), BITPIX -64 as the
    reference or -32, with CHECKSUM and DATASUM.  The reorder, conversion, byte
    swap and data sums run on the GPU."""
    if bitpix not in (-64, -32):
        raise ValueError("bitpix must be -64 or -32")
    dev = _is_cuda(model_map)
    if dev:
        m = model_map.contiguous()
        f64 = str(m.dtype) == "torch.float64"
        if not f64 and str(m.dtype) != "torch.float32":
            raise ValueError("model_map must be float32 or float64")
        ptr = C.c_void_p(m.data_ptr())
        import torch

        handle = torch.cuda.current_stream(m.device).cuda_stream
        stream = C.c_void_p(handle if handle else 1)
    else:
        m = np.asarray(model_map)
        if m.dtype not in (np.float32, np.float64):
            raise ValueError("model_map must be float32 or float64")
        m = np.ascontiguousarray(m)
        f64 = m.dtype == np.float64
        ptr = C.c_void_p(m.ctypes.data)
        stream = None
    if m.ndim != 4:
        raise ValueError("model_map must be [S, H, W, E]")
    S, H, W, E = (int(x) for x in m.shape)
    cnames = None
    if names is not None:
        if len(names) != S:
            raise ValueError("one name per source")
        enc = [str(n).encode("ascii") for n in names]
        cnames = (C.c_char_p * S)(*enc)
    flags = (L.XTS_DEVICE_PTRS if dev else 0) | (L.XTS_OUT_F64 if f64 else 0) | (L.XTS_FITS_F32 if bitpix == -32 else 0)
    L.check(L.lib().xts_write_src_model(str(filename).encode(), ptr, S, H, W, E, cnames, flags, stream))


def make_psf_kernel(kernel_wcs: Wcs, Nk: int, upsf):
    """Psf::make_kernel (psf/psf.make_kernel.cpp:8-90): one source's mean PSF
    ``upsf`` [401, E] sampled at the pixel centres of the Nk x Nk grid
    ``kernel_wcs`` (Nk odd) by separation from its CRVAL, each energy plane
    normalised to unit sum -> [E, Nk, Nk] (float64)."""
    like = _device_of(upsf)
    c = _Call(like is not None, like)
    up, u = c.inp(upsf)
    E = int(u.shape[-1])
    kp, k = c.out((E, int(Nk), int(Nk)))
    w = _wcs_struct(kernel_wcs)
    L.check(L.lib().xts_make_psf_kernel(C.byref(w), int(Nk), up, E, kp, c.flags, c.stream))
    return k


def convolve_map_psf(image, kernel):
    """FFT::convolve_map_psf (model_map/mm_fft/fft.convolve_map_psf.cpp:7-43): per
    energy plane, the full linear convolution of image [E, H, W] with kernel
    [E, K, K] -> [E, H + K - 1, W + K - 1] (float64, cuFFT)."""
    like = _device_of(image, kernel)
    c = _Call(like is not None, like)
    ip, im = c.inp(image)
    kp, ke = c.inp(kernel)
    E, H, W = (int(x) for x in im.shape)
    K = int(ke.shape[1])
    if tuple(ke.shape) != (E, K, K):
        raise ValueError("kernel must be [E, K, K] with the image's E")
    op, o = c.out((E, H + K - 1, W + K - 1))
    L.check(L.lib().xts_convolve_map_psf(ip, E, H, W, kp, K, op, c.flags, c.stream))
    return o


def cutout_windows(wcs: Wcs, src_sph, radius_deg):
    """Per-source cutout windows for radii ``radius_deg`` [S] (degrees): a structured
    array [S] of (h0, w0, nh, nw, offset) (xts_cutout) and the total pixel count of
    the ragged map.  Host function."""
    src = np.ascontiguousarray(np.asarray(src_sph, dtype=np.float64).reshape(-1, 2))
    rad = np.ascontiguousarray(np.asarray(radius_deg, dtype=np.float64).reshape(-1))
    S = src.shape[0]
    if rad.shape[0] != S:
        raise ValueError("one radius per source")
    cut = np.zeros(S, dtype=L.CUTOUT_DTYPE)
    total = C.c_longlong(0)
    w = _wcs_struct(wcs)
    L.check(L.lib().xts_cutout_windows(C.byref(w), C.c_void_p(src.ctypes.data), C.c_void_p(rad.ctypes.data), S,
                                       C.c_void_p(cut.ctypes.data), C.byref(total)))
    return cut, int(total.value)


def point_src_model_map_cutouts(wcs: Wcs, src_sph, cut, exposure, uPsf, partial_integrals, out=None,
                                with_info: bool = True):
    """ModelMap::point_src_model_map_wcs (model_map/model_map.point_src_model_map_wcs.cxx:6-45)
    on per-source cutouts ``cut`` (cutout_windows): source s's map is the reference's
    model map of its window's sub-map, stored [nh, nw, E] from pixel cut[s].offset of
    a ragged float32 map [total_pixels, E].  CUDA inputs run on the device (``cut``
    then as the uint8 CUDA tensor of the structured array's bytes, or the numpy
    array itself, which is copied).  Returns (map, SrcmapInfo or None)."""
    cut_np = None if _is_cuda(cut) else np.ascontiguousarray(np.asarray(cut, dtype=L.CUTOUT_DTYPE))
    like = _device_of(src_sph, exposure, uPsf)
    c = _Call(like is not None, like)
    sp, sa = c.inp(src_sph)
    S = int(sa.shape[0]) if sa.ndim == 2 else 0
    ep, ea = c.inp(exposure)
    E = int(ea.shape[1])
    up, _ = c.inp(uPsf)
    pp, _ = c.inp(partial_integrals)
    if cut_np is not None:
        total = int((cut_np["nh"].astype(np.int64) * cut_np["nw"]).sum())
    if c.device:
        if cut_np is not None:
            cut_d = c.torch.as_tensor(np.frombuffer(cut_np.tobytes(), dtype=np.uint8).copy(), device=c.dev)
        else:
            cut_d = cut
        c.keep.append(cut_d)
        cutp = C.c_void_p(cut_d.data_ptr())
        if out is None:
            if cut_np is None:
                raise ValueError("pass out (the ragged map) with a device-resident cut")
            out = c.torch.empty((total, E), dtype=c.torch.float32, device=c.dev)
        mp = C.c_void_p(out.data_ptr())
    else:
        cutp = C.c_void_p(cut_np.ctypes.data)
        if out is None:
            out = np.empty((total, E), dtype=np.float32)
        mp = C.c_void_p(out.ctypes.data)
    info = info_s = None
    if with_info:
        o = [c.out((S, E)), c.out((S, E)), c.out((S,)), c.out((S,), "i32")]
        info_s = L.XtsSrcmapInfo(*[x[0] for x in o])
        info = SrcmapInfo(*[x[1] for x in o])
    w = _wcs_struct(wcs)
    L.check(L.lib().xts_point_src_model_map_cutouts(C.byref(w), sp, S, cutp, ep, up, pp, E, mp,
                                                    C.byref(info_s) if info_s is not None else None, c.flags,
                                                    c.stream))
    return out, info


def rebin_wcs(wcs: Wcs, target_pix_size: float) -> Wcs:
    """rebin_wcs_config (sky_geom/sky_geom.hxx:352-371): the WCS of the same region at
    pixel size ``target_pix_size`` degrees (CDELT2 rebinned, where the reference
    stores CRPIX2)."""
    w = _wcs_struct(wcs)
    o = L.XtsWcs()
    L.check(L.lib().xts_rebin_wcs(C.byref(w), float(target_pix_size), C.byref(o)))
    return Wcs(int(o.naxis1), int(o.naxis2), o.crpix1, o.crpix2, o.crval1, o.crval2, o.cdelt1, o.cdelt2, o.crota2,
               wcs.proj, wcs.galactic)


def allsky_crop_range(allsky_wcs: Wcs, roi_wcs: Wcs) -> tuple:
    """The all-sky pixel range under the ROI of fits::read_allsky_cropped
    (fits/fits.read_allsky_cropped.cpp:150-194): (x_first, x_last, y_first, y_last),
    1-based and inclusive."""
    r = (C.c_long * 4)()
    a, b = _wcs_struct(allsky_wcs), _wcs_struct(roi_wcs)
    L.check(L.lib().xts_allsky_crop_range(C.byref(a), C.byref(b), r))
    return tuple(int(v) for v in r)


def crop_allsky(allsky, crop_range):
    """The block of an all-sky cube [E0, NY, NX] (float32) inside ``crop_range``
    (x_first, x_last, y_first, y_last; x_first > x_last wraps across the image's
    longitude seam) -> [E0, ny, nx]."""
    like = _device_of(allsky)
    c = _Call(like is not None, like)
    ap, a = c.inp(allsky, "f32")
    E0, NY, NX = (int(v) for v in a.shape)
    x0, x1, y0, y1 = (int(v) for v in crop_range)
    nx = x1 - x0 + 1 if x1 >= x0 else NX - x0 + 1 + x1
    op, o = c.out((E0, y1 - y0 + 1, nx), "f32")
    r = (C.c_long * 4)(x0, x1, y0, y1)
    L.check(L.lib().xts_crop_allsky(ap, E0, NY, NX, r, op, c.flags, c.stream))
    return o


def trilerp_ehw(src, shape):
    """Fermi::math::trilerpEHW (math/trilerp.hpp:7-59): src [E0, H0, W0] (float32)
    resampled trilinearly onto ``shape`` = (E1, H1, W1), corner-aligned axes."""
    like = _device_of(src)
    c = _Call(like is not None, like)
    sp, sa = c.inp(src, "f32")
    E0, H0, W0 = (int(v) for v in sa.shape)
    E1, H1, W1 = (int(v) for v in shape)
    dp, d = c.out((E1, H1, W1), "f32")
    L.check(L.lib().xts_trilerp_ehw(sp, E0, H0, W0, dp, E1, H1, W1, c.flags, c.stream))
    return d


def scale_model_map(wcs: Wcs, src_sph, exposure, uPsf, partial_integrals, means, with_info: bool = True):
    """The final scalings of the diffuse-source map (model_map.diffuse_src_model_map_wcs.cxx:76-95),
    those of point_src_model_map_wcs after its cubature: pixel means [S, H, W, E]
    (float32) -> mean * solid angle * exposure * correction, with the map
    integral and containment correction of the point-source path.  Returns
    (model_map, SrcmapInfo or None); a CUDA ``means`` is scaled in place."""
    like = _device_of(means, exposure, uPsf)
    c = _Call(like is not None, like)
    sp, sa = c.inp(src_sph)
    S = int(sa.shape[0]) if sa.ndim == 2 else 0
    ep, ea = c.inp(exposure)
    E = int(ea.shape[1])
    up, _ = c.inp(uPsf)
    pp, _ = c.inp(partial_integrals)
    if c.device:
        m = means
        if str(m.dtype) != "torch.float32" or not m.is_contiguous():
            raise ValueError("means must be a contiguous float32 tensor")
        mp = C.c_void_p(m.data_ptr())
    else:
        m = np.array(means, dtype=np.float32, copy=True, order="C")
        mp = C.c_void_p(m.ctypes.data)
    info = info_s = None
    if with_info:
        o = [c.out((S, E)), c.out((S, E)), c.out((S,)), c.out((S,), "i32")]
        info_s = L.XtsSrcmapInfo(*[x[0] for x in o])
        info = SrcmapInfo(*[x[1] for x in o])
    w = _wcs_struct(wcs)
    L.check(L.lib().xts_scale_model_map(C.byref(w), sp, S, ep, up, pp, E, mp,
                                        C.byref(info_s) if info_s is not None else None, c.flags, c.stream))
    return m, info


def compute_srcmaps(wcs: Wcs, src_sph, exp: XtExp, psf: XtPsf, out_dtype: str = "float32", out=None):
    """ModelMap::compute_srcmaps<PointSource> (model_map/model_map.compute_src_maps.cxx:6-22)."""
    m, _ = point_src_model_map_wcs(wcs, src_sph, exp.exposure, psf.uPsf, psf.partial_psf_integral,
                                   out_dtype=out_dtype, out=out, with_info=False)
    return m


TUNING_FIELDS = ("window_blocks_per_sm", "write_blocks_per_sm", "queue_blocks_per_sm", "mlp_blocks_per_sm", "chunk_sources")


def set_tuning(**fields) -> None:
    """Launch shapes for the following calls (xts_set_tuning); unnamed fields keep
    their current value, 0 means the default.  set_tuning() with no fields keeps
    everything; reset_tuning() restores the defaults."""
    t = L.XtsTuning()
    L.check(L.lib().xts_get_tuning(C.byref(t)))
    for k, v in fields.items():
        if k not in TUNING_FIELDS:
            raise ValueError(f"unknown tuning field {k!r}")
        setattr(t, k, int(v))
    L.check(L.lib().xts_set_tuning(C.byref(t)))


def reset_tuning() -> None:
    L.check(L.lib().xts_set_tuning(None))


def get_tuning() -> dict:
    t = L.XtsTuning()
    L.check(L.lib().xts_get_tuning(C.byref(t)))
    return {k: int(getattr(t, k)) for k in TUNING_FIELDS}


def init(device: int = 0) -> None:
    L.check(L.lib().xts_init(int(device)))


def profile_enable(on: bool = True, keep: bool = False) -> None:
    """Time every library kernel with CUDA events.  ``keep`` keeps the record
    across reads, for launches captured into a CUDA graph (each read then
    reports the latest replay)."""
    L.check(L.lib().xts_profile_enable(2 if (on and keep) else int(bool(on))))


def profile_read() -> dict:
    """Per-kernel {name: (launches, total_ms)} since profiling was enabled (then cleared)."""
    import json

    buf = C.create_string_buffer(1 << 16)
    n = L.lib().xts_profile_read(buf, len(buf))
    if n < 0:
        L.check(n)
    return {k: (int(v[0]), float(v[1])) for k, v in json.loads(buf.value.decode()).items()}


def release() -> None:
    L.lib().xts_release()


def point_src_model_map_wcs_surrogate(wcs: Wcs, src_sph, exposure, uPsf, partial_integrals, logEs, net,
                                      check_tol: float = 1e-4, with_info: bool = True, out=None,
                                      stats: bool = True):
    """point_src_model_map_wcs with the pixel means from the learned surrogate
    (xtsrcmaps_b200.surrogate.Surrogate) where it applies and the FP64 12-point
    rule elsewhere; CUDA tensors.  Returns (maps, SrcmapInfo or None, stats or
    None); with stats=False the call does not synchronise."""
    from .surrogate import model_map

    return model_map(wcs, src_sph, exposure, uPsf, partial_integrals, logEs, net, check_tol, with_info, out=out,
                     stats=stats)
