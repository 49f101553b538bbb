"""The learned surrogate of the pixel cubature (no counterpart in the reference).

A perceptron 5 -> 128 -> 128 -> 128 -> 1 with tanh-form GELU maps five features
of a (source, pixel, energy) value -- log10 of the centre's separation in pixel
sizes, the centre's offset between the two rows of the separation table that
bracket it, log10 of the pixel's solid angle, log10 of the energy and the log
slope of the mean PSF's table segment at the centre -- to y = ln(m / u_c) rho^2, where m is the 12-point rule mean of the mean PSF over
the pixel (the plain path's cubature, model_map/mm_cubature/cubature.implementation.cxx:21-55)
and u_c the mean PSF at the centre.  Training samples come from the same FP64
rule on synthetic pixels (``samples``: separations log-uniform in 0.001-30 deg,
pixel sizes 0.025-0.2 deg); the network is trained on the GPU by the library's
own kernels (forward on tcgen05 with BF16 operands, backward GEMMs on tcgen05,
Adam).  ``Surrogate.calibrate`` then measures the network's largest error on
held-out samples per cell of (log10 rho, segment slope) and keeps the cells
within half the error bound.  The model map (``model_map``) takes the network's
values in those cells (and inside the training range), the rule's elsewhere,
evaluates every 16th pixel by the rule as well (those pixels keep the rule's
values) and redoes by the rule every map whose check exceeds the tolerance.

All tensors live on the CUDA device; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np

from . import _lib as L


def _torch():
    import torch

    return torch


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _stream(dev) -> C.c_void_p:
    torch = _torch()
    h = torch.cuda.current_stream(dev).cuda_stream
    return C.c_void_p(h if h else 1)  # 0 would mean the library's own stream


def samples(upsf, logEs, n: int, seed: int = 1, rho_min: float = 0.0):
    """Training samples from mean-PSF tables upsf [S, 401, E] (float64, CUDA) and
    log10 energies [E]: features X [n, 5] and targets Y [n] (float32, CUDA)."""
    torch = _torch()
    upsf = upsf.to(torch.float64).contiguous()
    logEs = torch.as_tensor(logEs, dtype=torch.float64, device=upsf.device).contiguous()
    S, D, E = upsf.shape
    if D != L.ND:
        raise ValueError(f"upsf must be [S, {L.ND}, E], got {tuple(upsf.shape)}")
    X = torch.empty((n, L.MLP_IN), dtype=torch.float32, device=upsf.device)
    Y = torch.empty((n,), dtype=torch.float32, device=upsf.device)
    L.check(L.lib().xts_surrogate_samples(_ptr(upsf), _ptr(logEs), S, E, int(n), int(seed) & (2**64 - 1),
                                          float(rho_min), _ptr(X), _ptr(Y), _stream(upsf.device)))
    return X, Y


def gemm_bf16(A, B, M: int, K: int, a_trans: bool = False, b_trans: bool = False, c_trans: bool = False,
              out=None, accumulate: bool = False):
    """C = A B^T on tcgen05 (BF16 operands, FP32 result); A [M, K] (or [K, M] with
    a_trans), B [128, K] (or [K, 128]), C [M, 128] (or [128, M] with c_trans)."""
    torch = _torch()
    if out is None:
        out = torch.zeros((128, M) if c_trans else (M, 128), dtype=torch.float32, device=A.device)
    A = A.contiguous()
    B = B.contiguous()
    L.check(L.lib().xts_gemm_bf16(_ptr(A), int(a_trans), _ptr(B), int(b_trans), int(M), int(K), _ptr(out),
                                  int(c_trans), int(accumulate), _stream(A.device)))
    return out


class Surrogate:
    """Parameters (FP32 master copy, BF16 copies of the hidden layers), Adam
    state and standardisation of one surrogate network."""

    def __init__(self, device=None, seed: int = 0, rho_min: float = 0.0):
        torch = _torch()
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        rng = np.random.default_rng(seed)
        p = np.zeros(L.MLP_NPARAM, dtype=np.float32)
        H, I = L.MLP_HID, L.MLP_IN

        def glorot(fan_in, fan_out, size):
            a = math.sqrt(6.0 / (fan_in + fan_out))
            return rng.uniform(-a, a, size).astype(np.float32)

        p[L.MLP_W1:L.MLP_B1] = glorot(I, H, H * I)
        p[L.MLP_W2:L.MLP_B2] = glorot(H, H, H * H)
        p[L.MLP_W3:L.MLP_B3] = glorot(H, H, H * H)
        p[L.MLP_W4:L.MLP_B4] = glorot(H, 1, H)
        self.params = torch.as_tensor(p, device=self.device)
        self.wbf16 = torch.empty(2 * H * H, dtype=torch.int16, device=self.device)
        self.refresh_bf16()
        self.adam_m = torch.zeros_like(self.params)
        self.adam_v = torch.zeros_like(self.params)
        self.grads = torch.zeros_like(self.params)
        self.step = 0
        self.in_mu = np.zeros(I, np.float32)
        self.in_sd = np.ones(I, np.float32)
        self.out_mu, self.out_sd = 0.0, 1.0
        self.lo = np.full(I, -np.inf, np.float32)
        self.hi = np.full(I, np.inf, np.float32)
        self.rho_min = float(rho_min)
        # error cells over (log10 rho, segment slope); None until calibrated: no restriction
        self.cell_lo = np.zeros(2, np.float32)
        self.cell_hi = np.ones(2, np.float32)
        self.cell_ok = None  # uint8 CUDA tensor [NR * NS]
        self.cell_err = None  # float64 numpy [NR, NS]: held-out max relative error per cell

    def refresh_bf16(self) -> None:
        """BF16 copies of W2 and W3 from the FP32 parameters (round to nearest even)."""
        torch = _torch()
        H = L.MLP_HID
        w = torch.cat([self.params[L.MLP_W2:L.MLP_B2], self.params[L.MLP_W3:L.MLP_B3]])
        self.wbf16.copy_(w.to(torch.bfloat16).view(torch.int16))
        assert self.wbf16.numel() == 2 * H * H

    def struct(self) -> L.XtsMlp:
        f5 = C.c_float * L.MLP_IN
        f2 = C.c_float * 2
        cells = _ptr(self.cell_ok) if self.cell_ok is not None else None
        return L.XtsMlp(_ptr(self.params), _ptr(self.wbf16), f5(*self.in_mu), f5(*self.in_sd),
                        float(self.out_mu), float(self.out_sd), f5(*self.lo), f5(*self.hi), float(self.rho_min),
                        f2(*self.cell_lo), f2(*self.cell_hi), cells)

    def calibrate(self, X, Y, tol: float = 1e-4, margin: float = 0.5, min_count: int = 200) -> dict:
        """Error cells from held-out samples X [n, 5], Y [n] (not used in training):
        per cell of (log10 rho, segment slope) the largest relative error of the
        pixel mean, |exp((y_net - y) / rho^2) - 1|; the network takes values only in
        cells with at least ``min_count`` samples whose largest error is within
        ``margin * tol``.  Returns the share of held-out samples in accepted cells
        and their largest error."""
        torch = _torch()
        NR, NS = L.MLP_CELL_NR, L.MLP_CELL_NS
        yp = self.predict(X).double()
        Xd = X.double()
        rho2 = (10.0 ** Xd[:, 0]) ** 2
        err = torch.expm1((yp - Y.double()) / rho2).abs()
        err = torch.where(torch.isfinite(err), err, torch.full_like(err, float("inf")))
        lo = np.array([float(self.lo[0]), float(self.lo[4])], np.float64)
        hi = np.array([float(self.hi[0]), float(self.hi[4])], np.float64)
        hi = np.where(hi > lo, hi, lo + 1.0)
        self.cell_lo = lo.astype(np.float32)
        self.cell_hi = (hi + 1e-6 * (hi - lo)).astype(np.float32)  # the training maximum falls inside
        a = ((Xd[:, 0] - float(self.cell_lo[0])) * (NR / float(self.cell_hi[0] - self.cell_lo[0]))).floor().long()
        b = ((Xd[:, 4] - float(self.cell_lo[1])) * (NS / float(self.cell_hi[1] - self.cell_lo[1]))).floor().long()
        inside = (a >= 0) & (a < NR) & (b >= 0) & (b < NS)
        cell = (a.clamp(0, NR - 1) * NS + b.clamp(0, NS - 1))[inside]
        e_in = err[inside]
        count = torch.zeros(NR * NS, dtype=torch.float64, device=X.device).index_add_(0, cell, torch.ones_like(e_in))
        worst = torch.zeros(NR * NS, dtype=torch.float64, device=X.device).scatter_reduce_(
            0, cell, e_in, reduce="amax", include_self=True)
        ok = (count >= min_count) & (worst <= margin * tol)
        self.cell_ok = ok.to(torch.uint8).contiguous()
        self.cell_err = worst.view(NR, NS).cpu().numpy()
        taken = ok[cell]
        return {"held_out": int(X.shape[0]), "share_in_accepted_cells": float(taken.double().mean()),
                "max_rel_err_in_accepted_cells": float(e_in[taken].max()) if bool(taken.any()) else 0.0,
                "cells_accepted": int(ok.sum()), "cells": NR * NS, "tol": tol, "margin": margin,
                "min_count": min_count}

    def fit_standardisation(self, X, Y) -> None:
        """Feature and target standardisation, and the accepted feature range, from
        a training set."""
        torch = _torch()
        Xd = X.to(torch.float64)
        self.in_mu = Xd.mean(0).cpu().numpy().astype(np.float32)
        sd = Xd.std(0).cpu().numpy()
        self.in_sd = np.where(sd > 1e-12, sd, 1.0).astype(np.float32)
        self.lo = Xd.min(0).values.cpu().numpy().astype(np.float32)
        self.hi = Xd.max(0).values.cpu().numpy().astype(np.float32)
        Yd = Y.to(torch.float64)
        self.out_mu = float(Yd.mean())
        self.out_sd = float(Yd.std()) or 1.0

    def predict(self, X):
        """Network output y (de-standardised) for features X [n, 5]."""
        torch = _torch()
        X = X.to(torch.float32).contiguous()
        y = torch.empty((X.shape[0],), dtype=torch.float32, device=X.device)
        s = self.struct()
        L.check(L.lib().xts_mlp_forward(C.byref(s), _ptr(X), int(X.shape[0]), _ptr(y), _stream(X.device)))
        return y

    def gradient(self, X, Y):
        """(grads [NPARAM], loss) of the standardised mean squared error on one batch
        (rows a multiple of 128)."""
        torch = _torch()
        g = torch.empty_like(self.params)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        s = self.struct()
        L.check(L.lib().xts_mlp_grads(C.byref(s), _ptr(X.contiguous()), _ptr(Y.contiguous()), int(X.shape[0]),
                                      _ptr(g), _ptr(loss), _stream(X.device)))
        torch.cuda.synchronize(X.device)
        return g, float(loss.item())

    def train(self, X, Y, epochs: int = 20, batch: int = 128 * 148 * 2, lr: float = 2e-3,
              lr_final: float = 2e-5, seed: int = 0, log=None):
        """Adam with a cosine learning-rate decay over shuffled batches; the
        standardisation is fitted first if not set.  Returns the loss per epoch."""
        torch = _torch()
        if not np.isfinite(self.lo).all():
            self.fit_standardisation(X, Y)
        n = int(X.shape[0])
        batch = max(128, (min(batch, n) // 128) * 128)
        steps_per_epoch = n // batch
        if steps_per_epoch < 1:
            raise ValueError("fewer training samples than one batch of 128")
        total = steps_per_epoch * epochs
        gen = torch.Generator(device=X.device)
        gen.manual_seed(seed)
        loss = torch.zeros(1, dtype=torch.float32, device=X.device)
        s = self.struct()
        stream = _stream(X.device)
        out = []
        k = 0
        for ep in range(epochs):
            perm = torch.randperm(n, device=X.device, generator=gen)
            loss.zero_()
            for b in range(steps_per_epoch):
                idx = perm[b * batch:(b + 1) * batch]
                xb = X.index_select(0, idx).contiguous()
                yb = Y.index_select(0, idx).contiguous()
                frac = k / max(1, total - 1)
                lr_k = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * frac))
                self.step += 1
                L.check(L.lib().xts_mlp_train_step(C.byref(s), _ptr(xb), _ptr(yb), batch, _ptr(self.grads),
                                                   _ptr(self.adam_m), _ptr(self.adam_v), self.step, float(lr_k),
                                                   _ptr(loss), stream))
                k += 1
            out.append(float(loss.item()) / steps_per_epoch)
            if log:
                log(f"epoch {ep}: loss {out[-1]:.3e}")
        return out

    def state(self) -> dict:
        st = {"params": self.params.cpu().numpy(), "in_mu": self.in_mu, "in_sd": self.in_sd,
              "out": np.array([self.out_mu, self.out_sd], np.float64), "lo": self.lo, "hi": self.hi,
              "rho_min": np.array(self.rho_min), "cell_lo": self.cell_lo, "cell_hi": self.cell_hi}
        if self.cell_ok is not None:
            st["cell_ok"] = self.cell_ok.cpu().numpy()
        return st

    def save(self, path: str) -> None:
        np.savez(path, **self.state())

    @classmethod
    def load(cls, path: str, device=None) -> "Surrogate":
        z = np.load(path)
        net = cls(device=device, rho_min=float(z["rho_min"]))
        net.params.copy_(_torch().as_tensor(z["params"], device=net.device))
        net.refresh_bf16()
        net.in_mu, net.in_sd = z["in_mu"].astype(np.float32), z["in_sd"].astype(np.float32)
        net.out_mu, net.out_sd = float(z["out"][0]), float(z["out"][1])
        net.lo, net.hi = z["lo"].astype(np.float32), z["hi"].astype(np.float32)
        if "cell_ok" in z:
            net.cell_lo, net.cell_hi = z["cell_lo"].astype(np.float32), z["cell_hi"].astype(np.float32)
            net.cell_ok = _torch().as_tensor(z["cell_ok"].astype(np.uint8), device=net.device)
        return net


def _stats_dict(st) -> dict:
    return {"values": st.values, "accepted": st.accepted, "checked": st.checked,
            "maps_fallback": st.maps_fallback, "max_check_err": st.max_check_err, "evaluated": st.evaluated}


def last_stats(device=None) -> dict:
    """Counts of the latest surrogate model map (waits for it on torch's current stream)."""
    torch = _torch()
    st = L.XtsSurrogateStats()
    L.check(L.lib().xts_surrogate_last_stats(C.byref(st), _stream(device or torch.device("cuda"))))
    return _stats_dict(st)


def model_map(wcs, src_sph, exposure, uPsf, partial_integrals, logEs, net: Surrogate,
              check_tol: float = 1e-4, with_info: bool = True, out=None, stats: bool = True):
    """point_src_model_map_wcs with the pixel means from the network where it
    applies (the 12-point rule elsewhere: the plain path's window and write passes
    for up to 52 energies, the FP64 rule per value above; the FP64 rule for every
    map whose check fails).  CUDA tensors in; returns (float32 maps [S, H, W, E], SrcmapInfo or
    None, stats dict or None).  With stats=False the call does not synchronise
    (and, once warm, can be captured into a CUDA graph); ``last_stats`` reads the
    counts afterwards."""
    torch = _torch()
    from .api import SrcmapInfo, _wcs_struct

    dev = uPsf.device
    t = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt, device=dev).contiguous()
    src, ex, up, pp, le = t(src_sph), t(exposure), t(uPsf), t(partial_integrals), t(logEs)
    S, E = int(src.shape[0]), int(ex.shape[1])
    maps = out if out is not None else torch.empty((S, int(wcs.naxis1), int(wcs.naxis2), E), dtype=torch.float32,
                                                   device=dev)
    info = info_s = None
    if with_info:
        o = [torch.empty((S, E), dtype=torch.float64, device=dev), torch.empty((S, E), dtype=torch.float64, device=dev),
             torch.empty((S,), dtype=torch.float64, device=dev), torch.empty((S,), dtype=torch.int32, device=dev)]
        info_s = L.XtsSrcmapInfo(*[_ptr(x) for x in o])
        info = SrcmapInfo(*o)
    st = L.XtsSurrogateStats() if stats else None
    s = net.struct()
    w = _wcs_struct(wcs)
    L.check(L.lib().xts_point_src_model_map_wcs_surrogate(
        C.byref(w), _ptr(src), S, _ptr(ex), _ptr(up), _ptr(pp), _ptr(le), E, C.byref(s), float(check_tol),
        _ptr(maps), C.byref(info_s) if info_s is not None else None, C.byref(st) if st is not None else None,
        _stream(dev)))
    return maps, info, (_stats_dict(st) if st is not None else None)
