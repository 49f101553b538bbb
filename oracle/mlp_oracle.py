"""CPU oracle of the surrogate network (test infrastructure only: the product
path never imports this file).

The network has no counterpart in the reference; this restates the library's
own definition (include/xtsrcmaps_b200.h, "Learned surrogate of the pixel
cubature") in numpy: 5 -> 128 -> 128 -> 128 -> 1, tanh-form GELU
(Hendrycks & Gimpel 2016), inputs standardised, loss the mean squared error of
the standardised output.  ``bf16=True`` rounds where the CUDA kernels round to
BF16 (the first- and output-layer weights, the hidden-layer weights and the
hidden activations h1, h2 that feed the tensor-core layers, and the back-
propagated dz that feed the backward GEMMs), with FP64 sums; ``bf16=False`` is
the plain FP64 network, which the finite-difference test pins.
"""
from __future__ import annotations

import numpy as np

IN, HID = 5, 128
W1 = 0
B1 = W1 + HID * IN
W2 = B1 + HID
B2 = W2 + HID * HID
W3 = B2 + HID
B3 = W3 + HID * HID
W4 = B3 + HID
B4 = W4 + HID
NPARAM = B4 + 1

K0 = 0.7978845608028654  # sqrt(2 / pi)
K1 = 0.044715


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(K0 * (z + K1 * z ** 3)))


def gelu_grad(z):
    th = np.tanh(K0 * (z + K1 * z ** 3))
    return 0.5 * (1.0 + th) + 0.5 * z * (1.0 - th * th) * K0 * (1.0 + 3.0 * K1 * z * z)


def _layers(p, use_bf16):
    r = bf16 if use_bf16 else (lambda x: np.asarray(x, np.float64))
    p = np.asarray(p, np.float64)
    return (r(p[W1:B1].reshape(HID, IN)), p[B1:W2], r(p[W2:B2].reshape(HID, HID)), p[B2:W3],
            r(p[W3:B3].reshape(HID, HID)), p[B3:W4], r(p[W4:B4]), p[B4])


def forward(p, X, in_mu, in_sd, use_bf16=True):
    """Standardised output yn [n] and the intermediates of the backward pass."""
    r = bf16 if use_bf16 else (lambda x: np.asarray(x, np.float64))
    w1, b1, w2, b2, w3, b3, w4, b4 = _layers(p, use_bf16)
    xn = (np.asarray(X, np.float32) - np.asarray(in_mu, np.float32)) / np.asarray(in_sd, np.float32)
    xn = xn.astype(np.float64)
    z1 = xn @ w1.T + b1
    h1 = r(gelu(z1))
    z2 = h1 @ w2.T + b2
    h2 = r(gelu(z2))
    z3 = h2 @ w3.T + b3
    h3 = gelu(z3)
    yn = h3 @ w4 + b4
    return yn, dict(xn=xn, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, h3=h3)


def predict(p, X, in_mu, in_sd, out_mu, out_sd, use_bf16=True):
    yn, _ = forward(p, X, in_mu, in_sd, use_bf16)
    return yn * out_sd + out_mu


def loss_and_grads(p, X, Y, in_mu, in_sd, out_mu, out_sd, use_bf16=True):
    """(loss, grads [NPARAM]) of L = mean((yn - (Y - out_mu) / out_sd)^2)."""
    r = bf16 if use_bf16 else (lambda x: np.asarray(x, np.float64))
    w1, b1, w2, b2, w3, b3, w4, b4 = _layers(p, use_bf16)
    yn, c = forward(p, X, in_mu, in_sd, use_bf16)
    n = len(yn)
    tgt = (np.asarray(Y, np.float32).astype(np.float64) - out_mu) / out_sd
    d = yn - tgt
    loss = float(np.mean(d * d))
    dy = 2.0 * d / n
    g = np.zeros(NPARAM, np.float64)
    g[W4:B4] = c["h3"].T @ dy
    g[B4] = dy.sum()
    dz3 = dy[:, None] * w4[None, :] * gelu_grad(c["z3"])
    g[B3:W4] = dz3.sum(0)
    dz3 = r(dz3)
    g[W3:B3] = (dz3.T @ c["h2"]).ravel()
    dh2 = dz3 @ w3
    dz2 = dh2 * gelu_grad(c["z2"])
    g[B2:W3] = dz2.sum(0)
    dz2 = r(dz2)
    g[W2:B2] = (dz2.T @ c["h1"]).ravel()
    dh1 = dz2 @ w2
    dz1 = dh1 * gelu_grad(c["z1"])
    g[B1:W2] = dz1.sum(0)
    g[W1:B1] = (dz1.T @ c["xn"]).ravel()
    return loss, g
