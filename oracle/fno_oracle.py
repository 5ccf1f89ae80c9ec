"""FP64 NumPy restatement of the warm-start surrogate -- TEST INFRASTRUCTURE.

Forward pass, masked MSE loss and backward pass of the Fourier neural operator
in curved_lbm/warmstart.py, written independently in float64 NumPy.  The
native path rounds the operands of its tensor-core GEMMs to bf16; with
`bf16=True` this restatement rounds the same operands (round to nearest
even), so the two agree to fp32-accumulation differences.  With
`bf16=False` it is a plain float64 model whose gradients the CPU tests check
against central finite differences.

Used only by tests/.
"""

from __future__ import annotations

import math

import numpy as np


def round_bf16(x) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    from math import erf

    e = np.vectorize(erf)(z / math.sqrt(2.0))
    return 0.5 * z * (1.0 + e)


def gelu_grad(z):
    from math import erf

    cdf = 0.5 * (1.0 + np.vectorize(erf)(z / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)
    return cdf + z * pdf


def pointwise(W, b, x):
    # x [B, Cin, G] -> [B, Cout, G]
    return np.einsum("oi,big->bog", W, x) + b[None, :, None]


def forward(params, x, phi, n_layers, bf16=True):
    """y and the cache of the backward pass.  phi: [G, M] basis."""
    rb = round_bf16 if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    phi_r = rb(phi)
    cache = {"x": x}
    h = pointwise(params["W0"], params["b0"], x)
    for l in range(1, n_layers + 1):
        a = np.einsum("bcg,gk->bck", rb(h), phi_r)
        bh = np.einsum("bik,kio->bok", a, params[f"R{l}"])
        s = np.einsum("bok,gk->bog", rb(bh), phi_r)
        z = pointwise(params[f"W{l}"], params[f"b{l}"], h) + s
        cache[l] = (h, a, z)
        h = gelu(z) if l < n_layers else z
    cache["h"] = h
    return pointwise(params["Wp"], params["bp"], h), cache


def mse(y, t, mask, wch):
    cnt = mask.sum() * y.shape[1]
    m = mask[:, None, :] * wch[None, :, None]
    e = y - t
    return float((m * e * e).sum() / cnt), 2.0 * m * e / cnt


def backward(params, cache, dy, phi, n_layers, bf16=True):
    rb = round_bf16 if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    phi_r = rb(phi)
    g = {}
    h = cache["h"]
    g["Wp"] = np.einsum("bog,big->oi", dy, h)
    g["bp"] = dy.sum(axis=(0, 2))
    dh = np.einsum("oi,bog->big", params["Wp"], dy)
    for l in range(n_layers, 0, -1):
        hl, a, z = cache[l]
        dz = dh * gelu_grad(z) if l < n_layers else dh
        g[f"W{l}"] = np.einsum("bog,big->oi", dz, hl)
        g[f"b{l}"] = dz.sum(axis=(0, 2))
        dprev = np.einsum("oi,bog->big", params[f"W{l}"], dz)
        dbh = np.einsum("bog,gk->bok", rb(dz), phi_r)
        g[f"R{l}"] = np.einsum("bik,bok->kio", a, dbh)
        da = np.einsum("kio,bok->bik", params[f"R{l}"], dbh)
        dprev = dprev + np.einsum("bik,gk->big", rb(da), phi_r)
        dh = dprev
    g["W0"] = np.einsum("bog,big->oi", dh, cache["x"])
    g["b0"] = dh.sum(axis=(0, 2))
    return g
