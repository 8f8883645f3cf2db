"""CPU oracle of the learned residual row filter (TEST INFRASTRUCTURE ONLY).

Restates the network of fdk_b200/csrc/learn.cu in numpy -- forward and an analytic backward --
in float64, optionally rounding the two hidden activations to bfloat16 exactly where the GPU
stores them, so the GPU gradients can be compared with a reference and the reference itself can
be checked by finite differences.  There is no reference (peng-ac/fdk) counterpart.
"""
from __future__ import annotations

import numpy as np

CH, K, HALO = 32, 9, 4
SIZES = [("W1", (CH, 1, K)), ("b1", (CH,)), ("W2", (CH, CH, K)), ("b2", (CH,)), ("W3", (1, CH, K)), ("b3", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(params):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([d[name].reshape(-1) for name, _ in SIZES])


def bf16(a):
    """Round float64 -> bfloat16 (round to nearest even) -> float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def conv(x, W, b):
    """'same' conv1d: x (rows, cin, L), W (cout, cin, K) -> (rows, cout, L); out[p] = sum_k W[k] x[p+k-4]."""
    rows, cin, L = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (HALO, HALO)))
    out = np.zeros((rows, W.shape[0], L)) + b[None, :, None]
    for k in range(K):
        out += np.einsum("oc,rcl->rol", W[:, :, k], xp[:, :, k:k + L])
    return out


def conv_t(g, W):
    """Transpose of conv for the input: g (rows, cout, L) -> (rows, cin, L)."""
    rows, cout, L = g.shape
    gp = np.pad(g, ((0, 0), (0, 0), (HALO, HALO)))
    out = np.zeros((rows, W.shape[1], L))
    for k in range(K):
        # x[q] feeds out[p] with q = p + k - 4  ->  p = q - k + 4
        out += np.einsum("oc,rol->rcl", W[:, :, k], gp[:, :, 2 * HALO - k:2 * HALO - k + L])
    return out


def conv_w(g, x):
    """Weight gradient: g (rows, cout, L), x (rows, cin, L) -> (cout, cin, K)."""
    rows, cin, L = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (HALO, HALO)))
    return np.stack([np.einsum("rol,rcl->oc", g, xp[:, :, k:k + L]) for k in range(K)], -1)


def forward(params, x, s, round_bf16=True):
    """x (rows, L) -> y (rows, L) and the cache."""
    P = unpack(params)
    r = bf16 if round_bf16 else (lambda a: a)
    xs = (np.asarray(x, np.float64) * s)[:, None, :]
    z1 = conv(xs, P["W1"], P["b1"])
    a1 = r(np.maximum(z1, 0))
    z2 = conv(a1, P["W2"], P["b2"])
    a2 = r(np.maximum(z2, 0))
    o = conv(a2, P["W3"], P["b3"])[:, 0, :]
    y = np.asarray(x, np.float64) + o / s
    return y, dict(xs=xs, z1=z1, a1=a1, z2=z2, a2=a2)


def backward(params, x, dy, s, round_bf16=True):
    """Gradient of sum(dy * y) w.r.t. the parameters (flat, float64)."""
    P = unpack(params)
    _, c = forward(params, x, s, round_bf16)
    d3 = (np.asarray(dy, np.float64) / s)[:, None, :]
    g = {"W3": conv_w(d3, c["a2"]), "b3": d3.sum((0, 2))}
    dz2 = conv_t(d3, P["W3"]) * (c["z2"] > 0)
    g["W2"] = conv_w(dz2, c["a1"])
    g["b2"] = dz2.sum((0, 2))
    dz1 = conv_t(dz2, P["W2"]) * (c["a1"] > 0)
    g["W1"] = conv_w(dz1, c["xs"])
    g["b1"] = dz1.sum((0, 2))
    return pack(g)
