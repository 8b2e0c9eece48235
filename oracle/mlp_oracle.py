"""CPU oracle of the warm-start network -- test infrastructure only, never on the product path.

Restates in NumPy what the library's bmc_mlp_forward / bmc_mlp_backward / bmc_mlp_adam_step compute:
the parameter layout of include/bmc_b200.h (per layer W [out][in] then b [out], dimensions padded to
64), GELU in its erf form, the mean squared error over the n_out outputs and Adam with bias
correction -- with the tensor-core path's roundings to bfloat16 at the same places (normalised
inputs, weights, hidden activations, back-propagated gradients), products and sums in float64.
`emulate=False` drops the roundings: that float64 network is checked against central finite
differences, which pins the backward pass's algebra; the GPU is then checked against
`emulate=True`.

BMC-JAX has no learned component, so there is no reference implementation to pin this against:
the network is specified by this restatement and its finite-difference check.
"""
from __future__ import annotations

from typing import List, NamedTuple

import numpy as np
from scipy.special import erf


def bf16(x):
    """Round to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).reshape(a.shape)


def rup(x, m):
    return (x + m - 1) // m * m


class Layer(NamedTuple):
    off_w: int
    off_b: int
    rows: int   # padded outputs
    cols: int   # padded inputs


def layout(n_in, n_hidden, n_layers, n_out) -> List[Layer]:
    """Parameter layout: hidden layers then the output layer, each W [rows][cols] then b [rows]."""
    in_pad, out_pad = rup(n_in, 64), rup(n_out, 64)
    dims = [(n_hidden, in_pad)] + [(n_hidden, n_hidden)] * (n_layers - 1) + [(out_pad, n_hidden)]
    out, off = [], 0
    for r, c in dims:
        out.append(Layer(off, off + r * c, r, c))
        off += r * c + r
    return out


def n_params(lay: List[Layer]) -> int:
    return lay[-1].off_b + lay[-1].rows


def init_params(n_in, n_hidden, n_layers, n_out, seed=0):
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) on the real (unpadded) weights and biases, zero padding."""
    lay = layout(n_in, n_hidden, n_layers, n_out)
    rng = np.random.default_rng(seed)
    p = np.zeros(n_params(lay), np.float32)
    fan_in = [n_in] + [n_hidden] * n_layers
    real_out = [n_hidden] * n_layers + [n_out]
    for L, fi, ro in zip(lay, fan_in, real_out):
        bound = 1.0 / np.sqrt(fi)
        W = np.zeros((L.rows, L.cols), np.float32)
        W[:ro, :fi] = rng.uniform(-bound, bound, (ro, fi))
        b = np.zeros(L.rows, np.float32)
        b[:ro] = rng.uniform(-bound, bound, ro)
        p[L.off_w:L.off_b] = W.ravel()
        p[L.off_b:L.off_b + L.rows] = b
    return p


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def _w(p, L):
    W = np.asarray(p[L.off_w:L.off_b], np.float64).reshape(L.rows, L.cols)
    b = np.asarray(p[L.off_b:L.off_b + L.rows], np.float64)
    return W, b


def forward(p, shape, x, shift=None, scale=None, emulate=True):
    """y [batch][n_out] and the cache for backward. shape = (n_in, n_hidden, n_layers, n_out)."""
    n_in, H, nl, n_out = shape
    lay = layout(*shape)
    rnd = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    x = np.asarray(x, np.float64)
    if shift is not None:
        x = x - np.asarray(shift, np.float64)
    if scale is not None:
        x = x * np.asarray(scale, np.float64)
    X = np.zeros((x.shape[0], lay[0].cols))
    X[:, :n_in] = rnd(x)
    acts, zs = [X], []
    h = X
    for L in lay[:-1]:
        W, b = _w(p, L)
        z = h @ np.asarray(rnd(W), np.float64).T + b
        zs.append(z)
        h = np.asarray(rnd(gelu(z)), np.float64)
        acts.append(h)
    W, b = _w(p, lay[-1])
    y = h @ np.asarray(rnd(W), np.float64).T + b
    return y[:, :n_out], dict(acts=acts, zs=zs, y=y, emulate=emulate)


def backward(p, shape, cache, target):
    """(grad [n_params], loss) of mean((y - t)^2) over the batch and the n_out outputs."""
    n_in, H, nl, n_out = shape
    lay = layout(*shape)
    rnd = bf16 if cache["emulate"] else (lambda a: np.asarray(a, np.float64))
    y = cache["y"][:, :n_out]
    B = y.shape[0]
    e = y - np.asarray(target, np.float64)
    loss = float(np.sum(e * e) / (B * n_out))
    g = np.zeros(n_params(lay))
    d = np.zeros((B, lay[-1].rows))
    d[:, :n_out] = np.asarray(rnd(2.0 * e / (B * n_out)), np.float64)
    for li in range(len(lay) - 1, -1, -1):
        L = lay[li]
        a_in = cache["acts"][li]
        g[L.off_w:L.off_b] = (d.T @ a_in).ravel()
        g[L.off_b:L.off_b + L.rows] = d.sum(axis=0)
        if li == 0:
            break
        W, _ = _w(p, L)
        dh = d @ np.asarray(rnd(W), np.float64)
        d = np.asarray(rnd(dh * gelu_grad(cache["zs"][li - 1])), np.float64)
    return g, loss


def adam(p, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step with bias correction; returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    lr_t = lr * np.sqrt(1 - b2 ** step) / (1 - b1 ** step)
    return p - lr_t * m / (np.sqrt(v) + eps), m, v
