"""CPU oracle for the warm-start network (libnir_mlp.so, include/nir_mlp.h).

TEST INFRASTRUCTURE ONLY: the tests use it to check the GPU network's
forward pass and gradients; nothing in the product imports it.  The
reference has no learned component, so this oracle restates the network
the header defines (dense layers, ReLU, mean-squared error weighted per
output) in numpy:

  * `loss_and_grads(..., emulate=True)` rounds to BF16 exactly where the
    device does (inputs, weight copies, hidden activations, the output
    gradient and the masked hidden gradients) and accumulates in float64,
    so the device's FP32 tensor-core sums must agree with it to a few FP32
    ulps of the sums, up to the rare element whose BF16 rounding flips;
  * `loss_and_grads(..., emulate=False)` is the exact float64 network, which
    `finite_difference` checks against central differences: that pins the
    oracle's backward formulas themselves.
"""
from __future__ import annotations

import numpy as np


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    # NaN/inf pass through unchanged
    bad = ~np.isfinite(f)
    out[bad] = f[bad]
    return out


def unpack(params: np.ndarray, dims: list[int]):
    """Flat layout of nir_mlp_get_params: per layer W (out x in) then b."""
    layers, o = [], 0
    for i in range(len(dims) - 1):
        n_in, n_out = dims[i], dims[i + 1]
        W = params[o:o + n_in * n_out].reshape(n_out, n_in).astype(np.float64)
        o += n_in * n_out
        b = params[o:o + n_out].astype(np.float64)
        o += n_out
        layers.append((W, b))
    assert o == params.size
    return layers


def forward(params, dims, X, emulate=True):
    q = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(np.asarray(params), dims)
    h = q(X)
    acts = [h]
    for li, (W, b) in enumerate(layers):
        z = h @ q(W).T + b
        if li + 1 < len(layers):
            h = q(np.maximum(z, 0.0))
            acts.append(h)
        else:
            out = z.astype(np.float32).astype(np.float64) if emulate else z
    return out, acts


def loss_and_grads(params, dims, X, T, w=None, emulate=True):
    """Weighted MSE, loss = sum w (y - t)^2 / (rows * sum w), and its
    gradients in the flat parameter layout."""
    q = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(np.asarray(params), dims)
    rows = X.shape[0]
    w = np.ones(dims[-1]) if w is None else np.asarray(w, dtype=np.float64)
    y, acts = forward(params, dims, X, emulate)
    d = y - np.asarray(T, dtype=np.float64)
    denom = rows * max(w.sum(), 1.0)
    loss = float((w * d * d).sum() / denom)
    g = q(2.0 / denom * (w * d))
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        W, _ = layers[li]
        a_in = acts[li]
        gW = g.T @ a_in
        gb = g.sum(axis=0)
        grads[li] = (gW, gb)
        if li > 0:
            g = q((g @ q(W)) * (acts[li] > 0))
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat


def finite_difference(params, dims, X, T, w=None, idx=None, h=1e-6):
    """Central differences of the exact float64 loss at parameter indices."""
    p = np.asarray(params, dtype=np.float64).copy()
    out = []
    for i in idx:
        old = p[i]
        p[i] = old + h
        lp, _ = loss_and_grads(p, dims, X, T, w, emulate=False)
        p[i] = old - h
        lm, _ = loss_and_grads(p, dims, X, T, w, emulate=False)
        p[i] = old
        out.append((lp - lm) / (2 * h))
    return np.array(out)
