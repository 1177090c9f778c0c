"""CPU restatement of the learned floor proposer (test infrastructure only).

The network has no counterpart in the reference; this numpy version defines
its arithmetic, and the CUDA forward / backward kernels are checked against
it (same parameters, same inputs):

    x (N, 1, 16, 16, 16)  density average-pooled to 16^3 (PyTorch adaptive
                          average-pool windows: [floor(i*n/16), ceil((i+1)*n/16)))
    conv 1->16, 3x3x3, stride 1, pad 1, ReLU   -> 16^3
    conv 16->16, 3x3x3, stride 2, pad 1, ReLU  -> 8^3
    conv 16->32, 3x3x3, stride 2, pad 1, ReLU  -> 4^3
    conv 32->32, 3x3x3, stride 2, pad 1, ReLU  -> 2^3
    mean over the 8 positions -> 32, concatenated with the 2 probe features
    dense 34 -> 3, softmax over the floor rungs; loss = mean cross-entropy.

Weights (not biases) are rounded to bfloat16 (round to nearest even) before
use; products accumulate in float32 (float64 here: the oracle is the exact
reference the float32 kernels are compared against within a tolerance).
Gradients are taken with respect to the rounded weights and applied to the
float32 master copy.
"""

from __future__ import annotations

import numpy as np

LAYERS = ((1, 16, 1), (16, 16, 2), (16, 32, 2), (32, 32, 2))  # (cin, cout, stride)
N_FEAT = 2
N_CLASS = 3
S0 = 16


def param_shapes():
    shapes = []
    for cin, cout, _ in LAYERS:
        shapes += [(cout, cin, 3, 3, 3), (cout,)]
    shapes += [(N_CLASS, LAYERS[-1][1] + N_FEAT), (N_CLASS,)]
    return shapes


def n_params() -> int:
    return int(sum(np.prod(s) for s in param_shapes()))


def unpack(theta: np.ndarray) -> list:
    out, o = [], 0
    for s in param_shapes():
        k = int(np.prod(s))
        out.append(theta[o:o + k].reshape(s))
        o += k
    return out


def bf16(w: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even) and back."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def pool16(density: np.ndarray, dims) -> np.ndarray:
    nx, ny, nz = dims
    d = np.asarray(density, dtype=np.float64).reshape(nx, ny, nz)
    out = np.empty((S0, S0, S0))
    w = [[(i * n // S0, -(-(i + 1) * n // S0)) for i in range(S0)] for n in (nx, ny, nz)]
    for a, (x0, x1) in enumerate(w[0]):
        for b, (y0, y1) in enumerate(w[1]):
            for c, (z0, z1) in enumerate(w[2]):
                out[a, b, c] = d[x0:x1, y0:y1, z0:z1].mean()
    return out.astype(np.float32)


def _conv(x, W, b, stride):
    """x (N, Cin, S, S, S), W (Cout, Cin, 3, 3, 3) -> (N, Cout, So, So, So); pad 1."""
    n, cin, s = x.shape[0], x.shape[1], x.shape[2]
    so = (s + 2 - 3) // stride + 1
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1), (1, 1)))
    cols = np.empty((n, cin, 3, 3, 3, so, so, so))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                cols[:, :, kz, ky, kx] = xp[:, :, kz:kz + stride * so:stride, ky:ky + stride * so:stride,
                                            kx:kx + stride * so:stride]
    y = np.einsum("ncijkpqr,ocijk->nopqr", cols, W) + b[None, :, None, None, None]
    return y, cols


def forward(theta, x, feats):
    """Returns (logits (N, 3), cache)."""
    p = unpack(np.asarray(theta, dtype=np.float64))
    h = np.asarray(x, dtype=np.float64)
    cache = []
    for li, (_, _, stride) in enumerate(LAYERS):
        W = bf16(p[2 * li]).astype(np.float64)
        y, cols = _conv(h, W, p[2 * li + 1].astype(np.float64), stride)
        a = np.maximum(y, 0.0)
        cache.append((cols, W, a, stride, h.shape))
        h = a
    g = h.mean(axis=(2, 3, 4))
    z = np.concatenate([g, np.asarray(feats, dtype=np.float64)], axis=1)
    Wfc = bf16(p[-2]).astype(np.float64)
    logits = z @ Wfc.T + p[-1].astype(np.float64)
    return logits, (cache, h, z, Wfc)


def loss_and_grad(theta, x, feats, labels):
    """Mean cross-entropy and its gradient with respect to every parameter."""
    logits, (cache, hlast, z, Wfc) = forward(theta, x, feats)
    n = logits.shape[0]
    m = logits.max(axis=1, keepdims=True)
    e = np.exp(logits - m)
    prob = e / e.sum(axis=1, keepdims=True)
    lab = np.asarray(labels, dtype=np.int64)
    loss = float(-np.log(prob[np.arange(n), lab]).mean())
    dlog = prob.copy()
    dlog[np.arange(n), lab] -= 1.0
    dlog /= n
    grads = [None] * (2 * len(LAYERS) + 2)
    grads[-2] = dlog.T @ z
    grads[-1] = dlog.sum(axis=0)
    dz = dlog @ Wfc
    c_last = hlast.shape[1]
    dh = np.broadcast_to(dz[:, :c_last, None, None, None] / 8.0, hlast.shape).copy()
    for li in range(len(LAYERS) - 1, -1, -1):
        cols, W, a, stride, in_shape = cache[li]
        dy = dh * (a > 0)
        grads[2 * li] = np.einsum("nopqr,ncijkpqr->ocijk", dy, cols)
        grads[2 * li + 1] = dy.sum(axis=(0, 2, 3, 4))
        if li == 0:
            break
        dcols = np.einsum("nopqr,ocijk->ncijkpqr", dy, W)
        n_, cin, s = in_shape[0], in_shape[1], in_shape[2]
        so = dy.shape[2]
        dxp = np.zeros((n_, cin, s + 2, s + 2, s + 2))
        for kz in range(3):
            for ky in range(3):
                for kx in range(3):
                    dxp[:, :, kz:kz + stride * so:stride, ky:ky + stride * so:stride,
                        kx:kx + stride * so:stride] += dcols[:, :, kz, ky, kx]
        dh = dxp[:, :, 1:-1, 1:-1, 1:-1]
    flat = np.concatenate([np.asarray(gr, dtype=np.float64).ravel() for gr in grads])
    return loss, flat


def init_params(seed: int) -> np.ndarray:
    """He-normal weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    out = []
    for s in param_shapes():
        if len(s) == 1:
            out.append(np.zeros(s))
        else:
            fan_in = int(np.prod(s[1:]))
            out.append(rng.standard_normal(s) * np.sqrt(2.0 / fan_in))
    return np.concatenate([o.ravel() for o in out]).astype(np.float32)
