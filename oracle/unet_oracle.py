"""CPU oracle of the learned warm start's network (test infrastructure).

numpy restatement, in FP64, of every layer of the U-Net that
``boilingsim_b200/learned.py`` runs on the GPU: the 3x3x3 zero-padded
convolution (channels-last activations act[i, j, k, c], weights
w[tap, co, ci] with tap = (di+1)*9 + (dj+1)*3 + (dk+1)), its data and weight
gradients, ReLU, 2x2x2 average pooling, nearest x2 upsampling, the additive
skips, the 16 -> 1 head and the masked mean-squared loss.  The GPU's forward
pass and every parameter gradient are checked against these on small grids.
Nothing in the product path imports this file.
"""
from __future__ import annotations

import numpy as np

TAPS = [(a - 1, b - 1, c - 1) for a in range(3) for b in range(3) for c in range(3)]


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (nearest even) and back, as the GPU stores them."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def _shift(x, d):
    """y[i, j, k] = x[i + di, j + dj, k + dk], zero outside."""
    di, dj, dk = d
    y = np.zeros_like(x)
    nx, ny, nz = x.shape[:3]
    si = slice(max(0, -di), nx - max(0, di))
    sj = slice(max(0, -dj), ny - max(0, dj))
    sk = slice(max(0, -dk), nz - max(0, dk))
    ti = slice(max(0, di), nx - max(0, -di))
    tj = slice(max(0, dj), ny - max(0, -dj))
    tk = slice(max(0, dk), nz - max(0, -dk))
    y[si, sj, sk] = x[ti, tj, tk]
    return y


def conv3(x, w, b=None):
    """out[v, co] = b[co] + sum_{tap, ci} x[v + d(tap), ci] w[tap, co, ci]."""
    out = np.zeros(x.shape[:3] + (w.shape[1],), np.float64)
    for t, d in enumerate(TAPS):
        out += np.einsum("ijkc,oc->ijko", _shift(x, d), w[t], optimize=True)
    if b is not None:
        out += b
    return out


def conv3_grad(x, w, g):
    """(dx, dw, db) of conv3 for the output gradient g."""
    dx = np.zeros(x.shape, np.float64)
    dw = np.zeros(w.shape, np.float64)
    for t, d in enumerate(TAPS):
        xs = _shift(x, d)
        dw[t] = np.einsum("ijko,ijkc->oc", g, xs, optimize=True)
        # x[v + d] feeds out[v]: dx[u] += g[u - d] w
        dx += _shift(np.einsum("ijko,oc->ijkc", g, w[t], optimize=True), tuple(-q for q in d))
    db = g.sum(axis=(0, 1, 2))
    return dx, dw, db


def pool(x):
    nx, ny, nz, c = x.shape
    return x.reshape(nx // 2, 2, ny // 2, 2, nz // 2, 2, c).mean(axis=(1, 3, 5))


def pool_grad(g):
    return np.repeat(np.repeat(np.repeat(g, 2, 0), 2, 1), 2, 2) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 0), 2, 1), 2, 2)


def up_grad(g):
    nx, ny, nz, c = g.shape
    return g.reshape(nx // 2, 2, ny // 2, 2, nz // 2, 2, c).sum(axis=(1, 3, 5))


LAYERS = [("e1a", 16, 16), ("e1b", 16, 16), ("e2a", 16, 32), ("e2b", 32, 32),
          ("e3a", 32, 64), ("e3b", 64, 64), ("bta", 64, 128), ("btb", 128, 128),
          ("u3a", 128, 64), ("u3b", 64, 64), ("u2a", 64, 32), ("u2b", 32, 32),
          ("u1a", 32, 16), ("u1b", 16, 16)]


def forward_backward(x0, P, fluid, target, scale, bf16=True, norm=None):
    """The network's forward pass and the gradient of its loss.

    x0: packed input (nx, ny, nz, 16); P: dict of parameters (name.w [27, co, ci],
    name.b [co], head.w [16], head.b [1]); fluid: bool mask; target: pressure;
    scale: S; norm: the loss divides the squared error by it (default: the
    number of fluid cells).  With ``bf16`` every activation and activation gradient is
    rounded to BF16 where the GPU stores one, and the convolution weights are
    the BF16 copies, so the comparison isolates summation order.  Returns
    (pred, loss, grads dict)."""
    q = (lambda a: bf16_round(a).astype(np.float64)) if bf16 else (lambda a: a)  # noqa: E731
    W = {k: (q(v) if k.endswith(".w") and not k.startswith("head") else v) for k, v in P.items()}
    relu = lambda z: np.maximum(z, 0.0)  # noqa: E731
    A = {}

    def cv(name, x):
        z = q(relu(conv3(x, W[name + ".w"], W[name + ".b"])))
        A[name] = (x, z)
        return z

    x0 = q(x0)
    e1 = cv("e1b", cv("e1a", x0))
    e2 = cv("e2b", cv("e2a", q(pool(e1))))
    e3 = cv("e3b", cv("e3a", q(pool(e2))))
    b4 = cv("btb", cv("bta", q(pool(e3))))
    u3 = cv("u3b", q(cv("u3a", up(b4)) + e3))
    u2 = cv("u2b", q(cv("u2a", up(u3)) + e2))
    u1 = cv("u1b", q(cv("u1a", up(u2)) + e1))
    y = u1 @ W["head.w"] + W["head.b"][0]
    pred = np.where(fluid, scale * y, 0.0)
    nfl = norm if norm is not None else max(int(fluid.sum()), 1)
    d = np.where(fluid, (pred - target) / scale, 0.0)
    loss = float((d * d).sum() / nfl)
    gy = 2.0 * d / nfl
    G = {"head.w": np.einsum("ijk,ijkc->c", gy, u1), "head.b": np.array([gy.sum()])}
    g = q(gy[..., None] * W["head.w"])

    def bw(name, g):
        x, z = A[name]
        gz = g * (z > 0)
        dx, dw, db = conv3_grad(x, W[name + ".w"], gz)
        G[name + ".w"], G[name + ".b"] = dw, db
        return q(dx)

    g = bw("u1b", g)
    g_e1 = g.copy()
    g = q(up_grad(bw("u1a", g)))
    g = bw("u2b", g)
    g_e2 = g.copy()
    g = q(up_grad(bw("u2a", g)))
    g = bw("u3b", g)
    g_e3 = g.copy()
    g = q(up_grad(bw("u3a", g)))
    g = bw("bta", bw("btb", g))
    g = bw("e3a", bw("e3b", q(g_e3 + pool_grad(g))))
    g = bw("e2a", bw("e2b", q(g_e2 + pool_grad(g))))
    bw("e1a", bw("e1b", q(g_e1 + pool_grad(g))))
    return pred, loss, G
