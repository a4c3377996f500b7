"""CPU oracle of the learned network (test infrastructure only).

Float64 numpy restatement of the network in pincflow.jl_b200/csrc/pcf_net.cu
(forward, residual-weighted loss, backward), used to check the GPU kernels'
outputs and gradients.  With bf=True it rounds to BF16 exactly where the
GPU stores BF16 (the gathered input, the activations and the convolution
windows that feed the tensor cores, the weight copies and the upstream
gradients); with bf=False it is the exact float64 network, whose analytic
gradient tests/test_oracle_kat.py pins against finite differences.

The network, per column c of the nx x ny grid (x = the column resampled to
L = 64 levels), with periodic 3 x 3 windows im2col(v)[c] = (v[nbr(c, t)])_t:
    a  = relu(C1 im2col(x) + c1)        64     C1: 64 x (9 * 64)
    h1 = relu(W1 a + b1)                256
    h2 = relu(W2 h1 + b2)               256
    z  = W3 h2 + b3                     64
    y  = z + C2 im2col(z) + c2          64     C2: 64 x (9 * 64)
Tap t = (dj + 1) * 3 + (di + 1) is the neighbour (i + di, j + dj).

The network has no counterpart in the reference; its oracle is written from
the architecture, not from reference code.
"""
from __future__ import annotations

import numpy as np

L, HID, TAPS = 64, 256, 9
KC = TAPS * L  # 576: the im2col width
SIZES = [("C1", (L, KC)), ("c1", (L,)), ("W1", (HID, L)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
         ("W3", (L, HID)), ("b3", (L,)), ("C2", (L, KC)), ("c2", (L,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)
BIASES = ("c1", "b1", "b2", "b3", "c2")


def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SIZES])


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _interp_weights(n_in, n_out):
    l = np.arange(n_out)
    if n_in == n_out:
        return l, l, np.zeros(n_out)
    pos = (l + 0.5) * n_in / n_out - 0.5
    pos = np.clip(pos.astype(np.float32), 0, n_in - 1).astype(np.float64)
    k0 = np.floor(pos).astype(int)
    k1 = np.minimum(k0 + 1, n_in - 1)
    return k0, k1, (pos - k0)


def gather(field):
    """(nz, ny, nx) field -> (C, L) columns resampled to L levels."""
    nz, ny, nx = field.shape
    cols = field.reshape(nz, ny * nx).T
    k0, k1, f = _interp_weights(nz, L)
    return (1 - f) * cols[:, k0] + f * cols[:, k1]


def scatter(Y, nz, ny, nx):
    l0, l1, f = _interp_weights(L, nz)
    cols = (1 - f) * Y[:, l0] + f * Y[:, l1]
    return cols.T.reshape(nz, ny, nx)


def _shift(H, ny, nx, tap):
    """H[nbr(c, tap)] for all c (periodic)."""
    di, dj = tap % 3 - 1, tap // 3 - 1
    G = H.reshape(ny, nx, -1)
    return np.roll(np.roll(G, -dj, axis=0), -di, axis=1).reshape(ny * nx, -1)


def im2col(H, ny, nx):
    return np.concatenate([_shift(H, ny, nx, t) for t in range(TAPS)], axis=1)


def col2im(D, ny, nx):
    """Adjoint of im2col: sum over taps of the window gradients sent back to
    the columns they were read from."""
    F = D.shape[1] // TAPS
    return sum(_shift(D[:, t * F:(t + 1) * F], ny, nx, TAPS - 1 - t) for t in range(TAPS))


def forward(p, b, bf=True):
    P = unpack(p)
    nz, ny, nx = b.shape
    r = bf16 if bf else (lambda x: np.asarray(x, dtype=np.float64))
    C1, W1, W2, W3, C2 = r(P["C1"]), r(P["W1"]), r(P["W2"]), r(P["W3"]), r(P["C2"])
    x0 = r(gather(b))
    xi = im2col(x0, ny, nx)
    a = r(np.maximum(xi @ C1.T + P["c1"], 0))
    h1 = r(np.maximum(a @ W1.T + P["b1"], 0))
    h2 = r(np.maximum(h1 @ W2.T + P["b2"], 0))
    z = r(h2 @ W3.T + P["b3"])
    zi = im2col(z, ny, nx)
    y = z + zi @ C2.T + P["c2"]
    cache = dict(x0=x0, xi=xi, a=a, h1=h1, h2=h2, z=z, zi=zi, y=y, C1=C1, W1=W1, W2=W2, W3=W3, C2=C2,
                 shape=(nz, ny, nx))
    return scatter(y, nz, ny, nx), cache


def loss_and_grad(p, b, x, bf=True):
    """Residual-weighted loss sum (y - t)^2 / sum t^2 on the L-level columns and
    its gradient with respect to the packed parameters (BF16 roundings are
    passed through unchanged by the gradient)."""
    r = bf16 if bf else (lambda v: np.asarray(v, dtype=np.float64))
    _, c = forward(p, b, bf)
    nz, ny, nx = c["shape"]
    t = gather(x).astype(np.float32).astype(np.float64) if bf else gather(x)
    d = c["y"] - t
    st2 = np.sum(t * t)
    loss = np.sum(d * d) / st2
    dy = 2 * d / st2
    dyb = r(dy)
    g = {}
    g["c2"] = dy.sum(0)
    g["C2"] = dyb.T @ c["zi"]
    dz = dy + col2im(dyb @ c["C2"], ny, nx)
    dzb = r(dz)
    g["b3"] = dz.sum(0)
    g["W3"] = dzb.T @ c["h2"]
    dg2 = (dzb @ c["W3"]) * (c["h2"] > 0)
    dg2b = r(dg2)
    g["b2"] = dg2.sum(0)
    g["W2"] = dg2b.T @ c["h1"]
    dg1 = (dg2b @ c["W2"]) * (c["h1"] > 0)
    dg1b = r(dg1)
    g["b1"] = dg1.sum(0)
    g["W1"] = dg1b.T @ c["a"]
    dga = (dg1b @ c["W1"]) * (c["a"] > 0)
    dgab = r(dga)
    g["c1"] = dga.sum(0)
    g["C1"] = dgab.T @ c["xi"]
    return loss, pack(g)
