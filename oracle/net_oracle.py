"""CPU oracle of the learned warm-start network (test infrastructure only).

Float64 numpy restatement of the network in pincflow.jl_b200/csrc/pcf_net.cu
(forward, residual-weighted loss, backward), used to check the GPU kernels'
outputs and gradients.  With bf16=True it rounds to BF16 exactly where the
GPU stores BF16 (inputs and activations that feed the tensor-core GEMMs, the
weight copies and the upstream gradients dY, dZ); with bf16=False it is the
exact float64 network, whose analytic gradient tests/test_oracle_kat.py
pins against finite differences.

The network has no counterpart in the reference; its oracle is written from
the architecture, not from reference code.
"""
from __future__ import annotations

import numpy as np

L, HID, TAPS = 64, 256, 9
SIZES = [("W1", (HID, L)), ("b1", (HID,)), ("K1", (HID, TAPS)), ("W2", (HID, HID)), ("b2", (HID,)),
         ("K2", (HID, TAPS)), ("W3", (L, HID)), ("b3", (L,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


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


def conv(H, K, ny, nx):
    return H + sum(K[:, t][None, :] * _shift(H, ny, nx, t) for t in range(TAPS))


def forward(p, b, bf=True):
    P = unpack(p)
    nz, ny, nx = b.shape
    r = bf16 if bf else (lambda x: np.asarray(x, dtype=np.float64))
    W1, W2, W3 = r(P["W1"]), r(P["W2"]), r(P["W3"])
    x0 = r(gather(b))
    h1 = r(np.maximum(x0 @ W1.T + P["b1"], 0))
    h1c = r(conv(h1, P["K1"], ny, nx))
    h2 = r(np.maximum(h1c @ W2.T + P["b2"], 0))
    h2c = r(conv(h2, P["K2"], ny, nx))
    y = h2c @ W3.T + P["b3"]
    cache = dict(x0=x0, h1=h1, h1c=h1c, h2=h2, h2c=h2c, y=y, W1=W1, W2=W2, W3=W3, shape=(nz, ny, nx))
    return scatter(y, nz, ny, nx), cache


def loss_and_grad(p, b, x, bf=True):
    """Residual-weighted loss sum (y - t)^2 / sum t^2 on the L-level columns and
    its gradient with respect to the packed parameters."""
    P = unpack(p)
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
    g["b3"] = dy.sum(0)
    g["W3"] = dyb.T @ c["h2c"]
    dh2c = dyb @ c["W3"]

    def conv_bwd(dhc, h, K):
        dh = dhc + sum(K[:, TAPS - 1 - t][None, :] * _shift(dhc, ny, nx, t) for t in range(TAPS))
        dK = np.stack([np.sum(dhc * _shift(h, ny, nx, t), axis=0) for t in range(TAPS)], axis=1)
        dz = dh * (h > 0)
        return dz, dK

    dz2, g["K2"] = conv_bwd(dh2c, c["h2"], P["K2"])
    g["b2"] = dz2.sum(0)
    dz2b = r(dz2)
    g["W2"] = dz2b.T @ c["h1c"]
    dh1c = dz2b @ c["W2"]
    dz1, g["K1"] = conv_bwd(dh1c, c["h1"], P["K1"])
    g["b1"] = dz1.sum(0)
    dz1b = r(dz1)
    g["W1"] = dz1b.T @ c["x0"]
    return loss, pack(g)
