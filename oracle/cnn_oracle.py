"""CPU restatement of the warm-start network (test infrastructure only).

FP64 numpy forward and backward passes of the 4-layer 3x3x3 network that
am-cfd_b200/csrc/k_cnn.cu runs on the tensor cores, with the same parameter
layout (per layer W[27][cout][cin] then b[cout]; tap = 9(dk+1) + 3(dj+1) +
(di+1)), the same zero-padding rule (activations held at zero on boundary
nodes) and the same points of BF16 rounding (input features, packed weights,
every stored activation and stored gradient), so that the GPU kernels can be
checked to BF16 accuracy.  The network has no counterpart in the reference;
this file is the checker for its gradients.
"""
from __future__ import annotations

import numpy as np

CIN = (16, 32, 32, 32)
COUT = (32, 32, 32, 16)
NFEAT, NOUT = 11, 2


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def layer_slices():
    out, o = [], 0
    for ci, co in zip(CIN, COUT):
        nw = 27 * co * ci
        out.append((slice(o, o + nw), slice(o + nw, o + nw + co)))
        o += nw + co
    return out


def param_count():
    return sum(27 * ci * co + co for ci, co in zip(CIN, COUT))


def interior_mask(ni, nj, nk):
    m = np.zeros((nk, nj, ni), dtype=bool)
    m[1:-1, 1:-1, 1:-1] = True
    return m.reshape(-1)


def offsets(ni, nj):
    return [dk * ni * nj + dj * ni + di for dk in (-1, 0, 1) for dj in (-1, 0, 1) for di in (-1, 0, 1)]


def shift(x, off):
    """y[c] = x[c + off] (zero outside [0, ncell))."""
    n = x.shape[0]
    y = np.zeros_like(x)
    if off >= 0:
        y[: n - off] = x[off:]
    else:
        y[-off:] = x[: n + off]
    return y


def conv(x, w, offs):
    """z[c][co] = sum_t sum_ci x[c + off_t][ci] w[t][co][ci]."""
    z = np.zeros((x.shape[0], w.shape[1]))
    for t, off in enumerate(offs):
        z += shift(x, off) @ w[t].T
    return z


def forward(params, feat, dims):
    """Returns (y [ncell][2], activations list) for features [ncell][11]."""
    ni, nj, nk = dims
    offs = offsets(ni, nj)
    inner = interior_mask(ni, nj, nk)[:, None]
    x = np.zeros((feat.shape[0], 16))
    x[:, :NFEAT] = feat
    x = bf16(x) * inner
    acts = [x]
    y = None
    for l, (ws, bs) in enumerate(layer_slices()):
        w = bf16(params[ws]).reshape(27, COUT[l], CIN[l])
        z = conv(acts[-1], w, offs) + params[bs][None, :].astype(np.float64)
        if l < 3:
            z = np.maximum(z, 0.0)
        z = z * inner
        if l == 3:
            y = z[:, :NOUT].copy()
        acts.append(bf16(z))
    return y, acts


def backward(params, acts, y, target, dims):
    """MSE over interior cells and the 2 outputs; returns (loss, grads)."""
    ni, nj, nk = dims
    offs = offsets(ni, nj)
    inner = interior_mask(ni, nj, nk)
    nint = inner.sum() * NOUT
    d = (y - target) * inner[:, None]
    loss = float((d ** 2).sum() / nint)
    dz = np.zeros((y.shape[0], COUT[3]))
    dz[:, :NOUT] = 2.0 * d / nint
    dz = bf16(dz)
    grads = np.zeros(param_count())
    sl = layer_slices()
    for l in range(3, -1, -1):
        ws, bs = sl[l]
        x = acts[l]
        gw = np.zeros((27, COUT[l], CIN[l]))
        for t, off in enumerate(offs):
            gw[t] = dz.T @ shift(x, off)
        grads[ws] = gw.reshape(-1)
        grads[bs] = dz.sum(axis=0)
        if l > 0:
            w = bf16(params[ws]).reshape(27, COUT[l], CIN[l])
            dx = np.zeros((x.shape[0], CIN[l]))
            for t, off in enumerate(offs):
                dx += shift(dz @ w[t], -off)
            dx = dx * (acts[l] > 0) * inner[:, None]
            dz = bf16(dx)
    return loss, grads
