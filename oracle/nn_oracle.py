"""FP64 CPU restatement of the control-variate surrogate network's kernels.

TEST INFRASTRUCTURE ONLY: tests/ use it to check the forward values and the
gradients of the CUDA kernels (jmultislicelib_b200/csrc/jms_nn.cu); the
product never calls it.  Same definitions as the kernels: 3x3 convolutions
of stride 2 and padding 1 with ReLU, activations [B][C][H][W], weights
[Co][Ci][3][3], a global average pool and a linear layer, mean squared error.
BF16 storage is emulated where the kernels store BF16 (round to nearest even).
"""
from __future__ import annotations

import numpy as np


def bf16_round(a) -> np.ndarray:
    """float -> nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def conv_fwd(x, w, b, relu=True):
    """y = relu(b + conv3x3_s2_p1(x, w)) in FP64 (x, w as given)."""
    B, Ci, H, W = x.shape
    Co = w.shape[0]
    Ho, Wo = H // 2, W // 2
    xp = np.zeros((B, Ci, H + 2, W + 2))
    xp[:, :, 1:H + 1, 1:W + 1] = x
    y = np.broadcast_to(np.asarray(b, np.float64)[None, :, None, None], (B, Co, Ho, Wo)).copy()
    for ky in range(3):
        for kx in range(3):
            y += np.einsum("bchw,oc->bohw", xp[:, :, ky:ky + 2 * Ho:2, kx:kx + 2 * Wo:2], w[:, :, ky, kx])
    return np.maximum(y, 0.0) if relu else y


def conv_bwd(x, w, y, dy, relu=True):
    """(dx, dw, db) of conv_fwd from dL/dy taken before the ReLU mask y > 0."""
    B, Ci, H, W = x.shape
    Ho, Wo = H // 2, W // 2
    g = dy * (y > 0) if relu else dy
    xp = np.zeros((B, Ci, H + 2, W + 2))
    xp[:, :, 1:H + 1, 1:W + 1] = x
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w, dtype=np.float64)
    for ky in range(3):
        for kx in range(3):
            sl = (slice(None), slice(None), slice(ky, ky + 2 * Ho, 2), slice(kx, kx + 2 * Wo, 2))
            dxp[sl] += np.einsum("bohw,oc->bchw", g, w[:, :, ky, kx])
            dw[:, :, ky, kx] = np.einsum("bohw,bchw->oc", g, xp[sl])
    return dxp[:, :, 1:H + 1, 1:W + 1], dw, g.sum(axis=(0, 2, 3))


def pool_linear_fwd(h, wl, bl):
    return h.mean(axis=(2, 3)) @ wl.T + bl


def pool_linear_bwd(h, wl, dout):
    B, C, Hh, Ww = h.shape
    pooled = h.mean(axis=(2, 3))
    dh = np.broadcast_to((dout @ wl)[:, :, None, None] / (Hh * Ww), h.shape).copy()
    return dh, dout.T @ pooled, dout.sum(axis=0)


def mse(out, t):
    d = out - t
    return float((d * d).mean()), 2.0 * d / d.size
