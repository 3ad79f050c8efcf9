"""CPU oracle of the warm-start U-Net (test infrastructure only).

A numpy restatement of every layer the BF16 kernels in
smili_b200/csrc/unet.cu compute, and of the whole network's forward and
backward pass, used to check the GPU gradients.  Arrays are NHWC; weights are
[Cout][3][3][Cin].  ``bf16`` rounds float32 values to bfloat16 (round to
nearest even), which is where the GPU stores activations, gradients and
weights; the contractions here accumulate in float64 (the GPU accumulates in
float32).  The U-Net has no reference counterpart, so this oracle is pinned
by finite differences of its own backward pass (tests/test_unet.py).
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


# ------------------------------------------------------------------ layers
def conv3x3(x, w, b=None, relu=False):
    """y[n,h,w,o] = sum_{ky,kx,c} x[n,h+ky-1,w+kx-1,c] w[o,ky,kx,c] (+ b[o])."""
    N, H, W, _ = x.shape
    xp = np.pad(np.asarray(x, np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
    w = np.asarray(w, np.float64)
    y = np.zeros((N, H, W, w.shape[0]))
    for ky in range(3):
        for kx in range(3):
            y += np.einsum("nhwc,oc->nhwo", xp[:, ky:ky + H, kx:kx + W, :], w[:, ky, kx, :], optimize=True)
    if b is not None:
        y += np.asarray(b, np.float64)
    return np.maximum(y, 0.0) if relu else y


def conv3x3_dgrad(dy, w):
    """Gradient of conv3x3 with respect to its input."""
    N, H, W, _ = dy.shape
    dyp = np.pad(np.asarray(dy, np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
    w = np.asarray(w, np.float64)
    dx = np.zeros((N, H, W, w.shape[3]))
    for ky in range(3):
        for kx in range(3):
            dx += np.einsum("nhwo,oc->nhwc", dyp[:, 2 - ky:2 - ky + H, 2 - kx:2 - kx + W, :], w[:, ky, kx, :],
                            optimize=True)
    return dx


def conv3x3_wgrad(x, dy):
    """dw[o,ky,kx,c] = sum_{n,h,w} dy[n,h,w,o] x[n,h+ky-1,w+kx-1,c]."""
    N, H, W, C = x.shape
    xp = np.pad(np.asarray(x, np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
    dy = np.asarray(dy, np.float64)
    dw = np.zeros((dy.shape[3], 3, 3, C))
    for ky in range(3):
        for kx in range(3):
            dw[:, ky, kx, :] = np.einsum("nhwo,nhwc->oc", dy, xp[:, ky:ky + H, kx:kx + W, :], optimize=True)
    return dw


def flip_weights(w):
    """wt[c,ky,kx,o] = w[o,2-ky,2-kx,c]: conv3x3(dy, wt) == conv3x3_dgrad(dy, w)."""
    return np.ascontiguousarray(np.transpose(w[:, ::-1, ::-1, :], (3, 1, 2, 0)))


def avgpool2(x):
    N, H, W, C = x.shape
    return np.asarray(x, np.float64).reshape(N, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def avgpool2_bwd(dy):
    return 0.25 * np.repeat(np.repeat(np.asarray(dy, np.float64), 2, axis=1), 2, axis=2)


def upsample2(x):
    return np.repeat(np.repeat(np.asarray(x, np.float64), 2, axis=1), 2, axis=2)


def upsample2_bwd(dy):
    N, H, W, C = dy.shape
    return np.asarray(dy, np.float64).reshape(N, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def mse(y, t):
    """loss = sum (y - t)^2 and dy = 2 (y - t) / n (the kernel's convention)."""
    r = np.asarray(y, np.float64) - np.asarray(t, np.float64)
    return float(np.sum(r * r)), 2.0 * r / r.size


def adam(w, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    upd = (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w * (1 - lr * wd) - lr * upd, m, v


# ------------------------------------------------------------------ network
def unet_layers(c=(24, 48, 96, 192), cin=1, cout=1):
    """(name, Cin, Cout, relu) of every 3x3 convolution, in forward order."""
    c1, c2, c3, c4 = c
    return [("e1a", cin, c1, True), ("e1b", c1, c1, True),
            ("e2a", c1, c2, True), ("e2b", c2, c2, True),
            ("e3a", c2, c3, True), ("e3b", c3, c3, True),
            ("ba", c3, c4, True), ("bb", c4, c4, True),
            ("d3a", c4 + c3, c3, True), ("d3b", c3, c3, True),
            ("d2a", c3 + c2, c2, True), ("d2b", c2, c2, True),
            ("d1a", c2 + c1, c1, True), ("d1b", c1, c1, True),
            ("head", c1, cout, False)]


def unet_forward(params, x, rnd=bf16):
    """Forward pass; returns (output, activations).  ``rnd`` is applied where
    the GPU stores a tensor (bf16), or the identity for an exact float64 pass."""
    P = params
    A = {"x": rnd(x)}

    def conv(name, inp, relu=True):
        w, b = P[name]
        return rnd(conv3x3(inp, w, b, relu))

    A["e1a"] = conv("e1a", A["x"]); A["e1b"] = conv("e1b", A["e1a"])
    A["p1"] = rnd(avgpool2(A["e1b"]))
    A["e2a"] = conv("e2a", A["p1"]); A["e2b"] = conv("e2b", A["e2a"])
    A["p2"] = rnd(avgpool2(A["e2b"]))
    A["e3a"] = conv("e3a", A["p2"]); A["e3b"] = conv("e3b", A["e3a"])
    A["p3"] = rnd(avgpool2(A["e3b"]))
    A["ba"] = conv("ba", A["p3"]); A["bb"] = conv("bb", A["ba"])
    A["cat3"] = np.concatenate([upsample2(A["bb"]), A["e3b"]], axis=3)
    A["d3a"] = conv("d3a", A["cat3"]); A["d3b"] = conv("d3b", A["d3a"])
    A["cat2"] = np.concatenate([upsample2(A["d3b"]), A["e2b"]], axis=3)
    A["d2a"] = conv("d2a", A["cat2"]); A["d2b"] = conv("d2b", A["d2a"])
    A["cat1"] = np.concatenate([upsample2(A["d2b"]), A["e1b"]], axis=3)
    A["d1a"] = conv("d1a", A["cat1"]); A["d1b"] = conv("d1b", A["d1a"])
    A["out"] = conv("head", A["d1b"], relu=False)
    return A["out"], A


def unet_backward(params, A, dout, rnd=bf16):
    """Gradients of every (w, b) given the output gradient, in the order and
    with the storage rounding of the GPU backward pass."""
    P = params
    G = {}

    def back(name, inp_key, dy, out_key=None, need_dx=True):
        """conv layer backward: mask by the layer's ReLU output, then dw, db, dx."""
        w, _ = P[name]
        if out_key is not None:
            dy = np.where(A[out_key] > 0, dy, 0.0)
        dy = rnd(dy)
        G[name] = (conv3x3_wgrad(A[inp_key], dy), dy.sum(axis=(0, 1, 2)))
        return rnd(conv3x3_dgrad(dy, w)) if need_dx else None

    c1 = P["e1b"][0].shape[0]
    c2 = P["e2b"][0].shape[0]
    c3 = P["e3b"][0].shape[0]
    d = back("head", "d1b", dout)
    d = back("d1b", "d1a", d, "d1b")
    dcat1 = back("d1a", "cat1", d, "d1a")
    d = rnd(upsample2_bwd(dcat1[..., :c2]))
    d = back("d2b", "d2a", d, "d2b")
    dcat2 = back("d2a", "cat2", d, "d2a")
    d = rnd(upsample2_bwd(dcat2[..., :c3]))
    d = back("d3b", "d3a", d, "d3b")
    dcat3 = back("d3a", "cat3", d, "d3a")
    d = rnd(upsample2_bwd(dcat3[..., :dcat3.shape[3] - c3]))
    d = back("bb", "ba", d, "bb")
    dp3 = back("ba", "p3", d, "ba")
    de3b = rnd(dcat3[..., dcat3.shape[3] - c3:] + avgpool2_bwd(dp3))
    d = back("e3b", "e3a", de3b, "e3b")
    dp2 = back("e3a", "p2", d, "e3a")
    de2b = rnd(dcat2[..., dcat2.shape[3] - c2:] + avgpool2_bwd(dp2))
    d = back("e2b", "e2a", de2b, "e2b")
    dp1 = back("e2a", "p1", d, "e2a")
    de1b = rnd(dcat1[..., dcat1.shape[3] - c1:] + avgpool2_bwd(dp1))
    d = back("e1b", "e1a", de1b, "e1b")
    back("e1a", "x", d, "e1a", need_dx=False)
    return G


def init_params(rng, c=(24, 48, 96, 192), cin=1, cout=1):
    """He-normal weights (bf16-representable), zero biases."""
    P = {}
    for name, ci, co, relu in unet_layers(c, cin, cout):
        std = np.sqrt(2.0 / (9 * ci)) * (1.0 if relu else 0.1)
        P[name] = (bf16(rng.standard_normal((co, 3, 3, ci)) * std), np.zeros(co, np.float32))
    return P
