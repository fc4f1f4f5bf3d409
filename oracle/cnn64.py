"""FP64 numpy restatement of the warm-start network (gpair_b200/warmstart.py):
forward pass, loss and the analytic gradient of every parameter.

TEST INFRASTRUCTURE ONLY: the checker of the CUDA training and inference
kernels (gpair_b200/csrc/warmstart_cnn.cu). The reference has no learned
component, so this oracle restates the library's own network definition.
3x3 weights are rounded to bfloat16 first (round to nearest even), as the
CUDA path uses them; everything else is FP64.
"""
from __future__ import annotations

import numpy as np

from gpair_b200.warmstart import HEAD_C, LAYERS, param_layout


def bf16_round(x: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def unpack(params: np.ndarray, round_bf16: bool = True) -> dict:
    out = {}
    shapes = {name: (cin, cout) for name, cin, cout in LAYERS}
    for name, off, n in param_layout():
        v = np.asarray(params[off:off + n], np.float32)
        lname, kind = name.split(".")
        if lname != "head" and kind == "w":
            cin, cout = shapes[lname]
            v = (bf16_round(v) if round_bf16 else v).reshape(cout, cin, 3, 3)
        out[name] = v.astype(np.float64)
    return out


def conv3(x, w, b, skip=None, relu=True):
    B, Cin, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    y = np.zeros((B, w.shape[0], H, W))
    for ky in range(3):
        for kx in range(3):
            y += np.einsum("oc,bchw->bohw", w[:, :, ky, kx], xp[:, :, ky:ky + H, kx:kx + W])
    y += b[None, :, None, None]
    if skip is not None:
        y += skip
    return np.maximum(y, 0.0) if relu else y


def conv3_bwd(x, w, gy):
    """gy: gradient of the pre-activation. Returns (gx, gw, gb)."""
    B, Cin, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    gw = np.zeros_like(w)
    gxp = np.zeros_like(xp)
    for ky in range(3):
        for kx in range(3):
            gw[:, :, ky, kx] = np.einsum("bohw,bchw->oc", gy, xp[:, :, ky:ky + H, kx:kx + W])
            gxp[:, :, ky:ky + H, kx:kx + W] += np.einsum("oc,bohw->bchw", w[:, :, ky, kx], gy)
    return gxp[:, :, 1:-1, 1:-1], gw, gy.sum(axis=(0, 2, 3))


def pool(x):
    B, C, H, W = x.shape
    return x.reshape(B, C, H // 2, 2, W // 2, 2).mean(axis=(3, 5))


def pool_bwd(g):
    return np.repeat(np.repeat(g, 2, axis=2), 2, axis=3) * 0.25


def up(x):
    return np.repeat(np.repeat(x, 2, axis=2), 2, axis=3)


def up_bwd(g):
    B, C, H, W = g.shape
    return g.reshape(B, C, H // 2, 2, W // 2, 2).sum(axis=(3, 5))


def softplus(z):
    return np.where(z > 20, z, np.log1p(np.exp(np.minimum(z, 20))))


def forward(P: dict, x: np.ndarray):
    a = {"x": x}

    def c(name, inp, skip=None):
        return conv3(inp, P[name + ".w"], P[name + ".b"], skip)

    a["e1a"] = c("e1a", x)
    a["e1"] = c("e1b", a["e1a"])
    a["p1"] = pool(a["e1"])
    a["e2a"] = c("e2a", a["p1"])
    a["e2"] = c("e2b", a["e2a"])
    a["p2"] = pool(a["e2"])
    a["e3a"] = c("e3a", a["p2"])
    a["e3"] = c("e3b", a["e3a"])
    a["p3"] = pool(a["e3"])
    a["e4a"] = c("e4a", a["p3"])
    a["e4"] = c("e4b", a["e4a"])
    a["u3"] = up(a["e4"])
    a["s3"] = c("d3a", a["u3"], a["e3"])
    a["d3"] = c("d3b", a["s3"])
    a["u2"] = up(a["d3"])
    a["s2"] = c("d2a", a["u2"], a["e2"])
    a["d2"] = c("d2b", a["s2"])
    a["u1"] = up(a["d2"])
    a["s1"] = c("d1a", a["u1"], a["e1"])
    a["d1"] = c("d1b", a["s1"])
    B, _, H, W = x.shape
    z = np.einsum("c,bchw->bhw", P["head.w"], a["d1"]).reshape(B, -1) + P["head.b"][0]
    sp = softplus(z)
    S = sp.sum(axis=1, keepdims=True)
    a["z"], a["S"], a["out"] = z, S, sp / S
    return a["out"], a


def loss(out, target, mode=1):
    """Batch mean of the per-image loss: mode 0 npix sum (out - t)^2, mode 1 sum (out - t)^2 / sum t^2."""
    HW = out.shape[1]
    e2 = np.sum((out - target) ** 2, axis=1)
    return float(np.mean(HW * e2 if mode == 0 else e2 / np.sum(target ** 2, axis=1)))


def backward(P: dict, a: dict, target: np.ndarray, mode=1) -> dict:
    """Gradient of loss(out, target, mode) with respect to every parameter block."""
    G = {}
    out, z, S = a["out"], a["z"], a["S"]
    B, HW = out.shape
    if mode == 0:
        gout = 2.0 * HW * (out - target) / B
    else:
        gout = 2.0 * (out - target) / np.sum(target ** 2, axis=1, keepdims=True) / B
    dot = np.sum(gout * out, axis=1, keepdims=True)
    gz = (gout - dot) / S / (1.0 + np.exp(-z))
    _, _, H, W = a["x"].shape
    gz4 = gz.reshape(B, H, W)
    G["head.w"] = np.einsum("bhw,bchw->c", gz4, a["d1"])
    G["head.b"] = np.array([gz.sum()])
    gd1 = P["head.w"][None, :, None, None] * gz4[:, None]

    def cb(name, xin, yout, gy):
        gy = gy * (yout > 0)
        gx, gw, gb = conv3_bwd(xin, P[name + ".w"], gy)
        G[name + ".w"], G[name + ".b"] = gw, gb
        return gx, gy

    gs1, _ = cb("d1b", a["s1"], a["d1"], gd1)
    gu1, ge1 = cb("d1a", a["u1"], a["s1"], gs1)
    gd2 = up_bwd(gu1)
    gs2, _ = cb("d2b", a["s2"], a["d2"], gd2)
    gu2, ge2 = cb("d2a", a["u2"], a["s2"], gs2)
    gd3 = up_bwd(gu2)
    gs3, _ = cb("d3b", a["s3"], a["d3"], gd3)
    gu3, ge3 = cb("d3a", a["u3"], a["s3"], gs3)
    ge4 = up_bwd(gu3)
    ge4a, _ = cb("e4b", a["e4a"], a["e4"], ge4)
    gp3, _ = cb("e4a", a["p3"], a["e4a"], ge4a)
    ge3 = ge3 + pool_bwd(gp3)
    ge3a, _ = cb("e3b", a["e3a"], a["e3"], ge3)
    gp2, _ = cb("e3a", a["p2"], a["e3a"], ge3a)
    ge2 = ge2 + pool_bwd(gp2)
    ge2a, _ = cb("e2b", a["e2a"], a["e2"], ge2)
    gp1, _ = cb("e2a", a["p1"], a["e2a"], ge2a)
    ge1 = ge1 + pool_bwd(gp1)
    ge1a, _ = cb("e1b", a["e1a"], a["e1"], ge1)
    cb("e1a", a["x"], a["e1a"], ge1a)
    return G


def flat_grad(G: dict) -> np.ndarray:
    from gpair_b200.warmstart import n_params
    g = np.zeros(n_params())
    for name, off, n in param_layout():
        g[off:off + n] = np.asarray(G[name]).ravel()
    return g


assert HEAD_C == 16
