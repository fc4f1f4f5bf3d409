"""Learned warm start for CG: a small convolutional encoder/decoder that maps
feature maps of a problem (dirty images and the gridded uv density) to a
positive, unit-flux start image.

The reference has no learned component; CG from the flat prior stays the
fallback. Everything that computes runs in the library's own CUDA kernels
(csrc/warmstart_cnn.cu) through the C ABI; torch only holds device memory and
supplies the stream.

Network (channels 16-32-64-128, 3x3 convolutions, ReLU, BF16 weights with
FP32 accumulation):

    x [4,H,W] -> e1 (2 convs, 16) -> pool -> e2 (32) -> pool -> e3 (64) -> pool -> e4 (128)
    e4 -> up -> conv 64 + e3 -> conv 64 -> up -> conv 32 + e2 -> conv 32
       -> up -> conv 16 + e1 -> conv 16 -> 1x1 conv -> softplus -> / sum

H and W must be multiples of 8.

Inputs of one problem (:func:`features`), each scaled to max |value| 1:
  channel 0  dirty image: -d chi2 / dI at the flat start image (the adjoint
             DFT of the residuals, the library's own gradient path);
  channel 1  V2 dirty map: the adjoint DFT of the V2 data, sum_k V2_k
             cos(phase_k(x - N/2, y - N/2)) -- the image's autocorrelation as
             the uv coverage samples it, centred (gpair_adjoint_image);
  channel 2  uv density: the (u, v) points and their conjugates gridded on the
             image's Fourier grid (cell = u * pixel size * N), log(1 + count),
             zero frequency at the centre;
  channel 3  probe gradient: -d chi2 / dI at a centred Gaussian of FWHM N/4
             pixels with the prior's flux. Its visibilities are non-zero on
             every baseline, so the closure-phase residuals reach the gradient
             (at the flat image they nearly vanish).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from . import api
from .synth import ArrayConfig, Component, Scene, make_oifits

RPMAS = (math.pi / 180.0) / 3600000.0
N_FEATURES = 4
LAYERS: Tuple[Tuple[str, int, int], ...] = (
    ("e1a", N_FEATURES, 16), ("e1b", 16, 16), ("e2a", 16, 32), ("e2b", 32, 32), ("e3a", 32, 64), ("e3b", 64, 64),
    ("e4a", 64, 128), ("e4b", 128, 128), ("d3a", 128, 64), ("d3b", 64, 64), ("d2a", 64, 32), ("d2b", 32, 32),
    ("d1a", 32, 16), ("d1b", 16, 16))
HEAD_C = 16
LOSS_ABSOLUTE, LOSS_RELATIVE = 0, 1
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_cnn.npz")


def _declare(L):
    if getattr(L, "_cnn_declared", False):
        return
    vp, i, f, ll = C.c_void_p, C.c_int, C.c_float, C.c_longlong
    L.gpair_cnn_conv3x3.argtypes = [vp, vp, vp, vp, vp, i, i, i, i, i, i, vp]
    L.gpair_cnn_conv3x3_bwd_data.argtypes = [vp, vp, vp, i, i, i, i, i, i, vp]
    L.gpair_cnn_conv3x3_bwd_weight.argtypes = [vp, vp, vp, vp, vp, ll, i, i, i, i, i, vp]
    L.gpair_cnn_relu_mask.argtypes = [vp, vp, ll, vp]
    L.gpair_cnn_pool2.argtypes = [vp, vp, ll, i, i, vp]
    L.gpair_cnn_pool2_bwd.argtypes = [vp, vp, ll, i, i, i, vp]
    L.gpair_cnn_up2.argtypes = [vp, vp, ll, i, i, vp]
    L.gpair_cnn_up2_bwd.argtypes = [vp, vp, ll, i, i, vp]
    L.gpair_cnn_head.argtypes = [vp, vp, vp, vp, vp, vp, i, i, i, vp]
    L.gpair_cnn_head_bwd.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, i, i, i, vp]
    L.gpair_cnn_mse.argtypes = [vp, vp, vp, vp, i, i, f, i, vp]
    L.gpair_cnn_adam.argtypes = [vp, vp, vp, vp, vp, i, f, f, f, f, i, vp]
    L.gpair_cnn_to_bf16.argtypes = [vp, vp, i, vp]
    L._cnn_declared = True


def _ptr(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


def param_layout() -> List[Tuple[str, int, int]]:
    """(name, offset, count) of every parameter block in the flat FP32 vector."""
    out, off = [], 0
    for name, cin, cout in LAYERS:
        out.append((name + ".w", off, cout * cin * 9))
        off += cout * cin * 9
        out.append((name + ".b", off, cout))
        off += cout
    out.append(("head.w", off, HEAD_C))
    off += HEAD_C
    out.append(("head.b", off, 1))
    off += 1
    return out


def n_params() -> int:
    name, off, n = param_layout()[-1]
    return off + n


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal 3x3 weights, zero biases, small head (FP32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(n_params(), np.float32)
    lay = {name: (off, n) for name, off, n in param_layout()}
    for name, cin, cout in LAYERS:
        off, n = lay[name + ".w"]
        p[off:off + n] = rng.normal(0.0, math.sqrt(2.0 / (cin * 9)), n)
    off, n = lay["head.w"]
    p[off:off + n] = rng.normal(0.0, math.sqrt(1.0 / HEAD_C), n)
    return p


class WarmStartNet:
    """The network on one CUDA device; parameters in one flat FP32 vector (+ its
    BF16 working copy), gradients and Adam moments alike."""

    loss_mode = LOSS_RELATIVE

    def __init__(self, params: Optional[np.ndarray] = None, device: int = 0, seed: int = 0):
        import torch
        self.torch = torch
        self.L = api.lib()
        _declare(self.L)
        self.dev = torch.device("cuda", device)
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        assert p.size == n_params()
        self.p = torch.from_numpy(p.copy()).to(self.dev)
        self.pbf = torch.empty(p.size, dtype=torch.bfloat16, device=self.dev)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step = 0
        self.lay = {name: (off, n) for name, off, n in param_layout()}
        self._scratch = torch.empty(1 << 22, dtype=torch.float32, device=self.dev)
        self._loss = torch.zeros(4096, dtype=torch.float64, device=self.dev)
        self.sync_bf16()

    # ---------------------------------------------------------------- utils
    @property
    def stream(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def _chk(self, rc):
        if rc != 0:
            raise api.GpairError(f"warm-start kernel failed ({rc})")

    def sync_bf16(self):
        self._chk(self.L.gpair_cnn_to_bf16(self.p.data_ptr(), self.pbf.data_ptr(), self.p.numel(), self.stream))

    def _w(self, name):
        off, n = self.lay[name + ".w"]
        return self.pbf[off:off + n]

    def _b(self, name):
        off, n = self.lay[name + ".b"]
        return self.p[off:off + n]

    def _gw(self, name):
        off, n = self.lay[name + ".w"]
        return self.g[off:off + n]

    def _gb(self, name):
        off, n = self.lay[name + ".b"]
        return self.g[off:off + n]

    def params_numpy(self) -> np.ndarray:
        return self.p.detach().cpu().numpy().copy()

    def save(self, path: str, meta: Optional[dict] = None):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, params=self.params_numpy(), **{k: np.asarray(v) for k, v in (meta or {}).items()})

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, device: int = 0) -> "WarmStartNet":
        with np.load(path) as z:
            return cls(z["params"], device)

    # -------------------------------------------------------------- forward
    def _conv(self, name, x, cin, cout, H, W, skip=None, relu=True):
        B = x.shape[0]
        y = self.torch.empty((B, cout, H, W), dtype=self.torch.float32, device=self.dev)
        self._chk(self.L.gpair_cnn_conv3x3(x.data_ptr(), self._w(name).data_ptr(), self._b(name).data_ptr(),
                                           _ptr(skip), y.data_ptr(), B, cin, cout, H, W, int(relu), self.stream))
        return y

    def _pool(self, x):
        B, Cc, H, W = x.shape
        y = self.torch.empty((B, Cc, H // 2, W // 2), dtype=self.torch.float32, device=self.dev)
        self._chk(self.L.gpair_cnn_pool2(x.data_ptr(), y.data_ptr(), B * Cc, H, W, self.stream))
        return y

    def _up(self, x):
        B, Cc, H, W = x.shape
        y = self.torch.empty((B, Cc, 2 * H, 2 * W), dtype=self.torch.float32, device=self.dev)
        self._chk(self.L.gpair_cnn_up2(x.data_ptr(), y.data_ptr(), B * Cc, H, W, self.stream))
        return y

    def forward(self, x, keep: bool = False):
        """x: float32 [B, N_FEATURES, H, W] on the device -> unit-flux images [B, H, W]."""
        t = self.torch
        x = x.contiguous()
        B, _, H, W = x.shape
        if H % 8 or W % 8:
            raise ValueError("image size must be a multiple of 8")
        a = {"x": x}
        h = [H, H // 2, H // 4, H // 8]
        w = [W, W // 2, W // 4, W // 8]
        a["e1a"] = self._conv("e1a", x, N_FEATURES, 16, h[0], w[0])
        a["e1"] = self._conv("e1b", a["e1a"], 16, 16, h[0], w[0])
        a["p1"] = self._pool(a["e1"])
        a["e2a"] = self._conv("e2a", a["p1"], 16, 32, h[1], w[1])
        a["e2"] = self._conv("e2b", a["e2a"], 32, 32, h[1], w[1])
        a["p2"] = self._pool(a["e2"])
        a["e3a"] = self._conv("e3a", a["p2"], 32, 64, h[2], w[2])
        a["e3"] = self._conv("e3b", a["e3a"], 64, 64, h[2], w[2])
        a["p3"] = self._pool(a["e3"])
        a["e4a"] = self._conv("e4a", a["p3"], 64, 128, h[3], w[3])
        a["e4"] = self._conv("e4b", a["e4a"], 128, 128, h[3], w[3])
        a["u3"] = self._up(a["e4"])
        a["s3"] = self._conv("d3a", a["u3"], 128, 64, h[2], w[2], skip=a["e3"])
        a["d3"] = self._conv("d3b", a["s3"], 64, 64, h[2], w[2])
        a["u2"] = self._up(a["d3"])
        a["s2"] = self._conv("d2a", a["u2"], 64, 32, h[1], w[1], skip=a["e2"])
        a["d2"] = self._conv("d2b", a["s2"], 32, 32, h[1], w[1])
        a["u1"] = self._up(a["d2"])
        a["s1"] = self._conv("d1a", a["u1"], 32, 16, h[0], w[0], skip=a["e1"])
        a["d1"] = self._conv("d1b", a["s1"], 16, 16, h[0], w[0])
        z = t.empty((B, H * W), dtype=t.float32, device=self.dev)
        out = t.empty((B, H * W), dtype=t.float32, device=self.dev)
        asum = t.empty(B, dtype=t.float32, device=self.dev)
        hw_off, _ = self.lay["head.w"]
        hb_off, _ = self.lay["head.b"]
        self._chk(self.L.gpair_cnn_head(a["d1"].data_ptr(), self.p[hw_off:].data_ptr(), self.p[hb_off:].data_ptr(),
                                        z.data_ptr(), out.data_ptr(), asum.data_ptr(), B, HEAD_C, H * W, self.stream))
        a["z"], a["out"], a["asum"] = z, out, asum
        if keep:
            self._acts = a
        return out.view(B, H, W)

    # ------------------------------------------------------------- backward
    def _conv_bwd(self, name, x_in, y_out, gy, cin, cout, H, W, gx=None, accumulate=False, need_gx=True):
        """Backward of y = relu(conv(x) [+ skip]): masks gy in place, writes the
        weight/bias gradients, returns dL/dx (into gx when given)."""
        B = gy.shape[0]
        self._chk(self.L.gpair_cnn_relu_mask(y_out.data_ptr(), gy.data_ptr(), gy.numel(), self.stream))
        self._chk(self.L.gpair_cnn_conv3x3_bwd_weight(x_in.data_ptr(), gy.data_ptr(), self._gw(name).data_ptr(),
                                                      self._gb(name).data_ptr(), self._scratch.data_ptr(),
                                                      self._scratch.numel(), B, cin, cout, H, W, self.stream))
        if not need_gx:
            return None
        if gx is None:
            gx = self.torch.empty((B, cin, H, W), dtype=self.torch.float32, device=self.dev)
            accumulate = False
        self._chk(self.L.gpair_cnn_conv3x3_bwd_data(gy.data_ptr(), self._w(name).data_ptr(), gx.data_ptr(), B, cin,
                                                    cout, H, W, int(accumulate), self.stream))
        return gx

    def _pool_bwd(self, gy, gx, accumulate):
        B, Cc, H, W = gx.shape
        self._chk(self.L.gpair_cnn_pool2_bwd(gy.data_ptr(), gx.data_ptr(), B * Cc, H, W, int(accumulate),
                                             self.stream))

    def _up_bwd(self, gy):
        B, Cc, H2, W2 = gy.shape
        gx = self.torch.empty((B, Cc, H2 // 2, W2 // 2), dtype=self.torch.float32, device=self.dev)
        self._chk(self.L.gpair_cnn_up2_bwd(gy.data_ptr(), gx.data_ptr(), B * Cc, H2 // 2, W2 // 2, self.stream))
        return gx

    def backward(self, gout):
        """gout: dL/d(out) [B, H*W]; fills self.g (every parameter's gradient)."""
        t = self.torch
        a = self._acts
        B, _, H, W = a["x"].shape
        h = [H, H // 2, H // 4, H // 8]
        w = [W, W // 2, W // 4, W // 8]
        gd1 = t.empty_like(a["d1"])
        hw_off, _ = self.lay["head.w"]
        self._chk(self.L.gpair_cnn_head_bwd(a["d1"].data_ptr(), self.p[hw_off:].data_ptr(), a["z"].data_ptr(),
                                            a["out"].data_ptr(), a["asum"].data_ptr(), gout.contiguous().data_ptr(),
                                            gd1.data_ptr(), self.g[hw_off:].data_ptr(), self._scratch.data_ptr(), B,
                                            HEAD_C, H * W, self.stream))
        gs1 = self._conv_bwd("d1b", a["s1"], a["d1"], gd1, 16, 16, h[0], w[0])
        # s1 = relu(conv(u1) + e1): the masked gradient flows to e1 and to conv(u1)
        gu1 = self._conv_bwd("d1a", a["u1"], a["s1"], gs1, 32, 16, h[0], w[0])
        ge1 = gs1  # masked in place above: this is dL/d e1 from the skip
        gd2 = self._up_bwd(gu1)
        gs2 = self._conv_bwd("d2b", a["s2"], a["d2"], gd2, 32, 32, h[1], w[1])
        gu2 = self._conv_bwd("d2a", a["u2"], a["s2"], gs2, 64, 32, h[1], w[1])
        ge2 = gs2
        gd3 = self._up_bwd(gu2)
        gs3 = self._conv_bwd("d3b", a["s3"], a["d3"], gd3, 64, 64, h[2], w[2])
        gu3 = self._conv_bwd("d3a", a["u3"], a["s3"], gs3, 128, 64, h[2], w[2])
        ge3 = gs3
        ge4 = self._up_bwd(gu3)
        ge4a = self._conv_bwd("e4b", a["e4a"], a["e4"], ge4, 128, 128, h[3], w[3])
        gp3 = self._conv_bwd("e4a", a["p3"], a["e4a"], ge4a, 64, 128, h[3], w[3])
        self._pool_bwd(gp3, ge3, accumulate=True)
        ge3a = self._conv_bwd("e3b", a["e3a"], a["e3"], ge3, 64, 64, h[2], w[2])
        gp2 = self._conv_bwd("e3a", a["p2"], a["e3a"], ge3a, 32, 64, h[2], w[2])
        self._pool_bwd(gp2, ge2, accumulate=True)
        ge2a = self._conv_bwd("e2b", a["e2a"], a["e2"], ge2, 32, 32, h[1], w[1])
        gp1 = self._conv_bwd("e2a", a["p1"], a["e2a"], ge2a, 16, 32, h[1], w[1])
        self._pool_bwd(gp1, ge1, accumulate=True)
        ge1a = self._conv_bwd("e1b", a["e1a"], a["e1"], ge1, 16, 16, h[0], w[0])
        self._conv_bwd("e1a", a["x"], a["e1a"], ge1a, N_FEATURES, 16, h[0], w[0], need_gx=False)

    def loss_and_grad(self, out, target, want_grad=True):
        """Per-image losses (LOSS_ABSOLUTE: npix sum (out - t)^2; LOSS_RELATIVE:
        sum (out - t)^2 / sum t^2) and the gradient of their batch mean."""
        t = self.torch
        B = out.shape[0]
        HW = out[0].numel()
        g = t.empty((B, HW), dtype=t.float32, device=self.dev) if want_grad else None
        self._chk(self.L.gpair_cnn_mse(out.contiguous().data_ptr(), target.contiguous().data_ptr(), _ptr(g),
                                       self._loss.data_ptr(), B, HW, 1.0 / B, self.loss_mode, self.stream))
        return self._loss[:B], g

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        self._chk(self.L.gpair_cnn_adam(self.p.data_ptr(), self.pbf.data_ptr(), self.g.data_ptr(), self.m.data_ptr(),
                                        self.v.data_ptr(), self.p.numel(), lr, b1, b2, eps, self.step, self.stream))

    def train_step(self, x, target, lr):
        out = self.forward(x, keep=True)
        loss, g = self.loss_and_grad(out.view(out.shape[0], -1), target)
        self.backward(g)
        self.adam(lr)
        return loss


# ------------------------------------------------------------ problem features

def uv_density(p: api.Problem) -> np.ndarray:
    """The problem's (u, v) points and their conjugates gridded on the N x N
    Fourier grid of the image, log(1 + count) scaled to max 1, centred."""
    N = p.width
    k = p.uv[:, 0].astype(np.float64) * RPMAS * p.pixellation * N
    l = p.uv[:, 1].astype(np.float64) * RPMAS * p.pixellation * N
    iu = np.concatenate([np.rint(k), np.rint(-k)]).astype(np.int64) + N // 2
    iv = np.concatenate([np.rint(l), np.rint(-l)]).astype(np.int64) + N // 2
    ok = (iu >= 0) & (iu < N) & (iv >= 0) & (iv < N)
    grid = np.zeros((N, N), np.float64)
    np.add.at(grid, (iv[ok], iu[ok]), 1.0)
    grid = np.log1p(grid)
    m = grid.max()
    return (grid / m if m > 0 else grid).astype(np.float32)


def dirty_image(rec: api.Reconstructor, p: api.Problem) -> np.ndarray:
    """-d chi2/dI at the flat start image, scaled to max |value| 1 (device gradient path)."""
    rec.set_image(p.start_image())
    rec.criterion()
    rec.gradient(alpha=0.0)
    g = -rec.data_gradient().astype(np.float64)
    m = np.abs(g).max()
    return (g / m if m > 0 else g).reshape(p.width, p.width).astype(np.float32)


def v2_dirty_map(rec: api.Reconstructor, p: api.Problem) -> np.ndarray:
    """Adjoint DFT of the V2 data, centred on the image (device adjoint path)."""
    N = p.width
    u = p.uv[:, 0].astype(np.float64)
    v = p.uv[:, 1].astype(np.float64)
    # conj(Fx[k][N/2] Fy[k][N/2]) moves the origin of the map to the image centre
    ph = -2.0 * np.pi * RPMAS * p.pixellation * (u - v) * (N // 2)
    w = np.zeros(p.nuv, np.complex128)
    w[:p.npow] = np.maximum(p.data[:p.npow].astype(np.float64), 0.0)
    w *= np.exp(1j * ph)
    img = rec.adjoint_image(w.astype(np.complex64)).astype(np.float64)
    m = np.abs(img).max()
    return (img / m if m > 0 else img).reshape(N, N).astype(np.float32)


def probe_gradient(rec: api.Reconstructor, p: api.Problem) -> np.ndarray:
    """-d chi2/dI at a centred Gaussian (FWHM N/4 pixels, the prior's flux), max |value| 1."""
    N = p.width
    y, x = np.mgrid[0:N, 0:N].astype(np.float64)
    sig = (N / 4.0) / 2.3548
    gauss = np.exp(-((x - N // 2) ** 2 + (y - N // 2) ** 2) / (2 * sig * sig))
    img = gauss / gauss.sum() * float(np.sum(p.start_image(), dtype=np.float64))
    rec.set_image(np.maximum(img, 1e-8).astype(np.float32).ravel())
    rec.criterion()
    rec.gradient(alpha=0.0)
    g = -rec.data_gradient().astype(np.float64)
    m = np.abs(g).max()
    return (g / m if m > 0 else g).reshape(N, N).astype(np.float32)


def features(rec: api.Reconstructor, p: api.Problem) -> np.ndarray:
    return np.stack([dirty_image(rec, p), v2_dirty_map(rec, p), uv_density(p), probe_gradient(rec, p)])


def warm_start(net: WarmStartNet, rec: api.Reconstructor, p: api.Problem, feats: Optional[np.ndarray] = None):
    """Start image (float32 [N*N], total flux = the prior's) predicted by the network."""
    t = net.torch
    f = features(rec, p) if feats is None else feats
    x = t.from_numpy(f[None]).to(net.dev)
    out = net.forward(x)[0].reshape(-1)
    flux = float(np.sum(p.start_image(), dtype=np.float64))
    img = (out * flux).cpu().numpy().astype(np.float32)
    return np.maximum(img, np.float32(1e-8))


# ------------------------------------------------------------ training scenes

def training_scene(rng: np.random.Generator, field_mas: float) -> Scene:
    """1-10 components (Gaussians, uniform disks, points), total flux 1."""
    comps = []
    n = int(rng.integers(1, 11))
    half = 0.3 * field_mas
    for _ in range(n):
        kind = ("gauss", "disk", "point")[int(rng.integers(0, 3))]
        x, y = float(rng.uniform(-half, half)), float(rng.uniform(-half, half))
        f = float(rng.uniform(0.1, 1.0))
        if kind == "point":
            comps.append(Component("point", f, x=x, y=y))
        elif kind == "disk":
            comps.append(Component("disk", f, x=x, y=y, size=float(rng.uniform(0.04, 0.25) * field_mas)))
        else:
            comps.append(Component("gauss", f, x=x, y=y, size=float(rng.uniform(0.03, 0.2) * field_mas),
                                   ratio=float(rng.uniform(0.3, 1.0)), pa=float(rng.uniform(0, np.pi))))
    tot = sum(c.flux for c in comps)
    for c in comps:
        c.flux /= tot
    return Scene(comps)


def training_array(rng: np.random.Generator) -> ArrayConfig:
    """4-12 telescopes in a 150-400 m disk, 8-16 hour angles, 3 channels."""
    return ArrayConfig(int(rng.integers(4, 13)), float(rng.uniform(150.0, 400.0)), int(rng.integers(8, 17)),
                       [1.5e-6, 1.65e-6, 1.8e-6], "all")


@dataclass
class TrainingCase:
    seed: int
    width: int
    problem: api.Problem


def training_case(seed: int, width: int) -> TrainingCase:
    """Seeded scene + array + noise (independent streams) -> problem at `width`
    (64 -> 0.1 mas/pixel, 128 -> 0.05 mas/pixel: a 6.4 mas field)."""
    ss = np.random.SeedSequence(seed)
    s_scene, s_array, s_obs, s_noise = ss.spawn(4)
    pix = 6.4 / width
    scene = training_scene(np.random.default_rng(s_scene), 6.4)
    cfg = training_array(np.random.default_rng(s_array))
    oi = make_oifits(cfg, scene, int(s_obs.generate_state(1)[0]), int(s_noise.generate_state(1)[0]))
    p = api.problem_from_oifits(oi, width, pix, 1e-3)
    return TrainingCase(seed, width, p)
