"""Learned warm start for transmission EM.

A small BF16 U-Net (4 levels, 32 base channels, ~1.95M parameters) maps an
FBP reconstruction to an image that tEM starts from, instead of the uniform
start the reference uses (em_methods.py:117-122).  The network runs on the
library's own tensor-core kernels (raft_unet_* in libraft.so) for inference
and training; PyTorch only provides device memory and streams.  Plain EM
from a uniform start remains the fallback and the judge: the figure of merit
is the time tEM needs to reach the data residual of plain 100-iteration EM.

Everything here works on device tensors (torch CUDA).  Geometry: images on
the EM grid (em_RT_kernel.cu:97-99); the FBP input is flipped in y and scaled
by (N-1)/2 to that grid before entering the network.
"""
import ctypes
import math
import time

import numpy as np

from . import synthetic as S
from .rafttypes import _ptr, check_error, libraft

_P, _I, _F, _Z = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_size_t
libraft.raft_unet_conv_fwd.argtypes = [_P, _I, _P, _I, _P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P]
libraft.raft_unet_conv_wgrad.argtypes = [_P, _P, _I, _P, _I, _P, _P, _I, _I, _I, _I, _P]
libraft.raft_unet_flip_weights.argtypes = [_P, _P, _I, _I, _P]
libraft.raft_unet_relu_bwd.argtypes = [_P, _P, _P, _Z, _P]
libraft.raft_unet_pool.argtypes = [_I, _P, _P, _I, _I, _I, _I, _P]
libraft.raft_unet_upsample.argtypes = [_I, _P, _P, _I, _I, _I, _I, _P]
libraft.raft_unet_input.argtypes = [_P, _P, _P, _I, _I, _I, _I, _P]
libraft.raft_unet_head.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _P]
libraft.raft_unet_mse.argtypes = [_P, _P, _P, _P, _P, _I, _I, _P]
libraft.raft_unet_adam.argtypes = [_P, _P, _P, _P, _P, _Z, _F, _F, _F, _F, _I, _P]
libraft.raft_unet_add.argtypes = [_P, _P, _Z, _P]
libraft.raft_unet_to_bf16.argtypes = [_P, _P, _Z, _P]
libraft.raft_radon_device.argtypes = [_I, _P, _P, _P, _I, _I, _I, _I, _I, _F, _F, _P]
libraft.raft_radon_device.restype = _I
for _f in ("raft_unet_conv_fwd", "raft_unet_conv_wgrad", "raft_unet_flip_weights", "raft_unet_relu_bwd",
           "raft_unet_pool", "raft_unet_upsample", "raft_unet_input", "raft_unet_head", "raft_unet_mse",
           "raft_unet_adam", "raft_unet_add", "raft_unet_to_bf16"):
    getattr(libraft, _f).restype = _I


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _ok(rc, what):
    if rc:
        raise RuntimeError(f"sscRaft.warmstart: {what} failed (bad sizes or CUDA error)")


class UNet:
    """4-level U-Net, base 32 channels, 3x3 convolutions + ReLU, 2x2 average
    pooling, nearest 2x upsampling, skip connections by channel concatenation,
    1x1 head with a residual connection to the (scaled) input image."""

    LAYERS = [("e0a", 32, 0, 32), ("e0b", 32, 0, 32), ("e1a", 32, 0, 64), ("e1b", 64, 0, 64),
              ("e2a", 64, 0, 128), ("e2b", 128, 0, 128), ("e3a", 128, 0, 256), ("e3b", 256, 0, 256),
              ("d2a", 256, 128, 128), ("d2b", 128, 0, 128), ("d1a", 128, 64, 64), ("d1b", 64, 0, 64),
              ("d0a", 64, 32, 32), ("d0b", 32, 0, 32)]

    def __init__(self, device, seed=0):
        import torch
        self.torch = torch
        self.dev = device
        g = torch.Generator().manual_seed(seed)
        self.w, self.b, self.wb = {}, {}, {}
        self.m, self.v = {}, {}
        for name, c0, c1, co in self.LAYERS:
            cin = c0 + c1
            std = math.sqrt(2.0 / (9 * cin))
            w = (torch.randn((co, 3, 3, cin), generator=g) * std).to(device)
            if name == "e0a":
                w[:, :, :, 1:] = 0.0          # only channel 0 of the packed input carries data
            self.w[name] = w.contiguous()
            self.b[name] = torch.zeros(co, device=device)
        self.w["head"] = (torch.randn(32, generator=g) * 1e-3).to(device)
        self.b["head"] = torch.zeros(1, device=device)
        for k in self.w:
            self.m[k] = (torch.zeros_like(self.w[k]), torch.zeros_like(self.b[k]))
            self.v[k] = (torch.zeros_like(self.w[k]), torch.zeros_like(self.b[k]))
        self._sync_bf16()
        self.step_count = 0
        self.stream = None

    def n_params(self):
        return sum(t.numel() for t in self.w.values()) + sum(t.numel() for t in self.b.values())

    def _sync_bf16(self):
        for name, *_ in self.LAYERS:
            self.wb[name] = self.w[name].to(self.torch.bfloat16).contiguous()

    def _st(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    # ----------------------------------------------------------- layers --
    def _conv(self, name, x0, x1, N, H, W, relu=True):
        _, c0, c1, co = next(l for l in self.LAYERS if l[0] == name)
        y = self.torch.empty((N, H, W, co), dtype=self.torch.bfloat16, device=self.dev)
        _ok(libraft.raft_unet_conv_fwd(_p(x0), c0, _p(x1), c1, _p(self.wb[name]), _p(self.b[name]), _p(y), None, 0,
                                       N, H, W, co, 1 if relu else 0, self._st()), "conv_fwd " + name)
        return y

    def _pool(self, x, N, H, W, C):
        y = self.torch.empty((N, H // 2, W // 2, C), dtype=self.torch.bfloat16, device=self.dev)
        _ok(libraft.raft_unet_pool(0, _p(x), _p(y), N, H, W, C, self._st()), "pool")
        return y

    def _up(self, x, N, H, W, C):
        y = self.torch.empty((N, 2 * H, 2 * W, C), dtype=self.torch.bfloat16, device=self.dev)
        _ok(libraft.raft_unet_upsample(0, _p(x), _p(y), N, H, W, C, self._st()), "upsample")
        return y

    def forward(self, img, scale, keep=False):
        """img [N,H,W] fp32 (EM grid), scale [N] fp32 -> output [N,H,W] fp32 in scaled units.
        H, W must be multiples of 8."""
        torch = self.torch
        N, H, W = img.shape
        x = torch.empty((N, H, W, 32), dtype=torch.bfloat16, device=self.dev)
        _ok(libraft.raft_unet_input(_p(img), _p(scale), _p(x), N, H, W, 32, self._st()), "input")
        A = {"x": x}
        A["e0a"] = self._conv("e0a", x, None, N, H, W)
        A["s0"] = self._conv("e0b", A["e0a"], None, N, H, W)
        A["p0"] = self._pool(A["s0"], N, H, W, 32)
        h1, w1 = H // 2, W // 2
        A["e1a"] = self._conv("e1a", A["p0"], None, N, h1, w1)
        A["s1"] = self._conv("e1b", A["e1a"], None, N, h1, w1)
        A["p1"] = self._pool(A["s1"], N, h1, w1, 64)
        h2, w2 = h1 // 2, w1 // 2
        A["e2a"] = self._conv("e2a", A["p1"], None, N, h2, w2)
        A["s2"] = self._conv("e2b", A["e2a"], None, N, h2, w2)
        A["p2"] = self._pool(A["s2"], N, h2, w2, 128)
        h3, w3 = h2 // 2, w2 // 2
        A["e3a"] = self._conv("e3a", A["p2"], None, N, h3, w3)
        A["bt"] = self._conv("e3b", A["e3a"], None, N, h3, w3)
        A["u2"] = self._up(A["bt"], N, h3, w3, 256)
        A["d2a"] = self._conv("d2a", A["u2"], A["s2"], N, h2, w2)
        A["d2"] = self._conv("d2b", A["d2a"], None, N, h2, w2)
        A["u1"] = self._up(A["d2"], N, h2, w2, 128)
        A["d1a"] = self._conv("d1a", A["u1"], A["s1"], N, h1, w1)
        A["d1"] = self._conv("d1b", A["d1a"], None, N, h1, w1)
        A["u0"] = self._up(A["d1"], N, h1, w1, 64)
        A["d0a"] = self._conv("d0a", A["u0"], A["s0"], N, H, W)
        A["d0"] = self._conv("d0b", A["d0a"], None, N, H, W)
        out = torch.empty((N, H, W), dtype=torch.float32, device=self.dev)
        _ok(libraft.raft_unet_head(0, _p(A["d0"]), _p(self.w["head"]), _p(self.b["head"]), _p(img), _p(scale),
                                   _p(out), None, None, None, N, H * W, 32, self._st()), "head")
        self._acts = (A, (N, H, W), img, scale) if keep else None
        return out

    # --------------------------------------------------------- backward --
    def _conv_bwd(self, name, x0, x1, y, gy, N, H, W, need_dx=True):
        torch = self.torch
        _, c0, c1, co = next(l for l in self.LAYERS if l[0] == name)
        st = self._st()
        dpre = torch.empty_like(gy)
        _ok(libraft.raft_unet_relu_bwd(_p(y), _p(gy), _p(dpre), gy.numel(), st), "relu_bwd")
        _ok(libraft.raft_unet_conv_wgrad(_p(dpre), _p(x0), c0, _p(x1), c1, _p(self.gw[name]), _p(self.gb[name]),
                                         N, H, W, co, st), "wgrad " + name)
        if not need_dx:
            return None, None
        cin = c0 + c1
        wt = torch.empty((cin, 3, 3, co), dtype=torch.bfloat16, device=self.dev)
        _ok(libraft.raft_unet_flip_weights(_p(self.wb[name]), _p(wt), co, cin, st), "flip")
        dx0 = torch.empty((N, H, W, c0), dtype=torch.bfloat16, device=self.dev)
        dx1 = torch.empty((N, H, W, c1), dtype=torch.bfloat16, device=self.dev) if c1 else None
        _ok(libraft.raft_unet_conv_fwd(_p(dpre), co, None, 0, _p(wt), None, _p(dx0), _p(dx1), c0 if c1 else 0,
                                       N, H, W, cin, 0, st), "dgrad " + name)
        return dx0, dx1

    def _upb(self, g, N, H, W, C):
        y = self.torch.empty((N, H, W, C), dtype=self.torch.bfloat16, device=self.dev)
        _ok(libraft.raft_unet_upsample(1, _p(g), _p(y), N, H, W, C, self._st()), "upsample_bwd")
        return y

    def _poolb(self, g, N, H, W, C):
        y = self.torch.empty((N, H, W, C), dtype=self.torch.bfloat16, device=self.dev)
        _ok(libraft.raft_unet_pool(1, _p(g), _p(y), N, H, W, C, self._st()), "pool_bwd")
        return y

    def _add(self, y, x):
        _ok(libraft.raft_unet_add(_p(y), _p(x), y.numel(), self._st()), "add")
        return y

    def backward(self, gout):
        """gout [N,H,W] fp32 = dLoss/dOutput; fills self.gw / self.gb."""
        torch = self.torch
        A, (N, H, W), img, scale = self._acts
        self.gw = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.gb = {k: torch.zeros_like(v) for k, v in self.b.items()}
        st = self._st()
        g_d0 = torch.empty_like(A["d0"])
        _ok(libraft.raft_unet_head(1, _p(A["d0"]), _p(self.w["head"]), None, None, None, _p(gout), _p(g_d0),
                                   _p(self.gw["head"]), _p(self.gb["head"]), N, H * W, 32, st), "head_bwd")
        h1, w1, h2, w2, h3, w3 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8
        g, _ = self._conv_bwd("d0b", A["d0a"], None, A["d0"], g_d0, N, H, W)
        g_u0, g_s0 = self._conv_bwd("d0a", A["u0"], A["s0"], A["d0a"], g, N, H, W)
        g = self._upb(g_u0, N, h1, w1, 64)
        g, _ = self._conv_bwd("d1b", A["d1a"], None, A["d1"], g, N, h1, w1)
        g_u1, g_s1 = self._conv_bwd("d1a", A["u1"], A["s1"], A["d1a"], g, N, h1, w1)
        g = self._upb(g_u1, N, h2, w2, 128)
        g, _ = self._conv_bwd("d2b", A["d2a"], None, A["d2"], g, N, h2, w2)
        g_u2, g_s2 = self._conv_bwd("d2a", A["u2"], A["s2"], A["d2a"], g, N, h2, w2)
        g = self._upb(g_u2, N, h3, w3, 256)
        g, _ = self._conv_bwd("e3b", A["e3a"], None, A["bt"], g, N, h3, w3)
        g, _ = self._conv_bwd("e3a", A["p2"], None, A["e3a"], g, N, h3, w3)
        g = self._add(self._poolb(g, N, h2, w2, 128), g_s2)
        g, _ = self._conv_bwd("e2b", A["e2a"], None, A["s2"], g, N, h2, w2)
        g, _ = self._conv_bwd("e2a", A["p1"], None, A["e2a"], g, N, h2, w2)
        g = self._add(self._poolb(g, N, h1, w1, 64), g_s1)
        g, _ = self._conv_bwd("e1b", A["e1a"], None, A["s1"], g, N, h1, w1)
        g, _ = self._conv_bwd("e1a", A["p0"], None, A["e1a"], g, N, h1, w1)
        g = self._add(self._poolb(g, N, H, W, 32), g_s0)
        g, _ = self._conv_bwd("e0b", A["e0a"], None, A["s0"], g, N, H, W)
        self._conv_bwd("e0a", A["x"], None, A["e0a"], g, N, H, W, need_dx=False)

    def adam_step(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        st = self._st()
        for k in self.w:
            wb = self.wb.get(k)
            _ok(libraft.raft_unet_adam(_p(self.w[k]), _p(self.m[k][0]), _p(self.v[k][0]), _p(self.gw[k]),
                                       _p(wb), self.w[k].numel(), lr, b1, b2, eps, self.step_count, st), "adam")
            _ok(libraft.raft_unet_adam(_p(self.b[k]), _p(self.m[k][1]), _p(self.v[k][1]), _p(self.gb[k]), None,
                                       self.b[k].numel(), lr, b1, b2, eps, self.step_count, st), "adam")
        if "e0a" in self.w:
            self.w["e0a"][:, :, :, 1:] = 0.0
            self.wb["e0a"][:, :, :, 1:] = 0.0

    def train_step(self, img, target, scale, lr):
        """One Adam step on MSE(out, target*scale); returns the loss (device tensor)."""
        torch = self.torch
        N, H, W = img.shape
        out = self.forward(img, scale, keep=True)
        g = torch.empty_like(out)
        loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        _ok(libraft.raft_unet_mse(_p(out), _p(target), _p(scale), _p(g), _p(loss), N, H * W, self._st()), "mse")
        self.backward(g)
        self.adam_step(lr)
        self._acts = None
        return loss

    def predict(self, img, batch=16):
        """Warm-start estimate on the EM grid: out/scale, clamped to a small positive floor."""
        torch = self.torch
        res = torch.empty_like(img)
        for i in range(0, img.shape[0], batch):
            x = img[i:i + batch]
            sc = input_scale(x)
            o = self.forward(x, sc) / sc[:, None, None]
            floor = 1e-3 * torch.clamp(x.abs().mean(dim=(1, 2)), min=1e-12)
            res[i:i + batch] = torch.maximum(o, floor[:, None, None])
        return res

    def state(self):
        return {k: v.detach().cpu().numpy() for k, v in list(self.w.items())} | \
               {k + ".bias": v.detach().cpu().numpy() for k, v in self.b.items()}

    def load(self, state):
        torch = self.torch
        for k in self.w:
            self.w[k] = torch.as_tensor(state[k], device=self.dev).contiguous()
            self.b[k] = torch.as_tensor(state[k + ".bias"], device=self.dev).contiguous()
        self._sync_bf16()


def input_scale(img):
    """Per-image normalisation: 1 / mean |input|."""
    return (1.0 / img.abs().mean(dim=(1, 2)).clamp(min=1e-12)).float().contiguous()


# ------------------------------------------------------------------ data --
def perlin(N, seed, cells=8, device=None):
    """Seeded 2-D gradient (Perlin) noise on an N x N grid, values ~[-1, 1]."""
    import torch
    g = torch.Generator().manual_seed(seed)
    ang = torch.rand((cells + 1, cells + 1), generator=g) * 2 * math.pi
    gx, gy = torch.cos(ang).to(device), torch.sin(ang).to(device)
    t = (torch.arange(N, device=device, dtype=torch.float32) + 0.5) * (cells / N)
    i0 = t.floor().long().clamp(max=cells - 1)
    f = t - i0
    fy, fx = f[:, None], f[None, :]
    iy, ix = i0[:, None], i0[None, :]

    def dot(oy, ox):
        return gx[iy + oy, ix + ox] * (fx - ox) + gy[iy + oy, ix + ox] * (fy - oy)

    def fade(u):
        return u * u * u * (u * (u * 6 - 15) + 10)

    u, v = fade(fx), fade(fy)
    n0 = dot(0, 0) * (1 - u) + dot(0, 1) * u
    n1 = dot(1, 0) * (1 - u) + dot(1, 1) * u
    return (n0 * (1 - v) + n1 * v) * 1.4


def make_pairs(n, seed0, device, N=512, A=720, em_iters=200, chunk=64, i0_range=(1e3, 1e5), gpu=0):
    """(input, label, transmission) triples made by the method itself:
    ellipse + Perlin-texture phantoms on the EM grid, scaled so the largest
    line integral is 3; Radon projections; Poisson counts at I0 ~ U[i0_range];
    FBP (linear operator, Hann) of -log(transmission) mapped to the EM grid as
    the network input; `em_iters`-iteration tEM from a uniform start as the
    label.  Everything stays on the device."""
    import torch
    ang = S.uniform_angles(A)
    angp = np.ascontiguousarray(ang)
    inputs = torch.empty((n, N, N), dtype=torch.float32, device=device)
    labels = torch.empty((n, N, N), dtype=torch.float32, device=device)
    trans = torch.empty((n, A, N), dtype=torch.float32, device=device)
    st = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    rng = np.random.Generator(np.random.PCG64(seed0))
    for c0 in range(0, n, chunk):
        m = min(chunk, n - c0)
        ph = torch.empty((m, N, N), dtype=torch.float32, device=device)
        for k in range(m):
            s = seed0 + c0 + k
            img = S.phantom_image(S.ellipse_params(s, 20), N, xp=torch, device=device)
            tex = perlin(N, s, device=device)
            ph[k] = img * (1.0 + 0.3 * tex) * (img > 0)
        proj = torch.empty((m, A, N), dtype=torch.float32, device=device)
        _ok(libraft.raft_radon_device(gpu, _p(proj), _p(ph), _ptr(angp), N, N, N, A, m, 1.0, 1.0, st), "radon")
        scl = 3.0 / proj.amax(dim=(1, 2)).clamp(min=1e-12)
        proj *= scl[:, None, None]
        i0 = torch.as_tensor(rng.uniform(i0_range[0], i0_range[1], m), dtype=torch.float64, device=device)
        gen = torch.Generator(device=device).manual_seed(seed0 + c0)
        counts = torch.poisson(i0[:, None, None] * torch.exp(-proj.double()), generator=gen)
        t = (counts.clamp(min=1.0) / i0[:, None, None]).float().contiguous()
        trans[c0:c0 + m] = t
        sino = (-torch.log(t)).contiguous()
        fbp = torch.empty((m, N, N), dtype=torch.float32, device=device)
        pf = np.array([0, 0, 1, 0, 1, 1, 0], np.float32)
        pi = np.array([N, A, m, N, 2, 0, 0, 5, 0, 0], np.int32)
        rc = libraft.raft_fbp_device(gpu, _p(fbp), _p(sino), _ptr(angp), _ptr(pf), _ptr(pi), 1, 1, st)
        if rc:
            check_error("fbp")
        inputs[c0:c0 + m] = torch.flip(fbp, dims=(1,)) * ((N - 1) / 2.0)
        obj = torch.ones((m, N, N), dtype=torch.float32, device=device)
        flat = torch.ones((m, N), dtype=torch.float32, device=device)
        rc = libraft.raft_em_device(0, gpu, _p(obj), _p(t), _p(flat), _ptr(angp), N, A, m, em_iters, None, 1, st)
        if rc:
            check_error("tem")
        labels[c0:c0 + m] = obj
    torch.cuda.synchronize(device)
    return inputs, labels, trans, ang


def train(net, inputs, labels, epochs=4, batch=8, lr=1e-3, log=None):
    """Adam on MSE between the network output and the EM label (both scaled
    by the input's normalisation), cosine learning-rate decay."""
    import torch
    n = inputs.shape[0]
    steps = epochs * ((n + batch - 1) // batch)
    k = 0
    perm_g = torch.Generator().manual_seed(1234)
    losses = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=perm_g)
        for i in range(0, n - batch + 1, batch):
            idx = perm[i:i + batch].to(inputs.device)
            x = inputs[idx].contiguous()
            y = labels[idx].contiguous()
            sc = input_scale(x)
            cur = lr * 0.5 * (1 + math.cos(math.pi * k / max(1, steps)))
            losses.append(net.train_step(x, y, sc, cur))
            k += 1
        if log:
            log(f"epoch {ep}: loss {float(torch.stack(losses[-10:]).mean()):.4g}")
    return [float(l) for l in losses]


def em_residuals(obj, trans, ang, iters, gpu=0):
    """Run `iters` tEM iterations from `obj` (in place) and return the data
    residual ||exp(-Ax_k) - y|| / ||y|| of the iterate entering each iteration
    (per slice, [iters, n]) and the device time per iteration (ms)."""
    import torch
    n, A, N = trans.shape
    dev = trans.device
    met = torch.zeros((iters, n, 3), dtype=torch.float64, device=dev)
    flat = torch.ones((n, N), dtype=torch.float32, device=dev)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rc = libraft.raft_em_device(0, gpu, _p(obj), _p(trans), _p(flat), _ptr(np.ascontiguousarray(ang)), N, A, n,
                                iters, _p(met), 1, st)
    e1.record()
    if rc:
        check_error("tem")
    torch.cuda.synchronize(dev)
    m = met.cpu().numpy()
    res = np.sqrt(m[:, :, 0]) / np.sqrt(m[:, :, 1])
    return res, e0.elapsed_time(e1) / max(1, iters)


def evaluate(net, inputs, trans, ang, plain_iters=100, max_warm_iters=100, tol=0.01, gpu=0):
    """Time-to-residual of warm-started vs plain tEM on held-out samples.

    target r* = data residual of plain EM after `plain_iters` iterations (per
    slice); plain EM needs `plain_iters` iterations by definition (and may cross
    (1+tol) r* earlier, reported too); warm start = network inference + the
    iterations until the residual is within (1+tol) r*."""
    import torch
    n, A, N = trans.shape
    obj = torch.ones((n, N, N), dtype=torch.float32, device=trans.device)
    res_plain, t_iter = em_residuals(obj, trans, ang, plain_iters + 1, gpu)
    target = res_plain[plain_iters] * (1.0 + tol)
    first_plain = np.array([int(np.argmax(res_plain[:, j] <= target[j])) for j in range(n)])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    x0 = net.predict(inputs)
    e1.record()
    torch.cuda.synchronize()
    t_net = e0.elapsed_time(e1)
    res_warm, t_iter_w = em_residuals(x0.clone(), trans, ang, max_warm_iters + 1, gpu)
    reached = res_warm <= target[None, :]
    k_warm = np.where(reached.any(0), reached.argmax(0), max_warm_iters + 1)
    t_plain = plain_iters * t_iter
    k_all = int(k_warm.max())
    t_warm = t_net + k_all * t_iter_w
    return {"samples": n, "ms_per_iteration_batch": t_iter, "unet_ms_batch": t_net,
            "plain_iterations": plain_iters, "plain_first_within_tol_median": float(np.median(first_plain)),
            "warm_iterations_median": float(np.median(k_warm)), "warm_iterations_max": k_all,
            "warm_reached_fraction": float(reached.any(0).mean()),
            "time_plain_ms": t_plain, "time_warm_ms": t_warm, "speedup": t_plain / t_warm,
            "residual_plain100_median": float(np.median(res_plain[plain_iters])),
            "residual_start_warm_median": float(np.median(res_warm[0])),
            "residual_start_plain_median": float(np.median(res_plain[0]))}
