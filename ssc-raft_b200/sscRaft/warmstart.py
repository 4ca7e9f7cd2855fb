"""Learned warm start for transmission EM.

A small BF16 U-Net (4 levels, 32 base channels, ~1.95M parameters) maps an
FBP reconstruction to an image that tEM starts from, instead of the uniform
start the reference uses (em_methods.py:117-122).  The network runs on the
library's own tensor-core kernels (raft_unet_* in libraft.so) for inference
and training; PyTorch only provides device memory and streams.  Plain EM
from a uniform start remains the fallback and sets the bar: the figure of
merit is the time tEM needs to reach the data residual of plain 100-iteration
EM.

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
libraft.raft_unet_input_conv.argtypes = [_P, _P, _P, _I, _P, _P, _I, _I, _I, _P]
libraft.raft_unet_input_wgrad.argtypes = [_P, _P, _P, _P, _I, _P, _P, _Z, _I, _I, _I, _P]
libraft.raft_unet_head.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _P]
libraft.raft_unet_mse.argtypes = [_P, _P, _P, _P, _P, _I, _I, _P]
libraft.raft_unet_adam.argtypes = [_P, _P, _P, _P, _P, _Z, _F, _F, _F, _F, _I, _P]
libraft.raft_unet_add.argtypes = [_P, _P, _Z, _P]
libraft.raft_unet_to_bf16.argtypes = [_P, _P, _Z, _P]
libraft.raft_unet_set_conv_path.argtypes = [_I]
libraft.raft_unet_set_conv_halo.argtypes = [_I]
libraft.raft_unet_set_wgrad_nine.argtypes = [_I]
libraft.raft_unet_conv_error.argtypes = []
for _f in ("raft_unet_set_conv_path", "raft_unet_set_conv_halo", "raft_unet_set_wgrad_nine", "raft_unet_conv_error", "raft_unet_conv_fwd", "raft_unet_conv_wgrad", "raft_unet_flip_weights", "raft_unet_relu_bwd",
           "raft_unet_pool", "raft_unet_upsample", "raft_unet_input", "raft_unet_input_conv", "raft_unet_input_wgrad",
           "raft_unet_head",
           "raft_unet_mse",
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
        # the first layer straight from the one-channel image (bit-identical to
        # convolving a packed 32-channel input whose other channels are zero)
        A = {"e0a": torch.empty((N, H, W, 32), dtype=torch.bfloat16, device=self.dev)}
        _ok(libraft.raft_unet_input_conv(_p(img), _p(scale), _p(self.wb["e0a"]), 32, _p(self.b["e0a"]),
                                         _p(A["e0a"]), N, H, W, self._st()), "input_conv")
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
        # first layer: weight (channel 0) and bias gradients from the image itself
        dpre = torch.empty_like(g)
        _ok(libraft.raft_unet_relu_bwd(_p(A["e0a"]), _p(g), _p(dpre), g.numel(), st), "relu_bwd")
        work = torch.empty(N * H * 320, dtype=torch.float32, device=self.dev)
        _ok(libraft.raft_unet_input_wgrad(_p(img), _p(scale), _p(dpre), _p(self.gw["e0a"]), 32, _p(self.gb["e0a"]),
                                          _p(work), work.numel(), N, H, W, st), "wgrad e0a")

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
        self.check()
        return res

    def check(self):
        """Raises if a bounded wait of the tensor-core convolution ran out since
        the last check (synchronises the device)."""
        _ok(libraft.raft_unet_conv_error(), "tensor-core convolution: a pipeline wait timed out")

    def state(self):
        return {k: v.detach().cpu().numpy() for k, v in list(self.w.items())} | \
               {k + ".bias": v.detach().cpu().numpy() for k, v in self.b.items()}

    def load(self, state):
        torch = self.torch
        for k in self.w:
            self.w[k] = torch.as_tensor(state[k], device=self.dev).contiguous()
            self.b[k] = torch.as_tensor(state[k + ".bias"], device=self.dev).contiguous()
        self._sync_bf16()

    def save(self, path, **meta):
        """Weights file: 3x3 convolution weights as BF16 bit patterns (the
        precision inference runs in), biases and the head in FP32, plus
        free-form metadata (training recipe)."""
        torch = self.torch
        arr = {}
        for k, v in self.w.items():
            if k == "head":
                arr[k] = v.detach().cpu().numpy().astype(np.float32)
            else:
                arr[k + ".bf16"] = v.detach().to(torch.bfloat16).view(torch.int16).cpu().numpy()
        for k, v in self.b.items():
            arr[k + ".bias"] = v.detach().cpu().numpy().astype(np.float32)
        arr["meta"] = np.array(repr(meta))
        np.savez_compressed(path, **arr)

    @classmethod
    def from_file(cls, path, device):
        """A network with the weights `save` wrote (FP32 masters = the BF16 values)."""
        import torch
        net = cls(device, seed=0)
        z = np.load(path)
        st = {}
        for k in net.w:
            if k == "head":
                st[k] = z[k]
            else:
                st[k] = torch.from_numpy(z[k + ".bf16"]).view(torch.bfloat16).float().numpy()
            st[k + ".bias"] = z[k + ".bias"]
        net.load(st)
        net.meta = str(z["meta"])
        return net


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


def fbp_input(trans, ang, gpu=0, out=None):
    """Network input from normalised transmissions t [n, A, N] (device):
    FBP (linear-interpolation backprojector, Hann filter, pad 2) of -log t,
    flipped in y and scaled by (N-1)/2 onto the EM grid."""
    import torch
    n, A, N = trans.shape
    dev = trans.device
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    sino = (-torch.log(trans)).contiguous()
    fbp = torch.empty((n, N, N), dtype=torch.float32, device=dev)
    pf = np.array([0, 0, 1, 0, 1, 1, 0], np.float32)
    pi = np.array([N, A, n, N, 2, 0, 0, 5, 0, 0], np.int32)
    rc = libraft.raft_fbp_device(gpu, _p(fbp), _p(sino), _ptr(np.ascontiguousarray(ang)), _ptr(pf), _ptr(pi),
                                 1, 1, st)
    if rc:
        check_error("fbp")
    res = torch.flip(fbp, dims=(1,))
    res *= (N - 1) / 2.0
    if out is None:
        return res
    out.copy_(res)
    return out


def make_transmissions(n, seed0, device, N=512, A=720, chunk=64, i0_range=(1e3, 1e5), gpu=0, out=None):
    """Normalised transmissions t = counts/I0 [n, A, N] of seeded phantoms:
    random ellipses (seed s = seed0 + i) with seeded Perlin texture on the EM
    grid, Radon projections scaled so the largest line integral is 3, Poisson
    counts at I0 ~ U[i0_range] per slice."""
    import torch
    angp = np.ascontiguousarray(S.uniform_angles(A))
    trans = out if out is not None else torch.empty((n, A, N), dtype=torch.float32, device=device)
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
        trans[c0:c0 + m] = (counts.clamp(min=1.0) / i0[:, None, None]).float()
    return trans


def em_label(trans, iters, gpu=0):
    """`iters` tEM iterations from the uniform start (the reference's default
    initial guess), [n, N, N] on the EM grid."""
    import torch
    n, A, N = trans.shape
    dev = trans.device
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    ang = np.ascontiguousarray(S.uniform_angles(A))
    obj = torch.ones((n, N, N), dtype=torch.float32, device=dev)
    flat = torch.ones((n, N), dtype=torch.float32, device=dev)
    rc = libraft.raft_em_device(0, gpu, _p(obj), _p(trans), _p(flat), _ptr(ang), N, A, n, iters, None, 1, st)
    if rc:
        check_error("tem")
    return obj


def make_pairs(n, seed0, device, N=512, A=720, em_iters=200, chunk=64, i0_range=(1e3, 1e5), gpu=0,
               keep_trans=True):
    """(input, label, transmission) triples made by the method itself:
    make_transmissions' seeded data, the FBP input of fbp_input, and
    `em_iters`-iteration tEM from a uniform start as the label.  Everything
    stays on the device; with keep_trans=False only one chunk of
    transmissions is held at a time and None is returned in its place."""
    import torch
    ang = S.uniform_angles(A)
    inputs = torch.empty((n, N, N), dtype=torch.float32, device=device)
    labels = torch.empty((n, N, N), dtype=torch.float32, device=device)
    trans = torch.empty((n, A, N), dtype=torch.float32, device=device) if keep_trans else None
    for c0 in range(0, n, chunk):
        m = min(chunk, n - c0)
        t = make_transmissions(m, seed0 + c0, device, N, A, chunk=m, i0_range=i0_range, gpu=gpu)
        if keep_trans:
            trans[c0:c0 + m] = t
        fbp_input(t, ang, gpu, out=inputs[c0:c0 + m])
        labels[c0:c0 + m] = em_label(t, em_iters, gpu)
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


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _em_timed(obj, trans, ang, iters, gpu=0):
    """`iters` tEM iterations in place (no metrics, graph-captured loop), device ms."""
    import torch
    n, A, N = trans.shape
    flat = torch.ones((n, N), dtype=torch.float32, device=trans.device)
    st = ctypes.c_void_p(torch.cuda.current_stream(trans.device).cuda_stream)
    e0, e1 = _events()
    e0.record()
    rc = 0
    if iters > 0:
        rc = libraft.raft_em_device(0, gpu, _p(obj), _p(trans), _p(flat), _ptr(np.ascontiguousarray(ang)), N, A, n,
                                    iters, None, 1, st)
    e1.record()
    if rc:
        check_error("tem")
    torch.cuda.synchronize(trans.device)
    return e0.elapsed_time(e1)


def _first_within(res, target, cap):
    """Per slice: first iterate index whose residual is <= target (cap + 1 if none)."""
    ok = res <= target[None, :]
    return np.where(ok.any(0), ok.argmax(0), cap + 1)


def fbp_start(x):
    """The FBP image itself as an EM start (ablation without the network):
    clamped to the same positive floor predict() uses."""
    import torch
    floor = 1e-3 * torch.clamp(x.abs().mean(dim=(1, 2)), min=1e-12)
    return torch.maximum(x, floor[:, None, None])


def evaluate_wall(net, trans, ang, plain_iters=100, tol=0.01, max_iters=100, gpu=0, batch=16):
    """Wall time to the plain-EM data residual, learned start vs plain EM.

    For every held-out slice the target is r* = (1 + tol) x the data residual
    ||exp(-A x_k) - y|| / ||y|| of plain tEM after `plain_iters` iterations
    from the uniform start.  Iteration counts come from FP64-metric runs;
    the times are separate device-timed runs of the same work without
    metrics, all slices batched as EM runs them:
      plain   = `plain_iters` EM iterations from the uniform start;
      learned = FBP of the data + U-Net inference + k EM iterations, k = the
                largest per-slice count the warm start needs to reach r*;
      fbp     = FBP + k' EM iterations from the clamped FBP image (the
                method without the network, reported beside it)."""
    import torch
    n, A, N = trans.shape
    dev = trans.device
    # iteration counts (metric runs)
    res_plain, _ = em_residuals(torch.ones((n, N, N), device=dev), trans, ang, plain_iters + 1, gpu)
    target = res_plain[plain_iters] * (1.0 + tol)
    x = fbp_input(trans, ang, gpu)
    warm = net.predict(x, batch=batch)
    res_warm, _ = em_residuals(warm.clone(), trans, ang, max_iters + 1, gpu)
    res_fbp, _ = em_residuals(fbp_start(x), trans, ang, max_iters + 1, gpu)
    k_warm = _first_within(res_warm, target, max_iters)
    k_fbp = _first_within(res_fbp, target, max_iters)
    kw, kf = int(k_warm.max()), int(k_fbp.max())
    # wall times (no metrics): warm-up once, then time
    for _ in range(2):
        t_plain = _em_timed(torch.ones((n, N, N), device=dev), trans, ang, plain_iters, gpu)
    for _ in range(2):
        e0, e1 = _events()
        e0.record()
        x = fbp_input(trans, ang, gpu)
        e1.record()
        torch.cuda.synchronize(dev)
        t_fbp = e0.elapsed_time(e1)
        e0.record()
        warm = net.predict(x, batch=batch)
        e1.record()
        torch.cuda.synchronize(dev)
        t_net = e0.elapsed_time(e1)
        t_em_w = _em_timed(warm, trans, ang, min(kw, max_iters), gpu)
        t_em_f = _em_timed(fbp_start(x), trans, ang, min(kf, max_iters), gpu)
    t_learned = t_fbp + t_net + t_em_w
    t_fbponly = t_fbp + t_em_f
    return {"samples": n, "plain_iterations": plain_iters, "tol": tol,
            "residual_plain_median": float(np.median(res_plain[plain_iters])),
            "residual_start_uniform_median": float(np.median(res_plain[0])),
            "residual_start_learned_median": float(np.median(res_warm[0])),
            "residual_start_fbp_median": float(np.median(res_fbp[0])),
            "learned_iterations_median": float(np.median(k_warm)), "learned_iterations_max": kw,
            "learned_reached_fraction": float((k_warm <= max_iters).mean()),
            "fbp_iterations_median": float(np.median(k_fbp)), "fbp_iterations_max": kf,
            "fbp_reached_fraction": float((k_fbp <= max_iters).mean()),
            "ms_plain": t_plain, "ms_fbp": t_fbp, "ms_unet": t_net, "ms_em_learned": t_em_w,
            "ms_learned": t_learned, "ms_fbp_start": t_fbponly,
            "speedup_learned_vs_plain": t_plain / t_learned, "speedup_fbp_start_vs_plain": t_plain / t_fbponly,
            "all_reached": bool((k_warm <= max_iters).all())}


TRAIN_SEED0 = 100_000       # training phantoms: seeds 100000 + i
HELDOUT_SEED0 = 900_000     # evaluation phantoms: seeds 900000 + i (disjoint)


def default_weights():
    import os
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "unet_tem_512x720.npz")


def train_recipe(pairs=20000, epochs=3, batch=16, lr=1e-3, N=512, A=720, em_iters=200, val=64, chunk=256,
                 seed=0, device=None, log=print):
    """The training recipe of the shipped weights: `pairs` (FBP, em_iters-tEM)
    pairs from seeds TRAIN_SEED0 + i, Adam with cosine decay; validation MSE
    (network vs FBP input, both against the label) on `val` held-out pairs."""
    import torch
    dev = device or torch.device("cuda", 0)
    t0 = time.time()
    inputs, labels, _, _ = make_pairs(pairs, TRAIN_SEED0, dev, N=N, A=A, em_iters=em_iters, chunk=chunk,
                                      keep_trans=False)
    vx, vy, _, _ = make_pairs(val, HELDOUT_SEED0 + 500_000, dev, N=N, A=A, em_iters=em_iters, chunk=val,
                              keep_trans=False)
    log(f"pairs: {pairs} + {val} in {time.time() - t0:.1f} s")
    net = UNet(dev, seed=seed)

    def val_mse():
        sc = input_scale(vx)
        out = torch.cat([net.forward(vx[i:i + batch].contiguous(), sc[i:i + batch]) for i in range(0, val, batch)])
        return (float(((out - vy * sc[:, None, None]) ** 2).mean()),
                float((((vx - vy) * sc[:, None, None]) ** 2).mean()))
    log(f"val mse before: net {val_mse()[0]:.4g}, fbp input {val_mse()[1]:.4g}")
    t0 = time.time()
    losses = train(net, inputs, labels, epochs=epochs, batch=batch, lr=lr, log=log)
    torch.cuda.synchronize(dev)
    log(f"trained {len(losses)} steps in {time.time() - t0:.1f} s; val mse net {val_mse()[0]:.4g}")
    meta = {"pairs": pairs, "epochs": epochs, "batch": batch, "lr": lr, "N": N, "A": A, "em_iters": em_iters,
            "train_seed0": TRAIN_SEED0, "init_seed": seed, "final_train_loss": float(np.mean(losses[-50:])),
            "val_mse": val_mse()[0], "val_mse_fbp_input": val_mse()[1]}
    del inputs, labels
    return net, meta


def main(argv=None):
    import argparse
    import json
    import torch
    ap = argparse.ArgumentParser(description="train / evaluate the tEM warm-start U-Net")
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--em-iters", type=int, default=200)
    ap.add_argument("--chunk", type=int, default=256)
    ap.add_argument("--samples", type=int, default=256)
    ap.add_argument("--weights", default=default_weights())
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    if a.cmd == "train":
        net, meta = train_recipe(a.pairs, a.epochs, a.batch, a.lr, em_iters=a.em_iters, chunk=a.chunk, device=dev,
                                 log=lambda m: print(m, flush=True))
        net.save(a.out or a.weights, **meta)
        print(json.dumps(meta), flush=True)
    else:
        net = UNet.from_file(a.weights, dev)
        trans = torch.empty((a.samples, 720, 512), dtype=torch.float32, device=dev)
        for c0 in range(0, a.samples, 64):
            m = min(64, a.samples - c0)
            make_transmissions(m, HELDOUT_SEED0 + c0, dev, chunk=m, out=trans[c0:c0 + m])
        r = evaluate_wall(net, trans, S.uniform_angles(720))
        print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
