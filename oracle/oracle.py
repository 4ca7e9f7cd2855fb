"""ctypes binding of the FP64 CPU oracle (oracle/raft_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker.  The CUDA
product (ssc-raft_b200/sscRaft) never imports this module.

Every function takes numpy arrays in the reference layouts
(sinogram [slices, angles, rays], image [slices, N, N]) and returns float64
results.  See raft_oracle.c for the reference file:line each routine follows.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

MODE_REF = 0
MODE_LIN = 1


def build(force=False):
    """Compile raft_oracle.c into liboracle.so (gcc + OpenMP)."""
    src = os.path.join(HERE, "raft_oracle.c")
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src):
        return LIB_PATH
    cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
           "-o", LIB_PATH, src, "-lm"]
    subprocess.check_call(cmd)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        F = ctypes.c_float
        _lib.oracle_filter_spectrum.argtypes = [I, I, I, D, D, D, D, P, P]
        _lib.oracle_filter_rows.argtypes = [I, I, I, I, I, D, D, D, D, P, P]
        _lib.oracle_lowpass.argtypes = [I, I, I, I, I, D, D, D, P, P]
        _lib.oracle_fbp_backproject.argtypes = [I, I, I, I, I, F, F, P, P, P, P, P]
        _lib.oracle_fbp_backproject_f32.argtypes = [I, I, I, I, I, F, F, P, P, P, P, P]
        _lib.oracle_fbp.argtypes = [I, I, I, I, I, I, D, D, D, F, F, P, P, P, P, P]
        _lib.oracle_fbp_f32.argtypes = [I, I, I, I, I, I, D, D, D, F, F, P, P, P]
        _lib.oracle_radon_rt.argtypes = [I, I, I, I, I, F, F, P, P, P, P, P]
        _lib.oracle_em_forward.argtypes = [I, I, I, I, P, P, P, P, P]
        _lib.oracle_em_backproject.argtypes = [I, I, I, I, P, P, P, P, P]
        _lib.oracle_tem.argtypes = [I, I, I, I, I, P, P, P, P, P, P, P, P]
        _lib.oracle_eem.argtypes = [I, I, I, I, I, P, P, P, P, P, P, P]
        _lib.oracle_tem_metrics.argtypes = [I, I, I, I, P, P, P, P, P, P, P, P]
        _lib.oracle_conv3x3_fwd.argtypes = [P, P, P, P, I, I, I, I, I, I]
        _lib.oracle_conv3x3_wgrad.argtypes = [P, P, P, I, I, I, I, I]
        _lib.oracle_conv3x3_dgrad.argtypes = [P, P, P, I, I, I, I, I]
        _lib.oracle_background.argtypes = [P, P, P, I, I, I, I, I, P]
        _lib.oracle_bst.argtypes = [P, I, I, I, I, I, D, D, I, F, P]
        _lib.oracle_centersino.argtypes = [P, P, P, P, I, I, I]
        _lib.oracle_centersino.restype = D
        _lib.oracle_rotaxis.argtypes = [P, I, I, F, P]
        _lib.oracle_temfq.argtypes = [P, P, P, P, I, I, I, I, I, I, F, P]
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _as3(a):
    a = np.asarray(a)
    return a[None] if a.ndim == 2 else a


def _trig(tr):
    """(cos, sin) float32 arrays to use for the nearest-sample index rule, or
    None for libm's.  Keeps the arrays alive in the returned tuple."""
    if tr is None:
        return None, None, None
    c, s = _f32(tr[0]), _f32(tr[1])
    return (c, s), _p(c), _p(s)


def filter_spectrum(mode, ftype, Np, paganin=0.0, reg=0.0, offset=0.0, pixel=1.0):
    hre = np.zeros(Np)
    him = np.zeros(Np)
    lib().oracle_filter_spectrum(mode, ftype, Np, paganin, reg, offset, pixel, _p(hre), _p(him))
    return hre + 1j * him


def filter_rows(sino, mode, ftype, pad, paganin=0.0, reg=0.0, offset=0.0, pixel=1.0):
    """Filtered, edge-padded rows: [..., Np] float64."""
    s = _f32(sino)
    N = s.shape[-1]
    nrows = s.size // N
    Np = N * (1 + pad)
    q = np.zeros(s.shape[:-1] + (Np,))
    lib().oracle_filter_rows(mode, ftype, N, nrows, pad, paganin, reg, offset, pixel, _p(s), _p(q))
    return q


def lowpass(sino, mode, ftype, pad, paganin=0.0, reg=0.0, pixel=1.0):
    s = _f32(sino)
    N = s.shape[-1]
    out = np.zeros(s.shape)
    lib().oracle_lowpass(mode, ftype, N, s.size // N, pad, paganin, reg, pixel, _p(s), _p(out))
    return out


def fbp(sino, angles, mode, ftype, pad, paganin=0.0, reg=0.0, offset=0.0, pixel=1.0,
        f32=False, trig=None):
    """FBP of sino [B, A, N] -> [B, N, N] (float64, or float32 if f32).
    trig = (cos, sin) overrides libm's values in the nearest-sample index rule."""
    s = _f32(_as3(sino))
    B, A, N = s.shape
    ang = _f32(angles)
    keep, pc, ps = _trig(trig)
    if f32:
        img = np.zeros((B, N, N), dtype=np.float32)
        lib().oracle_fbp_f32(mode, ftype, N, A, B, pad, paganin, reg, offset, pixel, pixel,
                             _p(ang), _p(s), _p(img))
    else:
        img = np.zeros((B, N, N))
        lib().oracle_fbp(mode, ftype, N, A, B, pad, paganin, reg, offset, pixel, pixel,
                         _p(ang), _p(s), _p(img), pc, ps)
    return img


def fbp_backproject(q, angles, mode, N, pad, pixel=1.0, trig=None):
    q = _f64(_as3(q))
    B, A, Np = q.shape
    img = np.zeros((B, N, N))
    keep, pc, ps = _trig(trig)
    lib().oracle_fbp_backproject(mode, N, A, B, pad, pixel, pixel, _p(_f32(angles)), _p(q), _p(img), pc, ps)
    return img


def radon_rt(img, angles, nrays=None, ax=1.0, ay=1.0, trig=None):
    """Radon_RT_version_sscRadon (without the Python-side N*pixel/2 scale)."""
    im = _f32(_as3(img))
    B, ny, nx = im.shape
    nrays = nx if nrays is None else nrays
    ang = _f32(angles)
    out = np.zeros((B, len(ang), nrays))
    keep, pc, ps = _trig(trig)
    lib().oracle_radon_rt(nx, ny, nrays, len(ang), B, ax, ay, _p(ang), _p(im), _p(out), pc, ps)
    return out


def em_forward(img, angles, nrays, trig=None):
    im = _f64(_as3(img))
    B, N, _ = im.shape
    ang = _f32(angles)
    out = np.zeros((B, len(ang), nrays))
    keep, pc, ps = _trig(trig)
    lib().oracle_em_forward(N, nrays, len(ang), B, _p(ang), _p(im), _p(out), pc, ps)
    return out


def em_backproject(sino, angles, N, trig=None):
    s = _f64(_as3(sino))
    ang = _f32(angles)
    B, A, nrays = s.shape
    img = np.zeros((B, N, N))
    keep, pc, ps = _trig(trig)
    lib().oracle_em_backproject(N, nrays, A, B, _p(ang), _p(s), _p(img), pc, ps)
    return img


def em_backproject_ones(angles, N, nrays, nslices=1, trig=None):
    ang = _f32(angles)
    img = np.zeros((nslices, N, N))
    keep, pc, ps = _trig(trig)
    lib().oracle_em_backproject(N, nrays, len(ang), nslices, _p(ang), None, _p(img), pc, ps)
    return img


def tem(counts_exp, flat, angles, niter, obj=None, fwd_trig=None, bp_trig=None):
    """tEM on counts already mapped through exp(-x) (em_methods.py:109).
    fwd_trig / bp_trig: (cos, sin) for the projector and the backprojector."""
    c = _f32(_as3(counts_exp))
    B, A, nrays = c.shape
    N = nrays
    fl = _f32(np.asarray(flat).reshape(B, nrays))
    o = np.ones((B, N, N)) if obj is None else _f64(_as3(obj)).copy()
    k1, fc, fs = _trig(fwd_trig)
    k2, bc, bs = _trig(bp_trig)
    lib().oracle_tem(N, nrays, A, B, niter, _p(_f32(angles)), _p(c), _p(fl), _p(o), fc, fs, bc, bs)
    return o


def eem(tomo, angles, niter, obj=None, fwd_trig=None, bp_trig=None):
    t = _f32(_as3(tomo))
    B, A, nrays = t.shape
    N = nrays
    o = np.ones((B, N, N)) if obj is None else _f64(_as3(obj)).copy()
    k1, fc, fs = _trig(fwd_trig)
    k2, bc, bs = _trig(bp_trig)
    lib().oracle_eem(N, nrays, A, B, niter, _p(_f32(angles)), _p(t), _p(o), fc, fs, bc, bs)
    return o


def tem_metrics(counts_exp, flat, angles, obj, fwd_trig=None):
    c = _f32(_as3(counts_exp))
    B, A, nrays = c.shape
    N = nrays
    fl = _f32(np.asarray(flat).reshape(B, nrays))
    o = _f64(_as3(obj))
    res = np.zeros(B)
    nll = np.zeros(B)
    k1, fc, fs = _trig(fwd_trig)
    lib().oracle_tem_metrics(N, nrays, A, B, _p(_f32(angles)), _p(c), _p(fl), _p(o), _p(res), _p(nll),
                             fc, fs)
    return res, nll


# ----------------------------------------------------------- U-Net convs --
def conv3x3(x, w, b=None, relu=False):
    """x [N,H,W,Cin], w [Cout,3,3,Cin] -> y [N,H,W,Cout], FP64."""
    x, w = _f64(x), _f64(w)
    N, H, W, Cin = x.shape
    Cout = w.shape[0]
    y = np.zeros((N, H, W, Cout))
    bb = None if b is None else _f64(b)
    lib().oracle_conv3x3_fwd(_p(x), _p(w), None if bb is None else _p(bb), _p(y), N, H, W, Cin, Cout, int(relu))
    return y


def conv3x3_wgrad(dy, x):
    dy, x = _f64(dy), _f64(x)
    N, H, W, Cout = dy.shape
    Cin = x.shape[-1]
    dw = np.zeros((Cout, 3, 3, Cin))
    lib().oracle_conv3x3_wgrad(_p(dy), _p(x), _p(dw), N, H, W, Cin, Cout)
    return dw


def conv3x3_dgrad(dy, w):
    dy, w = _f64(dy), _f64(w)
    N, H, W, Cout = dy.shape
    Cin = w.shape[-1]
    dx = np.zeros((N, H, W, Cin))
    lib().oracle_conv3x3_dgrad(_p(dy), _p(w), _p(dx), N, H, W, Cin, Cout)
    return dx


def background(frames, flat, dark, is_log):
    """Flat/dark correction (+ -log), background_correction.cu:15-47 / opt.cu:196-214.
    frames [B, A, N], flat [B, F, N] (or [B, N]), dark [B, N]; FP64 result."""
    fr = _as3(_f32(frames))
    B, A, N = fr.shape
    fl = _f32(flat).reshape(B, -1, N)
    dk = _f32(dark).reshape(B, N)
    out = np.empty((B, A, N), np.float64)
    lib().oracle_background(_p(fr), _p(np.ascontiguousarray(fl)), _p(dk), N, A, B, fl.shape[1], int(bool(is_log)),
                            _p(out))
    return out.reshape(np.shape(frames))


def bst(tomo, ftype, pad, paganin=0.0, reg=0.0, offset=0, pixel=1.0):
    """FBP by the backprojection slice theorem (bst.cu:251-312, 534-642 and
    filters.cu:295-390); tomo [B, A, N] -> [B, N, N] FP64.  offset: integer
    axis offset (the reference truncates it)."""
    t = _as3(_f32(tomo))
    B, A, N = t.shape
    out = np.empty((B, N, N), np.float64)
    lib().oracle_bst(_p(t), N, A, B, int(pad), int(ftype), float(paganin), float(reg), int(offset), float(pixel),
                     _p(out))
    return out if np.ndim(tomo) == 3 else out[0]


def centersino(frame0, frame180, dark, flat, subpixel=False):
    """Rotation-axis offset by phase correlation (rotation_axis.cu:14-46,221-360):
    the reference's integer (int) or sub-pixel (float) result."""
    fr = [_f32(a) for a in (frame0, frame180, dark, flat)]
    sy, sx = fr[0].shape
    v = lib().oracle_centersino(*[_p(a) for a in fr], sx, sy, int(bool(subpixel)))
    return float(v) if subpixel else int(v)


def rotaxis(tomo, offset):
    """Sub-pixel axis shift of every row (rotation_axis.cu:455-526); FP64 result."""
    t = _f32(tomo)
    N = t.shape[-1]
    out = np.empty(t.shape, np.float64)
    lib().oracle_rotaxis(_p(t), N, int(t.size // N), float(offset), _p(out))
    return out


def temfq(counts, flat, angles, zpad, interp, niter, obj=None, dx=0.0, trig=None):
    """tEMFQ (em_frequency.cu:13-87 with radon_fst.cu:544-637 and bst.cu:100-249):
    counts [B, A, N], flat [B, N], niter iterations from obj (default ones);
    trig = (cos, sin) of the angles as the GPU computes them (default libm's)."""
    c = _as3(_f32(counts))
    B, A, N = c.shape
    fl = _f32(flat).reshape(B, N)
    if trig is None:
        a = np.asarray(angles, np.float32)
        cs, sn = np.cos(a).astype(np.float32), np.sin(a).astype(np.float32)
    else:
        cs, sn = _f32(trig[0]), _f32(trig[1])
    x = np.ones((B, N, N), np.float64) if obj is None else _f64(obj).reshape(B, N, N).copy()
    lib().oracle_temfq(_p(c), _p(fl), _p(cs), _p(sn), N, A, B, int(zpad), int(interp), int(niter), float(dx), _p(x))
    return x
