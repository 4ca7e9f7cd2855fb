"""Generate golden fixtures by running the REFERENCE ssc-raft CUDA library.

Runs on a GPU box: loads oracle/_ref/libraft_ref.so (built from the
reference sources by oracle/build_ref.sh) and calls its own C ABI
(getFBPMultiGPU, getFilterLowPassMultiGPU, getRadonRTMultiGPU,
get_tEM_RT_MultiGPU, get_eEM_RT_MultiGPU, getBackgroundCorrectionMultiGPU, getBSTMultiGPU,
the rotation-axis finders and correction, get_tEM_FQ_MultiGPU)
with the packing of the reference Python wrappers, on small seeded inputs.
Inputs and outputs are saved together in tests/golden/ref_<case>.npz (or
under --out); --only PREFIX writes only the cases whose names start with it.

    python tests/golden/make_golden.py [--out DIR] [--only PREFIX]
"""
import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "ssc-raft_b200"))
sys.path.insert(0, os.path.join(REPO, "tests"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

from helpers import fbp_params, phantom_case, sino_case, temfq_counts  # noqa: E402


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def load_ref():
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libraft_ref.so"))
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    lib.getFBPMultiGPU.argtypes = [P, I, P, P, P, P, P]
    lib.getFilterLowPassMultiGPU.argtypes = [P, I, P, P, P]
    lib.getRadonRTMultiGPU.argtypes = [P, I, P, P, P, I, I, I, I, I, F, F]
    lib.get_tEM_RT_MultiGPU.argtypes = [P, I, P, P, P, P, P, P]
    lib.get_eEM_RT_MultiGPU.argtypes = [P, I, P, P, P, P, P]
    lib.getBackgroundCorrectionMultiGPU.argtypes = [P, I, P, P, P, I, I, I, I, I, I]
    lib.getBSTMultiGPU.argtypes = [P, I, P, P, P, P, P, I]
    lib.findcentersino.argtypes = [P, P, P, P, I, I]
    lib.findcentersino.restype = I
    lib.findcentersino16.argtypes = [P, P, P, P, I, I]
    lib.findcentersino16.restype = I
    lib.findcentersino_subpixel.argtypes = [P, P, P, P, I, I]
    lib.findcentersino_subpixel.restype = F
    lib.getRotAxisCorrectionMultiGPU.argtypes = [P, I, P, F, I, I, I, I]
    lib.get_tEM_FQ_MultiGPU.argtypes = [P, I, P, P, P, P, P, P]
    return lib


GPUS = np.array([0], np.intc)

# (name, N, A, nslices, pad, ftype, pixel, offset, reg, angle_span)
FBP_CASES = [
    ("fbp_ramp_n64", 64, 90, 2, 2, 7, 1.0, 0.0, 0.0, np.pi),
    ("fbp_hann_off", 96, 120, 2, 2, 5, 1.0, 3.5, 0.0, np.pi),
    ("fbp_hamming_px", 50, 64, 1, 2, 6, 0.5, 1.25, 0.0, np.pi),
    ("fbp_ramp_pad1_2pi", 80, 100, 1, 1, 7, 1.0, 0.0, 0.0, 2 * np.pi),
    ("fbp_none", 64, 60, 1, 2, 0, 1.0, 0.0, 0.0, np.pi),
    ("fbp_gaussian", 64, 45, 1, 2, 1, 1.0, 0.0, 2.0, np.pi),
    ("fbp_lorentz", 64, 45, 1, 2, 2, 1.0, -2.0, 3.0, np.pi),
    ("fbp_cosine", 64, 45, 1, 2, 3, 1.0, 0.0, 0.0, np.pi),
    ("fbp_rectangle", 64, 45, 1, 2, 4, 1.0, 0.0, 1.5, np.pi),
    ("fbp_ramp_pad0_odd", 63, 37, 1, 0, 7, 1.0, 0.0, 0.0, np.pi),
    ("fbp_ramp_n200", 200, 180, 1, 2, 7, 1.0, 0.0, 0.0, np.pi),
]


def fbp_case(lib, name, N, A, B, pad, ftype, pixel, offset, reg, span, seed):
    ang = (np.arange(A, dtype=np.float64) * (span / A)).astype(np.float32)
    sino, _ = sino_case(N, A, B, seed=seed, pixel=pixel, angles=ang)
    pf, pi = fbp_params(N, A, B, pad=pad, ftype=ftype, pixel=pixel, offset=offset, reg=reg, blocksize=B)
    obj = np.zeros((B, N, N), np.float32)
    s = sino.copy()
    lib.getFBPMultiGPU(ptr(GPUS), 1, ptr(obj), ptr(s), ptr(ang), ptr(pf), ptr(pi))
    return dict(kind="fbp", sino=sino, angles=ang, paramf=pf, parami=pi, out=obj)


def index_probe(lib, N, pad, pixel, thetas):
    """Filter 'none', two angles (theta, theta + 2^-10), bin values = bin index
    on the first row: the output is exactly idx(theta) * 2^-10 per pixel."""
    Np = N * (1 + pad)
    off = (pad * N) // 2
    out = []
    for th in thetas:
        ang = np.array([th, th + 2.0 ** -10], np.float32)
        sino = np.zeros((1, 2, N), np.float32)
        # padded bin b holds sino[clamp(b - off)]: make the raw row encode b for b in [off, off+N)
        sino[0, 0, :] = np.arange(N, dtype=np.float32) + off
        pf, pi = fbp_params(N, 2, 1, pad=pad, ftype=0, pixel=pixel)
        obj = np.zeros((1, N, N), np.float32)
        lib.getFBPMultiGPU(ptr(GPUS), 1, ptr(obj), ptr(sino), ptr(ang), ptr(pf), ptr(pi))
        out.append(obj[0])
    return dict(kind="index_probe", N=N, pad=pad, pixel=pixel, thetas=np.asarray(thetas, np.float32),
                out=np.stack(out), Np=Np)


def background_case(lib, B, A, N, nflats, is_log, seed):
    """Raw frames from a phantom's projections: dark + (flat - dark) * exp(-p)
    plus noise, some samples below the dark (the 0.5 clamp) and above the flat."""
    rng = np.random.default_rng(seed)
    sino, ang = sino_case(N, A, B, seed=seed)
    p = sino / max(float(sino.max()), 1e-6) * 2.5
    flat = rng.uniform(800.0, 1200.0, (B, nflats, N)).astype(np.float32)
    dark = rng.uniform(50.0, 150.0, (B, N)).astype(np.float32)
    w = (np.arange(A, dtype=np.float64) / A)[None, :, None]
    ft = flat[:, :1, :] * (1 - w) + w * flat[:, min(1, nflats - 1):min(1, nflats - 1) + 1, :]
    frames = dark[:, None, :] + (ft - dark[:, None, :]) * np.exp(-p) + rng.normal(0, 5.0, (B, A, N))
    frames[:, ::7, ::5] = dark[:, None, ::5] - 20.0        # below the dark: clamped to 0.5
    frames[:, 3::11, 2::9] += 400.0                       # above the flat
    frames = frames.astype(np.float32)
    out = frames.copy()
    lib.getBackgroundCorrectionMultiGPU(ptr(GPUS), 1, ptr(out), ptr(flat), ptr(dark), N, A, B, nflats, is_log, 0)
    return dict(kind="background", frames=frames, flat=flat, dark=dark, is_log=is_log, out=out)


# BST cases (name, N, nslices, pad, ftype, integer offset, reg); nangles == N, the
# setting in which the reference's padding call (sized by N rows) covers every row.
BST_CASES = [
    ("bst_ramp_n64", 64, 2, 2, 7, 0, 0.0),
    ("bst_hann_off2_n96", 96, 1, 2, 5, 2, 0.0),
    ("bst_none_pad1_n64", 64, 1, 1, 0, 0, 0.0),
    ("bst_gauss_n80", 80, 1, 2, 1, -1, 2.0),
]


def bst_case(lib, name, N, B, pad, ftype, offset, reg, seed):
    """One BST case through the reference's getBSTMultiGPU.  Run in a fresh
    process: the reference zero-pads its half-rays with freshly allocated,
    never-cleared device memory, which a new process receives zeroed."""
    A = N
    ang = np.linspace(0.0, np.pi, A, endpoint=False).astype(np.float32)
    sino, _ = sino_case(N, A, B, seed=seed, angles=ang)
    pf, pi = fbp_params(N, A, B, pad=pad, ftype=ftype, offset=float(offset), reg=reg)
    obj = np.zeros((B, N, N), np.float32)
    t = sino.copy()
    lib.getBSTMultiGPU(ptr(GPUS), 1, ptr(obj), ptr(t), ptr(ang), ptr(pf), ptr(pi), 0)
    return dict(kind="bst", sino=sino, angles=ang, paramf=pf, parami=pi, out=obj)


def frame_pair(sizex, sizey, axis, seed):
    """Raw 0 and 180 degree frames [sizey][sizex] of a smooth random object whose
    rotation axis sits at ray `axis` (the 180 degree frame is the 0 degree one
    mirrored about it), with flat 1e4 + 100, dark 100 and Poisson noise."""
    rng = np.random.default_rng(seed)
    x = np.arange(sizex, dtype=np.float64)
    p0 = np.zeros((sizey, sizex))
    for _ in range(6):
        c, w, a = rng.uniform(0.3, 0.7) * sizex, rng.uniform(4, 20), rng.uniform(0.2, 1.0)
        tilt = rng.uniform(0.5, 1.5, sizey)[:, None]
        p0 += a * tilt * np.exp(-((x[None, :] - c) ** 2) / (2 * w * w))
    p180 = np.array([np.interp(2 * axis - x, x, r) for r in p0])
    dark = np.full((sizey, sizex), 100.0)
    flat = dark + 1e4
    f0 = dark + rng.poisson(1e4 * np.exp(-p0))
    f1 = dark + rng.poisson(1e4 * np.exp(-p180))
    return [a.astype(np.float32) for a in (f0, f1, dark, flat)]


ROT_CASES = [("rot_256x128", 256, 128, 131.0), ("rot_240x96", 240, 96, 111.5), ("rot_160x64", 160, 64, 84.0)]


def rot_case(lib, name, sizex, sizey, axis, seed):
    f0, f1, dk, ft = frame_pair(sizex, sizey, axis, seed)
    c = lib.findcentersino(ptr(f0), ptr(f1), ptr(dk), ptr(ft), sizex, sizey)
    sp = lib.findcentersino_subpixel(ptr(f0), ptr(f1), ptr(dk), ptr(ft), sizex, sizey)
    u = [a.astype(np.uint16) for a in (f0, f1, dk, ft)]
    c16 = lib.findcentersino16(*[ptr(a) for a in u], sizex, sizey)
    return dict(kind="centersino", frame0=f0, frame180=f1, dark=dk, flat=ft, out=np.int32(c),
                out_subpixel=np.float32(sp), out16=np.int32(c16))


def rotaxis_case(lib, seed):
    tomo, _ = sino_case(64, 10, 2, seed=seed)
    out = {}
    for off in (1.7, -2.3):
        t = tomo.copy()
        lib.getRotAxisCorrectionMultiGPU(ptr(GPUS), 1, ptr(t), off, 64, 10, 2, 0)
        out[f"out_{off:+.1f}"] = t
    return dict(kind="rotaxis", tomo=tomo, offsets=np.array([1.7, -2.3], np.float32),
                out_a=out["out_+1.7"], out_b=out["out_-2.3"])


# (name, N, A, nslices, zpad, interpolation, iterations, dx).  Sizes keep N^2 B,
# N A B, N (1+zpad) A and N (1+zpad) A B / 2 multiples of 1024 (the reference's
# element-wise grids are size/1024 blocks and skip a tail otherwise), zpad with
# a convBST grid that covers every sampled frequency, angles k pi / A in [0, pi)
# with A not a multiple of 3 (no cos/sin of exactly 1/2, so nearest-neighbour
# rounding never meets a tie that the GPU's fast cosine could break otherwise).
TEMFQ_CASES = [
    ("temfq_n64_z1_bilinear", 64, 64, 2, 1, 1, 4, 0.02),
    ("temfq_n64_z1_nearest", 64, 64, 1, 1, 0, 3, 0.02),
    ("temfq_n64_z2_bilinear", 64, 64, 2, 2, 1, 3, 0.02),
    ("temfq_n128_z3_nearest", 128, 80, 1, 3, 0, 2, 0.01),
]


def temfq_case(lib, name, N, A, B, zpad, interp, niter, dx, seed):
    """One tEMFQ case through the reference's get_tEM_FQ_MultiGPU, packed as
    tEMFQ_GPU_ (em_methods.py:154-232) packs it, initial guess ones.  Run in a
    fresh process, like the BST cases (the half-ray padding is never-cleared
    device memory)."""
    counts, flat, ang = temfq_counts(N, A, B, dx, seed)
    obj = np.ones((B, N, N), np.float32)
    pi = np.array([N, A, B, N, zpad, 0, 0, B, niter, interp, 0], np.int32)
    pf = np.array([dx, dx, 0.0], np.float32)
    c, f = counts.copy(), flat.copy()
    lib.get_tEM_FQ_MultiGPU(ptr(GPUS), 1, ptr(c), ptr(obj), ptr(ang), ptr(f), ptr(pf), ptr(pi))
    return dict(kind="temfq", counts=counts, flat=flat, angles=ang, zpad=np.int32(zpad), interpolation=np.int32(interp),
                iterations=np.int32(niter), dx=np.float32(dx), out=obj)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default="")
    ap.add_argument("--bst-case", default="", help=argparse.SUPPRESS)
    ap.add_argument("--temfq-case", default="", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.temfq_case:
        i = [c[0] for c in TEMFQ_CASES].index(args.temfq_case)
        d = temfq_case(load_ref(), *TEMFQ_CASES[i], seed=1100 + i)
        np.savez_compressed(os.path.join(args.out, f"ref_{args.temfq_case}.npz"), **d)
        return
    if args.only.startswith("temfq"):
        import subprocess
        for c in TEMFQ_CASES:
            if c[0].startswith(args.only):
                subprocess.run([sys.executable, os.path.abspath(__file__), "--out", args.out, "--temfq-case", c[0]],
                               check=True)
        print("wrote", len([c for c in TEMFQ_CASES if c[0].startswith(args.only)]), "tEMFQ fixtures to", args.out)
        return
    if args.bst_case:
        i = [c[0] for c in BST_CASES].index(args.bst_case)
        d = bst_case(load_ref(), *BST_CASES[i], seed=800 + i)
        np.savez_compressed(os.path.join(args.out, f"ref_{args.bst_case}.npz"), **d)
        return
    if args.only.startswith("bst"):
        import subprocess
        for c in BST_CASES:
            if c[0].startswith(args.only):
                subprocess.run([sys.executable, os.path.abspath(__file__), "--out", args.out, "--bst-case", c[0]],
                               check=True)
        print("wrote", len([c for c in BST_CASES if c[0].startswith(args.only)]), "BST fixtures to", args.out)
        return
    os.makedirs(args.out, exist_ok=True)
    lib = load_ref()
    cases = {}
    for i, c in enumerate(FBP_CASES):
        cases[c[0]] = fbp_case(lib, *c, seed=100 + i)
    # index probes (bit-exact nearest-sample rule)
    rng = np.random.default_rng(7)
    th = np.concatenate([[0.0, np.pi / 4, np.pi / 2, 1.0], rng.uniform(0, np.pi, 12)])
    cases["probe_px1"] = index_probe(lib, 48, 2, 1.0, th)
    cases["probe_px07"] = index_probe(lib, 40, 1, 0.7, th[:8])
    # lowpass
    for name, N, A, pad, ftype in (("lowpass_ramp", 64, 30, 2, 7), ("lowpass_hann_pad1", 72, 24, 1, 5)):
        sino, ang = sino_case(N, A, 2, seed=300)
        pf, pi = fbp_params(N, A, 2, pad=pad, ftype=ftype)
        t = sino.copy()
        lib.getFilterLowPassMultiGPU(ptr(GPUS), 1, ptr(t), ptr(pf), ptr(pi))
        cases[name] = dict(kind="lowpass", sino=sino, angles=ang, paramf=pf, parami=pi, out=t)
    # Radon RT
    img = phantom_case(64, 2, seed=400)
    ang = (np.arange(90) * (np.pi / 90)).astype(np.float32)
    proj = -np.ones((2, 90, 64), np.float32)
    lib.getRadonRTMultiGPU(ptr(GPUS), 1, ptr(proj), ptr(img), ptr(ang), 64, 64, 64, 90, 2, 1.0, 1.0)
    cases["radon_n64"] = dict(kind="radon", img=img, angles=ang, out=proj)
    # tEM: blocksize == nangles == nslices and a constant flat, the setting in which the
    # reference's angle-indexed flat buffer (em_rt.cu:107,134) is fully initialised
    N, A, B, it = 48, 32, 32, 4
    img = phantom_case(N, B, seed=500, scale=0.02)
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    import oracle as O  # only to make the transmission data from a forward projection
    p = O.em_forward(img.astype(np.float64), ang, N)
    counts = np.exp(-p).astype(np.float32)            # exp(-data) as em_methods.py:109 produces
    flat = np.ones((B, N), np.float32)
    obj = np.ones((B, N, N), np.float32)
    pi = np.array([N, A, B, N, 0, 0, 0, B, it, A], np.int32)
    pf = np.array([0], np.float32)
    c = counts.copy()
    lib.get_tEM_RT_MultiGPU(ptr(GPUS), 1, ptr(obj), ptr(c), ptr(flat), ptr(ang), ptr(pf), ptr(pi))
    cases["tem_n48"] = dict(kind="tem", counts=counts, flat=flat, angles=ang, iterations=it, out=obj)
    # eEM
    N, A, B, it = 48, 40, 2, 5
    img = phantom_case(N, B, seed=600)
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    tomo = O.em_forward(img.astype(np.float64), ang, N).astype(np.float32)
    obj = np.ones((B, N, N), np.float32)
    pi = np.array([N, A, B, N, 0, 0, 0, 1, it, 0], np.int32)
    t = tomo.copy()
    lib.get_eEM_RT_MultiGPU(ptr(GPUS), 1, ptr(obj), ptr(t), ptr(ang), ptr(pf), ptr(pi))
    cases["eem_n48"] = dict(kind="eem", tomo=tomo, angles=ang, iterations=it, out=obj)
    # flat/dark correction: two flats + log (odd row length), one flat no log, three flats + log
    cases["bg_log_2flats"] = background_case(lib, 3, 50, 70, 2, 1, seed=700)
    cases["bg_nolog_1flat"] = background_case(lib, 2, 33, 64, 1, 0, seed=701)
    cases["bg_log_3flats"] = background_case(lib, 2, 20, 40, 3, 1, seed=702)
    # rotation axis: finders on frame pairs with known axes, sub-pixel axis correction
    for i, (name, sx, sy, axis) in enumerate(ROT_CASES):
        cases[name] = rot_case(lib, name, sx, sy, axis, seed=900 + i)
    cases["rotaxis_n64"] = rotaxis_case(lib, seed=950)
    # the fast-intrinsic sin/cos values the reference's index rules use, as data
    # for the oracle: kind 0 = __sinf/__cosf, kind 1 = __sincosf
    from sscRaft.rafttypes import fast_sincos
    for name, d in cases.items():
        if "angles" in d:
            d["fcos"], d["fsin"] = fast_sincos(d["angles"], 0)
            d["bcos"], d["bsin"] = fast_sincos(d["angles"], 1)
        elif d["kind"] == "index_probe":
            allang = np.concatenate([[t, np.float32(t) + np.float32(2.0 ** -10)] for t in d["thetas"]])
            allang = allang.astype(np.float32)
            d["fcos"], d["fsin"] = fast_sincos(allang, 0)
    cases = {k: v for k, v in cases.items() if k.startswith(args.only)}
    for name, d in cases.items():
        np.savez_compressed(os.path.join(args.out, f"ref_{name}.npz"), **d)
    print("wrote", len(cases), "fixtures to", args.out)


if __name__ == "__main__":
    main()
