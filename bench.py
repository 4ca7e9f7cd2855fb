"""Benchmark: batched parallel-beam FBP at 2048^2 x 1800 angles.

Workload (one "step"): FBP of a 512-slice volume, 2048 detector bins, 1800
angles over [0, pi), rotation-axis offset +3.5 px, Hann filter, padding 2,
synthetic data (50 seeded random ellipses per slice, Poisson noise at
I0 = 1e4 photons/ray, converted to -log transmission).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:      `value` = slices/s with the sinogram already resident in HBM
           (raft_fbp_device), `e2e` = slices/s through the public drop-in API
           sscRaft.fbp (-> getFBPMultiGPU) with pinned host buffers, H2D and
           D2H inside the timed region.  Headline operator: the reference's
           nearest-sample FBP (bit-faithful index rule), FP32.  The linear-
           interpolation operator (FP32 and BF16 storage) is reported under
           "variants".
reference: the reference's own CUDA library (oracle/_ref/libraft_ref.so, built
           from its sources for sm_100a) through its C ABI getFBPMultiGPU with
           host buffers, on a bounded sample of the same workload.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "ssc-raft_b200"))

N_RAYS, N_ANGLES, N_SLICES = 2048, 1800, 512
OFFSET, PAD, FILTER_ID = 3.5, 2, 5          # Hann
I0 = 1.0e4
# DRAM bytes (read + write) of one 32-slice nearest backprojector launch at
# 2048^2 x 1800 angles (four slices per CTA on slice-interleaved rows),
# measured with ncu (1.08x the algorithmic bytes).
BP_TRAFFIC_PER_LAUNCH = 783_763_456 + 518_802_944
WORKLOAD = ("batched FBP: 512 slices x 2048^2, 1800 angles over [0,pi), 2048 bins, "
            "axis offset +3.5 px, Hann, padding 2")
METRIC = "FBP slices/s at 2048^2 x 1800 angles"
DATA = ("synthetic: 50 seeded random ellipses per slice, exact projections, Poisson I0=1e4, "
        "-log transmission (no public dataset exists for this path)")


def bench_config(ws):
    """The `config` of both arms' lines (identical: the same workload; each
    line's `slices_per_step` says how many of its slices one step covers)."""
    return {"workload": WORKLOAD, "operator": "nearest-sample FBP (the reference's index rule), FP32",
            "parallelism": f"slab x{ws}, no collective",
            "l2": "inputs 7.5 GB/GPU > 126 MB L2: no flush needed"}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x, device=None):
    """Max of a per-rank float over all ranks (the timing reduction); identity
    without an initialised process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def slice_seed_base(rank, nslices):
    """Per-rank seed base: every rank reconstructs its own distinct slices."""
    return 2_000_000 + rank * nslices


# ------------------------------------------------------------------ data --
def synthetic_module():
    """sscRaft/synthetic.py (numpy only) loaded by its file path, so that
    making inputs does not import the sscRaft package and load its library
    (the reference arm must map no library of this repository)."""
    import importlib.util
    name = "raft_bench_synthetic"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            name, os.path.join(REPO, "ssc-raft_b200", "sscRaft", "synthetic.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules[name] = mod
    return sys.modules[name]


def make_sinograms_gpu(nslices, seed_base, device):
    """Exact ellipse projections (50 ellipses/slice) + Poisson noise, on the GPU."""
    import torch
    S = synthetic_module()
    ang = S.uniform_angles(N_ANGLES)
    th = torch.as_tensor(ang.astype(np.float64), device=device)[None, :, None]
    R = N_RAYS / 2.0
    c0 = (PAD * N_RAYS) // 2 - N_RAYS * (1 + PAD) / 2.0
    t = ((torch.arange(N_RAYS, device=device, dtype=torch.float64) + c0) / R)[None, None, :]
    cth, sth = torch.cos(th), torch.sin(th)
    out = torch.empty((nslices, N_ANGLES, N_RAYS), dtype=torch.float32, device=device)
    gen = torch.Generator(device=device)
    for k in range(nslices):
        prm = torch.as_tensor(S.ellipse_params(seed_base + k, 50), device=device)
        x0, y0, a, b, phi, rho = [prm[:, i][:, None, None] for i in range(6)]
        c = cth * torch.cos(phi) - sth * torch.sin(phi)
        s = sth * torch.cos(phi) + cth * torch.sin(phi)
        s2 = (a * c) ** 2 + (b * s) ** 2
        tau = t - (x0 * cth - y0 * sth)
        p = (rho * 2.0 * a * b * torch.sqrt(torch.clamp(s2 - tau * tau, min=0.0)) / s2).sum(0) * R
        sc = 3.0 / float(p.max())
        gen.manual_seed(seed_base + k)
        counts = torch.poisson(I0 * torch.exp(-p * sc), generator=gen)
        out[k] = (-torch.log(torch.clamp(counts, min=1.0) / I0)).float()
    return out, ang


def fbp_params(nslices, blocksize=0):
    pi = np.array([N_RAYS, N_ANGLES, nslices, N_RAYS, PAD, 0, 0, FILTER_ID, 0, blocksize], np.int32)
    pf = np.array([0.0, 0.0, 1.0, 0.0, 1.0, 1.0, OFFSET], np.float32)
    return pf, pi


# ------------------------------------------------------------- EM data --
EM_N, EM_A, EM_SLICES, EM_ITERS, EM_I0 = 1024, 900, 64, 100, 1.0e4


def make_tem_data(nslices, seed_base, device, N=EM_N, A=EM_A, I0=EM_I0, n_ell=20, radon_lib=None):
    """Transmission data: ellipse phantoms with attenuation U[0,0.02] per pixel,
    projected with the library's own ray-tracing Radon transform (same geometry
    as the EM forward operator when nrays = N), each slice scaled so that its
    largest line integral is 3 (transmission >= 5%; unscaled 1024-pixel paths
    reach ~20 and starve the detector at I0 = 1e4), Poisson counts at flat I0,
    returned as transmission max(counts,1)/I0 (what tEM consumes after the
    wrapper's exp(-x)) together with the phantom in EM units.  `radon_lib`:
    another library with the same getRadonRTMultiGPU export (the reference
    arm passes the reference's) instead of this package's."""
    import torch
    S = synthetic_module()
    if radon_lib is None:
        from sscRaft.rafttypes import libraft, check_error
    else:
        libraft, check_error = radon_lib, (lambda what: None)

    def _ptr(a):
        return a.ctypes.data_as(ctypes.c_void_p)
    ang = S.uniform_angles(A)
    imgs = torch.stack([S.phantom_image(S.ellipse_params(seed_base + k, n_ell, intensity=(0.0, 0.02)), N,
                                        xp=torch, device=device) for k in range(nslices)]).cpu().numpy()
    # EM units: the forward operator sums x * dt per pixel step, dt = 2/(N-1)
    x_true = imgs * ((N - 1) / 2.0)
    proj = -np.ones((nslices, A, N), np.float32)
    g = np.array([0 if device.index is None else device.index], np.intc)
    libraft.getRadonRTMultiGPU(_ptr(g), 1, _ptr(proj), _ptr(np.ascontiguousarray(x_true)), _ptr(ang),
                               N, N, N, A, nslices, 1.0, 1.0)
    check_error("radon")
    sc = 3.0 / np.maximum(proj.reshape(nslices, -1).max(1), 1e-12)
    proj *= sc[:, None, None].astype(np.float32)
    x_true *= sc[:, None, None].astype(np.float32)
    p = torch.from_numpy(proj).to(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed_base)
    counts = torch.poisson(I0 * torch.exp(-p.double()), generator=gen)
    trans = (torch.clamp(counts, min=1.0) / I0).float()
    return trans, ang, x_true


def run_tem(local, dev, nslices=EM_SLICES, iters=EM_ITERS, warm_iters=3):
    """Plain tEM from a uniform start, the loop captured as one CUDA graph,
    device-resident; returns timing and the per-iteration data residual."""
    import torch
    from sscRaft.rafttypes import libraft, check_error, _ptr
    trans, ang, _ = make_tem_data(nslices, 3_000_000, dev)
    flat = torch.ones((nslices, EM_N), dtype=torch.float32, device=dev)
    obj = torch.ones((nslices, EM_N, EM_N), dtype=torch.float32, device=dev)
    met = torch.zeros((iters, nslices, 3), dtype=torch.float64, device=dev)
    angp = np.ascontiguousarray(ang)
    st = torch.cuda.current_stream(dev).cuda_stream

    def em(n, m):
        rc = libraft.raft_em_device(0, local, ctypes.c_void_p(obj.data_ptr()), ctypes.c_void_p(trans.data_ptr()),
                                    ctypes.c_void_p(flat.data_ptr()), _ptr(angp), EM_N, EM_A, nslices, n,
                                    ctypes.c_void_p(m.data_ptr()) if m is not None else None, 1, ctypes.c_void_p(st))
        if rc:
            check_error("raft_em_device")

    em(warm_iters, None)
    torch.cuda.synchronize()
    obj.fill_(1.0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    em(iters, met)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    m = met.cpu().numpy()
    res = np.sqrt(m[:, :, 0].sum(1)) / np.sqrt(m[:, :, 1].sum(1))
    upd = 2.0 * nslices * EM_N * EM_N * EM_A * iters
    return {"workload": f"tEM {nslices} x {EM_N}^2, {EM_A} angles x {EM_N} bins, flat I0=1e4, "
                        f"{iters} iterations from a uniform start, one CUDA graph; ellipse attenuation "
                        f"U[0,0.02]/px scaled per slice to a maximum line integral of 3",
            "ms_total": ms, "ms_per_iteration": ms / iters, "gups": upd / (ms / 1e3) / 1e9,
            "residual_first": float(res[0]), "residual_last": float(res[-1]),
            "metrics": "FP64 data residual ||flat*exp(-Ax)-y||/||y|| and Poisson NLL per iteration"}


def run_radon(dev, sm_mhz, nslices=EM_SLICES, reps=5, warm=3):
    """Radon transform (the ray-driven Radon_RT projector of getRadonRTMultiGPU)
    of nslices seeded random 1024^2 images at 900 angles x 1024 bins.
    Device-resident through raft_radon_device (slice-interleaved re-layout +
    projector; median of reps CUDA-event timings) and end to end through
    getRadonRTMultiGPU with pinned host buffers.  Roofline: one sample-update
    moves 4 B through the L1/shared-memory data pipe (a 32-byte sector serves
    8 slices) and costs one FP32 add -- the gather roofline of the
    backprojector."""
    import torch
    from sscRaft.rafttypes import libraft, check_error, _ptr
    N, A = EM_N, EM_A
    g = torch.Generator(device=dev).manual_seed(4242)
    img = torch.rand((nslices, N, N), generator=g, device=dev)
    out = torch.empty((nslices, A, N), device=dev)
    ang = np.ascontiguousarray(np.linspace(0.0, np.pi, A, endpoint=False).astype(np.float32))
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    times = []
    for r in range(warm + reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rc = libraft.raft_radon_device(dev.index or 0, p(out), p(img), _ptr(ang), N, N, N, A, nslices, 1.0, 1.0, st)
        e1.record()
        if rc:
            check_error("raft_radon_device")
        torch.cuda.synchronize(dev)
        if r >= warm:
            times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    upd = float(nslices) * A * N * N
    gups = upd / (ms / 1e3) / 1e9
    peak = gather_peak_gups(4, 1, sm_mhz)
    h_img = torch.empty((nslices, N, N), dtype=torch.float32, pin_memory=True)
    h_img.copy_(img)
    h_out = torch.empty((nslices, A, N), dtype=torch.float32, pin_memory=True)
    hi, ho = h_img.numpy(), h_out.numpy()
    gl = np.array([dev.index or 0], np.intc)
    e2e = []
    for r in range(3):
        t0 = time.perf_counter()
        libraft.getRadonRTMultiGPU(_ptr(gl), 1, _ptr(ho), _ptr(hi), _ptr(ang), N, N, N, A, nslices, 1.0, 1.0)
        e2e.append(time.perf_counter() - t0)
        check_error("getRadonRTMultiGPU")
    spot = float((torch.from_numpy(ho[nslices // 2]).to(dev) - out[nslices // 2]).abs().max())
    ms_e2e = 1e3 * statistics.median(e2e)
    return {"workload": f"Radon transform {nslices} x {N}^2 -> {A} angles x {N} bins, uniform random images",
            "ms_per_step": ms, "slices_per_s": nslices / (ms / 1e3), "gups": gups,
            "gather_roofline": {"achieved_gups": gups, "peak_gups": peak, "frac": gups / peak,
                                "bytes_per_update": 4, "fp32_ops_per_update": 1, "sm_mhz": sm_mhz},
            "e2e": {"slices_per_s": nslices / (ms_e2e / 1e3), "ms_per_step": ms_e2e,
                    "api": "getRadonRTMultiGPU, pinned host buffers",
                    "h2d_bytes_per_step": nslices * N * N * 4, "d2h_bytes_per_step": nslices * A * N * 4,
                    "max_abs_diff_vs_device_path": spot}}


def run_aux(dev, sino, reps=3):
    """Timings of the remaining drop-in operators through their Python entry
    points with pinned host arrays, on the FBP workload's shapes: lowpass
    (getFilterLowPassMultiGPU: Hann, padding 2, in place) and the sub-pixel
    rotation-axis correction (getRotAxisCorrectionMultiGPU, 1.5 rays) of 64 x
    1800 x 2048 sinograms (host -> device -> host inside the timed call), and
    the rotation-axis search (findcentersino, findcentersino_subpixel) on one
    2048 x 2048 frame pair of a smooth object mirrored about ray 1061 --
    through the host entries and on device frames (raft_centersino_device)."""
    import torch
    import sscRaft
    from sscRaft.processing import Centersino, Centersino_subpixel, correct_rotation_axis
    from sscRaft.rafttypes import libraft, check_error
    gpu = dev.index or 0
    n = min(64, sino.shape[0])
    A, N = sino.shape[1], sino.shape[2]
    h_base = torch.empty((n, A, N), dtype=torch.float32, pin_memory=True)
    h_base.copy_(sino[:n])
    h_work = torch.empty_like(h_base).pin_memory()
    base, work = h_base.numpy(), h_work.numpy()

    def timed(fn):
        ts = []
        for r in range(reps + 1):
            np.copyto(work, base)
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        return 1e3 * statistics.median(ts[1:])

    ms_lp = timed(lambda: sscRaft.lowpass(work, dic={"gpu": [gpu], "filter": "hann", "padding": 2}))
    ms_ax = timed(lambda: correct_rotation_axis(work, 1.5, gpus=[gpu]))
    io = {"h2d_bytes_per_step": n * A * N * 4, "d2h_bytes_per_step": n * A * N * 4}

    sx = sy = 2048
    axis = sx // 2 + 37
    rng = np.random.default_rng(2024)
    x = np.arange(sx, dtype=np.float64)
    p0 = np.zeros((sy, sx))
    for _ in range(6):
        c, w, a = rng.uniform(0.3, 0.7) * sx, rng.uniform(8, 40), rng.uniform(0.2, 1.0)
        p0 += a * rng.uniform(0.5, 1.5, sy)[:, None] * np.exp(-((x[None, :] - c) ** 2) / (2 * w * w))
    src = (2 * axis - np.arange(sx))
    ok = (src >= 0) & (src < sx)
    p180 = np.zeros_like(p0)
    p180[:, ok] = p0[:, src[ok]]
    dark = np.full((sy, sx), 100.0, np.float32)
    flat = dark + 1e4
    f0 = (dark + 1e4 * np.exp(-p0)).astype(np.float32)
    f1 = (dark + 1e4 * np.exp(-p180)).astype(np.float32)
    ts, tsp = [], []
    for r in range(reps + 1):
        t0 = time.perf_counter()
        off = Centersino(f0, f1, flat, dark)
        t1 = time.perf_counter()
        off_sp = Centersino_subpixel(f0, f1, flat, dark)
        t2 = time.perf_counter()
        if r:
            ts.append(t1 - t0)
            tsp.append(t2 - t1)
    d = [torch.from_numpy(a).to(dev) for a in (f0, f1, dark, flat)]
    res = ctypes.c_double(0)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    td = []
    for r in range(reps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        rc = libraft.raft_centersino_device(gpu, *[ctypes.c_void_p(t.data_ptr()) for t in d], sx, sy, 0,
                                            ctypes.byref(res), st)
        if rc:
            check_error("raft_centersino_device")
        if r:
            td.append(time.perf_counter() - t0)
    return {"lowpass": {"workload": f"{n} x {A} x {N} sinograms, Hann, padding 2, in place", "ms": ms_lp,
                        "slices_per_s": n / (ms_lp / 1e3), "api": "sscRaft.lowpass -> getFilterLowPassMultiGPU",
                        **io},
            "axis_correction": {"workload": f"{n} x {A} x {N} sinograms shifted by 1.5 rays, in place", "ms": ms_ax,
                                "slices_per_s": n / (ms_ax / 1e3),
                                "api": "correct_rotation_axis -> getRotAxisCorrectionMultiGPU", **io},
            "centersino": {"workload": f"one {sx} x {sy} frame pair mirrored about ray {axis}",
                           "ms_host": 1e3 * statistics.median(ts), "ms_host_subpixel": 1e3 * statistics.median(tsp),
                           "ms_device_frames": 1e3 * statistics.median(td), "offset": int(off),
                           "offset_subpixel": float(off_sp), "offset_device": float(res.value),
                           "api": "Centersino / Centersino_subpixel (findcentersino*), raft_centersino_device"}}


def run_fbp_noalloc(dev, sino, ang, nslices=32, reps=3):
    """The headline FBP of `nslices` slices through raft_fbp_device_noalloc
    (working memory from the library's fixed device array, planar
    backprojector) and through raft_fbp_device (grow-only workspaces,
    slice-interleaved backprojector) on the same device-resident sinograms:
    device time per call and the largest difference of the two images."""
    import torch
    from sscRaft.rafttypes import libraft, check_error, _ptr
    src = sino[:nslices]
    pf, pi = fbp_params(nslices)
    angp = np.ascontiguousarray(ang)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    outs, ms = {}, {}
    for name in ("raft_fbp_device_noalloc", "raft_fbp_device"):
        fn = getattr(libraft, name)
        out = torch.empty((nslices, N_RAYS, N_RAYS), dtype=torch.float32, device=dev)
        ts = []
        for r in range(reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            rc = fn(dev.index or 0, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(src.data_ptr()), _ptr(angp),
                    _ptr(pf), _ptr(pi), 0, 0, st)
            e1.record()
            if rc:
                check_error(name)
            torch.cuda.synchronize(dev)
            if r:
                ts.append(e0.elapsed_time(e1))
        ms[name] = statistics.median(ts)
        outs[name] = out
    return {"workload": f"{nslices} slices of the headline FBP workload, device-resident",
            "ms": ms, "slices_per_s": {k: nslices / (v / 1e3) for k, v in ms.items()},
            "max_abs_diff": float((outs["raft_fbp_device_noalloc"] - outs["raft_fbp_device"]).abs().max())}


# ---------------------------------------------------------------- tEMFQ --
TEMFQ_ZPAD, TEMFQ_ITERS = 2, 10


def temfq_inputs(nslices, dev, radon_lib=None):
    """tEMFQ inputs on the tEM workload (nslices x 1024^2, 900 angles over
    [0, pi), flat I0 = 1e4): counts, flat, a uniform start at the phantoms'
    mean attenuation, and the pixel size 2/(N-1) that puts the Fourier-slice
    projection in the units of the tEM data."""
    import torch
    trans, ang, x_true = make_tem_data(nslices, 3_000_000, dev, radon_lib=radon_lib)
    counts = (trans * EM_I0).contiguous()
    flat = torch.full((nslices, EM_N), EM_I0, dtype=torch.float32, device=dev)
    x0 = float(np.mean(x_true))
    return counts, flat, np.ascontiguousarray(ang), x0, 2.0 / (EM_N - 1)


def run_temfq(dev, nslices=EM_SLICES, iters=TEMFQ_ITERS, warm_iters=1):
    """tEMFQ (Fourier-slice projector + BST back-projector) on the tEM
    workload, padding 2 (3072-point transforms) and bilinear sampling, the
    reference's defaults: device-resident (raft_temfq_device) and through the
    drop-in API with pinned host buffers (sscRaft.em -> get_tEM_FQ_MultiGPU)."""
    import torch
    import sscRaft
    from sscRaft.rafttypes import libraft, check_error, _ptr
    counts, flat, ang, x0, dx = temfq_inputs(nslices, dev)
    obj = torch.full((nslices, EM_N, EM_N), x0, dtype=torch.float32, device=dev)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    pf = np.array([dx, dx, 0.0], np.float32)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def em(n):
        pi = np.array([EM_N, EM_A, nslices, EM_N, TEMFQ_ZPAD, 0, 0, nslices, n, 1, 0], np.int32)
        if libraft.raft_temfq_device(dev.index or 0, p(obj), p(counts), p(flat), _ptr(ang), _ptr(pf), _ptr(pi), st):
            check_error("raft_temfq_device")

    em(warm_iters)
    torch.cuda.synchronize(dev)
    obj.fill_(x0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    em(iters)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    dev_obj = obj.cpu().numpy()
    h_counts = torch.empty(counts.shape, dtype=torch.float32, pin_memory=True)
    h_counts.copy_(counts)
    h_flat = flat.cpu().numpy()
    h_obj = torch.empty(obj.shape, dtype=torch.float32, pin_memory=True)
    dic = {"gpu": [dev.index or 0], "method": "tEMFQ", "iterations": iters, "padding": TEMFQ_ZPAD,
           "interpolation": "bilinear", "detectorPixel[m]": dx}
    h_obj.fill_(x0)
    t0 = time.perf_counter()
    sscRaft.em(h_counts.numpy(), flat=h_flat, angles=ang, obj=h_obj.numpy(), dic=dict(dic))
    ms_e2e = (time.perf_counter() - t0) * 1e3
    return {"workload": f"tEMFQ {nslices} x {EM_N}^2, {EM_A} angles over [0,pi) x {EM_N} bins, flat I0=1e4, "
                        f"padding {TEMFQ_ZPAD} ({EM_N * (1 + TEMFQ_ZPAD)}-point transforms), bilinear, "
                        f"{iters} iterations from a uniform start",
            "ms_total": ms, "ms_per_iteration": ms / iters,
            "slice_iterations_per_s": nslices * iters / (ms / 1e3),
            "e2e_ms": ms_e2e, "e2e_api": "sscRaft.em(method='tEMFQ') -> get_tEM_FQ_MultiGPU, pinned host buffers",
            "e2e_max_abs_diff_vs_device_path": float(np.abs(h_obj.numpy() - dev_obj).max())}


# ---------------------------------------------------------- flat / dark --
def run_flat_dark(dev, sino, reps=3, hbm_peak=None):
    """Flat/dark correction + -log of a raw-count volume of the FBP workload's
    shape (flat ~ 1e4 +- 2 %, dark ~ 100 +- 10, two flats interpolated over the
    angles): device-resident (raft_background_device, in place) and through
    the drop-in API with pinned host buffers (getBackgroundCorrectionMultiGPU).
    Algorithmic bytes: one 4-byte read + one 4-byte write per element."""
    import torch
    import sscRaft
    from sscRaft.rafttypes import libraft, check_error
    B, A, N = sino.shape
    g = torch.Generator(device=dev).manual_seed(77)
    flat = (1e4 * (1 + 0.02 * torch.randn((B, 2, N), generator=g, device=dev))).float().contiguous()
    dark = (100 + 10 * torch.randn((B, N), generator=g, device=dev)).float().contiguous()
    w = (torch.arange(A, device=dev, dtype=torch.float32) / A)[None, :, None]
    raw = dark[:, None, :] + (flat[:, :1, :] * (1 - w) + w * flat[:, 1:, :] - dark[:, None, :]) * torch.exp(-sino)
    raw = raw.contiguous()
    work = torch.empty_like(raw)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    times = []
    for r in range(reps + 2):
        work.copy_(raw)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rc = libraft.raft_background_device(dev.index or 0, p(work), p(flat), p(dark), N, A, B, 2, 1, st)
        e1.record()
        if rc:
            check_error("raft_background_device")
        torch.cuda.synchronize(dev)
        if r >= 2:
            times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    err = float((work - sino).abs().max())
    nbytes = 8.0 * B * A * N
    h_raw = torch.empty((B, A, N), dtype=torch.float32, pin_memory=True)
    h_raw.copy_(raw)
    h_work = torch.empty_like(h_raw).pin_memory()
    hf, hd = flat.cpu().numpy(), dark.cpu().numpy()
    e2e = []
    for r in range(3):
        h_work.copy_(h_raw)
        t0 = time.perf_counter()
        sscRaft.correct_background(h_work.numpy(), hf, hd, gpus=[dev.index or 0], is_log=True)
        e2e.append((time.perf_counter() - t0) * 1e3)
    gbs = nbytes / (ms / 1e3) / 1e9
    out = {"workload": f"flat/dark + -log, {B} x {A} x {N} raw counts, 2 flats", "ms": ms, "gb_per_s": gbs,
           "slices_per_s": B / (ms / 1e3), "e2e_ms": statistics.median(e2e[1:]),
           "e2e_slices_per_s": B / (statistics.median(e2e[1:]) / 1e3),
           "max_abs_diff_vs_generating_sinogram": err}
    if hbm_peak:
        out["roofline"] = {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak}
    return out


# ------------------------------------------------------- learned warm start --
def run_warm(dev, samples=256):
    """Learned warm start for tEM at 512^2 x 720 angles: the shipped U-Net
    (trained on 20k (FBP, 200-iteration tEM) pairs) on `samples` held-out
    seeds; wall time to the plain-EM-100 data residual (+1%), learned start
    vs plain EM from the uniform start, with the FBP-only start beside it."""
    import torch
    from sscRaft import synthetic as S
    from sscRaft import warmstart as W
    net = W.UNet.from_file(W.default_weights(), dev)
    trans = torch.empty((samples, 720, 512), dtype=torch.float32, device=dev)
    for c0 in range(0, samples, 64):
        m = min(64, samples - c0)
        W.make_transmissions(m, W.HELDOUT_SEED0 + c0, dev, chunk=m, out=trans[c0:c0 + m])
    r = W.evaluate_wall(net, trans, S.uniform_angles(720))
    r["workload"] = (f"tEM warm start: {samples} held-out 512^2 ellipse+Perlin phantoms (seeds "
                     f"{W.HELDOUT_SEED0}+i), 720 angles, I0 ~ U[1e3,1e5]; target = plain EM-100 residual +1%")
    r["weights"] = os.path.relpath(W.default_weights(), REPO)
    r["unet_params"] = net.n_params()
    return r


def unet_flops_per_image(net, H=512, W=512):
    """2 * 9 * Cin * Cout * pixels summed over the 3x3 convolutions; the first
    layer counted with its one real input channel (its packed input's other
    31 channels are zero, and inference convolves the image directly)."""
    level = {"0": 1, "1": 2, "2": 4, "3": 8}
    return sum(2.0 * 9 * (1 if name == "e0a" else c0 + c1) * co * (H // level[name[1]]) * (W // level[name[1]])
               for name, c0, c1, co in net.LAYERS)


def run_unet(dev, samples=256, reps=3):
    """U-Net inference (the warm start's network) on `samples` 512^2 images in
    batches of 16: device time per image on the tcgen05 convolution and on the
    mma.sync convolution, the convolutions' TFLOP/s, and the largest output
    difference between the two."""
    import torch
    from sscRaft import warmstart as W
    from sscRaft.rafttypes import libraft
    net = W.UNet.from_file(W.default_weights(), dev)
    g = torch.Generator(device=dev).manual_seed(12)
    img = torch.rand((samples, 512, 512), generator=g, device=dev) * 0.01
    out, ms = {}, {}
    for name, path in (("tcgen05", 0), ("mma_sync", 1)):
        libraft.raft_unet_set_conv_path(path)
        try:
            net.predict(img[:16])
            ts = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                o = net.predict(img)
                e1.record()
                torch.cuda.synchronize(dev)
                ts.append(e0.elapsed_time(e1))
            ms[name] = statistics.median(ts)
            out[name] = o
        finally:
            libraft.raft_unet_set_conv_path(0)
    fl = unet_flops_per_image(net)
    return {"workload": f"U-Net inference, {samples} x 512^2, batches of 16 (4 levels, 32 base channels)",
            "ms_per_image": {k: v / samples for k, v in ms.items()},
            "tflops_network": {k: fl * samples / (v / 1e3) / 1e12 for k, v in ms.items()},
            "speedup_tcgen05_vs_mma_sync": ms["mma_sync"] / ms["tcgen05"],
            "max_abs_diff": float((out["tcgen05"] - out["mma_sync"]).abs().max()),
            "max_abs_output": float(out["mma_sync"].abs().max())}


def run_unet_train(dev, batch=16, reps=5):
    """One training step of the warm-start U-Net (forward, MSE, backward with
    the tcgen05 convolutions and weight gradients, Adam) on a batch of 512^2
    images: device time per step, and the same with the weight gradient on
    the mma.sync kernel for comparison."""
    import torch
    from sscRaft import warmstart as W
    from sscRaft.rafttypes import libraft
    net = W.UNet(dev, seed=1)
    g = torch.Generator(device=dev).manual_seed(3)
    img = torch.rand((batch, 512, 512), generator=g, device=dev) * 0.01
    tgt = torch.rand((batch, 512, 512), generator=g, device=dev) * 0.01
    scale = torch.ones((batch,), device=dev)
    ms = {}
    for name, path in (("tcgen05", 0), ("mma_sync", 1)):
        libraft.raft_unet_set_conv_path(path)
        try:
            for _ in range(2):
                net.train_step(img, tgt, scale, 1e-5)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                net.train_step(img, tgt, scale, 1e-5)
            e1.record()
            torch.cuda.synchronize(dev)
            ms[name] = e0.elapsed_time(e1) / reps
        finally:
            libraft.raft_unet_set_conv_path(0)
    net.check()
    return {"workload": f"U-Net training step, batch {batch} x 512^2 (forward, MSE, backward, Adam)",
            "ms_per_step": ms, "speedup_tcgen05_vs_mma_sync": ms["mma_sync"] / ms["tcgen05"]}


# ----------------------------------------------------------- ragged batch --
def run_ragged(dev, nreq=96, seed=5_000_000, em_iters=30):
    """96 requests, side log-uniform in [256, 2048], angles U[180, 1800], bins =
    side; alternate FBP (Hann, padding 2) and 30-iteration eEM; device-resident,
    one batch call.  Returns p50/p99 request latency and aggregate GUPS."""
    import torch
    from sscRaft import synthetic as S
    from sscRaft.geometries.parallel.batch_methods import reconstruct_ragged
    from sscRaft.rafttypes import libraft, check_error, _ptr
    rng = np.random.Generator(np.random.PCG64(seed))
    sides = np.exp(rng.uniform(np.log(256), np.log(2048), nreq)).astype(int)
    nangs = rng.integers(180, 1801, nreq)
    reqs, updates = [], 0.0
    for i in range(nreq):
        N, A = int(sides[i]), int(nangs[i])
        ang = S.uniform_angles(A)
        prm = S.ellipse_params(seed + i, 20)
        if i % 2 == 0:
            sino = S.ellipse_sinogram(prm, ang, N, xp=torch, device=dev).float().contiguous()
            reqs.append({"kind": "fbp", "data": sino, "out": torch.empty((N, N), dtype=torch.float32, device=dev),
                         "angles": ang, "filter": "hann", "padding": 2})
            updates += float(N) * N * A
        else:
            img = S.phantom_image(prm, N, xp=torch, device=dev).cpu().numpy()[None]
            proj = -np.ones((1, A, N), np.float32)
            g = np.array([dev.index or 0], np.intc)
            libraft.getRadonRTMultiGPU(_ptr(g), 1, _ptr(proj), _ptr(np.ascontiguousarray(img)), _ptr(ang),
                                       N, N, N, A, 1, 1.0, 1.0)
            check_error("radon")
            reqs.append({"kind": "eem", "data": torch.from_numpy(proj[0]).to(dev),
                         "out": torch.ones((N, N), dtype=torch.float32, device=dev), "angles": ang,
                         "iterations": em_iters})
            updates += 2.0 * N * N * A * em_iters
    reconstruct_ragged(reqs)            # warm-up (plans, tuning, graph capture paths)
    for r in reqs:
        if r["kind"] == "eem":
            r["out"].fill_(1.0)
    torch.cuda.synchronize()
    lat, total = reconstruct_ragged(reqs)
    fbp_lat = lat[0::2]
    em_lat = lat[1::2]
    return {"workload": f"{nreq} requests, side log-uniform [256,2048], angles U[180,1800], bins = side, "
                        f"alternating FBP (Hann) and {em_iters}-iteration eEM, one ragged batch",
            "total_ms": total, "gups": updates / (total / 1e3) / 1e9,
            "latency_ms_p50": float(np.percentile(lat, 50)), "latency_ms_p99": float(np.percentile(lat, 99)),
            "fbp_latency_ms_p50": float(np.percentile(fbp_lat, 50)),
            "eem_latency_ms_p50": float(np.percentile(em_lat, 50)),
            "updates": updates}


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            self.path = f"/tmp/raft_clocks_{os.getpid()}.csv"
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        loaded = [v for v in sm if v > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "power_w_max": max(power), "samples": len(sm)}


# --------------------------------------------------------------- helpers --
def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("sm_max_mhz", 1965.0), "measured"
    return 6650.0, 1965.0, "fallback"


def gather_peak_gups(store_bytes, ops, sm_mhz, n_sm=148):
    """Backprojection gather roofline: SMs x clock x min(smem bytes/clk / bytes
    per update, FP32 lanes / FP32 ops per update)."""
    per_clk = min(128.0 / store_bytes, 128.0 / ops)
    return n_sm * sm_mhz * 1e6 * per_clk / 1e9


def cpu_baseline(sino_host, ang):
    """The FP32 OpenMP restatement of the same operator (oracle), on a bounded
    sample of slices, timed on the host cores."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    done, t_total = 0, 0.0
    while done < sino_host.shape[0] and (t_total < 10.0 or done == 0):
        t0 = time.perf_counter()
        oracle.fbp(sino_host[done:done + 1], ang, oracle.MODE_REF, FILTER_ID, PAD, offset=OFFSET, f32=True)
        t_total += time.perf_counter() - t0
        done += 1
    return {"value": done / t_total, "unit": "slices/s", "cores": cores, "kind": "port",
            "sample": f"{done} of 512 slices (2048^2 x 1800, nearest operator, FP32 OpenMP oracle port), "
                      f"{t_total:.1f} s"}


# -------------------------------------------------------------- our arm --
def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    import sscRaft
    from sscRaft.rafttypes import libraft, check_error, _ptr, GEOMETRY, STORE, autotune_table

    nsl = args.slices
    t0 = time.perf_counter()
    sino, ang = make_sinograms_gpu(nsl, slice_seed_base(rank, nsl), dev)
    torch.cuda.synchronize()
    log(f"[rank {rank}] generated {nsl} sinograms in {time.perf_counter() - t0:.1f} s")
    img = torch.empty((nsl, N_RAYS, N_RAYS), dtype=torch.float32, device=dev)
    pf, pi = fbp_params(nsl)
    angp = np.ascontiguousarray(ang)

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def ranks_max(x):
        return max_over_ranks(x, dev)

    def device_step(geometry, store):
        st = torch.cuda.current_stream(dev).cuda_stream
        rc = libraft.raft_fbp_device(local, ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(sino.data_ptr()),
                                     _ptr(angp), _ptr(pf), _ptr(pi), geometry, store, ctypes.c_void_p(st))
        if rc:
            check_error("raft_fbp_device")

    def time_device(geometry, store, K, W):
        for _ in range(W):
            device_step(geometry, store)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        n0 = libraft.raft_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(K):
            device_step(geometry, store)
        e1.record()
        torch.cuda.synchronize()
        barrier()
        launches = libraft.raft_launch_count() - n0
        return ranks_max(e0.elapsed_time(e1) / K), launches

    def bst_step():
        st = torch.cuda.current_stream(dev).cuda_stream
        rc = libraft.raft_bst_device(local, ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(sino.data_ptr()),
                                     _ptr(pf), _ptr(pi), ctypes.c_void_p(st))
        if rc:
            check_error("raft_bst_device")

    def time_bst(K, W):
        for _ in range(W):
            bst_step()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(K):
            bst_step()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        return ranks_max(e0.elapsed_time(e1) / K)

    def profile_bp(geometry, store):
        libraft.raft_profile_enable(1)
        device_step(geometry, store)
        torch.cuda.synchronize()
        libraft.raft_profile_enable(0)
        ms = (ctypes.c_double * 3)()
        cnt = (ctypes.c_longlong * 3)()
        libraft.raft_profile_read(ms, cnt, 3)
        return ms[0], cnt[0], ms[1], cnt[1]

    hbm_peak, sm_max, peak_kind = peaks()
    if args.quick and args.op == "ragged":
        r = run_ragged(dev)
        if rank == 0:
            print(json.dumps({"quick": True, "op": "ragged", **r}), flush=True)
        return
    if args.quick and args.op == "bst":
        ms = time_bst(args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"quick": True, "op": "bst", "slices": nsl, "ms_per_step": ms,
                              "slices_per_s": ws * nsl / (ms / 1e3)}), flush=True)
        return
    if args.quick and args.op == "flat_dark":
        r = run_flat_dark(dev, sino, reps=args.steps, hbm_peak=hbm_peak)
        if rank == 0:
            print(json.dumps({"quick": True, "op": "flat_dark", **r}), flush=True)
        return
    if args.quick and args.op == "unet":
        r = run_unet(dev, samples=args.slices, reps=max(1, args.steps))
        if rank == 0:
            print(json.dumps({"quick": True, "op": "unet", **r}), flush=True)
        return
    if args.quick and args.op == "unet_train":
        r = run_unet_train(dev, reps=max(1, args.steps))
        if rank == 0:
            print(json.dumps({"quick": True, "op": "unet_train", **r}), flush=True)
        return
    if args.quick and args.op == "warm":
        r = run_warm(dev, samples=args.slices)
        if rank == 0:
            print(json.dumps({"quick": True, "op": "warm", **r}), flush=True)
        return
    if args.quick and args.op == "temfq":
        r = run_temfq(dev, nslices=args.slices, iters=args.steps, warm_iters=args.warmup)
        if rank == 0:
            print(json.dumps({"quick": True, "op": "temfq", **r}), flush=True)
        return
    if args.quick and args.op == "aux":
        r = run_aux(dev, sino, reps=max(1, args.steps))
        if rank == 0:
            print(json.dumps({"quick": True, "op": "aux", **r}), flush=True)
        return
    if args.quick and args.op == "radon":
        r = run_radon(dev, sm_max, nslices=args.slices, reps=max(1, args.steps), warm=max(1, args.warmup))
        if rank == 0:
            print(json.dumps({"quick": True, "op": "radon", **r}), flush=True)
        return
    if args.quick and args.op == "tem":
        # profiling mode: a short tEM run (args.slices x 1024^2, 900 angles)
        r = run_tem(local, dev, nslices=args.slices, iters=args.steps, warm_iters=args.warmup)
        if rank == 0:
            print(json.dumps({"quick": True, "op": "tem", **r}), flush=True)
        return
    if args.quick:
        # profiling mode: only the device-resident FBP of the chosen operator
        g, s = {"nearest": (0, 0), "linear": (1, 1), "linear_bf16": (1, 2)}[args.op]
        ms, launches = time_device(g, s, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"quick": True, "op": args.op, "slices": nsl, "ms_per_step": ms,
                              "slices_per_s": ws * nsl / (ms / 1e3), "gpu_launches": int(launches),
                              "autotune": autotune_table()}), flush=True)
        return
    result = {}
    with ClockSampler(local) as clk:
        ms_dev, launches = time_device(0, 0, args.steps, args.warmup)
        # end-to-end through the public drop-in API with pinned host buffers
        h_sino = torch.empty((nsl, N_ANGLES, N_RAYS), dtype=torch.float32, pin_memory=True)
        h_sino.copy_(sino)
        h_img = torch.empty((nsl, N_RAYS, N_RAYS), dtype=torch.float32, pin_memory=True)
        hs, hi = h_sino.numpy(), h_img.numpy()
        dic = {"gpu": [local], "angles[rad]": angp, "filter": "hann", "padding": PAD,
               "rotation axis offset": OFFSET}
        for _ in range(args.warmup):
            sscRaft.fbp(hs, dic=dict(dic), obj=hi)
        barrier()
        t_e2e = []
        for _ in range(args.steps):
            t1 = time.perf_counter()
            sscRaft.fbp(hs, dic=dict(dic), obj=hi)
            t_e2e.append(time.perf_counter() - t1)
        barrier()
        ms_e2e = ranks_max(1e3 * sum(t_e2e) / len(t_e2e))
        # parity spot check of the e2e output against the device-path output
        spot = float((torch.from_numpy(hi[nsl // 2]).to(dev) - img[nsl // 2]).abs().max())
        variants = {}
        for name, g, s in (("linear_fp32", 1, 1), ("linear_bf16", 1, 2)):
            ms_v, _ = time_device(g, s, max(1, args.steps), max(3, args.warmup))
            variants[name] = {"value": ws * nsl / (ms_v / 1e3), "ms_per_step": ms_v}
        ms_b = time_bst(max(1, args.steps), max(3, args.warmup))
        variants["bst"] = {"value": ws * nsl / (ms_b / 1e3), "ms_per_step": ms_b,
                           "operator": "backprojection slice theorem (Fourier regridding), Hann, axis offset "
                                       "truncated to 3 as the reference does, padding 2 (6144-point transforms)"}
    clocks = clk.summary()

    # dominant kernel: the backprojector; one profiled pass of the headline operator
    f_ms, f_n, bp_ms, bp_n = profile_bp(0, 0)
    chunk = min(nsl, 32)
    upd_per_launch = chunk * N_RAYS * N_RAYS * N_ANGLES
    bp_avg_s = bp_ms / bp_n / 1e3
    # algorithmic bytes per launch: the filtered detector bins the image can
    # reach (ceil(sqrt(2) N) per angle, 4 B) read once + the image written once
    reach = int(math.ceil(math.sqrt(2) * N_RAYS))
    alg_bytes = chunk * N_ANGLES * reach * 4 + chunk * N_RAYS * N_RAYS * 4
    sm_mhz = (clocks or {}).get("sm_mhz") or sm_max
    gups_bp = upd_per_launch / bp_avg_s / 1e9
    peak_gups = gather_peak_gups(4, 4, sm_mhz)
    # f32 pairs: 8 B + 5 FP32 ops per update; bf16 pairs on slice-interleaved rows:
    # 4 B + 4 ops (two FP32, two integer to unpack the pair)
    for name, (g, s, bytes_upd, ops) in (("linear_fp32", (1, 1, 8, 5)), ("linear_bf16", (1, 2, 4, 4))):
        _, _, vms, vn = profile_bp(g, s)
        vg = upd_per_launch / (vms / vn / 1e3) / 1e9
        pk = gather_peak_gups(bytes_upd, ops, sm_mhz)
        variants[name].update({"bp_gups": vg, "gather_roofline": {"achieved_gups": vg, "peak_gups": pk,
                                                                   "frac": vg / pk}})

    radon_result = None if args.no_radon else run_radon(dev, sm_mhz)
    em_result = None if args.no_em else run_tem(local, dev)
    ragged_result = None if args.no_ragged else run_ragged(dev)
    warm_result = None if args.no_warm else run_warm(dev)
    if warm_result is not None:
        warm_result["training_step"] = run_unet_train(dev)
    flat_dark_result = None if args.no_flat_dark else run_flat_dark(dev, sino, hbm_peak=hbm_peak)
    temfq_result = None if args.no_temfq else run_temfq(dev)
    aux_result = None if args.no_aux else run_aux(dev, sino)
    if aux_result is not None:
        aux_result["fbp_noalloc"] = run_fbp_noalloc(dev, sino, ang)

    if rank == 0:
        value = ws * nsl / (ms_dev / 1e3)
        updates_step = nsl * N_RAYS * N_RAYS * N_ANGLES
        result = {
            "metric": METRIC,
            "value": value,
            "unit": "slices/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_dev,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": DATA,
            "config": bench_config(ws),
            "slices_per_step": nsl,
            "gups": ws * updates_step / (ms_dev / 1e3) / 1e9,
            "e2e": {"value": ws * nsl / (ms_e2e / 1e3), "unit": "slices/s", "ms_per_step": ms_e2e,
                    "api": "sscRaft.fbp -> getFBPMultiGPU, pinned host buffers",
                    "h2d_bytes_per_step": nsl * N_ANGLES * N_RAYS * 4,
                    "d2h_bytes_per_step": nsl * N_RAYS * N_RAYS * 4,
                    "max_abs_diff_vs_device_path": spot},
            "roofline": {"bound": "smem-gather", "achieved": gups_bp, "peak": peak_gups, "unit": "GUPS",
                         "frac": gups_bp / peak_gups,
                         "kernel": "bp_kernel_s4<nearest,f32,interleaved>",
                         "kernel_ms_per_launch": bp_avg_s * 1e3,
                         "updates_per_launch": upd_per_launch,
                         "peak_def": "148 SMs x SM clock (median sampled) x 32 updates/clk: 128 B/clk of "
                                     "shared-memory data pipe / 4 B per update",
                         "sm_mhz": sm_mhz,
                         "traffic": BP_TRAFFIC_PER_LAUNCH if chunk == 32 else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 32-slice "
                                           "launch (S4 interleaved, AB16), --set full capture",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "hbm": {"achieved_gbs": alg_bytes / bp_avg_s / 1e9, "peak_gbs": hbm_peak,
                                 "frac": alg_bytes / bp_avg_s / 1e9 / hbm_peak, "peak_kind": peak_kind}},
            "gather_roofline": {"achieved_gups": gups_bp, "peak_gups": peak_gups, "frac": gups_bp / peak_gups,
                                "bytes_per_update": 4, "fp32_ops_per_update": 4, "sm_mhz": sm_mhz},
            "kernel_ms": {"filter_per_launch": f_ms / max(1, f_n), "bp_per_launch": bp_ms / max(1, bp_n),
                          "launches_per_step": {"filter": f_n, "bp": bp_n}},
            "variants": variants,
            "autotune": autotune_table(),
            "radon": radon_result,
            "em": em_result,
            "ragged": ragged_result,
            "warm_start": warm_result,
            "flat_dark": flat_dark_result,
            "temfq": temfq_result,
            "aux": aux_result,
            "clocks": clocks,
            "gpu_launches": int(launches),
        }
        if ws == 1 and not args.no_cpu:
            sino_host = sino[: 4].cpu().numpy()
            result["cpu_baseline"] = cpu_baseline(sino_host, angp)
        print(json.dumps(result), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# -------------------------------------------------------- reference arm --
def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return
    lib_path = os.path.join(REPO, "oracle", "_ref", "libraft_ref.so")
    if not os.path.exists(lib_path):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libraft_ref.so not built"}))
        return
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.ref_op == "temfq":
        run_reference_temfq(args, lib_path, dev, local)
        return
    S = args.ref_slices
    sino, ang = make_sinograms_gpu(S, 2_000_000, dev)
    h_sino = sino.cpu().numpy()
    del sino
    torch.cuda.empty_cache()
    lib = ctypes.CDLL(lib_path)
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.getFBPMultiGPU.argtypes = [P, I, P, P, P, P, P]
    g = np.array([local], np.intc)
    # blocksize 0: the reference chooses its own slice block (process.cu:31-66)
    pf, pi = fbp_params(S, blocksize=0)
    obj = np.zeros((S, N_RAYS, N_RAYS), np.float32)
    angp = np.ascontiguousarray(ang)

    def p(a):
        return a.ctypes.data_as(ctypes.c_void_p)

    def step():
        lib.getFBPMultiGPU(p(g), 1, p(obj), p(h_sino), p(angp), p(pf), p(pi))

    for _ in range(args.warmup):
        step()
    ts = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            step()
            ts.append(time.perf_counter() - t0)
    ms = 1e3 * sum(ts) / len(ts)
    value = S / (ms / 1e3)
    sample = (f"{S} of the workload's 512 slices per step through the reference's own getFBPMultiGPU "
              f"(its CUDA sources built for sm_100a, host buffers, blocksize chosen by the reference)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "slices/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": DATA, "config": bench_config(1),
        "slices_per_step": S,
        "cpu_baseline": {"value": value, "unit": "slices/s", "cores": 1, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "slices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "the reference's call takes host buffers: its copies are inside every step"},
        "clocks": clk.summary(),
    }), flush=True)


def run_reference_temfq(args, lib_path, dev, local):
    """The reference's get_tEM_FQ_MultiGPU on `--ref-slices` slices of the
    tEMFQ workload (host buffers), for comparison with the ours arm's temfq
    section; prints its own line."""
    S = args.ref_slices
    lib = ctypes.CDLL(lib_path)
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    lib.get_tEM_FQ_MultiGPU.argtypes = [P, I, P, P, P, P, P, P]
    lib.getRadonRTMultiGPU.argtypes = [P, I, P, P, P, I, I, I, I, I, F, F]
    counts, flat, ang, x0, dx = temfq_inputs(S, dev, radon_lib=lib)
    h_counts, h_flat = counts.cpu().numpy(), flat.cpu().numpy()
    g = np.array([local], np.intc)
    pi = np.array([EM_N, EM_A, S, EM_N, TEMFQ_ZPAD, 0, 0, S, TEMFQ_ITERS, 1, S], np.int32)
    pf = np.array([dx, dx, 0.0], np.float32)
    obj = np.empty((S, EM_N, EM_N), np.float32)

    def p(a):
        return a.ctypes.data_as(ctypes.c_void_p)

    ts = []
    for k in range(args.warmup + args.steps):
        obj.fill(x0)
        t0 = time.perf_counter()
        lib.get_tEM_FQ_MultiGPU(p(g), 1, p(h_counts), p(obj), p(ang), p(h_flat), p(pf), p(pi))
        if k >= args.warmup:
            ts.append(time.perf_counter() - t0)
    ms = 1e3 * sum(ts) / len(ts)
    print(json.dumps({"impl": "reference", "op": "temfq", "slices": S, "iterations": TEMFQ_ITERS,
                      "ms_per_call": ms, "ms_per_slice_iteration": ms / (S * TEMFQ_ITERS),
                      "slice_iterations_per_s": S * TEMFQ_ITERS / (ms / 1e3)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--slices", type=int, default=N_SLICES)
    ap.add_argument("--ref-slices", type=int, default=32)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-radon", action="store_true")
    ap.add_argument("--no-em", action="store_true")
    ap.add_argument("--no-ragged", action="store_true")
    ap.add_argument("--no-warm", action="store_true")
    ap.add_argument("--no-flat-dark", action="store_true")
    ap.add_argument("--no-temfq", action="store_true")
    ap.add_argument("--no-aux", action="store_true")
    ap.add_argument("--ref-op", default="fbp", choices=["fbp", "temfq"],
                    help="reference arm: the headline FBP, or tEMFQ on the tEM workload (comparison only)")
    ap.add_argument("--quick", action="store_true", help="device timing of one operator only (profiling)")
    ap.add_argument("--op", default="nearest", choices=["nearest", "linear", "linear_bf16", "radon", "aux", "tem", "ragged", "flat_dark", "bst",
                                                        "temfq", "unet", "unet_train", "warm"])
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
