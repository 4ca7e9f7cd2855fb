"""GPU tests of transmission EM with the Fourier-slice projector (tEMFQ):
get_tEM_FQ_MultiGPU, raft_temfq_device, sscRaft.em(method='tEMFQ').

Tolerances (rel-L2 of the object after two to four iterations): <= 5e-6
against the reference library's own outputs (measured <= 7.8e-7) and against
the FP64 oracle (measured <= 5.2e-7).  All three
regrid in float with the same geometry and fast sine/cosine; the transforms
are float here (own FFT) and in the reference (cuFFT), FP64 in the oracle,
and the EM update multiplies their rounding into the object each iteration.
Nearest-neighbour cases use angle sets whose samples stay at least 4e-4 away
from a rounding tie, so the fast and the libm cosine pick the same sample.
Chunked, whole, Python and device-entry runs are bit-identical.  Lengths with
a prime factor above 7 (Bluestein transforms): <= 2e-5 against the oracle."""
import ctypes
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2
from helpers import temfq_counts

pytestmark = pytest.mark.gpu


def _temfq(counts, flat, ang, zpad, interp, niter, dx, blocksize=0, obj=None):
    from sscRaft.rafttypes import libraft, check_error
    B, A, N = counts.shape
    obj = np.ones((B, N, N), np.float32) if obj is None else np.ascontiguousarray(obj, np.float32).copy()
    pi = np.array([N, A, B, N, zpad, 0, 0, B, niter, interp, blocksize], np.int32)
    pf = np.array([dx, dx, 0.0], np.float32)
    g = np.array([0], np.intc)
    c = np.ascontiguousarray(counts, np.float32)
    f = np.ascontiguousarray(flat, np.float32)
    a = np.ascontiguousarray(ang, np.float32)
    libraft.get_tEM_FQ_MultiGPU(g.ctypes.data, 1, c.ctypes.data, obj.ctypes.data, a.ctypes.data, f.ctypes.data,
                                pf.ctypes.data, pi.ctypes.data)
    check_error("temfq")
    return obj


def test_temfq_vs_reference_fixtures():
    files = sorted(glob.glob(os.path.join(GOLDEN, "ref_temfq_*.npz")))
    assert files, "tEMFQ fixtures missing"
    for f in files:
        d = np.load(f)
        counts = d["counts"].copy()
        out = _temfq(counts, d["flat"], d["angles"], int(d["zpad"]), int(d["interpolation"]),
                     int(d["iterations"]), float(d["dx"]))
        assert np.array_equal(counts, d["counts"])                 # counts are not modified
        assert rel_l2(out, d["out"]) <= 5e-6, (os.path.basename(f), rel_l2(out, d["out"]))


@pytest.mark.parametrize("N,A,B,zpad,interp,niter", [(64, 64, 2, 1, 1, 4), (100, 100, 1, 1, 1, 3),
                                                     (96, 80, 2, 2, 0, 3), (72, 50, 1, 3, 1, 2)])
def test_temfq_vs_oracle(oracle, N, A, B, zpad, interp, niter):
    counts, flat, ang = temfq_counts(N, A, B, 0.02, seed=N + A + zpad)
    out = _temfq(counts, flat, ang, zpad, interp, niter, 0.02)
    ref = oracle.temfq(counts, flat, ang, zpad, interp, niter, dx=0.02)
    assert rel_l2(out, ref) <= 5e-6, rel_l2(out, ref)


def test_temfq_zero_pixel_size_and_initial_guess(oracle):
    # dx <= 0: scale 1 / (N (1 + zpad)), i.e. attenuation per pixel; counts whose
    # attenuation is about 0.01 per pixel and a uniform initial guess near it
    counts, flat, ang = temfq_counts(64, 64, 1, 1.0 / 128, seed=3)
    guess = np.full((1, 64, 64), 0.01, np.float32)
    out = _temfq(counts, flat, ang, 1, 1, 3, 0.0, obj=guess)
    ref = oracle.temfq(counts, flat, ang, 1, 1, 3, obj=guess, dx=0.0)
    assert rel_l2(out, ref) <= 5e-6, rel_l2(out, ref)


def test_temfq_chunking_python_and_device_entry():
    import torch
    import sscRaft
    from sscRaft.rafttypes import libraft
    N, A, B = 64, 64, 5
    counts, flat, ang = temfq_counts(N, A, B, 0.02, seed=11)
    whole = _temfq(counts, flat, ang, 1, 1, 3, 0.02)
    chunked = _temfq(counts, flat, ang, 1, 1, 3, 0.02, blocksize=2)
    assert np.array_equal(whole, chunked)
    py = sscRaft.em(counts, flat=flat, angles=ang, dic={"gpu": [0], "method": "tEMFQ", "iterations": 3,
                                                       "padding": 1, "interpolation": "bilinear",
                                                       "detectorPixel[m]": 0.02})
    assert np.array_equal(py, whole)
    d_obj = torch.ones((B, N, N), device="cuda")
    d_counts = torch.from_numpy(counts).cuda()
    d_flat = torch.from_numpy(flat).cuda()
    pi = np.array([N, A, B, N, 1, 0, 0, B, 3, 1, 0], np.int32)
    pf = np.array([0.02, 0.02, 0.0], np.float32)
    assert libraft.raft_temfq_device(0, ctypes.c_void_p(d_obj.data_ptr()), ctypes.c_void_p(d_counts.data_ptr()),
                                     ctypes.c_void_p(d_flat.data_ptr()), ang.ctypes.data, pf.ctypes.data,
                                     pi.ctypes.data, None) == 0
    assert np.array_equal(d_obj.cpu().numpy(), whole)
    assert np.array_equal(d_counts.cpu().numpy(), counts)


def test_temfq_prime_factor_lengths_vs_oracle(oracle):
    # N = 44 = 4 x 11, zpad 1: 88- and 44-point transforms by Bluestein's algorithm
    counts, flat, ang = temfq_counts(44, 44, 1, 0.02, seed=44)
    out = _temfq(counts, flat, ang, 1, 1, 3, 0.02)
    ref = oracle.temfq(counts, flat, ang, 1, 1, 3, dx=0.02)
    assert rel_l2(out, ref) <= 2e-5, rel_l2(out, ref)


def test_temfq_too_long_length_raises():
    # 7342 = 2 x 3671: Bluestein would need a transform beyond shared memory
    counts = np.ones((1, 1, 7342), np.float32)
    with pytest.raises(RuntimeError):
        _temfq(counts, np.ones((1, 7342), np.float32), np.zeros(1, np.float32), 0, 1, 1, 0.0)
