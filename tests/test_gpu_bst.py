"""GPU tests of FBP by the backprojection slice theorem (getBSTMultiGPU,
raft_bst_device, sscRaft.fbp(method='BST')).

Tolerances: rel-L2 <= 5e-6 against the reference library's own outputs
(fixtures with nangles == nrays; measured <= 4.7e-7) and <= 1e-5 against the
FP64 oracle; the regridding geometry is float in all three, the FFTs float
here and in the reference, FP64 in the oracle.
Chunked / whole / device-entry runs are bit-identical.  Lengths with a prime
factor above 7 (Bluestein transforms): <= 1e-5 against both."""
import ctypes
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2
from helpers import fbp_params, sino_case

pytestmark = pytest.mark.gpu


def _bst(sino, pad, ftype, offset=0, reg=0.0, pixel=1.0, blocksize=0):
    from sscRaft.rafttypes import libraft, check_error
    B, A, N = sino.shape
    pf, pi = fbp_params(N, A, B, pad=pad, ftype=ftype, offset=float(offset), reg=reg, pixel=pixel,
                        blocksize=blocksize)
    obj = np.zeros((B, N, N), np.float32)
    g = np.array([0], np.intc)
    s = np.ascontiguousarray(sino, np.float32)
    ang = np.linspace(0, np.pi, A, endpoint=False).astype(np.float32)
    libraft.getBSTMultiGPU(g.ctypes.data, 1, obj.ctypes.data, s.ctypes.data, ang.ctypes.data, pf.ctypes.data,
                           pi.ctypes.data, 0)
    check_error("bst")
    return obj


def test_bst_vs_reference_fixtures():
    files = sorted(glob.glob(os.path.join(GOLDEN, "ref_bst_*.npz")))
    assert files, "BST fixtures missing"
    for f in files:
        d = np.load(f)
        pi, pf = d["parami"], d["paramf"]
        out = _bst(d["sino"], int(pi[4]), int(pi[7]), int(pf[6]), float(pf[1]), float(pf[4]))
        assert rel_l2(out, d["out"]) <= 5e-6, (os.path.basename(f), rel_l2(out, d["out"]))


@pytest.mark.parametrize("N,A,pad,ftype,offset", [(100, 90, 2, 7, 0), (64, 120, 1, 5, -2), (128, 128, 2, 6, 3)])
def test_bst_vs_oracle(oracle, N, A, pad, ftype, offset):
    ang = np.linspace(0, np.pi, A, endpoint=False).astype(np.float32)
    sino, _ = sino_case(N, A, 2, seed=N + A, angles=ang)
    out = _bst(sino, pad, ftype, offset)
    ref = oracle.bst(sino, ftype, pad, offset=offset)
    assert rel_l2(out, ref) <= 1e-5, rel_l2(out, ref)


def test_bst_python_entry_and_chunking():
    import torch
    import sscRaft
    from sscRaft.rafttypes import libraft
    N, A, B = 96, 96, 5
    ang = np.linspace(0, np.pi, A, endpoint=False).astype(np.float32)
    sino, _ = sino_case(N, A, B, seed=9, angles=ang)
    whole = _bst(sino, 2, 5, 1)
    chunked = _bst(sino, 2, 5, 1, blocksize=2)
    assert np.array_equal(whole, chunked)
    py = sscRaft.fbp(sino, dic={"gpu": [0], "method": "BST", "filter": "hann", "rotation axis offset": 1.6})
    assert np.array_equal(py, whole)          # offset 1.6 -> 1, as the reference truncates it
    d_in = torch.from_numpy(sino).cuda()
    d_out = torch.empty((B, N, N), device="cuda")
    pf, pi = fbp_params(N, A, B, pad=2, ftype=5, offset=1.0)
    assert libraft.raft_bst_device(0, ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_in.data_ptr()),
                                   pf.ctypes.data, pi.ctypes.data, None) == 0
    assert np.array_equal(d_out.cpu().numpy(), whole)


def test_bst_prime_factor_length_vs_oracle_and_reference(oracle, tmp_path):
    """N = 88 = 8 x 11 at padding 2: 264-point transforms by Bluestein's
    algorithm (the reference runs them through cuFFT), vs the FP64 oracle and
    the reference's own getBSTMultiGPU in a fresh process."""
    import subprocess
    import sys
    from conftest import REF_LIB, REPO
    N = A = 88
    ang = np.linspace(0, np.pi, A, endpoint=False).astype(np.float32)
    sino, _ = sino_case(N, A, 2, seed=88, angles=ang)
    out = _bst(sino, 2, 5, 1)
    ref = oracle.bst(sino, 5, 2, offset=1)
    assert rel_l2(out, ref) <= 1e-5, rel_l2(out, ref)
    if not os.path.exists(REF_LIB):
        pytest.skip("reference library not built (oracle/build_ref.sh)")
    pf, pi = fbp_params(N, A, 2, pad=2, ftype=5, offset=1.0)
    src, dst = tmp_path / "in.npz", tmp_path / "out.npz"
    np.savez(src, sino=sino, angles=ang, paramf=pf, parami=pi)
    subprocess.run([sys.executable, os.path.join(REPO, "tests", "ref_runner.py"), "bst", str(src), str(dst)],
                   check=True, timeout=600)
    err = rel_l2(out, np.load(dst)["out"])
    assert err <= 1e-5, err


def test_bst_too_long_length_raises():
    sino = np.zeros((1, 4, 3671), np.float32)
    with pytest.raises(RuntimeError):
        _bst(sino, 1, 7)                     # Np = 2 x 3671: its transform would not fit shared memory


def test_bst_4096_pad2_vs_reference_library(tmp_path):
    """A 4096-bin detector at the default padding 2 (12288-point transforms,
    above what one CTA held before the row kernel parked the second row's
    half-rays): vs the reference's own getBSTMultiGPU on the same inputs, run
    in a fresh process (its half-ray padding is freshly allocated device
    memory, zero there); angles = rays, as the reference's padding needs."""
    import subprocess
    import sys
    from conftest import REF_LIB, REPO
    N = A = 4096
    ang = np.linspace(0, np.pi, A, endpoint=False).astype(np.float32)
    sino, _ = sino_case(N, A, 1, seed=4096, angles=ang, n_ell=12)
    out = _bst(sino, 2, 5, 1)
    assert np.all(np.isfinite(out))
    if not os.path.exists(REF_LIB):
        pytest.skip("reference library not built (oracle/build_ref.sh)")
    pf, pi = fbp_params(N, A, 1, pad=2, ftype=5, offset=1.0)
    src, dst = tmp_path / "in.npz", tmp_path / "out.npz"
    np.savez(src, sino=sino, angles=ang, paramf=pf, parami=pi)
    subprocess.run([sys.executable, os.path.join(REPO, "tests", "ref_runner.py"), "bst", str(src), str(dst)],
                   check=True, timeout=600)
    ref = np.load(dst)["out"]
    err = rel_l2(out, ref)
    print(f"BST 4096^2 pad 2 vs reference library: rel-L2 {err:.3e}")
    assert err <= 1e-5, err
