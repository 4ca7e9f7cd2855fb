"""The transform kernels compiled for fixed lengths (1024, 1536, 2048, 3072,
4096, 6144, 8192, 12288 points: FBP filter rows, BST, tEMFQ) against the generic ones,
through the C ABI.

The fixed-length kernels keep the generic kernels' radix order, twiddle
expressions and butterflies, with every rounding explicit (no multiply-add
left for the compiler to fuse), so whole reconstructions with
raft_filter_set_fixed(1) and (0) must be equal bit for bit, for every row
format the filter writes: single floats in the four-slice interleaved layout
(nearest operator), the same in the planar layout (nearest, backprojector
forced to S = 2), FP32 (mid, diff) pairs (linear) and BF16 pairs in the
interleaved layout (linear).  An odd angle count leaves a single row in each slice's last pair, five slices
leave three zero slices in the last group of four, jittered angles make the
angle weights unequal, and padding 0 with an axis offset puts window elements
outside the padded row.  BST (rows, half-rays and grid all of the padded
length; filtered and with the 'none' filter) and tEMFQ (Fourier-slice
projector transforms of L = N (1 + zpad) points, BST core of other lengths;
two EM iterations) must be equal bit for bit as well."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # N, pad -> padded length
    (512, 1),    # 1024
    (512, 2),    # 1536
    (1024, 1),   # 2048
    (2048, 0),   # 2048, window beyond the row
    (1024, 2),   # 3072
    (2048, 1),   # 4096
    (2048, 2),   # 6144
    (4096, 1),   # 8192
    (4096, 2),   # 12288
]
FORMATS = [
    # geometry, store, RAFT_BP_TUNE
    (0, 0, None),      # nearest, single floats, interleaved rows
    (0, 0, "2,16"),    # nearest, single floats, planar rows
    (1, 1, None),      # linear, FP32 pairs, planar rows
    (1, 2, None),      # linear, BF16 pairs, interleaved rows
]


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture
def restore():
    from sscRaft.rafttypes import libraft
    old = os.environ.get("RAFT_BP_TUNE")
    yield
    libraft.raft_filter_set_fixed(1)
    if old is None:
        os.environ.pop("RAFT_BP_TUNE", None)
    else:
        os.environ["RAFT_BP_TUNE"] = old


@pytest.mark.parametrize("N,pad", CASES)
def test_fixed_length_filter_bit_identical_to_generic(N, pad, restore):
    import torch
    from sscRaft.rafttypes import _ptr, libraft
    A, n = 21, 5
    rng = np.random.default_rng(N + pad)
    ang = np.sort((np.arange(A) + rng.uniform(-0.3, 0.3, A)) * (np.pi / A)).astype(np.float32)
    sino = torch.from_numpy(rng.standard_normal((n, A, N)).astype(np.float32)).cuda()
    pf = np.array([0, 0, 1, 0, 1, 1, 3.5], np.float32)
    pi = np.array([N, A, n, N, pad, 0, 0, 5, 0, 0], np.int32)
    for geometry, store, tune in FORMATS:
        if tune is None:
            os.environ.pop("RAFT_BP_TUNE", None)
        else:
            os.environ["RAFT_BP_TUNE"] = tune
        outs = []
        for fixed in (1, 0):
            libraft.raft_filter_set_fixed(fixed)
            out = torch.empty((n, N, N), device="cuda")
            assert libraft.raft_fbp_device(0, _p(out), _p(sino), _ptr(ang), _ptr(pf), _ptr(pi), geometry, store,
                                           None) == 0
            outs.append(out)
        assert torch.isfinite(outs[0]).all()
        assert torch.equal(outs[0], outs[1]), (N, pad, geometry, store, tune,
                                               float((outs[0] - outs[1]).abs().max()))


@pytest.mark.parametrize("N,pad,ftype", [(512, 2, 5), (1024, 1, 7), (1024, 2, 5), (2048, 1, 5), (2048, 2, 5), (2048, 2, 0),
                                         (4096, 1, 7)])
def test_fixed_length_bst_matches_generic(N, pad, ftype, restore):
    from sscRaft.rafttypes import check_error, libraft
    A, n = 33, 2
    rng = np.random.default_rng(N + pad + ftype)
    sino = np.ascontiguousarray(rng.standard_normal((n, A, N)).astype(np.float32))
    ang = np.linspace(0, np.pi, A, endpoint=False).astype(np.float32)
    pi = np.array([N, A, n, N, pad, 0, 0, ftype, 0, 0], np.int32)
    pf = np.array([0, 0, 1, 0, 1, 1, 2.0], np.float32)
    g = np.array([0], np.intc)
    outs = []
    for fixed in (1, 0):
        libraft.raft_filter_set_fixed(fixed)
        obj = np.zeros((n, N, N), np.float32)
        libraft.getBSTMultiGPU(g.ctypes.data, 1, obj.ctypes.data, sino.ctypes.data, ang.ctypes.data,
                               pf.ctypes.data, pi.ctypes.data, 0)
        check_error("bst")
        outs.append(obj)
    assert np.all(np.isfinite(outs[0]))
    np.testing.assert_array_equal(outs[0], outs[1])


@pytest.mark.parametrize("N,zpad,interp", [(512, 2, 1), (1024, 1, 1), (1024, 2, 1), (1024, 2, 0), (2048, 1, 1)])
def test_fixed_length_temfq_matches_generic(N, zpad, interp, restore):
    from sscRaft.rafttypes import check_error, libraft
    A, B, niter, dx = 45, 2, 2, 0.02
    rng = np.random.default_rng(N + zpad + interp)
    flat = np.ascontiguousarray(1e4 * (1 + 0.05 * rng.random((B, N))), np.float32)
    counts = np.ascontiguousarray(rng.poisson(flat[:, None, :] * np.exp(-rng.random((B, A, N)))), np.float32)
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    pi = np.array([N, A, B, N, zpad, 0, 0, B, niter, interp, 0], np.int32)
    pf = np.array([dx, dx, 0.0], np.float32)
    g = np.array([0], np.intc)
    outs = []
    for fixed in (1, 0):
        libraft.raft_filter_set_fixed(fixed)
        obj = np.ones((B, N, N), np.float32)
        libraft.get_tEM_FQ_MultiGPU(g.ctypes.data, 1, counts.ctypes.data, obj.ctypes.data, ang.ctypes.data,
                                    flat.ctypes.data, pf.ctypes.data, pi.ctypes.data)
        check_error("temfq")
        outs.append(obj)
    assert np.all(np.isfinite(outs[0]))
    np.testing.assert_array_equal(outs[0], outs[1])
