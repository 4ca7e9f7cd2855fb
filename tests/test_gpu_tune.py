"""Every backprojector launch shape the autotuner may pick (S slices per CTA,
AB angles per pipeline stage) gives bit-identical images: the per-pixel
accumulation order over angles does not depend on the shape.  The shape is
forced with RAFT_BP_TUNE="S,AB"."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CANDIDATES = ["1,32", "1,16", "2,32", "2,16", "2,8", "4,16", "4,8"]


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture
def restore_env():
    old = os.environ.get("RAFT_BP_TUNE")
    yield
    if old is None:
        os.environ.pop("RAFT_BP_TUNE", None)
    else:
        os.environ["RAFT_BP_TUNE"] = old


def test_fbp_shapes_bit_identical(restore_env):
    import torch
    from sscRaft import synthetic as S
    from sscRaft.rafttypes import _ptr, libraft
    N, A, n = 384, 300, 5
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    img = torch.stack([S.phantom_image(S.ellipse_params(40 + k, 12), N, xp=torch, device="cuda")
                       for k in range(n)]).contiguous()
    sino = torch.empty((n, A, N), device="cuda")
    assert libraft.raft_radon_device(0, _p(sino), _p(img), _ptr(ang), N, N, N, A, n, 1.0, 1.0, None) == 0
    pf = np.array([0, 0, 1, 0, 1, 1, 3.5], np.float32)     # pixel 1, rotation-axis offset 3.5
    pi = np.array([N, A, n, N, 2, 0, 0, 5, 0, 0], np.int32)
    for geometry, store in ((0, 0), (1, 1), (1, 2)):
        outs = {}
        for c in CANDIDATES:
            os.environ["RAFT_BP_TUNE"] = c
            out = torch.empty((n, N, N), device="cuda")
            assert libraft.raft_fbp_device(0, _p(out), _p(sino), _ptr(ang), _ptr(pf), _ptr(pi), geometry, store,
                                           None) == 0
            outs[c] = out
        for c in CANDIDATES[1:]:
            assert torch.equal(outs[c], outs[CANDIDATES[0]]), (geometry, store, c)


def test_em_shapes_bit_identical(restore_env):
    import torch
    from sscRaft import synthetic as S
    from sscRaft.rafttypes import _ptr, libraft
    N, A, n, iters = 256, 180, 5, 4
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    ph = torch.stack([S.phantom_image(S.ellipse_params(60 + k, 12), N, xp=torch, device="cuda")
                      for k in range(n)]).contiguous()
    proj = torch.empty((n, A, N), device="cuda")
    assert libraft.raft_radon_device(0, _p(proj), _p(ph), _ptr(ang), N, N, N, A, n, 1.0, 1.0, None) == 0
    trans = torch.exp(-proj * (3.0 / proj.amax())).contiguous()
    flat = torch.ones((n, N), device="cuda")
    outs = {}
    for c in CANDIDATES:
        os.environ["RAFT_BP_TUNE"] = c
        obj = torch.ones((n, N, N), device="cuda")
        assert libraft.raft_em_device(0, 0, _p(obj), _p(trans), _p(flat), _ptr(ang), N, A, n, iters, None, 1,
                                      None) == 0
        outs[c] = obj
    for c in CANDIDATES[1:]:
        assert torch.equal(outs[c], outs[CANDIDATES[0]]), c
