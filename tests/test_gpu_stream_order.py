"""Stream ordering of the device-pointer entry points.

PyTorch's default stream is the legacy default stream, whose handle is 0,
so Python callers pass a NULL stream.  The library then runs on its own
non-blocking stream, which must first wait for the work already queued on
the legacy stream.  Each test queues a bounded spin kernel and, behind it,
the copy that produces the input, calls the entry point at once with a NULL
stream, and requires the result to equal (bit for bit) a run whose inputs
were complete before the call.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPIN_CYCLES = 200_000_000      # about 0.1 s of a bounded spin on the default stream


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _late_copy(src):
    """A tensor that becomes `src` only after a spin kernel queued before it."""
    import torch
    dst = torch.zeros_like(src)
    torch.cuda.synchronize()
    torch.cuda._sleep(SPIN_CYCLES)
    dst.copy_(src)
    return dst


def _phantom(n, N, seed):
    import torch
    from sscRaft import synthetic as S
    return torch.stack([S.phantom_image(S.ellipse_params(seed + k, 10), N, xp=torch, device="cuda")
                        for k in range(n)]).contiguous()


def test_radon_device_null_stream_waits():
    import torch
    from sscRaft.rafttypes import _ptr, libraft
    N, A, n = 256, 180, 4
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    img = _phantom(n, N, 11)
    ref = torch.empty((n, A, N), device="cuda")
    assert libraft.raft_radon_device(0, _p(ref), _p(img), _ptr(ang), N, N, N, A, n, 1.0, 1.0, None) == 0
    late = _late_copy(img)
    out = torch.zeros_like(ref)
    assert libraft.raft_radon_device(0, _p(out), _p(late), _ptr(ang), N, N, N, A, n, 1.0, 1.0, None) == 0
    torch.cuda.synchronize()
    assert torch.equal(out, ref)


def test_fbp_device_null_stream_waits():
    import torch
    from sscRaft.rafttypes import _ptr, libraft
    N, A, n = 256, 180, 4
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    sino = torch.empty((n, A, N), device="cuda")
    img = _phantom(n, N, 21)
    assert libraft.raft_radon_device(0, _p(sino), _p(img), _ptr(ang), N, N, N, A, n, 1.0, 1.0, None) == 0
    pf = np.array([0, 0, 1, 0, 1, 1, 0], np.float32)
    pi = np.array([N, A, n, N, 2, 0, 0, 5, 0, 0], np.int32)
    for geometry, store in ((0, 0), (1, 1)):
        ref = torch.empty((n, N, N), device="cuda")
        assert libraft.raft_fbp_device(0, _p(ref), _p(sino), _ptr(ang), _ptr(pf), _ptr(pi), geometry, store,
                                       None) == 0
        late = _late_copy(sino)
        out = torch.zeros_like(ref)
        assert libraft.raft_fbp_device(0, _p(out), _p(late), _ptr(ang), _ptr(pf), _ptr(pi), geometry, store,
                                       None) == 0
        torch.cuda.synchronize()
        assert torch.equal(out, ref), (geometry, store)


def test_em_device_null_stream_waits():
    import torch
    from sscRaft.rafttypes import _ptr, libraft
    N, A, n, iters = 128, 90, 4, 5
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    ph = _phantom(n, N, 31) * 0.02
    proj = torch.empty((n, A, N), device="cuda")
    assert libraft.raft_radon_device(0, _p(proj), _p(ph), _ptr(ang), N, N, N, A, n, 1.0, 1.0, None) == 0
    trans = torch.exp(-proj * (2.0 / (N - 1))).contiguous()
    flat = torch.ones((n, N), device="cuda")
    ref = torch.ones((n, N, N), device="cuda")
    assert libraft.raft_em_device(0, 0, _p(ref), _p(trans), _p(flat), _ptr(ang), N, A, n, iters, None, 1,
                                  None) == 0
    late = _late_copy(trans)
    obj = torch.empty((n, N, N), device="cuda")
    obj.fill_(1.0)                       # queued behind the spin as well
    assert libraft.raft_em_device(0, 0, _p(obj), _p(late), _p(flat), _ptr(ang), N, A, n, iters, None, 1,
                                  None) == 0
    torch.cuda.synchronize()
    assert torch.equal(obj, ref)
